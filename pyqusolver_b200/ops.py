"""The library's hot-path entry points registered as PyTorch operators (``torch.ops.qes_b200.*``).

Each operator is a thin shim over one C-ABI call (through ``device.py``); there is no other
implementation behind it: on a CPU tensor or without the library the call raises.  Fake
(meta) implementations give output shapes and dtypes, so the operators can be traced.

    torch.ops.qes_b200.rbm_forward(flat, bits, ns, nh)            -> (tanh theta, log psi)
    torch.ops.qes_b200.log_derivatives(flat, bits, tanh, ns, nh)  -> O (rows x P)
    torch.ops.qes_b200.logpsi_vjp(flat, bits, tanh, g, ns, nh)    -> O^H g (float64 / complex128)
    torch.ops.qes_b200.sr_matvec(flat, bits, tanh, v, ns, nh, shift) -> (S + shift) v
    torch.ops.qes_b200.sr_solve_cg(flat, bits, tanh, eloc, ns, nh, shift, rtol, maxiter) -> x
    torch.ops.qes_b200.loss_stats(eloc)                            -> [mean_re, mean_im, var, std]
"""

from __future__ import annotations

from typing import Tuple

import torch

from . import device as dv

_NS = "qes_b200"


def _vec_dtype(dt):
    return torch.complex128 if dt == torch.complex64 else torch.float64


@torch.library.custom_op(f"{_NS}::rbm_forward", mutates_args=(), device_types="cuda")
def rbm_forward(flat: torch.Tensor, bits: torch.Tensor, ns: int, nh: int) -> Tuple[torch.Tensor, torch.Tensor]:
    _, tn, lp = dv.rbm_forward(flat, ns, nh, bits, theta=False, tanh=True, logpsi=True)
    return tn, lp


@rbm_forward.register_fake
def _(flat, bits, ns, nh):
    n = bits.shape[0]
    return flat.new_empty((n, nh)), flat.new_empty((n,))


@torch.library.custom_op(f"{_NS}::log_derivatives", mutates_args=(), device_types="cuda")
def log_derivatives(flat: torch.Tensor, bits: torch.Tensor, tanh_theta: torch.Tensor, ns: int, nh: int) -> torch.Tensor:
    return dv.log_derivatives(flat, ns, nh, bits, tanh_theta)


@log_derivatives.register_fake
def _(flat, bits, tanh_theta, ns, nh):
    return flat.new_empty((bits.shape[0], dv.n_params(ns, nh)))


@torch.library.custom_op(f"{_NS}::logpsi_vjp", mutates_args=(), device_types="cuda")
def logpsi_vjp(flat: torch.Tensor, bits: torch.Tensor, tanh_theta: torch.Tensor, g: torch.Tensor, ns: int,
               nh: int) -> torch.Tensor:
    return dv.logpsi_vjp(flat, ns, nh, bits, tanh_theta, g)


@logpsi_vjp.register_fake
def _(flat, bits, tanh_theta, g, ns, nh):
    return flat.new_empty((dv.n_params(ns, nh),), dtype=_vec_dtype(flat.dtype))


@torch.library.custom_op(f"{_NS}::sr_matvec", mutates_args=(), device_types="cuda")
def sr_matvec(flat: torch.Tensor, bits: torch.Tensor, tanh_theta: torch.Tensor, v: torch.Tensor, ns: int, nh: int,
              shift: float) -> torch.Tensor:
    return dv.sr_matvec(flat, ns, nh, bits, tanh_theta, v, shift=shift)


@sr_matvec.register_fake
def _(flat, bits, tanh_theta, v, ns, nh, shift):
    return torch.empty_like(v)


@torch.library.custom_op(f"{_NS}::sr_solve_cg", mutates_args=(), device_types="cuda")
def sr_solve_cg(flat: torch.Tensor, bits: torch.Tensor, tanh_theta: torch.Tensor, eloc: torch.Tensor, ns: int,
                nh: int, shift: float, rtol: float, maxiter: int) -> torch.Tensor:
    x, _ = dv.sr_solve_cg(flat, ns, nh, bits, tanh_theta, eloc, shift=shift, rtol=rtol, maxiter=maxiter)
    return x


@sr_solve_cg.register_fake
def _(flat, bits, tanh_theta, eloc, ns, nh, shift, rtol, maxiter):
    return flat.new_empty((dv.n_params(ns, nh),), dtype=_vec_dtype(flat.dtype))


@torch.library.custom_op(f"{_NS}::loss_stats", mutates_args=(), device_types="cuda")
def loss_stats(eloc: torch.Tensor) -> torch.Tensor:
    return dv.loss_stats(eloc)


@loss_stats.register_fake
def _(eloc):
    return eloc.new_empty((4,), dtype=torch.float64)
