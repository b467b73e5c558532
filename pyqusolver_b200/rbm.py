"""RBM ansatz on the GPU: parameters, forward, fast-update hooks, hand-written backward.

log psi(sigma) = sum_i a_i sigma_i + sum_m log cosh(theta_m),  theta = W^T sigma + b,
with sigma = +-1 obtained from the +-0.5 states (the reference's ``in_activation``,
``Python/tests/nqs/test_network_representation_consistency.py:121-156``).
P = N*M + N + M (``QES/NQS/src/network/presets.py:117-137``); the flat order is
[a, b, W] with W row-major.  Parameters live on the device as float32 or
complex64 (the working copy the kernels read) and as a float64/complex128
master copy that the SR update accumulates into.

Gradients: ``RBMLogPsi`` is a ``torch.autograd.Function`` whose backward is the
library's O^H g kernel (O_a = sigma, O_b = tanh theta, O_W = sigma tanh theta,
holomorphic for complex parameters).
"""

from __future__ import annotations

import numpy as np
import torch

from . import device as dv


class RBM:
    fast_update_supported_rules = {"LOCAL", "EXCHANGE"}
    family = "rbm"

    def __init__(self, input_shape, n_hidden=None, *, alpha=None, dtype="complex64", param_dtype=None, seed=0,
                 init_scale=0.01, device=None, **_):
        ns = int(np.prod(input_shape)) if not np.isscalar(input_shape) else int(input_shape)
        if n_hidden is None:
            n_hidden = int(round((alpha if alpha is not None else 1.0) * ns))
        self.ns, self.nh = ns, int(n_hidden)
        dt = param_dtype if param_dtype is not None else dtype
        self.is_complex = _is_complex(dt)
        self.dtype = torch.complex64 if self.is_complex else torch.float32
        self.master_dtype = torch.complex128 if self.is_complex else torch.float64
        self.device = torch.device("cuda") if device is None else torch.device(device)
        self.seed = seed
        self.init_scale = init_scale
        rng = np.random.default_rng(seed)
        P = self.n_params
        x = rng.normal(0.0, init_scale, size=P)
        if self.is_complex:
            x = x + 1j * rng.normal(0.0, init_scale, size=P)
        self._set_flat(x)

    # ------------------------------------------------------------------ parameters
    @property
    def n_params(self):
        return dv.n_params(self.ns, self.nh)

    def _set_flat(self, x):
        x = torch.as_tensor(np.asarray(x) if not isinstance(x, torch.Tensor) else x)
        self.master = x.to(device=self.device, dtype=self.master_dtype).contiguous().clone()
        self.flat = self.master.to(self.dtype).contiguous()
        self.version = getattr(self, "version", 0) + 1

    def get_params(self, unravel=False):
        """The parameter tree in the reference RBM's layout, ``{"visible_bias": a, "VisibleToHidden":
        {"kernel": W, "bias": b}}`` (``Python/tests/nqs/test_nqs_entropy_exact_sum.py:51-57``), or the
        flat [a, b, W] vector with ``unravel``."""
        if unravel:
            return self.master.clone()
        a, b, W = dv.split_params(self.master, self.ns, self.nh)
        return {"visible_bias": a.clone(), "VisibleToHidden": {"kernel": W.clone(), "bias": b.clone()}}

    def set_params(self, params):
        if isinstance(params, dict):
            a, b, W = rbm_leaves(params)
            flat = torch.cat([torch.as_tensor(x).reshape(-1).to(self.master_dtype).cpu() for x in (a, b, W)])
        else:
            flat = torch.as_tensor(params).reshape(-1)
        if flat.numel() != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {flat.numel()}")
        self._set_flat(flat)

    def bump(self):
        """Mark the device copy as changed (tables depending on W are rebuilt lazily)."""
        self.version += 1

    @property
    def params_shapes(self):
        return [(self.ns,), (self.nh,), (self.ns, self.nh)]

    @property
    def params_sizes(self):
        return [self.ns, self.nh, self.ns * self.nh]

    @property
    def params_cpx(self):
        return [self.is_complex] * 3

    # ------------------------------------------------------------------ evaluation
    def bits(self, states):
        if isinstance(states, torch.Tensor) and states.dtype == torch.int32 and states.dim() == 2 \
                and states.shape[1] == dv.n_words(self.ns) and states.is_cuda:
            return states
        return dv.pack_states(states, self.device)

    def __call__(self, states):
        return self.log_psi(states)

    def log_psi(self, states):
        bits = self.bits(states)
        return dv.rbm_forward(self.flat, self.ns, self.nh, bits, theta=False, tanh=False, logpsi=True)[2]

    def theta(self, states):
        return dv.rbm_forward(self.flat, self.ns, self.nh, self.bits(states), theta=True, tanh=False,
                              logpsi=False)[0]

    def init_log_psi_delta_cache(self, params, states):
        return self.theta(states)

    def log_psi_delta(self, params, current_val, states, update_info, cache=None):
        """Delta log psi for flipping the listed sites (sequentially; a masked entry is skipped)."""
        st = states.detach().cpu().numpy() if isinstance(states, torch.Tensor) else np.asarray(states)
        st = np.atleast_2d(np.array(st, dtype=np.float32, copy=True))
        if isinstance(update_info, tuple):
            idx, valid = update_info
        else:
            idx, valid = update_info, None
        idx = np.atleast_2d(np.asarray(idx.cpu() if isinstance(idx, torch.Tensor) else idx))
        valid = np.ones_like(idx, dtype=bool) if valid is None else \
            np.atleast_2d(np.asarray(valid.cpu() if isinstance(valid, torch.Tensor) else valid))
        for r in range(st.shape[0]):
            for i, ok in zip(idx[r], valid[r]):
                if ok:
                    st[r, i] = -st[r, i]
        new = self.log_psi(st)
        cur = torch.as_tensor(current_val, device=self.device).to(new.dtype)
        delta = new - cur
        if cache is not None:
            return delta, self.theta(st)
        return delta

    def log_derivative(self, states):
        bits = self.bits(states)
        _, tn, _ = dv.rbm_forward(self.flat, self.ns, self.nh, bits, theta=False, tanh=True, logpsi=False)
        return dv.log_derivatives(self.flat, self.ns, self.nh, bits, tn)

    def log_psi_autograd(self, states, params=None):
        """log psi as a differentiable function of the flat parameter tensor."""
        p = self.flat.detach().requires_grad_(True) if params is None else params
        return RBMLogPsi.apply(p, self.bits(states), self), p


def rbm_leaves(params):
    """(a, b, W) of an RBM parameter tree: the reference's nested layout (``visible_bias``,
    ``VisibleToHidden/kernel``, ``VisibleToHidden/bias``), its flattened npz form with keys joined
    by "/", or the names ``visible_bias`` / ``hidden_bias`` / ``W``; a leading ``params/`` level is
    accepted.  Raises KeyError when a leaf is missing."""
    flat = {}

    def walk(d, prefix):
        for k, v in d.items():
            key = f"{prefix}/{k}" if prefix else str(k)
            if isinstance(v, dict):
                walk(v, key)
            else:
                flat[key] = v
    walk(params, "")
    flat = {(k[len("params/"):] if k.startswith("params/") else k): v for k, v in flat.items()}

    def pick(*names):
        for n in names:
            if n in flat:
                return flat[n]
        raise KeyError(f"RBM parameter tree has none of {names}; keys: {sorted(flat)}")
    return (pick("visible_bias"), pick("VisibleToHidden/bias", "hidden_bias"),
            pick("VisibleToHidden/kernel", "W"))


def _is_complex(dt):
    s = str(dt).lower()
    return "complex" in s


class RBMLogPsi(torch.autograd.Function):
    """log psi(flat params) with the library's hand-written O^H g backward."""

    @staticmethod
    def forward(ctx, flat, bits, net):
        _, tn, lp = dv.rbm_forward(flat.detach(), net.ns, net.nh, bits, theta=False, tanh=True, logpsi=True)
        ctx.save_for_backward(bits, tn)
        ctx.net = net
        ctx.flat_dtype = flat.dtype
        return lp

    @staticmethod
    def backward(ctx, g):
        bits, tn = ctx.saved_tensors
        net = ctx.net
        g = g.contiguous()
        if not torch.is_complex(g):
            g = g.to(torch.complex64)
        # PyTorch's complex convention: grad_in = conj(d logpsi / d p) * g  (holomorphic)
        flat_like = torch.empty(1, dtype=ctx.flat_dtype, device=bits.device)
        grad = dv.logpsi_vjp(flat_like, net.ns, net.nh, bits, tn, g)
        return grad.to(ctx.flat_dtype), None, None
