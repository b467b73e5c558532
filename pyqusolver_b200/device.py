"""Torch-tensor wrappers around the C ABI (one function per library entry point).

Tensors are CUDA tensors owned by the caller; every call is enqueued on the
current torch stream.  Packed spin words are stored in int32 tensors and
reinterpreted as uint32 by the library.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream_ptr


def _dev(device=None):
    return torch.device("cuda") if device is None else torch.device(device)


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.DTYPE_F32
    if t.dtype == torch.complex64:
        return _lib.DTYPE_C64
    raise TypeError(f"unsupported parameter dtype {t.dtype}")


def n_words(ns: int) -> int:
    return (ns + 31) // 32


def n_params(ns: int, nh: int) -> int:
    return ns + nh + ns * nh


def split_params(flat: torch.Tensor, ns: int, nh: int):
    a = flat[:ns]
    b = flat[ns:ns + nh]
    W = flat[ns + nh:].view(ns, nh)
    return a, b, W


# --------------------------------------------------------------------------------------
# configurations
# --------------------------------------------------------------------------------------

def init_chains(kind: int, n_chains: int, ns: int, seed: int, n_up: int = 0, chain_offset: int = 0, device=None):
    out = torch.empty((n_chains, n_words(ns)), dtype=torch.int32, device=_dev(device))
    call("qes_init_chains", int(kind), int(n_up), C.c_uint64(int(seed) & (2 ** 64 - 1)), int(chain_offset),
         int(n_chains), int(ns), ptr(out), stream_ptr())
    return out


def pack_states(states, device=None) -> torch.Tensor:
    """(B, ns) array of +-0.5 / +-1 / {0,1} values (positive = up) -> packed int32 words on the device."""
    s = states.detach().cpu().numpy() if isinstance(states, torch.Tensor) else np.asarray(states)
    s = np.atleast_2d(s) > 0
    B, ns = s.shape
    nw = n_words(ns)
    pad = np.zeros((B, nw * 32), dtype=bool)
    pad[:, :ns] = s
    words = np.packbits(pad.reshape(B, nw, 32), axis=2, bitorder="little").view(np.uint32).reshape(B, nw)
    return torch.from_numpy(words.view(np.int32).copy()).to(_dev(device))


def unpack_states(words: torch.Tensor, ns: int, value: float = 0.5) -> torch.Tensor:
    """Packed int32 words (B, nw) -> float32 (B, ns) with entries +-value (on the same device)."""
    nw = words.shape[-1]
    shifts = torch.arange(32, device=words.device, dtype=torch.int32)
    bits = (words.reshape(-1, nw, 1) >> shifts) & 1
    bits = bits.reshape(-1, nw * 32)[:, :ns]
    return (bits.to(torch.float32) * (2 * value) - value)


# --------------------------------------------------------------------------------------
# RBM
# --------------------------------------------------------------------------------------

def move_tables(flat_params, ns, nh, move_i, move_j, move_kind, move_major: bool):
    K = int(move_i.shape[0])
    a, b, W = split_params(flat_params, ns, nh)
    shape = (K, nh) if move_major else (nh, K)
    Ct = torch.empty(shape, dtype=flat_params.dtype, device=flat_params.device)
    St = torch.empty_like(Ct)
    A = torch.empty((K,), dtype=flat_params.dtype, device=flat_params.device)
    if K:
        call("qes_rbm_move_tables", dtype_code(flat_params), ns, nh, ptr(a), ptr(W), K, ptr(move_i), ptr(move_j),
             ptr(move_kind), 1 if move_major else 0, ptr(Ct), ptr(St), ptr(A), stream_ptr())
    return Ct, St, A


_FWD_WS = {}


def rbm_forward(flat_params, ns, nh, bits, theta=False, tanh=True, logpsi=True, tensor_cores=False):
    """theta, tanh(theta), log psi of a batch (CUDA cores, or tensor cores when ``tensor_cores``)."""
    n = int(bits.shape[0])
    a, b, W = split_params(flat_params, ns, nh)
    dt, dev = flat_params.dtype, flat_params.device
    th = torch.empty((n, nh), dtype=dt, device=dev) if theta else None
    tn = torch.empty((n, nh), dtype=dt, device=dev) if tanh else None
    lp = torch.empty((n,), dtype=dt, device=dev) if logpsi else None
    if tensor_cores and n > 0:
        nb = C.c_size_t(0)
        call("qes_rbm_forward_tc_workspace_bytes", dtype_code(flat_params), ns, nh, n, C.byref(nb))
        ws = _FWD_WS.get(dev)
        if ws is None or ws.numel() < nb.value:
            ws = torch.empty((int(nb.value),), dtype=torch.uint8, device=dev)
            _FWD_WS[dev] = ws
        call("qes_rbm_forward_tc", dtype_code(flat_params), ns, nh, n, ptr(bits), ptr(a), ptr(b), ptr(W), ptr(th),
             ptr(tn), ptr(lp), ptr(ws), int(ws.numel()), stream_ptr())
        return th, tn, lp
    call("qes_rbm_forward", dtype_code(flat_params), ns, nh, n, ptr(bits), ptr(a), ptr(b), ptr(W), ptr(th), ptr(tn),
         ptr(lp), stream_ptr())
    return th, tn, lp


def forward_uses_tensor_cores(flat_params, ns, nh, n) -> bool:
    """The training step's forward runs on the tensor cores in the mixed form (SR impl 0 or 2) when the
    shapes fit the tensor-core forward."""
    if _lib.sr_impl() in (_lib.SR_IMPL_CUDA_CORES, _lib.SR_IMPL_FP64) or n <= 0:
        return False
    nb = C.c_size_t(0)
    rc = call("qes_rbm_forward_tc_workspace_bytes", dtype_code(flat_params), ns, nh, int(n), C.byref(nb),
              allow=(_lib.QES_ERR_SIZE,))
    return rc == _lib.QES_OK


def rbm_forward_step(flat_params, ns, nh, bits, theta=False, tanh=True, logpsi=True):
    """Forward of the VMC step: tensor cores in the mixed form, CUDA cores in the plain form."""
    tc = forward_uses_tensor_cores(flat_params, ns, nh, int(bits.shape[0]))
    return rbm_forward(flat_params, ns, nh, bits, theta=theta, tanh=tanh, logpsi=logpsi, tensor_cores=tc)


def log_derivatives(flat_params, ns, nh, bits, tanh_theta, out=None):
    n = int(bits.shape[0])
    P = n_params(ns, nh)
    if out is None:
        out = torch.empty((n, P), dtype=flat_params.dtype, device=flat_params.device)
    call("qes_rbm_log_derivatives", dtype_code(flat_params), ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(out),
         int(out.stride(0)), stream_ptr())
    return out


# --------------------------------------------------------------------------------------
# Hamiltonian
# --------------------------------------------------------------------------------------

class DeviceHamiltonian:
    """Device copy of a lowered Hamiltonian and its C struct."""

    def __init__(self, lowered, device=None):
        dev = _dev(device)
        t = lambda x, dt: torch.as_tensor(np.ascontiguousarray(x), dtype=dt, device=dev)
        self.lowered = lowered
        self.ns = lowered.ns
        self.move_i = t(lowered.move_i, torch.int32)
        self.move_j = t(lowered.move_j, torch.int32)
        self.move_kind = t(lowered.move_kind, torch.int32)
        self.move_coef = t(lowered.move_coef.reshape(-1), torch.float32)
        self.zf_site = t(lowered.zf_site, torch.int32)
        self.zf_h = t(lowered.zf_h, torch.float32)
        self.zz_i = t(lowered.zz_i, torch.int32)
        self.zz_j = t(lowered.zz_j, torch.int32)
        self.zz_J = t(lowered.zz_J, torch.float32)
        self.struct = _lib.Hamiltonian(
            lowered.n_moves, ptr(self.move_i), ptr(self.move_j), ptr(self.move_kind), ptr(self.move_coef),
            int(self.zf_site.numel()), ptr(self.zf_site), ptr(self.zf_h),
            int(self.zz_i.numel()), ptr(self.zz_i), ptr(self.zz_j), ptr(self.zz_J))

    @property
    def n_moves(self):
        return self.lowered.n_moves


def local_energy_workspace(dtype_c, ns, nh, n, K):
    nb = C.c_size_t(0)
    call("qes_local_energy_workspace_bytes", dtype_c, ns, nh, n, K, C.byref(nb))
    return int(nb.value)


def local_energy(flat_params, ns, nh, bits, tanh_theta, ham: DeviceHamiltonian, tables, workspace=None):
    n = int(bits.shape[0])
    dc = dtype_code(flat_params)
    need = local_energy_workspace(dc, ns, nh, n, ham.n_moves)
    if workspace is None or workspace.numel() < need:
        workspace = torch.empty((max(need, 1),), dtype=torch.uint8, device=bits.device)
    Ct, St, A = tables
    out = torch.empty((n,), dtype=torch.complex64, device=bits.device)
    call("qes_local_energy", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), C.byref(ham.struct), ptr(Ct), ptr(St),
         ptr(A), ptr(workspace), int(workspace.numel()), ptr(out), stream_ptr())
    return out


def loss_stats(eloc, probs=None, workspace=None):
    n = int(eloc.shape[0])
    nb = C.c_size_t(0)
    call("qes_loss_stats_workspace_bytes", n, C.byref(nb))
    if workspace is None or workspace.numel() < nb.value:
        workspace = torch.empty((int(nb.value),), dtype=torch.uint8, device=eloc.device)
    out = torch.empty((4,), dtype=torch.float64, device=eloc.device)
    call("qes_loss_stats", n, ptr(eloc), ptr(probs), ptr(out), ptr(workspace), int(workspace.numel()), stream_ptr())
    return out


def loss_rhat(eloc, n_chains, workspace=None):
    """[r_hat, sigma2] (float64 device tensor) of E_loc split into n_chains contiguous blocks."""
    n = int(eloc.shape[0])
    nb = C.c_size_t(0)
    call("qes_loss_rhat_workspace_bytes", n, int(n_chains), C.byref(nb))
    if workspace is None or workspace.numel() < nb.value:
        workspace = torch.empty((int(nb.value),), dtype=torch.uint8, device=eloc.device)
    out = torch.empty((2,), dtype=torch.float64, device=eloc.device)
    call("qes_loss_rhat", n, int(n_chains), ptr(eloc), ptr(out), ptr(workspace), int(workspace.numel()), stream_ptr())
    return out


# --------------------------------------------------------------------------------------
# SR
# --------------------------------------------------------------------------------------

def vec_dtype(param_dtype):
    return torch.complex128 if param_dtype == torch.complex64 else torch.float64


def sr_workspace(dtype_c, ns, nh, n, device):
    nb = C.c_size_t(0)
    call("qes_sr_workspace_bytes", dtype_c, ns, nh, n, C.byref(nb))
    return torch.empty((int(nb.value),), dtype=torch.uint8, device=device)


def sample_weights(probs, n, device):
    """float32 device weights normalised to sum n (the reference's probs), or None for uniform sampling."""
    if probs is None:
        return None
    p = torch.as_tensor(probs, device=device).reshape(-1).to(torch.float64)
    if p.numel() != n:
        raise ValueError(f"probs has {p.numel()} entries for {n} samples")
    return (p * (n / p.sum())).to(torch.float32).contiguous()


def sr_force(flat_params, ns, nh, bits, tanh_theta, eloc, workspace=None, probs=None):
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_workspace(dc, ns, nh, n, bits.device)
    F = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    w = sample_weights(probs, n, bits.device)
    call("qes_sr_force_weighted", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(eloc), ptr(w), ptr(F), ptr(ws),
         int(ws.numel()), stream_ptr())
    return F


def sr_matvec(flat_params, ns, nh, bits, tanh_theta, v, shift=0.0, workspace=None, probs=None):
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_workspace(dc, ns, nh, n, bits.device)
    v = v.to(vec_dtype(flat_params.dtype)).contiguous()
    y = torch.empty_like(v)
    w = sample_weights(probs, n, bits.device)
    call("qes_sr_matvec_weighted", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(w), float(shift), ptr(v), ptr(y),
         ptr(ws), int(ws.numel()), stream_ptr())
    return y


def sr_solve_cg(flat_params, ns, nh, bits, tanh_theta, eloc, *, shift, rtol=1e-8, atol=0.0, maxiter=1000,
                check_every=16, rhs_prefactor=-1.0, workspace=None, allow_not_converged=True, x0=None, probs=None,
                precond=None, true_residual=True):
    """x0: initial guess of the unscaled system (S + shift) x = F (a previous solution divided by
    rhs_prefactor), float64 / complex128 of length P on the device; None starts from zero.
    probs: per-sample weights (any positive scale; normalised to sum Ns here), None = uniform.
    precond: None or "jacobi" (CG preconditioned by 1 / diag(S + shift), SciPy's cg(M=...)).
    true_residual: recompute ||F - (S + shift) x|| / ||F|| after the solve (one more matvec);
    info["true_residual"] is -1 when False."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_workspace(dc, ns, nh, n, bits.device)
    x = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    if x0 is not None:
        x0 = x0.to(device=bits.device, dtype=x.dtype).contiguous()
        if x0.numel() != x.numel():
            raise ValueError(f"x0 has {x0.numel()} entries, the parameter vector {x.numel()}")
    pc = {None: _lib.PRECOND_NONE, "none": _lib.PRECOND_NONE, "identity": _lib.PRECOND_NONE,
          "jacobi": _lib.PRECOND_JACOBI}.get(precond if precond is None else str(precond).lower())
    if pc is None:
        raise ValueError(f"preconditioner {precond!r}: None or 'jacobi'")
    opt = _lib.SROptions(float(shift), float(rtol), float(atol), int(maxiter), int(check_every), float(rhs_prefactor),
                         pc, 0 if true_residual else 1)
    res = _lib.SRResult()
    allow = (_lib.QES_ERR_NOT_CONVERGED,) if allow_not_converged else ()
    w = sample_weights(probs, n, bits.device)
    call("qes_sr_solve_cg_weighted", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(eloc), ptr(w), C.byref(opt),
         ptr(x0), ptr(x), C.byref(res), ptr(ws), int(ws.numel()), stream_ptr(), allow=allow)
    info = {"iterations": res.iterations, "converged": bool(res.converged), "residual": res.residual,
            "rhs_norm": res.rhs_norm, "e_mean": complex(res.e_mean_re, res.e_mean_im),
            "true_residual": res.true_residual}
    return x, info


def sr_solve_minres(flat_params, ns, nh, bits, tanh_theta, eloc, *, shift, rtol=1e-8, atol=0.0, maxiter=1000,
                    check_every=16, rhs_prefactor=-1.0, workspace=None, allow_not_converged=True, x0=None,
                    probs=None, true_residual=True):
    """The SR system solved by MINRES (``qes_sr_solve_minres_weighted``): arguments and stopping rule as
    sr_solve_cg; info["acond"] is the recurrence's condition estimate of S + shift."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_workspace(dc, ns, nh, n, bits.device)
    x = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    if x0 is not None:
        x0 = x0.to(device=bits.device, dtype=x.dtype).contiguous()
        if x0.numel() != x.numel():
            raise ValueError(f"x0 has {x0.numel()} entries, the parameter vector {x.numel()}")
    opt = _lib.SROptions(float(shift), float(rtol), float(atol), int(maxiter), int(check_every), float(rhs_prefactor),
                         _lib.PRECOND_NONE, 0 if true_residual else 1)
    res = _lib.SRResult()
    allow = (_lib.QES_ERR_NOT_CONVERGED,) if allow_not_converged else ()
    w = sample_weights(probs, n, bits.device)
    call("qes_sr_solve_minres_weighted", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(eloc), ptr(w), C.byref(opt),
         ptr(x0), ptr(x), C.byref(res), ptr(ws), int(ws.numel()), stream_ptr(), allow=allow)
    info = {"iterations": res.iterations, "converged": bool(res.converged), "residual": res.residual,
            "rhs_norm": res.rhs_norm, "e_mean": complex(res.e_mean_re, res.e_mean_im),
            "true_residual": res.true_residual, "acond": res.acond}
    return x, info


def sr_solve_minsr(flat_params, ns, nh, bits, tanh_theta, eloc, *, shift, rtol=1e-8, atol=0.0, maxiter=1000,
                   check_every=16, rhs_prefactor=-1.0, workspace=None, allow_not_converged=True):
    """MinSR: x = rhs_prefactor * O_c^H y with (O_c O_c^H / Ns + shift) y = E_c / Ns (sample-space CG)."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    nb = C.c_size_t(0)
    call("qes_sr_minsr_workspace_bytes", dc, ns, nh, n, C.byref(nb))
    ws = workspace if workspace is not None and workspace.numel() >= nb.value else torch.empty(
        (int(nb.value),), dtype=torch.uint8, device=bits.device)
    x = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    opt = _lib.SROptions(float(shift), float(rtol), float(atol), int(maxiter), int(check_every), float(rhs_prefactor))
    res = _lib.SRResult()
    allow = (_lib.QES_ERR_NOT_CONVERGED,) if allow_not_converged else ()
    call("qes_sr_solve_minsr", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(eloc), C.byref(opt), ptr(x),
         C.byref(res), ptr(ws), int(ws.numel()), stream_ptr(), allow=allow)
    info = {"iterations": res.iterations, "converged": bool(res.converged), "residual": res.residual,
            "rhs_norm": res.rhs_norm, "e_mean": complex(res.e_mean_re, res.e_mean_im)}
    return x, info, ws


def logpsi_vjp(flat_params, ns, nh, bits, tanh_theta, g, workspace=None):
    """grad = O^H g (hand-written backward of log psi)."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_workspace(dc, ns, nh, n, bits.device)
    g = g.to(torch.complex64).contiguous()
    out = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    call("qes_rbm_logpsi_vjp", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(g), ptr(out), ptr(ws),
         int(ws.numel()), stream_ptr())
    return out


def param_update(flat_params, master, x, lr):
    call("qes_param_update", dtype_code(flat_params), int(flat_params.numel()), float(lr), ptr(x), ptr(master),
         ptr(flat_params), stream_ptr())


# --------------------------------------------------------------------------------------
# sampler
# --------------------------------------------------------------------------------------

def sampler_run(flat_params, ns, nh, cfg: _lib.SamplerConfig, flip_tables, exch, chain_bits, chain_step, proposed,
                accepted, sample_bits, sample_logpsi, last_logpsi, chain_beta=None):
    a, b, W = split_params(flat_params, ns, nh)
    fC, fS = flip_tables if flip_tables is not None else (None, None)
    if exch is not None:
        nbr, nbr_pair, pi, pj, pC, pS = exch
        npairs = int(pi.numel())
    else:
        nbr = nbr_pair = pi = pj = pC = pS = None
        npairs = 0
    if chain_beta is not None:
        call("qes_sampler_run_betas", dtype_code(flat_params), C.byref(cfg), ptr(chain_beta), ptr(a), ptr(b), ptr(W),
             ptr(fC), ptr(fS), ptr(nbr), ptr(nbr_pair), ptr(pi), ptr(pj), npairs, ptr(pC), ptr(pS), ptr(chain_bits),
             ptr(chain_step), ptr(proposed), ptr(accepted), ptr(sample_bits), ptr(sample_logpsi), ptr(last_logpsi),
             stream_ptr())
        return
    call("qes_sampler_run", dtype_code(flat_params), C.byref(cfg), ptr(a), ptr(b), ptr(W), ptr(fC), ptr(fS),
         ptr(nbr), ptr(nbr_pair), ptr(pi), ptr(pj), npairs, ptr(pC), ptr(pS), ptr(chain_bits), ptr(chain_step),
         ptr(proposed), ptr(accepted), ptr(sample_bits), ptr(sample_logpsi), ptr(last_logpsi), stream_ptr())


# --------------------------------------------------------------------------------------
# formed SR matrix (tensor-core Gram) and its float64 Cholesky solve
# --------------------------------------------------------------------------------------

def sr_dense_workspace(dtype_c, ns, nh, n, device, gram_only=False):
    nb = C.c_size_t(0)
    call("qes_sr_dense_workspace_bytes", dtype_c, ns, nh, n, 1 if gram_only else 0, C.byref(nb))
    return torch.empty((int(nb.value),), dtype=torch.uint8, device=device)


def sr_gram(flat_params, ns, nh, bits, tanh_theta, probs=None, workspace=None):
    """S = O_c^H diag(p) O_c / Ns as a (P, P) float64 / complex128 device tensor (full Hermitian)."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    P = n_params(ns, nh)
    ws = workspace if workspace is not None else sr_dense_workspace(dc, ns, nh, n, bits.device, gram_only=True)
    S = torch.empty((P, P), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    w = sample_weights(probs, n, bits.device)
    call("qes_sr_gram", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(w), ptr(S), ptr(ws), int(ws.numel()),
         stream_ptr())
    return S


def sr_solve_dense(flat_params, ns, nh, bits, tanh_theta, eloc, *, shift, rhs_prefactor=-1.0, probs=None,
                   workspace=None, allow_not_pd=True):
    """x = rhs_prefactor (S + shift)^-1 F with S formed on the tensor cores and a float64 Cholesky solve."""
    dc = dtype_code(flat_params)
    n = int(bits.shape[0])
    ws = workspace if workspace is not None else sr_dense_workspace(dc, ns, nh, n, bits.device)
    x = torch.empty((n_params(ns, nh),), dtype=vec_dtype(flat_params.dtype), device=bits.device)
    opt = _lib.SROptions(float(shift), 0.0, 0.0, 0, 0, float(rhs_prefactor))
    res = _lib.SRResult()
    w = sample_weights(probs, n, bits.device)
    allow = (_lib.QES_ERR_NOT_CONVERGED,) if allow_not_pd else ()
    call("qes_sr_solve_dense", dc, ns, nh, n, ptr(bits), ptr(tanh_theta), ptr(eloc), ptr(w), C.byref(opt), ptr(x),
         C.byref(res), ptr(ws), int(ws.numel()), stream_ptr(), allow=allow)
    info = {"iterations": 0, "converged": bool(res.converged), "residual": res.residual, "rhs_norm": res.rhs_norm,
            "e_mean": complex(res.e_mean_re, res.e_mean_im), "true_residual": res.true_residual}
    return x, info, ws


def sr_dense_workspace_bytes(flat_params, ns, nh, n, gram_only=False):
    nb = C.c_size_t(0)
    call("qes_sr_dense_workspace_bytes", dtype_code(flat_params), ns, nh, int(n), 1 if gram_only else 0,
         C.byref(nb))
    return int(nb.value)
