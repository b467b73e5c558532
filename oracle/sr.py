"""Stochastic reconfiguration / TDVP solve (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``TDVP`` (``QES/NQS/src/tdvp.py``) with the normalisation pinned by
``Python/tests/nqs/test_tdvp_matrix_free_regressions.py:46-151``:

* centring of E_loc and O, promotion to float64/complex128 (``tdvp.py:1056-1085``);
* force F = O_c^H E_c / Ns (``tdvp.py:1099-1108``);
* standard SR solves (O_c^H O_c / Ns + shift I) x = F
  (GRAM form: s = O_c, s_p = O_c^H; MATVEC form v -> O_c^H (O_c v) / Ns);
* MinSR solves (O_c O_c^H / Ns + shift I) y = E_c / Ns and projects x = O_c^H y
  (``tdvp.py:1199-1226,1393-1408``);
* x <- rhs_prefactor * x (default -1), optional global-norm clip
  (``tdvp.py:882-907,1382-1422``);
* Euler / SGD update p <- p + lr * x (``nqs_train.py:1235-1262``).

The CG stopping rule is SciPy's (the reference's default ``lin_solver`` is
``scipy_cg``, ``QES/NQS/nqs.py:3014``): stop when ||r|| <= max(rtol*||b||, atol).
Centring with non-uniform sample weights is not pinned by the reference
(its SR module is in the empty submodule); the weighted form here uses the
weighted means and weights w_s / Ns in every sum.
"""

from __future__ import annotations

import numpy as np


def prepare(e_loc, O, probs=None):
    e = np.asarray(e_loc)
    O = np.asarray(O)
    dt = np.complex128 if (np.iscomplexobj(e) or np.iscomplexobj(O)) else np.float64
    e = e.astype(dt)
    O = O.astype(np.complex128 if np.iscomplexobj(O) else np.float64)
    ns = e.shape[0]
    if probs is None:
        w = np.ones(ns)
    else:
        w = np.asarray(probs, dtype=np.float64).reshape(-1)
    e_m = np.sum(w * e) / ns
    o_m = (w @ O) / ns
    return e - e_m, O - o_m[None, :], w, e_m, o_m


def force(O_c, e_c, w=None):
    ns = O_c.shape[0]
    w = np.ones(ns) if w is None else w
    return np.conj(O_c).T @ (w * e_c) / ns


def s_matrix(O_c, w=None):
    ns = O_c.shape[0]
    w = np.ones(ns) if w is None else w
    return np.conj(O_c).T @ (w[:, None] * O_c) / ns


def cg(matvec, b, *, rtol=1e-8, atol=0.0, maxiter=1000, x0=None, minv=None):
    """Conjugate gradients in float64/complex128.  Returns (x, iterations, residual_norm, converged).
    minv: the diagonal of a preconditioner M ~ A^-1 (SciPy's ``cg(M=...)``: z = M r, rho = r^H z);
    the stopping rule stays ||r|| <= max(rtol ||b||, atol)."""
    b = np.asarray(b)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=b.dtype)
    r = b - matvec(x) if x0 is not None else b.copy()
    z = r if minv is None else minv * r
    p = z.copy()
    rho = np.vdot(r, z).real
    bnorm = np.linalg.norm(b)
    thresh = max(rtol * bnorm, atol)
    if np.linalg.norm(r) <= thresh:
        return x, 0, np.linalg.norm(r), True
    for it in range(1, maxiter + 1):
        Ap = matvec(p)
        alpha = rho / np.vdot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        rn = np.linalg.norm(r)
        if rn <= thresh:
            return x, it, rn, True
        z = r if minv is None else minv * r
        rho_new = np.vdot(r, z).real
        p = z + (rho_new / rho) * p
        rho = rho_new
    return x, maxiter, np.linalg.norm(r), False


def minres(matvec, b, *, rtol=1e-8, atol=0.0, maxiter=1000, x0=None):
    """MINRES for a Hermitian operator (Paige & Saunders 1975; the recurrences of SciPy's ``minres``
    without a preconditioner), stopping when the recurrence's residual norm phibar <=
    max(rtol ||b||, atol), the rule of ``cg``.  The reference selects it with lin_solver 'minres' /
    'minres_qlp' (``QES/NQS/__init__.py:406``; the solvers live in the absent ``general_python``
    submodule).  Returns (x, iterations, phibar, converged, acond)."""
    b = np.asarray(b)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=b.dtype)
    r1 = b - matvec(x) if x0 is not None else b.copy()
    y = r1.copy()
    beta1 = np.sqrt(np.vdot(r1, y).real)
    thresh = max(rtol * np.linalg.norm(b), atol)
    if beta1 <= thresh:
        return x, 0, beta1, True, -1.0
    oldb, beta, dbar, epsln, phibar = 0.0, beta1, 0.0, 0.0, beta1
    cs, sn = -1.0, 0.0
    w = np.zeros_like(b)
    w2 = np.zeros_like(b)
    r2 = r1.copy()
    gmax, gmin = 0.0, np.inf
    for it in range(1, maxiter + 1):
        v = y / beta
        y = matvec(v)
        if it >= 2:
            y = y - (beta / oldb) * r1
        alfa = np.vdot(v, y).real
        y = y - (alfa / beta) * r2
        r1, r2 = r2, y
        oldb, beta = beta, np.sqrt(np.vdot(r2, r2).real)
        oldeps = epsln
        delta = cs * dbar + sn * alfa
        gbar = sn * dbar - cs * alfa
        epsln = sn * beta
        dbar = -cs * beta
        gamma = max(np.hypot(gbar, beta), np.finfo(float).tiny)
        cs, sn = gbar / gamma, beta / gamma
        phi, phibar = cs * phibar, sn * phibar
        w1, w2 = w2, w
        w = (v - oldeps * w1 - delta * w2) / gamma
        x = x + phi * w
        gmax, gmin = max(gmax, gamma), min(gmin, gamma)
        y = r2
        if phibar <= thresh or beta == 0.0:
            return x, it, phibar, True, gmax / gmin
    return x, maxiter, phibar, False, gmax / gmin


def jacobi_minv(O_c, w=None, shift=0.0):
    """Inverse diagonal of S + shift, diag(S)_k = sum_s w_s |O_c,sk|^2 / Ns: the Jacobi preconditioner
    named 'jacobi' by the reference's solver options (``QES/NQS/__init__.py:405-407``,
    ``tdvp.py:686-710``; its implementation lives in the absent ``general_python`` submodule, so this
    is the textbook diagonal of the same S)."""
    n = O_c.shape[0]
    w = np.ones(n) if w is None else np.asarray(w, dtype=np.float64)
    d = (w[:, None] * np.abs(O_c) ** 2).sum(axis=0) / n + shift
    return 1.0 / d


def solve_sr(e_loc, O, *, shift=1e-3, probs=None, method="dense", rtol=1e-8,
             maxiter=1000, rhs_prefactor=-1.0, grad_clip=None, use_minsr=False):
    """Return (x, info) with x already scaled by rhs_prefactor (and clipped)."""
    e_c, O_c, w, e_m, o_m = prepare(e_loc, O, probs)
    ns, npar = O_c.shape
    info = {"mean": e_m, "o_mean": o_m}
    if use_minsr:
        T = (np.sqrt(w)[:, None] * O_c) @ (np.conj(O_c).T * np.sqrt(w)[None, :]) / ns
        rhs = np.sqrt(w) * e_c / ns
        y = np.linalg.solve(T + shift * np.eye(ns), rhs)
        x = np.conj(O_c).T @ (np.sqrt(w) * y)
        info.update(iterations=0, converged=True)
    else:
        F = force(O_c, e_c, w)
        info["force"] = F
        if method == "dense":
            S = s_matrix(O_c, w)
            x = np.linalg.solve(S + shift * np.eye(npar), F)
            info.update(iterations=0, converged=True)
        elif method == "cg":
            def mv(v):
                return np.conj(O_c).T @ (w * (O_c @ v)) / ns + shift * v
            x, it, res, conv = cg(mv, F, rtol=rtol, maxiter=maxiter)
            info.update(iterations=it, residual=res, converged=conv)
        else:
            raise ValueError(method)
    x = rhs_prefactor * x
    if grad_clip is not None and grad_clip > 0:
        nrm = np.linalg.norm(x)
        if nrm > grad_clip:
            x = x * (grad_clip / (nrm + 1e-12))
    return x, info


# --------------------------------------------------------------------------------------
# Large shapes: O built chunk by chunk from the RBM (never whole), same normalisation
# --------------------------------------------------------------------------------------

def o_rows(params, sigma, tanh=None):
    """O rows [sigma, t, sigma (x) t] in float64 / complex128.  tanh=None evaluates t = tanh(theta)
    from the parameters in float64; given, t is the network's own (float32) output promoted, which
    is what the reference's SR receives (it promotes the network's O to float64,
    ``tdvp.py:827-858``)."""
    from . import rbm as rbm_mod
    if tanh is None:
        return rbm_mod.log_derivatives(params, sigma)
    t = np.asarray(tanh)
    t = t.astype(np.complex128 if np.iscomplexobj(t) else np.float64)
    sigma = np.atleast_2d(np.asarray(sigma, dtype=np.float64))
    ow = (sigma[:, :, None] * t[:, None, :]).reshape(sigma.shape[0], -1)
    return np.concatenate([sigma.astype(t.dtype), t, ow.astype(t.dtype)], axis=1)


def _o_chunks(params, sigma, chunk, tanh=None):
    for r0 in range(0, sigma.shape[0], chunk):
        yield r0, _o_chunks_one(params, sigma, r0, chunk, tanh)


def _o_chunks_one(params, sigma, r0, chunk, tanh=None):
    return o_rows(params, sigma[r0:r0 + chunk], None if tanh is None else tanh[r0:r0 + chunk])


def matvec_chunked(params, sigma, v, shift=0.0, chunk=64, probs=None, tanh=None):
    """(S + shift) v with S = O_c^H diag(w) O_c / Ns, O rebuilt per sample chunk (two passes)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    ns = sigma.shape[0]
    w = np.ones(ns) if probs is None else np.asarray(probs, dtype=np.float64)
    Ov = np.concatenate([O @ v for _, O in _o_chunks(params, sigma, chunk, tanh)])
    u = w * (Ov - np.sum(w * Ov) / ns) / ns
    y = shift * np.asarray(v, dtype=np.result_type(v, Ov))
    for r0, O in _o_chunks(params, sigma, chunk, tanh):
        y = y + np.conj(O).T @ u[r0:r0 + O.shape[0]]
    return y


def solve_sr_chunked(params, sigma, e_loc, shift, rhs_prefactor=-1.0, chunk=64, tanh=None):
    """Parameter-space SR solution through the sample-space identity
    (O_c^H O_c / Ns + shift)^-1 O_c^H E_c / Ns = O_c^H (O_c O_c^H / Ns + shift)^-1 E_c / Ns,
    with the Ns x Ns Gram matrix accumulated from O chunks; returns (x * rhs_prefactor, F)."""
    sigma = np.asarray(sigma, dtype=np.float64)
    ns = sigma.shape[0]
    e = np.asarray(e_loc)
    ec = e - e.mean()
    chunks = list(range(0, ns, chunk))
    om = None
    for _, O in _o_chunks(params, sigma, chunk, tanh):
        om = O.sum(axis=0) if om is None else om + O.sum(axis=0)
    om = om / ns
    G = np.zeros((ns, ns), dtype=np.complex128 if np.iscomplexobj(om) else np.float64)
    F = np.zeros_like(om)
    for a in chunks:
        Oa = _o_chunks_one(params, sigma, a, chunk, tanh) - om[None, :]
        F = F + np.conj(Oa).T @ ec[a:a + Oa.shape[0]]
        for b in chunks:
            if b < a:
                continue
            Ob = Oa if b == a else _o_chunks_one(params, sigma, b, chunk, tanh) - om[None, :]
            blk = Oa @ np.conj(Ob).T
            G[a:a + Oa.shape[0], b:b + Ob.shape[0]] = blk
            if b != a:
                G[b:b + Ob.shape[0], a:a + Oa.shape[0]] = np.conj(blk).T
    F = F / ns
    y = np.linalg.solve(G / ns + shift * np.eye(ns), ec / ns)
    x = np.zeros_like(om)
    for a in chunks:
        Oa = _o_chunks_one(params, sigma, a, chunk, tanh) - om[None, :]
        x = x + np.conj(Oa).T @ y[a:a + Oa.shape[0]]
    return rhs_prefactor * x, F
