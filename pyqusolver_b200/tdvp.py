"""TDVP / stochastic reconfiguration with the reference's options and conventions.

Mirrors ``QES/NQS/src/tdvp.py`` for the RBM path:

* centring and float64 promotion (``get_tdvp_standard`` ``:1056-1132``);
* force F = O_c^H E_c / Ns, standard SR (O_c^H O_c / Ns + shift) x = F in the
  GRAM / MATVEC form (``_solve_prepare_matvec`` ``:1138-1197``);
* x <- rhs_prefactor * x (default 1, as the reference's TDVP; NQS.train passes -1), optional global-norm clip
  (``_finalize_solution`` ``:1410-1422``, ``_apply_grad_clip`` ``:882-907``);
* ``use_sr=False`` returns x = -rhs_prefactor * F ... i.e. the reference's
  ``-final_b`` branch (``solve`` ``:1561-1569``);
* ``use_minsr=True`` solves the sample-space system (O_c O_c^H / Ns + shift) y = E_c / Ns
  and returns O_c^H y (``_solve_prepare_s_and_loss`` ``:1199-1226``, ``_project_minsr_result``
  ``:1393-1408``), matrix-free on the same kernels.

The solve runs on the GPU (``qes_sr_solve_cg_weighted``): the RBM's O is applied in
structured form and never materialised, CG vectors and dots are float64.  With the
sampler's reweighting factors (``probs``, when mu * beta != 1 / logprob_fact) the means
and sample sums of F and S are weighted (``vmc.py:1173-1184``).
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import device as dv


@dataclass
class TDVPStepInfo:
    mean_energy: complex
    std_energy: float
    iterations: int
    converged: bool
    residual: float


_SOLVERS_CG = ("scipy_cg", "cg")
_SOLVERS_MINRES = ("minres", "scipy_minres", "minres_qlp")
_SOLVERS_DIRECT = ("cholesky", "direct", "scipy_direct", "solve")


class TDVP:
    """Keyword arguments mirror ``TDVP.__init__`` (``tdvp.py:322-350``), defaults included
    (``rhs_prefactor=1.0``, ``sr_maxiter=100``; ``NQS.train`` passes the trainer's -1.0 / 1000).
    Options whose effect this path does not implement raise instead of being ignored; options that
    only tune solvers or features this path does not offer (the pseudo-inverse and SNR tolerances,
    backend, logger, timing) are accepted because they cannot change a CG result.  ``sr_tol`` /
    ``sr_atol`` (SciPy's rtol / atol), ``check_every``, ``use_old_result`` and ``true_residual`` are
    this package's additions; ``true_residual=True`` has every CG / MINRES solve recompute
    ||F - (S + shift) x|| / ||F|| with one more matvec (``last_info["true_residual"]``, -1 when off,
    the default: the reference computes no such diagnostic)."""

    def __init__(self, use_sr=True, use_minsr=False, rhs_prefactor=1.0, *, regularization=0.0,
                 sr_lin_solver=None, sr_precond=None, sr_snr_tol=1e-3, sr_pinv_tol=1e-14, sr_pinv_cutoff=1e-8,
                 sr_diag_shift=1e-3, sr_lin_solver_t="gram", sr_lin_x0=None, sr_maxiter=100, sr_form_matrix=False,
                 backend="default", logger=None, use_timing=False, dtype=None, grad_clip=None, verbose=False,
                 sr_tol=1e-8, sr_atol=0.0, check_every=16, use_old_result=False, true_residual=False):
        solver = "scipy_cg" if sr_lin_solver is None else str(getattr(sr_lin_solver, "name", sr_lin_solver)).lower()
        if solver not in _SOLVERS_CG + _SOLVERS_MINRES + _SOLVERS_DIRECT:
            raise NotImplementedError(f"linear solver {sr_lin_solver!r}: the GPU path implements CG (scipy_cg), "
                                      f"MINRES (minres, minres_qlp) and, on the formed matrix, a Cholesky solve")
        precond = None if sr_precond is None else str(getattr(sr_precond, "name", sr_precond)).lower()
        if precond in ("identity", "none"):
            precond = None
        if precond not in (None, "jacobi"):
            raise NotImplementedError(f"preconditioner {sr_precond!r}: the GPU path implements 'jacobi' "
                                      f"(1 / diag(S + shift)) and none")
        if precond is not None and use_minsr:
            raise NotImplementedError("a preconditioner on the MinSR (sample-space) system is not implemented")
        if precond is not None and solver in _SOLVERS_MINRES:
            raise NotImplementedError("a preconditioner on the MINRES path is not implemented (CG takes 'jacobi')")
        if solver in _SOLVERS_MINRES and (use_minsr or sr_form_matrix):
            raise NotImplementedError("MINRES runs on the matrix-free S v of the parameter-space SR system")
        if str(sr_lin_solver_t).lower() not in ("gram", "matvec", "matrix_free"):
            raise NotImplementedError(f"solver form {sr_lin_solver_t!r}: the GPU path applies S matrix-free")
        if solver in _SOLVERS_DIRECT and not sr_form_matrix:
            raise ValueError(f"linear solver {sr_lin_solver!r} needs the formed matrix (sr_form_matrix=True)")
        if sr_form_matrix and use_minsr:
            raise NotImplementedError("sr_form_matrix with MinSR (the Ns x Ns matrix) is not implemented")
        # formed matrix: S on the tensor cores, solved by a float64 Cholesky factorisation (the CG
        # solution it stands for is the same solution to within the CG tolerance)
        self.form_matrix = bool(sr_form_matrix)
        # Jacobi: CG on S + shift preconditioned by 1 / diag(S + shift) (a direct solve of the formed
        # matrix gives the same solution with or without it)
        self.sr_precond = precond
        self._dense_ws = None
        if regularization:
            raise NotImplementedError("regularization != 0 is not implemented on the GPU path")
        self.use_sr = bool(use_sr)
        self.use_minsr = bool(use_minsr)
        self._minsr_ws = None
        self.rhs_prefactor = float(rhs_prefactor)
        self.sr_lin_solver = solver
        self.sr_diag_shift = float(sr_diag_shift)
        self.sr_tol = float(sr_tol)
        self.sr_atol = float(sr_atol)
        self.sr_maxiter = int(sr_maxiter)
        self.grad_clip = grad_clip
        self.check_every = int(check_every)
        self.true_residual = bool(true_residual)
        self._workspace = None
        self.last_info = None
        # initial guess of the CG (QES/NQS/src/tdvp.py:1346-1380): a fixed vector sr_lin_x0, or with
        # use_old_result the previous solution (stored scaled, divided by rhs_prefactor for the
        # unscaled system); zeros when neither applies or the shape does not match
        self._x0 = sr_lin_x0
        self.use_old_result = bool(use_old_result)
        self._solution = None

    def set_diag_shift(self, shift):
        self.sr_diag_shift = float(shift)

    def _ws(self, net, n):
        dc = dv.dtype_code(net.flat)
        import ctypes as C
        from . import _lib
        nb = C.c_size_t(0)
        _lib.call("qes_sr_workspace_bytes", dc, net.ns, net.nh, n, C.byref(nb))
        if self._workspace is None or self._workspace.numel() < nb.value:
            self._workspace = torch.empty((int(nb.value),), dtype=torch.uint8, device=net.device)
        return self._workspace

    def _solve_handle_x0(self, P, use_old_result):
        x0 = self._x0
        if use_old_result and self._solution is not None:
            x0 = self._solution
            if self.rhs_prefactor != 1.0 and abs(self.rhs_prefactor) > 1e-12:
                x0 = x0 / self.rhs_prefactor
        if x0 is None or int(torch.as_tensor(x0).numel()) != P:
            return None
        return torch.as_tensor(x0)

    def solve(self, net, bits, tanh_theta, eloc, use_old_result=None, probs=None):
        """Parameter direction x (float64 / complex128, length P), already scaled by rhs_prefactor.
        probs: the sampler's reweighting factors (None when it samples |psi|^2): weighted means and
        sample sums in F and S (``qes_sr_solve_cg_weighted``)."""
        n = int(bits.shape[0])
        ws = self._ws(net, n)
        use_old = self.use_old_result if use_old_result is None else bool(use_old_result)
        if probs is not None and self.use_sr and self.use_minsr:
            raise NotImplementedError("MinSR with non-uniform sample weights is not implemented on the GPU path")
        if not self.use_sr:
            F = dv.sr_force(net.flat, net.ns, net.nh, bits, tanh_theta, eloc, workspace=ws, probs=probs)
            x = -(F * self.rhs_prefactor) if self.rhs_prefactor != 1.0 else -F
            self.last_info = {"iterations": 0, "converged": True, "residual": 0.0}
        elif self.form_matrix:
            x, info, self._dense_ws = dv.sr_solve_dense(
                net.flat, net.ns, net.nh, bits, tanh_theta, eloc, shift=self.sr_diag_shift,
                rhs_prefactor=self.rhs_prefactor, probs=probs,
                workspace=self._dense_ws if self._dense_ws is not None and self._dense_ws.numel() >=
                dv.sr_dense_workspace_bytes(net.flat, net.ns, net.nh, n) else None)
            self.last_info = info
            self._solution = x.detach().clone()
        elif self.use_minsr:
            x, info, self._minsr_ws = dv.sr_solve_minsr(
                net.flat, net.ns, net.nh, bits, tanh_theta, eloc, shift=self.sr_diag_shift, rtol=self.sr_tol,
                atol=self.sr_atol, maxiter=self.sr_maxiter, check_every=self.check_every,
                rhs_prefactor=self.rhs_prefactor, workspace=self._minsr_ws)
            self.last_info = info
        else:
            x0 = self._solve_handle_x0(dv.n_params(net.ns, net.nh), use_old)
            if self.sr_lin_solver in _SOLVERS_MINRES:
                # minres_qlp: MINRES iterates until the condition estimate (info["acond"]) passes
                # MINRES-QLP's switch threshold, which a positive shift keeps S + shift far from
                x, info = dv.sr_solve_minres(net.flat, net.ns, net.nh, bits, tanh_theta, eloc,
                                             shift=self.sr_diag_shift, rtol=self.sr_tol, atol=self.sr_atol,
                                             maxiter=self.sr_maxiter, check_every=self.check_every,
                                             rhs_prefactor=self.rhs_prefactor, workspace=ws, x0=x0, probs=probs,
                                             true_residual=self.true_residual)
            else:
                x, info = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tanh_theta, eloc, shift=self.sr_diag_shift,
                                         rtol=self.sr_tol, atol=self.sr_atol, maxiter=self.sr_maxiter,
                                         check_every=self.check_every, rhs_prefactor=self.rhs_prefactor,
                                         workspace=ws, x0=x0, probs=probs, precond=self.sr_precond,
                                         true_residual=self.true_residual)
            self.last_info = info
            self._solution = x.detach().clone()
        if self.grad_clip is not None and self.grad_clip > 0:
            nrm = torch.linalg.vector_norm(x)
            x = x * torch.clamp(self.grad_clip / (nrm + 1e-12), max=1.0)
        return x
