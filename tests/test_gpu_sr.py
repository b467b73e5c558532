"""SR solver paths through the C ABI: bounded-wait time-outs of the fused CG kernel.

A time-out is made on purpose with the library's barrier test hook (one arrival
that never comes and a short poll limit); every wait stays bounded, the kernel
records the time-out in a status word and the solve returns QES_ERR_TIMEOUT.
"""

import numpy as np
import pytest
import torch

import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.rbm import RBM

pytestmark = pytest.mark.gpu


def _small_problem(cplx, n=700, ns=9, nh=18, seed=6):
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=seed, init_scale=0.2)
    rng = np.random.default_rng(seed)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    return net, bits, tn, eloc


@pytest.mark.parametrize("device_loop", [0, 1])
@pytest.mark.parametrize("impl", [0, 1])
def test_fused_cg_barrier_timeout_is_reported_and_solver_recovers(impl, device_loop):
    net, bits, tn, eloc = _small_problem(cplx=True)
    _lib.set_sr_impl(impl)
    _lib.call("qes_set_cg_fused", 2)
    _lib.call("qes_set_cg_device_loop", device_loop)
    ref, info_ref = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10,
                                   maxiter=2000, check_every=4)
    try:
        _lib.call("qes_sr_set_barrier_test", 1, 1000)
        with pytest.raises(_lib.QESError) as ei:
            dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000,
                           check_every=4)
        assert ei.value.code == _lib.QES_ERR_TIMEOUT
    finally:
        _lib.call("qes_sr_set_barrier_test", 0, 0)
    try:
        x, info = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000,
                                 check_every=4)
        assert info["converged"] and info["iterations"] == info_ref["iterations"]
        assert torch.equal(x, ref)
    finally:
        _lib.call("qes_set_cg_fused", 1)
        _lib.call("qes_set_cg_device_loop", 1)
        _lib.set_sr_impl(0)


# ------------------------------------------------------------------------- sample weights
from oracle import rbm as orbm, sr as osr


def _oracle_params(net):
    flat = net.flat.detach().cpu().numpy().astype(np.complex128 if net.is_complex else np.float64)
    return orbm.RBMParams.from_flat(flat, net.ns, net.nh)


def rel_err(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-30, np.max(np.abs(b)))


@pytest.mark.parametrize("cplx,impl,big", [(True, 2, False), (True, 1, False), (False, 2, False), (False, 1, False),
                                           (False, 2, True)])
def test_weighted_sr_matches_oracle(cplx, impl, big):
    """probs-weighted force, matvec and CG solution (qes_sr_*_weighted) against the oracle's weighted
    centring F = O_c^H diag(p) E_c / Ns, S = O_c^H diag(p) O_c / Ns with means sum p X / Ns; the
    weights are the sampler's reweighting factors exp(c Re log psi), normalised to sum Ns.  `big`
    runs the M/N-tiled tensor-core O^H u (144 sites)."""
    if big:
        ns, nh, n = 144, 144, 512
        model = qb.TransverseFieldIsing(qb.SquareLattice(2, 12, 12), j=1.0, hx=1.5)
    else:
        ns, nh, n = 9, 18, 700
        model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=6, init_scale=0.2 if not big else 0.05)
    rng = np.random.default_rng(6)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=True)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    # reweighting factors as VMCSampler returns them (exponent 1: samples drawn from |psi|^1)
    lu = lp.real.double().cpu().numpy()
    pr = np.exp(lu - lu.max())
    probs = pr / pr.sum() * n
    probs_t = torch.as_tensor(probs.astype(np.float32)).cuda()
    w = probs_t.double().cpu().numpy()
    w = w / w.sum() * n                                        # the library renormalises the same way
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    # the oracle's SR on the network's own float32 tanh rows, promoted (what the reference's SR receives)
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    F = osr.force(Oc, ec, w_)
    S = osr.s_matrix(Oc, w_)
    _lib.set_sr_impl(impl)
    try:
        if impl == 2:
            assert _lib.sr_uses_tensor_cores(dv.dtype_code(net.flat), ns, nh, n)
        Fg = dv.sr_force(net.flat, ns, nh, bits, tn, eloc, probs=probs_t).cpu().numpy()
        assert rel_err(Fg, F) < 1e-4
        v = rng.normal(size=O.shape[1]) + (1j * rng.normal(size=O.shape[1]) if cplx else 0)
        y = dv.sr_matvec(net.flat, ns, nh, bits, tn, torch.as_tensor(v).cuda(), shift=1e-3, probs=probs_t)
        assert rel_err(y.cpu().numpy(), S @ v + 1e-3 * v) < 1e-4
        x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=3000,
                                 probs=probs_t)
        A = S + 1e-2 * np.eye(S.shape[0])
        xr = np.linalg.solve(A, F)
        assert info["converged"]
        xg = -x.cpu().numpy()
        resid = np.linalg.norm(A @ xg - F) / np.linalg.norm(F)
        assert resid < 1e-4 and 0.0 <= info["true_residual"] < 1e-4
        err = xg - xr
        assert np.sqrt(abs(np.vdot(err, A @ err)) / abs(np.vdot(xr, A @ xr))) < 1e-2
        # unit weights reproduce the unweighted entry points exactly
        ones = torch.ones(n, dtype=torch.float32, device="cuda")
        assert torch.equal(dv.sr_force(net.flat, ns, nh, bits, tn, eloc, probs=ones),
                           dv.sr_force(net.flat, ns, nh, bits, tn, eloc))
    finally:
        _lib.set_sr_impl(0)


def test_train_step_uses_the_sampler_weights():
    """NQS with s_mu = 1 (samples from |psi|^1): train_step's energy is the weighted mean and its
    SR direction the weighted solve of the same batch."""
    L = qb.SquareLattice(1, 10)
    model = qb.TransverseFieldIsing(L, j=1.0, hx=0.7)
    kw = dict(alpha=1, dtype="float32", seed=4, s_numchains=256, s_numsamples=2, s_therm_steps=4, s_sweep_steps=4,
              init_scale=0.2)
    nqs = qb.NQS("rbm", model, s_mu=1.0, **kw)
    assert not nqs.sampler.has_uniform_weights
    from pyqusolver_b200.tdvp import TDVP
    td = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_maxiter=2000, sr_tol=1e-10)
    flat0 = nqs.net.master.clone()
    # the same batch the step will draw: a twin NQS in the same state
    twin = qb.NQS("rbm", model, s_mu=1.0, **kw)
    bits, lp = twin.sampler.sample_bits()
    probs = twin.sampler.sample_probs(lp)
    _, tn, _ = dv.rbm_forward_step(twin.net.flat, 10, 10, bits, tanh=True, logpsi=False)
    eloc = twin.local_energy_bits(bits, tn)
    st = dv.loss_stats(eloc, probs).cpu().numpy()
    x_ref, _ = dv.sr_solve_cg(twin.net.flat, 10, 10, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000,
                              probs=probs)
    info = nqs.train_step(lr=0.1, tdvp=td)
    assert info["mean"] == pytest.approx(complex(st[0], st[1]), rel=1e-12)
    step = (nqs.net.master - flat0) / 0.1
    assert torch.allclose(step, x_ref, rtol=1e-9, atol=1e-12)


# ------------------------------------------------------------------------- fused S v kernel
@pytest.mark.parametrize("cplx", [True, False])
@pytest.mark.parametrize("n", [700, 19244])
def test_fused_sv_matches_kernel_pair_and_oracle(cplx, n):
    """The cooperative S v kernel (qes_sr_set_fused_sv(1)) against the O v + O^H u kernel pair (0, the
    default), with the single-product and the split-complex O v (qes_sr_set_ov_split), on the same
    weighted batch, and all against the oracle's weighted S v.  n = 19244 is
    151 sample tiles (the last one 44 samples): more tiles than CTAs, so some CTAs fold two tiles
    into their TMEM accumulators."""
    ns, nh = 9, 18
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=8, init_scale=0.2)
    rng = np.random.default_rng(8)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=True)
    lu = lp.real.double().cpu().numpy()
    pr = np.exp(lu - lu.max())
    probs_t = torch.as_tensor((pr / pr.sum() * n).astype(np.float32)).cuda()
    w = probs_t.double().cpu().numpy()
    w = w / w.sum() * n
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    _, Oc, w_, _, _ = osr.prepare(np.zeros(n), O, w)
    S = osr.s_matrix(Oc, w_)
    v = rng.normal(size=O.shape[1]) + (1j * rng.normal(size=O.shape[1]) if cplx else 0)
    vt = torch.as_tensor(v).cuda()
    ys = {}
    _lib.set_sr_impl(2)
    try:
        # (fused S v, split-complex O v): the fused kernel reads the single-product operand
        for fused, split in ((1, 0), (0, 0), (0, 1)):
            _lib.call("qes_sr_set_fused_sv", fused)
            _lib.call("qes_sr_set_ov_split", split)
            assert _lib.sr_uses_tensor_cores(dv.dtype_code(net.flat), ns, nh, n)
            plan = _lib.sr_tc_plan(dv.dtype_code(net.flat), ns, nh, n)
            assert plan["sv"] == fused
            ys[fused, split] = dv.sr_matvec(net.flat, ns, nh, bits, tn, vt, shift=1e-3, probs=probs_t).cpu().numpy()
            again = dv.sr_matvec(net.flat, ns, nh, bits, tn, vt, shift=1e-3, probs=probs_t).cpu().numpy()
            assert np.array_equal(ys[fused, split], again)      # fixed summation order: repeatable
    finally:
        _lib.call("qes_sr_set_fused_sv", 0)
        _lib.call("qes_sr_set_ov_split", 0)
        _lib.set_sr_impl(0)
    ref = S @ v + 1e-3 * v
    for key, y in ys.items():
        assert rel_err(y, ref) < 1e-4, key
        assert rel_err(y, ys[0, 0]) < 2e-5, key


# ------------------------------------------------------------------------- Jacobi-preconditioned CG
@pytest.mark.parametrize("cplx,impl,fused", [(True, 0, 0), (True, 0, 2), (True, 1, 0), (True, 3, 0), (False, 0, 0),
                                             (False, 1, 2), (False, 3, 0)])
def test_jacobi_pcg_matches_oracle(cplx, impl, fused):
    """qes_sr_solve_cg with QES_PRECOND_JACOBI (TDVP(sr_precond="jacobi")): the solution of the weighted
    SR system against a dense float64 solve (backward error, A-norm error); in the float64 form
    (impl 3) also the iteration count against the oracle's preconditioned CG on the same system,
    which checks the diagonal (weighted diag(S) + shift) and the recurrence.  The float32 forms take
    more iterations on these small, ill-conditioned systems (their operator's rounding slows any
    Krylov method), so for them the solution is the bar.  fused = 2 runs the vector updates in the
    cooperative CG kernel."""
    ns, nh, n = 9, 18, 700
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=5, init_scale=0.3)
    rng = np.random.default_rng(5)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=True)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    lu = lp.real.double().cpu().numpy()
    pr = np.exp(0.5 * (lu - lu.max()))
    probs_t = torch.as_tensor((pr / pr.sum() * n).astype(np.float32)).cuda()
    w = probs_t.double().cpu().numpy()
    w = w / w.sum() * n
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    F = osr.force(Oc, ec, w_)
    shift = 1e-2
    A = osr.s_matrix(Oc, w_) + shift * np.eye(O.shape[1])
    minv = osr.jacobi_minv(Oc, w_, shift)
    assert np.allclose(1.0 / minv, np.real(np.diag(A)), rtol=1e-12)
    _, it_ref, _, conv_ref = osr.cg(lambda v: A @ v, F, rtol=1e-5, maxiter=3000, minv=minv)
    _, it_plain, _, _ = osr.cg(lambda v: A @ v, F, rtol=1e-5, maxiter=3000)
    assert conv_ref
    _lib.set_sr_impl(impl)
    _lib.call("qes_set_cg_fused", fused)
    try:
        x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=1e-8, maxiter=3000,
                                 probs=probs_t, precond="jacobi", check_every=4)
        _, info5 = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=1e-5, maxiter=3000,
                                  probs=probs_t, precond="jacobi", check_every=1)
    finally:
        _lib.call("qes_set_cg_fused", 1)
        _lib.set_sr_impl(0)
    assert info["converged"]
    xg = -x.cpu().numpy()
    assert np.linalg.norm(A @ xg - F) / np.linalg.norm(F) < 1e-4
    xr = np.linalg.solve(A, F)
    err = xg - xr
    assert np.sqrt(abs(np.vdot(err, A @ err)) / abs(np.vdot(xr, A @ xr))) < 1e-3
    assert info5["converged"]
    if impl == 3:
        assert abs(info5["iterations"] - it_ref) <= max(3, 0.05 * it_ref), (info5["iterations"], it_ref, it_plain)


def test_tdvp_jacobi_option_reaches_the_solver():
    """TDVP(sr_precond="jacobi") and NQS.train(pre_solver="jacobi") run the preconditioned CG (the
    iteration count differs from the plain CG on the same batch); unknown preconditioners raise."""
    from pyqusolver_b200.tdvp import TDVP
    net, bits, tn, eloc = _small_problem(cplx=True)
    plain = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_maxiter=2000)
    jac = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_maxiter=2000, sr_precond="jacobi")
    _lib.set_sr_impl(3)               # float64 form: the two solutions agree to the CG tolerance
    try:
        x0 = plain.solve(net, bits, tn, eloc)
        x1 = jac.solve(net, bits, tn, eloc)
    finally:
        _lib.set_sr_impl(0)
    assert plain.last_info["converged"] and jac.last_info["converged"]
    assert plain.last_info["iterations"] != jac.last_info["iterations"]
    assert torch.allclose(x0, x1, rtol=1e-3, atol=1e-5 * float(x0.abs().max()))
    with pytest.raises(NotImplementedError):
        TDVP(sr_precond="ilu")


# ------------------------------------------------------------------------- MINRES
@pytest.mark.parametrize("cplx,impl", [(True, 0), (True, 1), (True, 3), (False, 0), (False, 1), (False, 3)])
def test_minres_matches_oracle(cplx, impl):
    """qes_sr_solve_minres_weighted (TDVP(sr_lin_solver="minres" / "minres_qlp")): solution against a dense
    float64 solve; in the float64 form (impl 3) also the iteration count and the condition estimate
    against the oracle's MINRES on the same weighted system.  With a float32 operator MINRES's
    attainable accuracy is about (operator rounding) x cond(A) (Sleijpen, van der Vorst and Modersitzki,
    SIAM J. Matrix Anal. Appl. 22 (2000) 726), larger than CG's, so its backward-error bar scales with
    the reported condition estimate."""
    ns, nh, n = 9, 18, 700
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=9, init_scale=0.3)
    rng = np.random.default_rng(9)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=True)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    lu = lp.real.double().cpu().numpy()
    pr = np.exp(0.5 * (lu - lu.max()))
    probs_t = torch.as_tensor((pr / pr.sum() * n).astype(np.float32)).cuda()
    w = probs_t.double().cpu().numpy()
    w = w / w.sum() * n
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    F = osr.force(Oc, ec, w_)
    shift = 1e-2
    A = osr.s_matrix(Oc, w_) + shift * np.eye(O.shape[1])
    _, it_ref, _, conv_ref, acond_ref = osr.minres(lambda v: A @ v, F, rtol=1e-5, maxiter=3000)
    assert conv_ref
    _lib.set_sr_impl(impl)
    try:
        x, info = dv.sr_solve_minres(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=1e-8, maxiter=3000,
                                     probs=probs_t, check_every=8)
        _, info5 = dv.sr_solve_minres(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=1e-5, maxiter=3000,
                                      probs=probs_t, check_every=1)
    finally:
        _lib.set_sr_impl(0)
    assert info["converged"]
    xg = -x.cpu().numpy()
    # operator rounding: ~1e-6 for the plain FP32 contractions, ~1e-5 for the BF16 hi/lo split (the dropped
    # lo*lo term is 2^-16 relative)
    bar = 1e-6 if impl == 3 else max(1e-4, (1e-5 if impl == 0 else 1e-6) * info["acond"])
    assert np.linalg.norm(A @ xg - F) / np.linalg.norm(F) < bar
    assert 0.0 <= info["true_residual"] < bar
    xr = np.linalg.solve(A, F)
    err = xg - xr
    assert np.sqrt(abs(np.vdot(err, A @ err)) / abs(np.vdot(xr, A @ xr))) < (1e-5 if impl == 3 else 1e-2)
    assert info5["converged"] and info5["acond"] > 1.0
    if impl == 3:
        assert abs(info5["iterations"] - it_ref) <= max(3, 0.05 * it_ref), (info5["iterations"], it_ref)
        # a rough estimate: the device takes alpha = v^H A v before the three-term subtraction (SciPy
        # after it), equal in exact arithmetic; the extreme gammas move by some 10% with rounding
        assert info5["acond"] == pytest.approx(acond_ref, rel=0.25)


def test_tdvp_minres_qlp_option():
    from pyqusolver_b200.tdvp import TDVP
    net, bits, tn, eloc = _small_problem(cplx=True)
    cg = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_maxiter=2000, sr_tol=1e-10)
    mr = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_maxiter=2000, sr_tol=1e-10, sr_lin_solver="minres_qlp")
    _lib.set_sr_impl(3)               # float64 form: CG and MINRES agree to their tolerance
    try:
        x0 = cg.solve(net, bits, tn, eloc)
        x1 = mr.solve(net, bits, tn, eloc)
    finally:
        _lib.set_sr_impl(0)
    assert mr.last_info["converged"] and mr.last_info["acond"] > 1.0
    assert torch.allclose(x0, x1, rtol=1e-4, atol=1e-6 * float(x0.abs().max()))
    with pytest.raises(NotImplementedError):
        TDVP(sr_lin_solver="minres", sr_precond="jacobi")


# ------------------------------------------------------------------------- Chronopoulos-Gear CG steps
@pytest.mark.parametrize("impl", [0, 1, 3])
@pytest.mark.parametrize("rtol", [1e-8, 1e-10])
def test_cg_single_reduction_matches_two_reduction_form(impl, rtol):
    """qes_set_cg_single_reduction(1) (Chronopoulos-Gear steps, the matvec of r with |r|^2 summed by
    its split reduction, one update kernel) against the standard steps (0, the default: matvec of
    p, x/r update with its |r|^2 reduction, p update) on the same weighted system, down to tight
    tolerances (the convergence test runs on the residual vector's norm in both): both converge;
    the standard form meets the dense solve's backward-error bar of 1e-4, the Chronopoulos-Gear
    form 1e-4 in float64 and 1e-3 in the float32 forms (its s = A p recurrence carries the
    operator's rounding forward, a wider residual gap); in the float64 form (impl 3) the iteration
    counts agree to within 3% and the solutions to 1e-6, in the float32 forms (0 = tensor cores,
    1 = CUDA cores, whose operator rounding makes late iterations sensitive to any change) the
    iteration counts to within 25%."""
    ns, nh, n = 10, 20, 700                      # P = 230: the vector form of the split reduction
    model = qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=15, init_scale=0.3)
    rng = np.random.default_rng(15)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=True)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    lu = lp.real.double().cpu().numpy()
    pr = np.exp(0.5 * (lu - lu.max()))
    probs_t = torch.as_tensor((pr / pr.sum() * n).astype(np.float32)).cuda()
    w = probs_t.double().cpu().numpy()
    w = w / w.sum() * n
    e = eloc.cpu().numpy().astype(np.complex128)
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    F = osr.force(Oc, ec, w_)
    shift = 1e-2
    A = osr.s_matrix(Oc, w_) + shift * np.eye(O.shape[1])
    out = {}
    _lib.set_sr_impl(impl)
    _lib.call("qes_set_cg_fused", 0)
    try:
        for single in (1, 0):
            _lib.call("qes_set_cg_single_reduction", single)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=rtol, maxiter=3000,
                                     probs=probs_t, check_every=8)
            out[single] = (-x.cpu().numpy(), info)
    finally:
        _lib.call("qes_set_cg_single_reduction", 0)
        _lib.call("qes_set_cg_fused", 1)
        _lib.set_sr_impl(0)
    (x1, i1), (x0, i0) = out[1], out[0]
    assert i1["converged"] and i0["converged"]
    assert i1["residual"] <= rtol * i1["rhs_norm"] * (1 + 1e-12)
    assert np.linalg.norm(A @ x0 - F) / np.linalg.norm(F) < 1e-4
    # the s = A p recurrence carries the float32 operator's rounding forward: a larger gap between
    # the recursive and the true residual in the float32 forms
    bar1 = 1e-4 if impl == 3 else 1e-3
    assert np.linalg.norm(A @ x1 - F) / np.linalg.norm(F) < bar1
    if impl == 3:
        assert abs(i1["iterations"] - i0["iterations"]) <= max(1, 0.03 * i0["iterations"]), (i1["iterations"],
                                                                                            i0["iterations"])
        assert np.max(np.abs(x1 - x0)) / np.max(np.abs(x0)) < 1e-6
    else:
        assert abs(i1["iterations"] - i0["iterations"]) <= max(2, 0.25 * i0["iterations"])
