"""Oracle parity at the benchmarked shapes, through the C ABI.

* heis10x10: Heisenberg XXX on the 10x10 periodic lattice (XXZ jxy = jz = -1), Sz = 0 samples,
  complex64 RBM alpha = 2 (M = 200, P = 20,300);
* tfim20x20: TFIM on the 20x20 periodic lattice, J = 1, hx = 3.04, real RBM alpha = 4
  (M = 1600, P = 642,000): the large tensor-core SR tiling (sites in 4 M tiles, hidden units in
  N chunks, sample chunks folded in TMEM).

Forward, E_loc and O are held to 1e-5 relative against the float64 oracle (the plain-FP32 bar).
The SR stage is checked against the oracle's SR applied to the network's own float32 tanh(theta)
rows promoted to float64 -- what the reference's SR receives, since it promotes the float32
network's O (tdvp.py:827-858) -- with O rebuilt chunk by chunk (never whole): force and matvec to
1e-4.  The SR checks run on the tensor cores (impl 2, the mixed form), on the CUDA cores in
float32 (impl 1, the plain form) and in float64 (impl 3, the reference's SR precision).

The CG solution is held to backward-error bars, not to an entrywise bar: at these shapes
(P >> Ns, shift 1e-3 / 1e-4) S + shift has condition numbers of 1e5-1e7, and a float32 or
BF16-split contraction (relative error ~1e-6-1e-5) limits the true residual of any Krylov solve to
about that level; the solution components along the near-null directions of S (eigenvalue ~ shift)
then differ from the float64 solve by up to residual / shift, while everything the update does to
the energy agrees.  Asserted for the float32 forms: the relative true residual in the oracle's
float64 operator below 1e-4, F^H x within 1e-5, and the error in the (S + shift)-norm (the norm
CG minimises) below 2e-2 of the solution's; the float64 form solves the same system as the
oracle and is held entrywise (1e-4).  Even the float32 rounding of T alone (the float64 oracle
fed tanh(theta) from float64 theta instead of the network's float32 rows) moves the true residual
of these systems to ~1e-5.
"""

import numpy as np
import pytest
import torch

from oracle import lattice as olat, hamiltonian as oH, rbm as orbm, estimator as oest, sampler as osm, sr as osr
import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.rbm import RBM

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b)))


def oracle_params(net):
    flat = net.flat.detach().cpu().numpy().astype(np.complex128 if net.is_complex else np.float64)
    return orbm.RBMParams.from_flat(flat, net.ns, net.nh)


def _heis10x10(init_scale):
    L, OL = qb.SquareLattice(2, 10, 10), olat.SquareLattice(2, 10, 10)
    model, terms = qb.XXZ(L, jxy=-1.0, jz=-1.0), oH.xxz_terms(OL, -1.0, -1.0)
    net = RBM((100,), alpha=2, dtype="complex64", seed=21, init_scale=init_scale)
    states = lambda n, seed: osm.init_states("RND_FIXED", n, 100, seed=seed, n_up=50) * 0.5
    return model, terms, net, states


def _tfim20x20(init_scale):
    L, OL = qb.SquareLattice(2, 20, 20), olat.SquareLattice(2, 20, 20)
    model, terms = qb.TransverseFieldIsing(L, j=1.0, hx=3.04, hz=0.0), oH.tfim_terms(OL, 1.0, 3.04, 0.0)
    net = RBM((400,), alpha=4, dtype="float32", seed=22, init_scale=init_scale)
    states = lambda n, seed: np.where(np.random.default_rng(seed).random((n, 400)) < 0.5, 0.5, -0.5)
    return model, terms, net, states


SHAPES = {"heis10x10": (_heis10x10, 256, 256, 256), "tfim20x20": (_tfim20x20, 64, 32, 16)}


@pytest.mark.parametrize("init_scale", [0.01, 0.05])
@pytest.mark.parametrize("shape", list(SHAPES))
def test_forward_local_energy_and_O_at_bench_shape(shape, init_scale):
    mk, n_fwd, n_el, n_o = SHAPES[shape]
    model, terms, net, states = mk(init_scale)
    ns, nh = net.ns, net.nh
    p = oracle_params(net)
    st = states(n_fwd, 11)
    bits = dv.pack_states(st)
    sig = orbm.to_sigma(st)
    th, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, theta=True, tanh=True, logpsi=True)
    assert rel_err(th.cpu().numpy(), orbm.theta(p, sig)) < RTOL
    th64 = th.cpu().numpy().astype(np.complex128 if net.is_complex else np.float64)
    assert rel_err(tn.cpu().numpy(), np.tanh(th64)) < RTOL
    lp_ref = orbm.log_psi(p, sig)
    assert np.max(np.abs(lp.cpu().numpy().real - lp_ref.real)) <= RTOL * max(1.0, np.max(np.abs(lp_ref.real)))
    # the mixed form's tensor-core forward (three-term BF16 split of W) at the same shape
    th2, tn2, lp2 = dv.rbm_forward(net.flat, ns, nh, bits, theta=True, tanh=True, logpsi=True, tensor_cores=True)
    assert rel_err(th2.cpu().numpy(), orbm.theta(p, sig)) < RTOL
    assert np.max(np.abs(lp2.cpu().numpy().real - lp_ref.real)) <= RTOL * max(1.0, np.max(np.abs(lp_ref.real)))
    # local energy
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    e = dv.local_energy(net.flat, ns, nh, bits[:n_el], tn[:n_el], h, tables).cpu().numpy()
    ref = oest.local_energy_full(p, terms, st[:n_el])
    assert np.max(np.abs(e - ref)) / max(1.0, np.max(np.abs(ref))) < RTOL
    # log-derivatives
    O = dv.log_derivatives(net.flat, ns, nh, bits[:n_o], tn[:n_o]).cpu().numpy()
    assert rel_err(O, orbm.log_derivatives(p, sig[:n_o])) < RTOL


SR_SHAPES = {"heis10x10": (_heis10x10, 1000, 1e-3, 64), "tfim20x20": (_tfim20x20, 256, 1e-4, 64)}


@pytest.fixture
def sr_impl():
    yield _lib.set_sr_impl
    _lib.set_sr_impl(0)


@pytest.mark.parametrize("impl", [2, 1, 3])
@pytest.mark.parametrize("shape", list(SR_SHAPES))
def test_sr_force_matvec_and_solution_at_bench_shape(sr_impl, shape, impl):
    """impl 2: tensor cores (mixed form), 1: CUDA cores in float32 (plain form), 3: CUDA cores in
    float64 (the reference's SR precision), whose solution is also held entrywise (1e-4)."""
    mk, n, shift, chunk = SR_SHAPES[shape]
    model, terms, net, states = mk(0.05)
    ns, nh = net.ns, net.nh
    st = states(n, 13)
    bits = dv.pack_states(st)
    sig = orbm.to_sigma(st)
    p = oracle_params(net)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    t32 = tn.cpu().numpy()                    # the network's float32 rows (forward checked above)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    e = eloc.cpu().numpy().astype(np.complex128)
    if not net.is_complex:
        e = e.real
    sr_impl(impl)
    if impl == 2:
        assert _lib.sr_uses_tensor_cores(dv.dtype_code(net.flat), ns, nh, n)
    rng = np.random.default_rng(7)
    P = dv.n_params(ns, nh)
    v = rng.normal(size=P) + (1j * rng.normal(size=P) if net.is_complex else 0)
    y = dv.sr_matvec(net.flat, ns, nh, bits, tn, torch.as_tensor(v).cuda(), shift=shift).cpu().numpy()
    y_ref = osr.matvec_chunked(p, sig, v, shift=shift, chunk=chunk, tanh=t32)
    assert rel_err(y, y_ref) < 1e-4
    x_ref, F_ref = osr.solve_sr_chunked(p, sig, e, shift, rhs_prefactor=-1.0, chunk=chunk, tanh=t32)
    F = dv.sr_force(net.flat, ns, nh, bits, tn, eloc).cpu().numpy()
    assert rel_err(F, F_ref) < 1e-4
    x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=shift, rtol=1e-8, maxiter=3000)
    assert info["converged"]
    xg = x.cpu().numpy()
    A = lambda u: osr.matvec_chunked(p, sig, u, shift=shift, chunk=chunk, tanh=t32)
    resid = np.linalg.norm(A(-xg) - F_ref) / np.linalg.norm(F_ref)          # x carries rhs_prefactor -1
    assert resid < 1e-4, resid
    fx = lambda u: np.vdot(F_ref, u)
    assert abs(fx(xg) - fx(x_ref)) <= 1e-5 * abs(fx(x_ref))
    err = xg - x_ref
    a_err = np.sqrt(abs(np.vdot(err, A(err)))) / np.sqrt(abs(np.vdot(x_ref, A(x_ref))))
    assert a_err < 2e-2, a_err
    # the library's own post-solve residual (in its own operator) is of the same small size
    assert 0.0 <= info["true_residual"] < 1e-4
    if impl == 3:
        # float64 contractions of the float32 network's T: the same system up to T's float32
        # rounding, so the solve reaches the oracle's solution entrywise
        assert resid < 1e-6, resid
        assert rel_err(xg, x_ref) < 1e-4


# ------------------------------------------------------------------------- public API: NQS.sample / NQS.step
@pytest.mark.parametrize("mu", [2.0, 1.0])
def test_nqs_sample_and_step_through_public_api(mu):
    """NQS.sample's ((last, last_logpsi), (configs, logpsi), probs) and NQS.step's NQSSingleStepResult
    (``QES/NQS/nqs.py:1896-1942,2353-2424``) against the oracle sampler, estimator and O; mu = 1
    samples |psi|^1 so that probs are the reweighting factors (``vmc.py:1173-1184``)."""
    L, OL = qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)
    model, terms = qb.XXZ(L, jxy=-1.0, jz=-1.0), oH.xxz_terms(OL, -1.0, -1.0)
    C, S = 128, 3
    nqs = qb.NQS("rbm", model, alpha=2, dtype="complex64", seed=31, s_upd_fun="EXCHANGE", s_initstate="RND_FIXED",
                 nparticles=8, s_numchains=C, s_numsamples=S, s_therm_steps=2, s_sweep_steps=5, s_seed=31,
                 s_mu=mu, init_scale=0.2)
    p = oracle_params(nqs.net)
    (last, last_lp), (cfg, lp), probs = nqs.sample()
    ref = osm.MetropolisSampler(16, C, rule="EXCHANGE", neighbor_table=olat.neighbor_table(OL), seed=31, mu=mu,
                                therm_steps=2, sweep_steps=5, init="RND_FIXED", n_up=8)
    cfg_ref, lp_ref, probs_ref = ref.sample(p, S)
    got = cfg.cpu().numpy()
    assert got.shape == (C * S, 16) and set(np.unique(got)) <= {-0.5, 0.5}
    tie = ref.min_margin <= 1e-4
    strict = ~tie[np.arange(C * S) % C]
    assert np.mean(tie) <= 0.15
    assert np.array_equal(got[strict], cfg_ref[strict] * 0.5)
    # log psi of the returned rows is log psi of those configurations
    lp_of_rows = orbm.log_psi(p, orbm.to_sigma(got))
    assert np.max(np.abs(lp.cpu().numpy().real - lp_of_rows.real)) < 1e-5 * max(1.0, np.abs(lp_of_rows.real).max())
    assert np.array_equal(last.cpu().numpy(), got[-C:])
    if mu == 2.0:
        assert probs is None and probs_ref is None
    else:
        pr_ref = oest.sample_probs(lp_of_rows, C * S, 1.0)
        assert rel_err(probs.cpu().numpy(), pr_ref) < 1e-5
    # NQS.step on the returned configurations, with and without probabilities
    for pr in (None, probs):
        res = nqs.step(configs=cfg, configs_ansatze=lp, probabilities=pr)
        e_ref = oest.local_energy_full(p, terms, got)
        assert rel_err(res.loss.cpu().numpy(), e_ref) < RTOL
        m_ref, s_ref = oest.loss_stats(e_ref, None if pr is None else pr.cpu().numpy())
        assert abs(complex(res.loss_mean.item()) - m_ref) < 1e-5 * abs(m_ref)
        assert float(res.loss_std) == pytest.approx(s_ref, rel=1e-4)
        assert rel_err(res.grad_flat.cpu().numpy(), orbm.log_derivatives(p, orbm.to_sigma(got))) < RTOL
        assert res.params_sizes == [16, 32, 16 * 32] and res.params_cpx == [True] * 3
    # step() without configurations draws its own batch from the sampler (the chains continue)
    res = nqs.step()
    assert res.loss.shape == (C * S,) and res.grad_flat.shape == (C * S, nqs.num_params)
