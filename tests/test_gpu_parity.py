"""CUDA path (through the C ABI) against the float64 oracle on identical inputs.

Tolerances: float32 kernels vs the float64 oracle -- 1e-5 relative for theta,
tanh, log psi, O and E_loc (the plain-FP32 bar), SR vectors 1e-4 relative
(float32 matvec inside a float64 CG).  Integer work (packed chains, sampler
trajectories, acceptance counters) is compared bit-exactly.
"""

import numpy as np
import pytest
import torch

from oracle import lattice as olat, hamiltonian as oH, rbm as orbm, estimator as oest, sampler as osm, sr as osr
from oracle import ed as oed
import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.rbm import RBM, RBMLogPsi
from pyqusolver_b200.sampler import VMCSampler

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def oracle_params(net: RBM):
    flat = net.flat.detach().cpu().numpy().astype(np.complex128 if net.is_complex else np.float64)
    return orbm.RBMParams.from_flat(flat, net.ns, net.nh)


def rand_states(n, ns, seed=0):
    rng = np.random.default_rng(seed)
    return np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)


def wrap_close(a, b, rtol=RTOL):
    """log psi comparison: real parts relative, imaginary parts modulo 2 pi."""
    a, b = np.asarray(a), np.asarray(b)
    scale = max(1.0, np.max(np.abs(b.real)))
    assert np.max(np.abs(a.real - b.real)) <= rtol * scale * 10
    if np.iscomplexobj(b):
        d = np.angle(np.exp(1j * (a.imag - b.imag)))
        assert np.max(np.abs(d)) <= rtol * scale * 10


def rel_err(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.max(np.abs(a - b)) / max(1e-30, np.max(np.abs(b)))


# A float32 Delta log psi (with the sampler's hardware-approximation tanh cache) can decide a
# Metropolis step the other way only where the float64 oracle's |log u - log_acc| is within its
# rounding; chains whose decisions all kept a larger margin must follow the oracle exactly.  The
# bound covers a few hundred float32 ratio factors (relative error ~1e-7 each) in Delta.
TIE = 1e-4


def assert_same_trajectories(got, cfg, ref, n_chains, accepted=None):
    """Rows are sample-major (row = sample * n_chains + chain).  Chains that never met a near-tie
    decision in the oracle must match row for row (and in their acceptance counts); the near-tie
    chains are a small minority."""
    tie = ref.min_margin <= TIE
    chain_of_row = np.arange(got.shape[0]) % n_chains
    strict = ~tie[chain_of_row]
    mism = np.any(got != cfg, axis=1)
    bad = np.flatnonzero(strict & mism)
    assert bad.size == 0, (bad[:10], ref.min_margin[chain_of_row[bad[:10]]])
    # near-tie chains (each decision has a ~TIE chance of one): a minority, most of them still exact
    assert np.mean(tie) <= 0.15, np.mean(tie)
    if accepted is not None:
        assert np.array_equal(accepted[~tie], ref.accepted[~tie])
    return strict


# ------------------------------------------------------------------------- chains
@pytest.mark.parametrize("ns", [16, 36, 100, 400])
def test_init_chains_match_oracle(ns):
    for kind, okind, nup in [(_lib.INIT_RND, "RND", 0), (_lib.INIT_RND_FIXED, "RND_FIXED", ns // 2)]:
        w = dv.init_chains(kind, 37, ns, seed=1234567, n_up=nup, chain_offset=5)
        got = dv.unpack_states(w, ns, 1.0).cpu().numpy()
        ref = osm.init_states(okind, 37, ns, seed=1234567, n_up=nup, chain_offset=5)
        assert np.array_equal(got, ref)


# ------------------------------------------------------------------------- forward
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("ns,nh", [(16, 16), (36, 144), (100, 200), (33, 70)])
def test_forward_matches_oracle(cplx, ns, nh):
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=3, init_scale=0.1)
    st = rand_states(300, ns, seed=1)
    bits = dv.pack_states(st)
    th, tn, lp = dv.rbm_forward(net.flat, ns, nh, bits, theta=True, tanh=True, logpsi=True)
    p = oracle_params(net)
    sig = orbm.to_sigma(st)
    th_ref = orbm.theta(p, sig)
    th_g = th.cpu().numpy()
    assert rel_err(th_g, th_ref) < RTOL
    # tanh is checked on the kernel's own theta: near the poles of complex tanh
    # (Im theta ~ pi/2) any float32 rounding of theta is amplified by sech^2
    t64 = np.tanh(th_g.astype(np.complex128 if cplx else np.float64))
    assert np.max(np.abs(tn.cpu().numpy() - t64) / np.maximum(1.0, np.abs(t64))) < RTOL
    wrap_close(lp.cpu().numpy(), orbm.log_psi(p, sig))


def test_forward_large_theta_is_finite():
    net = RBM((20,), n_hidden=8, dtype="complex64", seed=0, init_scale=3.0)
    st = rand_states(64, 20, seed=2)
    _, tn, lp = dv.rbm_forward(net.flat, 20, 8, dv.pack_states(st), tanh=True, logpsi=True)
    p = oracle_params(net)
    th = orbm.theta(p, orbm.to_sigma(st))
    assert torch.isfinite(torch.view_as_real(lp)).all()
    np.testing.assert_allclose(tn.cpu().numpy(), np.tanh(th), rtol=1e-4, atol=1e-5)


# ------------------------------------------------------------------------- local energy
def _model_cases():
    return [
        ("tfim1d", lambda: (qb.SquareLattice(1, 16), olat.SquareLattice(1, 16)),
         lambda L: qb.TransverseFieldIsing(L, j=1.0, hx=1.0, hz=0.0), lambda L: oH.tfim_terms(L, 1.0, 1.0, 0.0), 1.0),
        ("tfim2d_hz", lambda: (qb.SquareLattice(2, 4, 5), olat.SquareLattice(2, 4, 5)),
         lambda L: qb.TransverseFieldIsing(L, j=0.8, hx=3.04, hz=0.4), lambda L: oH.tfim_terms(L, 0.8, 3.04, 0.4), 2.0),
        ("xxx2d", lambda: (qb.SquareLattice(2, 6, 6), olat.SquareLattice(2, 6, 6)),
         lambda L: qb.XXZ(L, jxy=-1.0, jz=-1.0), lambda L: oH.xxz_terms(L, -1.0, -1.0), 2.0),
        ("xxz_hx", lambda: (qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)),
         lambda L: qb.XXZ(L, jxy=-1.0, jz=-0.5, hx=0.3), lambda L: oH.xxz_terms(L, -1.0, -0.5, hx=0.3), 2.0),
        ("j1j2", lambda: (qb.SquareLattice(2, 6, 6), olat.SquareLattice(2, 6, 6)),
         lambda L: qb.J1J2Model(L, J1=-1.0, J2=-0.5), lambda L: oH.j1j2_terms(L, -1.0, -0.5), 4.0),
        ("j1j2_hy", lambda: (qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)),
         lambda L: qb.J1J2Model(L, J1=-1.0, J2=-0.5, hx=0.2, hy=0.3), lambda L: oH.j1j2_terms(L, -1.0, -0.5, hx=0.2, hy=0.3), 2.0),
    ]


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("case", _model_cases(), ids=[c[0] for c in _model_cases()])
def test_local_energy_matches_oracle(case, cplx):
    name, lats, mk, mko, alpha = case
    L, OL = lats()
    model = mk(L)
    terms = mko(OL)
    ns = L.ns
    net = RBM((ns,), alpha=alpha, dtype="complex64" if cplx else "float32", seed=5, init_scale=0.05)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, net.nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    st = rand_states(200, ns, seed=4)
    if name.startswith("xxx") or name == "j1j2":
        st = osm.init_states("RND_FIXED", 200, ns, seed=9, n_up=ns // 2) * 0.5
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, net.nh, bits, tanh=True, logpsi=False)
    e = dv.local_energy(net.flat, ns, net.nh, bits, tn, h, tables).cpu().numpy()
    ref = oest.local_energy_full(oracle_params(net), terms, st)
    err = np.max(np.abs(e - ref)) / max(1.0, np.max(np.abs(ref)))
    assert err < RTOL, err


def test_local_energy_edge_cases():
    # one sample, K not a multiple of 32, trained-looking large weights (renormalisation path)
    L, OL = qb.SquareLattice(1, 7), olat.SquareLattice(1, 7)
    model = qb.TransverseFieldIsing(L, j=1.0, hx=0.5, hz=0.0)
    net = RBM((7,), n_hidden=300, dtype="complex64", seed=1, init_scale=0.6)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, 7, 300, h.move_i, h.move_j, h.move_kind, move_major=False)
    for n in (1, 33):
        st = rand_states(n, 7, seed=n)
        bits = dv.pack_states(st)
        _, tn, _ = dv.rbm_forward(net.flat, 7, 300, bits, tanh=True, logpsi=False)
        e = dv.local_energy(net.flat, 7, 300, bits, tn, h, tables).cpu().numpy()
        ref = oest.local_energy_full(oracle_params(net), oH.tfim_terms(OL, 1.0, 0.5, 0.0), st)
        assert np.max(np.abs(e - ref)) / max(1.0, np.max(np.abs(ref))) < 1e-4


def test_loss_stats_match_numpy():
    rng = np.random.default_rng(0)
    e = (rng.normal(size=5000) + 1j * rng.normal(size=5000)).astype(np.complex64) - 40.0
    w = rng.random(5000).astype(np.float32)
    w = w / w.sum() * 5000
    for probs in (None, w):
        out = dv.loss_stats(torch.as_tensor(e).cuda(), None if probs is None else torch.as_tensor(probs).cuda())
        mean, std = oest.loss_stats(e.astype(np.complex128), probs)
        o = out.cpu().numpy()
        assert abs(complex(o[0], o[1]) - mean) < 1e-9 * abs(mean)
        assert o[3] == pytest.approx(std, rel=1e-9)


@pytest.mark.parametrize("n,nch", [(16384, 4096), (5000, 8), (4096, 1), (4096, 5000), (5000, 3), (64, 64)])
def test_loss_rhat_matches_oracle(n, nch):
    rng = np.random.default_rng(n + nch)
    e = (rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex64) - 40.0
    e[: n // 2] += 0.3        # a between-block spread so R-hat differs from 1
    out = dv.loss_rhat(torch.as_tensor(e).cuda(), nch).cpu().numpy()
    ref = oest.step_rhat(e.astype(np.complex128), nch)
    if np.isnan(ref):
        assert np.isnan(out[0])
    else:
        assert out[0] == pytest.approx(ref, rel=1e-10)
    assert out[1] == pytest.approx(oest.step_sigma2(e.astype(np.complex128)), rel=1e-10)


# ------------------------------------------------------------------------- log-derivatives / backward
@pytest.mark.parametrize("cplx", [False, True])
def test_log_derivatives_match_oracle_and_finite_differences(cplx):
    ns, nh = 12, 24
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=2, init_scale=0.1)
    st = rand_states(50, ns, seed=3)
    O = net.log_derivative(st).cpu().numpy()
    p = oracle_params(net)
    Oref = orbm.log_derivatives(p, orbm.to_sigma(st))
    assert rel_err(O, Oref) < RTOL
    # central differences of the float64 log psi, step 1e-4
    flat = p.flat()
    sig = orbm.to_sigma(st)
    h = 1e-4
    rng = np.random.default_rng(0)
    for k in rng.choice(flat.size, 40, replace=False):
        e = np.zeros_like(flat)
        e[k] = h
        fd = (orbm.log_psi(orbm.RBMParams.from_flat(flat + e, ns, nh), sig)
              - orbm.log_psi(orbm.RBMParams.from_flat(flat - e, ns, nh), sig)) / (2 * h)
        np.testing.assert_allclose(O[:, k], fd, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("cplx", [False, True])
def test_autograd_backward_is_conj_O_transpose_g(cplx):
    ns, nh = 10, 20
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=4, init_scale=0.2)
    st = rand_states(64, ns, seed=5)
    lp, p = net.log_psi_autograd(st)
    rng = np.random.default_rng(1)
    g = rng.normal(size=64) + (1j * rng.normal(size=64) if cplx else 0)
    gt = torch.as_tensor(g.astype(np.complex64 if cplx else np.float32)).cuda()
    (grad,) = torch.autograd.grad(lp, p, grad_outputs=gt)
    O = orbm.log_derivatives(oracle_params(net), orbm.to_sigma(st))
    ref = np.conj(O).T @ g if cplx else O.T @ g
    assert rel_err(grad.cpu().numpy(), ref) < 1e-5


# ------------------------------------------------------------------------- SR
@pytest.mark.parametrize("cplx", [False, True])
def test_sr_force_matvec_and_cg_match_dense_oracle(cplx):
    ns, nh, n = 9, 18, 700
    L = qb.SquareLattice(2, 3, 3)
    model = qb.XXZ(L, jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=6, init_scale=0.2)
    st = rand_states(n, ns, seed=6)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    O = orbm.log_derivatives(oracle_params(net), orbm.to_sigma(st))
    ec, Oc, w, _, _ = osr.prepare(e, O)
    F = osr.force(Oc, ec)
    Fg = dv.sr_force(net.flat, ns, nh, bits, tn, eloc).cpu().numpy()
    assert rel_err(Fg, F) < 1e-4
    S = osr.s_matrix(Oc)
    v = np.random.default_rng(2).normal(size=O.shape[1]) + (1j if cplx else 0) * np.random.default_rng(3).normal(size=O.shape[1])
    y = dv.sr_matvec(net.flat, ns, nh, bits, tn, torch.as_tensor(v).cuda(), shift=1e-3).cpu().numpy()
    assert rel_err(y, S @ v + 1e-3 * v) < 1e-4
    x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000)
    xr = -np.linalg.solve(S + 1e-2 * np.eye(S.shape[0]), F)
    assert info["converged"]
    assert rel_err(x.cpu().numpy(), xr) < 1e-3


@pytest.mark.parametrize("cplx,impl", [(False, 1), (True, 1), (False, 0), (True, 0)])
def test_minsr_matches_oracle_and_push_through(sr_impl, cplx, impl):
    """MinSR (sample-space CG) against the oracle's dense MinSR solve and, by the push-through
    identity, against the parameter-space SR solution of the same data."""
    ns, nh, n = 9, 18, 400
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=16, init_scale=0.2)
    st = rand_states(n, ns, seed=17)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    O = orbm.log_derivatives(oracle_params(net), orbm.to_sigma(st))
    xr, _ = osr.solve_sr(e, O, shift=1e-2, use_minsr=True)
    sr_impl(impl)
    x, info, _ = dv.sr_solve_minsr(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=3000)
    assert info["converged"]
    assert rel_err(x.cpu().numpy(), xr) < 1e-3
    x_sr, _ = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=3000)
    assert rel_err(x.cpu().numpy(), x_sr.cpu().numpy()) < 1e-3


# ------------------------------------------------------------------------- sampler
def _gpu_sampler(net, rule, ns, chains, seed, therm, sweep, lattice=None, init=None, n_up=None):
    return VMCSampler(net, (ns,), upd_fun=rule, seed=seed, therm_steps=therm, sweep_steps=sweep, numchains=chains,
                      numsamples=1, lattice=lattice, initstate=init, n_particles=n_up)


@pytest.mark.parametrize("cplx,nh,wide", [(False, 20, 1), (True, 20, 1), (False, 600, 1), (True, 300, 1),
                                          (False, 600, 0), (True, 300, 0), (False, 1600, 1), (True, 1000, 1)])
def test_sampler_local_trajectory_matches_oracle(cplx, nh, wide):
    """Hidden layers wider than one warp's register cache (nh > 512 real / 256 complex) run chains of
    2-8 warps (wide = 1, the default: nh = 600 / 300 on two warps, 1600 / 1000 on four) or one warp per
    chain with the theta cache in shared memory (wide = 0)."""
    ns = 10
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=8,
              init_scale=0.3 if nh <= 32 else 0.05)
    _lib.call("qes_sampler_set_wide", wide)
    try:
        smp = _gpu_sampler(net, "LOCAL", ns, 64, seed=77, therm=2, sweep=5)
        bits, lp = smp.sample_bits(num_samples=6)
    finally:
        _lib.call("qes_sampler_set_wide", 1)
    got = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ref = osm.MetropolisSampler(ns, 64, rule="LOCAL", seed=77, therm_steps=2, sweep_steps=5)
    cfg, lp_ref, _ = ref.sample(oracle_params(net), 6)
    strict = assert_same_trajectories(got, cfg, ref, 64, accepted=smp.accepted.cpu().numpy())
    wrap_close(lp.cpu().numpy()[strict], lp_ref[strict])
    assert np.array_equal(smp.proposed.cpu().numpy(), ref.proposed)


@pytest.mark.parametrize("cplx,nh", [(False, 32), (True, 32), (True, 400), (False, 800)])
def test_sampler_exchange_trajectory_matches_oracle(cplx, nh):
    """nh = 400 (complex) / 800 (real): exchange moves on multi-warp chains."""
    L, OL = qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)
    ns = 16
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=9,
              init_scale=0.3 if nh <= 32 else 0.05)
    smp = _gpu_sampler(net, "EXCHANGE", ns, 64, seed=5, therm=1, sweep=7, lattice=L, init="RND_FIXED", n_up=8)
    bits, _ = smp.sample_bits(num_samples=5)
    got = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ref = osm.MetropolisSampler(ns, 64, rule="EXCHANGE", neighbor_table=olat.neighbor_table(OL), seed=5,
                                therm_steps=1, sweep_steps=7, init="RND_FIXED", n_up=8)
    cfg, _, _ = ref.sample(oracle_params(net), 5)
    assert np.all((got > 0).sum(1) == 8)
    assert_same_trajectories(got, cfg, ref, 64, accepted=smp.accepted.cpu().numpy())


@pytest.mark.parametrize("rule,cplx,nh", [("LOCAL", False, 64), ("EXCHANGE", True, 200), ("EXCHANGE", False, 20)])
def test_capped_sampler_kernel_is_bit_identical(rule, cplx, nh):
    """The register-capped sampler kernel (more chains resident per SM) and the uncapped one
    draw the same chains: identical samples, log-amplitudes and acceptance counts; the capped
    run also follows the oracle's trajectory."""
    L, OL = qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)
    ns = 16
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=19, init_scale=0.1)
    kw = dict(lattice=L, init="RND_FIXED", n_up=8) if rule == "EXCHANGE" else {}
    out = []
    try:
        for mode in (0, 2):
            _lib.call("qes_sampler_set_capped", mode)
            smp = _gpu_sampler(net, rule, ns, 256, seed=23, therm=2, sweep=6, **kw)
            bits, lp = smp.sample_bits(num_samples=4)
            out.append((bits.cpu().numpy(), lp.cpu().numpy(), smp.accepted.cpu().numpy()))
    finally:
        _lib.call("qes_sampler_set_capped", 1)
    for a, b in zip(out[0], out[1]):
        assert np.array_equal(a, b)
    okw = dict(neighbor_table=olat.neighbor_table(OL), init="RND_FIXED", n_up=8) if rule == "EXCHANGE" else {}
    ref = osm.MetropolisSampler(ns, 256, rule=rule, seed=23, therm_steps=2, sweep_steps=6, **okw)
    cfg, _, _ = ref.sample(oracle_params(net), 4)
    got = dv.unpack_states(torch.as_tensor(out[1][0]).cuda(), ns, 1.0).cpu().numpy()
    assert_same_trajectories(got, cfg, ref, 256, accepted=out[1][2])


def test_sampler_tanh_cache_error_bound():
    """The sampler's acceptance-cache tanh (hardware approximations) against float64 tanh of the
    same float32 inputs: absolute error below 1e-6, scaled by 1 + |t|^2 for complex arguments
    (the sensitivity of tanh near its poles); large |Im| exercises the reduction to [-pi, pi]."""
    rng = np.random.default_rng(5)
    xr = np.concatenate([np.linspace(-60, 60, 20001), rng.normal(scale=1e-3, size=4000),
                         [0.0, -0.0, 1e-30, -1e-30, 88.0, -88.0, 1e4, -1e4]]).astype(np.float32)
    yr = torch.empty(len(xr), dtype=torch.float32, device="cuda")
    _lib.call("qes_sampler_tanh_cache", _lib.DTYPE_F32, len(xr), _lib.ptr(torch.as_tensor(xr).cuda()), _lib.ptr(yr),
              _lib.stream_ptr())
    got = yr.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - np.tanh(xr.astype(np.float64)))) < 1e-6
    n = 200000
    z = (rng.uniform(-6, 6, n) + 1j * rng.uniform(-40, 40, n)).astype(np.complex64)
    z[:1000] = (rng.normal(scale=1e-3, size=1000) + 1j * rng.uniform(-3, 3, 1000)).astype(np.complex64)
    # the poles x = 0, y = pi/2 + k pi (in float32): the cache must stay finite there
    poles = np.float32(np.pi / 2) + np.float32(np.pi) * np.arange(-8, 8, dtype=np.float32)
    zt = torch.as_tensor(np.concatenate([z, 1j * poles.astype(np.complex64), 1j * np.nextafter(poles, np.float32(9))
                                         .astype(np.complex64)])).cuda()
    yt = torch.empty_like(zt)
    torch.cuda.synchronize()
    _lib.call("qes_sampler_tanh_cache", _lib.DTYPE_C64, int(zt.numel()), _lib.ptr(zt), _lib.ptr(yt),
              _lib.stream_ptr())
    got = yt.cpu().numpy().astype(np.complex128)
    assert np.all(np.isfinite(got))
    got = got[:n]
    ref = np.tanh(z.astype(np.complex128))
    err = np.abs(got - ref) / (1.0 + np.abs(ref) ** 2)
    assert np.max(err) < 1e-6, np.max(err)


@pytest.mark.parametrize("rule", ["LOCAL", "EXCHANGE"])
def test_sampler_matches_exact_distribution(rule):
    ns = 10
    L = qb.SquareLattice(1, ns)
    net = RBM((ns,), n_hidden=10, dtype="complex64", seed=12, init_scale=0.25)
    n_up = ns // 2 if rule == "EXCHANGE" else None
    smp = _gpu_sampler(net, rule, ns, 2048, seed=3, therm=20, sweep=20, lattice=L,
                       init="RND_FIXED" if rule == "EXCHANGE" else None, n_up=n_up)
    bits, _ = smp.sample_bits(num_samples=40)
    st = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ints = ((st > 0).astype(np.int64) * (1 << np.arange(ns - 1, -1, -1))).sum(1)
    basis, w = osm.exact_distribution(oracle_params(net), ns, n_up=n_up)
    hist = np.bincount(ints, minlength=1 << ns)[basis] / len(ints)
    tv = 0.5 * np.abs(hist - w).sum()
    # multinomial noise of 81920 samples over 252 / 1024 states is ~0.01-0.02
    assert tv < 0.03, tv


def test_sampler_exchange_process_matches_oracle_histogram():
    """Short, unthermalised exchange chains: GPU and oracle run the same Markov process."""
    ns = 10
    L, OL = qb.SquareLattice(1, ns), olat.SquareLattice(1, ns)
    net = RBM((ns,), n_hidden=10, dtype="complex64", seed=12, init_scale=0.5)
    smp = _gpu_sampler(net, "EXCHANGE", ns, 512, seed=3, therm=4, sweep=10, lattice=L, init="RND_FIXED", n_up=5)
    bits, _ = smp.sample_bits(num_samples=20)
    got = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ref = osm.MetropolisSampler(ns, 512, rule="EXCHANGE", neighbor_table=olat.neighbor_table(OL), seed=3,
                                therm_steps=4, sweep_steps=10, init="RND_FIXED", n_up=5)
    cfg, _, _ = ref.sample(oracle_params(net), 20)
    assert_same_trajectories(got, cfg, ref, 512, accepted=smp.accepted.cpu().numpy())


def test_sampler_continues_chains_without_rethermalising():
    ns = 12
    net = RBM((ns,), n_hidden=12, dtype="float32", seed=1)
    smp = _gpu_sampler(net, "LOCAL", ns, 16, seed=2, therm=3, sweep=4)
    smp.sample_bits(num_samples=2)
    assert int(smp.proposed[0]) == 3 * 4 * ns + 2 * 4
    smp.sample_bits(num_samples=3)
    assert int(smp.proposed[0]) == 3 * 4 * ns + 5 * 4


# ------------------------------------------------------------------------- end to end
def test_nqs_training_tfim_reaches_ed():
    L, OL = qb.SquareLattice(1, 8), olat.SquareLattice(1, 8)
    model = qb.TransverseFieldIsing(L, j=1.0, hx=1.0, hz=0.0)
    e0 = oed.ground_energy(oH.tfim_terms(OL, 1.0, 1.0, 0.0), 8)
    nqs = qb.NQS("rbm", model, alpha=1.0, dtype="float32", seed=1, s_numchains=256, s_numsamples=8,
                 s_therm_steps=10, s_sweep_steps=8)
    stats = nqs.train(n_epochs=150, lr=0.05, diag_shift=1e-3)
    tail = np.mean([h.real for h in stats.history[-10:]])
    assert abs(tail - e0) / abs(e0) < 5e-3, (tail, e0)


# ------------------------------------------------------------------------- tensor-core SR matvec
@pytest.fixture
def sr_impl():
    yield _lib.set_sr_impl
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)


@pytest.fixture
def ovz_switch():
    yield lambda on: _lib.call("qes_sr_set_ovz", int(on))
    _lib.call("qes_sr_set_ovz", 1)


@pytest.mark.parametrize("cplx,ns,nh,n", [(False, 16, 16, 300), (True, 9, 18, 700), (True, 36, 144, 1000),
                                           (False, 20, 40, 513), (True, 100, 200, 300),
                                           (False, 150, 300, 700), (True, 130, 100, 500),
                                           (True, 12, 21, 333), (False, 15, 30, 257), (True, 31, 255, 129)])
@pytest.mark.parametrize("ovz", [1, 0])
def test_sr_matvec_tensor_cores_match_oracle(sr_impl, ovz_switch, cplx, ns, nh, n, ovz):
    """The tensor-core S v against the float64 oracle, with O v through z = Sigma V (ovz = 1, where its
    operands fit: the default) and as the product over the hidden axis (ovz = 0).  Shapes include odd
    hidden-unit counts (T read element by element), sites + 1 on a 16 boundary, partial sample tiles
    and the M/N-tiled O^H u."""
    ovz_switch(ovz)
    if (ns, nh) in ((100, 200), (36, 144), (12, 21), (15, 30), (31, 255)):
        assert _lib.sr_tc_plan(_lib.DTYPE_C64 if cplx else _lib.DTYPE_F32, ns, nh, n)["ovz"] == ovz
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=21, init_scale=0.1)
    st = rand_states(n, ns, seed=22)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    O = orbm.log_derivatives(oracle_params(net), orbm.to_sigma(st))
    Oc = O - O.mean(0)
    rng = np.random.default_rng(5)
    v = rng.normal(size=O.shape[1]) + (1j * rng.normal(size=O.shape[1]) if cplx else 0)
    ref = np.conj(Oc).T @ (Oc @ v) / n + 1e-3 * v
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    y_tc = dv.sr_matvec(net.flat, ns, nh, bits, tn, torch.as_tensor(v).cuda(), shift=1e-3).cpu().numpy()
    sr_impl(_lib.SR_IMPL_CUDA_CORES)
    y_cc = dv.sr_matvec(net.flat, ns, nh, bits, tn, torch.as_tensor(v).cuda(), shift=1e-3).cpu().numpy()
    assert rel_err(y_cc, ref) < 1e-4
    assert rel_err(y_tc, ref) < 1e-4


@pytest.mark.parametrize("cplx,impl", [(False, 0), (True, 0), (True, 1)])
def test_sr_cg_initial_guess(sr_impl, cplx, impl):
    """CG from an initial guess (qes_sr_solve_cg_x0): from a random start it reaches the zero-start
    solution; from its own solution it stops at once; TDVP's use_old_result reuses the previous
    (scaled) solution."""
    from pyqusolver_b200.tdvp import TDVP
    ns, nh, n = 12, 24, 1500
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=71, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=72))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(impl)
    # tight tolerance: a random start reaches the zero-start solution
    kw = dict(shift=1e-2, rtol=1e-10, maxiter=3000, rhs_prefactor=-1.0)
    x_ref, info0 = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, **kw)
    assert info0["converged"] and info0["iterations"] > 5
    P = ns + nh + ns * nh
    rng = np.random.default_rng(73)
    # a random start of the solution's norm (the float32 contractions of A x0 carry errors
    # relative to |A x0|, so a start far larger than the solution costs accuracy)
    xr = torch.as_tensor(rng.normal(size=P) + (1j * rng.normal(size=P) if cplx else 0))
    xr = xr * (float(torch.linalg.vector_norm(x_ref.cpu())) / float(torch.linalg.vector_norm(xr)))
    x_rand, info2 = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, x0=xr, **kw)
    assert info2["converged"]
    assert rel_err(x_rand.cpu().numpy(), x_ref.cpu().numpy()) < 1e-4
    # a tolerance above the float32 floor of the contractions: from its own solution the CG stops
    # at once (at 1e-10 the true residual of a float32 matvec sits above the threshold)
    kl = dict(shift=1e-2, rtol=1e-5, maxiter=3000, rhs_prefactor=-1.0)
    x_l, info_l = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, **kl)
    x_l2, info_l2 = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, x0=x_l / -1.0, **kl)
    assert info_l2["converged"] and info_l2["iterations"] <= 2 < info_l["iterations"]
    assert rel_err(x_l2.cpu().numpy(), x_l.cpu().numpy()) < 1e-5
    td = TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-2, sr_tol=1e-5, sr_maxiter=3000, use_old_result=True)
    xa = td.solve(net, bits, tn, eloc)
    it_a = td.last_info["iterations"]
    xb = td.solve(net, bits, tn, eloc)
    assert td.last_info["iterations"] <= 2 < it_a
    assert rel_err(xb.cpu().numpy(), xa.cpu().numpy()) < 1e-5


@pytest.mark.parametrize("cplx", [False, True])
def test_cg_programmatic_launch_is_bit_identical(sr_impl, cplx):
    """Programmatic dependent launch only changes when the CG kernels start: the solution, its
    iteration count and residual are bit-identical with the attribute on and off (every reduction
    runs in a fixed order)."""
    ns, nh, n = 24, 48, 3000
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=81, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=82))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    out = []
    try:
        for on in (1, 0):
            _lib.call("qes_set_pdl", on)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=2000,
                                     check_every=8)
            out.append((x.cpu().numpy(), info["iterations"], info["residual"]))
    finally:
        _lib.call("qes_set_pdl", 1)
    assert out[0][1] == out[1][1] and out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("impl", [_lib.SR_IMPL_TENSOR_CORES, _lib.SR_IMPL_CUDA_CORES])
@pytest.mark.parametrize("fused", [0, 1])
def test_cg_iterations_after_convergence_change_nothing(sr_impl, impl, fused):
    """The host checks convergence every `check_every` iterations; the iterations launched after the
    converging one skip their work on the device (matvec, reduction and updates read the converged
    flag).  Solutions, iteration counts and residuals are bit-identical for check_every = 1 and 64,
    with the cooperative vector kernel and with the separate kernels."""
    ns, nh, n = 20, 40, 2500
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=91, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=92))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(impl)
    out = []
    try:
        _lib.call("qes_set_cg_fused", 2 if fused else 0)
        for ce in (1, 64):
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=2000,
                                     check_every=ce)
            out.append((x.cpu().numpy(), info["iterations"], info["residual"], info["converged"]))
    finally:
        _lib.call("qes_set_cg_fused", 1)
    assert out[0][3] and out[1][3]
    assert out[0][1] == out[1][1] and out[0][1] % 64 != 0
    assert out[0][2] == out[1][2]
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("impl", [_lib.SR_IMPL_TENSOR_CORES, _lib.SR_IMPL_CUDA_CORES])
@pytest.mark.parametrize("fused", [0, 2])
def test_cg_device_loop_matches_host_loop(sr_impl, impl, fused):
    """The CG chunks repeated on the device by a graph's WHILE node, against one host round trip
    per chunk: the same kernels in the same order, so the solution, iteration count and residual
    are bit-identical; a second solve reuses the loop graph."""
    ns, nh, n = 24, 48, 3000
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=71, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=72))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(impl)
    out = []
    try:
        _lib.call("qes_set_cg_fused", fused)
        for loop in (0, 1, 1):
            _lib.call("qes_set_cg_device_loop", loop)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=2000,
                                     check_every=8)
            out.append((x.cpu().numpy(), info["iterations"], info["residual"], info["converged"]))
    finally:
        _lib.call("qes_set_cg_fused", 1)
        _lib.call("qes_set_cg_device_loop", 1)
    assert all(o[3] for o in out) and out[0][1] > 16
    for o in out[1:]:
        assert o[1] == out[0][1] and o[2] == out[0][2]
        assert np.array_equal(o[0], out[0][0])


def test_cg_device_loop_respects_maxiter(sr_impl):
    """A solve that cannot converge within maxiter stops at maxiter with the device loop too."""
    ns, nh, n = 24, 48, 3000
    net = RBM((ns,), n_hidden=nh, dtype="float32", seed=73, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=74))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    res = []
    try:
        for loop in (0, 1):
            _lib.call("qes_set_cg_device_loop", loop)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-6, rtol=1e-14, maxiter=37,
                                     check_every=4)
            res.append((x.cpu().numpy(), info["iterations"], info["converged"]))
    finally:
        _lib.call("qes_set_cg_device_loop", 1)
    assert res[0][1] == res[1][1] == 37 and not res[0][2] and not res[1][2]
    assert np.array_equal(res[0][0], res[1][0])


@pytest.mark.parametrize("cplx", [False, True])
def test_ohu_cta_pairs_match_single_ctas(sr_impl, cplx):
    """O^H u as clusters of two CTAs that add their partials on chip (an odd chunk count, so one
    pair holds an empty padding chunk) against one partial per CTA: same matvec and SR solution."""
    ns, nh, n = 30, 60, 4800
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=61, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=62))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    P = ns + nh + ns * nh
    rng = np.random.default_rng(63)
    v = torch.as_tensor(rng.normal(size=P) + (1j * rng.normal(size=P) if cplx else 0)).cuda()
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    ys, xs, plans = [], [], []
    try:
        for on in (1, 0):
            _lib.call("qes_sr_set_ohu_pairs", on)
            plans.append(_lib.sr_tc_plan(dv.dtype_code(net.flat), ns, nh, n))
            ys.append(dv.sr_matvec(net.flat, ns, nh, bits, tn, v, shift=1e-3).cpu().numpy())
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000)
            assert info["converged"]
            xs.append(x.cpu().numpy())
    finally:
        _lib.call("qes_sr_set_ohu_pairs", 0)
    assert plans[0]["cl"] == 2 and plans[0]["n_chunks"] % 2 == 1 and plans[1]["cl"] == 1
    assert plans[0]["nsplit"] == (plans[1]["nsplit"] + 1) // 2
    assert rel_err(ys[0], ys[1]) < 1e-5
    assert rel_err(xs[0], xs[1]) < 1e-4


@pytest.mark.parametrize("cplx,ns,nh,n", [(False, 200, 800, 12000), (True, 140, 280, 12000),
                                           (False, 400, 1600, 2048)])
def test_sr_matvec_tensor_cores_large_match_cuda_cores(sr_impl, cplx, ns, nh, n):
    """Large shapes take the M/N-tiled tensor-core path (several sample chunks per CTA); the
    CUDA-core matvec, itself checked against the oracle above, is the reference."""
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=41, init_scale=0.05)
    bits = dv.pack_states(rand_states(n, ns, seed=42))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    P = ns + nh + ns * nh
    rng = np.random.default_rng(6)
    v = rng.normal(size=P) + (1j * rng.normal(size=P) if cplx else 0)
    vt = torch.as_tensor(v).cuda()
    dc = _lib.DTYPE_C64 if cplx else _lib.DTYPE_F32
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    assert _lib.sr_uses_tensor_cores(dc, ns, nh, n)
    y_tc = dv.sr_matvec(net.flat, ns, nh, bits, tn, vt, shift=1e-3).cpu().numpy()
    sr_impl(_lib.SR_IMPL_CUDA_CORES)
    y_cc = dv.sr_matvec(net.flat, ns, nh, bits, tn, vt, shift=1e-3).cpu().numpy()
    assert rel_err(y_tc, y_cc) < 1e-4


@pytest.mark.parametrize("cplx", [False, True])
def test_sr_force_and_cg_tensor_cores_match_cuda_cores(sr_impl, cplx):
    ns, nh, n = 16, 32, 2000
    L = qb.SquareLattice(2, 4, 4)
    model = qb.XXZ(L, jxy=-1.0, jz=-1.0, hx=0.3)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=23, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=24))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    out = {}
    for impl in (_lib.SR_IMPL_CUDA_CORES, _lib.SR_IMPL_TENSOR_CORES):
        sr_impl(impl)
        F = dv.sr_force(net.flat, ns, nh, bits, tn, eloc).cpu().numpy()
        x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-8, maxiter=1000)
        assert info["converged"]
        out[impl] = (F, x.cpu().numpy())
    assert rel_err(out[2][0], out[1][0]) < 1e-4
    assert rel_err(out[2][1], out[1][1]) < 1e-3


def test_cg_graph_replay_matches_direct_launches():
    ns, nh, n = 16, 32, 3000
    L = qb.SquareLattice(2, 4, 4)
    model = qb.XXZ(L, jxy=-1.0, jz=-1.0)
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=31, init_scale=0.2)
    bits = dv.init_chains(_lib.INIT_RND_FIXED, n, ns, seed=5, n_up=8)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    out = []
    try:
        for g in (0, 1, 1):
            _lib.call("qes_set_cg_graphs", g)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-3, rtol=1e-10, maxiter=400,
                                     check_every=8)
            out.append((x.cpu().numpy(), info["iterations"]))
    finally:
        _lib.call("qes_set_cg_graphs", 1)
    assert out[0][1] == out[1][1] == out[2][1]
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[1][0], out[2][0])


def test_torch_ops_match_direct_calls():
    import pyqusolver_b200.ops  # noqa: F401
    ns, nh, n = 12, 24, 200
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=51, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=52))
    tn, lp = torch.ops.qes_b200.rbm_forward(net.flat, bits, ns, nh)
    _, tn2, lp2 = dv.rbm_forward(net.flat, ns, nh, bits)
    assert torch.equal(tn, tn2) and torch.equal(lp, lp2)
    O = torch.ops.qes_b200.log_derivatives(net.flat, bits, tn, ns, nh)
    assert torch.equal(O, dv.log_derivatives(net.flat, ns, nh, bits, tn))
    g = torch.randn(n, dtype=torch.complex64, device="cuda")
    assert torch.allclose(torch.ops.qes_b200.logpsi_vjp(net.flat, bits, tn, g, ns, nh),
                          dv.logpsi_vjp(net.flat, ns, nh, bits, tn, g), rtol=1e-12, atol=1e-12)
    st = torch.ops.qes_b200.loss_stats(lp.to(torch.complex64))
    assert st.shape == (4,) and st.dtype == torch.float64


# ------------------------------------------------------------------------- parallel tempering
@pytest.mark.parametrize("rule", ["LOCAL", "EXCHANGE"])
def test_parallel_tempering_matches_oracle(rule):
    L, OL = qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)
    ns, C, betas = 16, 64, [1.0, 0.6, 0.35, 0.2]
    net = RBM((ns,), n_hidden=32, dtype="complex64", seed=61, init_scale=0.3)
    init, n_up = ("RND_FIXED", 8) if rule == "EXCHANGE" else (None, None)
    smp = VMCSampler(net, (ns,), upd_fun=rule, seed=9, therm_steps=1, sweep_steps=5, numchains=C, numsamples=1,
                     lattice=L, initstate=init, n_particles=n_up, pt_betas=betas)
    assert smp.is_pt and smp.n_replicas == 4
    bits, lp = smp.sample_bits(num_samples=4)
    got = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ref = osm.ParallelTemperingSampler(ns, C, betas, rule=rule, neighbor_table=olat.neighbor_table(OL), seed=9,
                                       therm_steps=1, sweep_steps=5, init=init or "RND", n_up=n_up)
    cfg, lp_ref, _ = ref.sample(oracle_params(net), 4)
    assert_same_trajectories(got, cfg, ref, C)
    gb = smp.chain_betas.cpu().numpy().astype(np.float64)
    strict = ref.min_margin > TIE
    assert np.array_equal(gb[:, strict], ref.betas[:, strict])
    assert smp._pt_round == ref.round


def test_parallel_tempering_ladder_and_weights():
    net = RBM((4,), n_hidden=3, dtype="float32", seed=37)
    smp = VMCSampler(net, (4,), seed=5, therm_steps=1, sweep_steps=1, numchains=2, numsamples=1, beta=0.8)
    smp.set_replicas(None, n_replicas=3)
    b = smp.pt_betas
    assert b[0] == pytest.approx(0.8) and b[-1] == pytest.approx(0.08)
    smp2 = VMCSampler(net, (4,), seed=5, therm_steps=1, sweep_steps=1, numchains=2, numsamples=1)
    smp2.set_pt_betas([1.0, 0.5, 0.25])
    assert smp2.is_pt and smp2.n_replicas == 3
    (last, _), _, probs = smp2.sample()
    assert tuple(last.shape) == (3, 2, 4)
    assert smp2.has_uniform_weights and probs is None


def test_parallel_tempering_matches_exact_distribution():
    ns = 10
    net = RBM((ns,), n_hidden=10, dtype="complex64", seed=12, init_scale=0.4)
    smp = VMCSampler(net, (ns,), seed=3, therm_steps=20, sweep_steps=20, numchains=2048, numsamples=1,
                     pt_betas=[1.0, 0.5, 0.25])
    bits, _ = smp.sample_bits(num_samples=40)
    st = dv.unpack_states(bits, ns, 1.0).cpu().numpy()
    ints = ((st > 0).astype(np.int64) * (1 << np.arange(ns - 1, -1, -1))).sum(1)
    basis, w = osm.exact_distribution(oracle_params(net), ns)
    hist = np.bincount(ints, minlength=1 << ns)[basis] / len(ints)
    assert 0.5 * np.abs(hist - w).sum() < 0.03


# ------------------------------------------------------------------------- overlaps and Renyi-2
def _exact_psi(net, ns):
    basis = np.arange(1 << ns)
    sig = np.where(((basis[:, None] >> np.arange(ns - 1, -1, -1)) & 1) == 1, 1.0, -1.0)
    lp = orbm.log_psi(oracle_params(net), sig)
    psi = np.exp(lp - np.max(np.real(lp)))
    return psi / np.linalg.norm(psi)


def test_renyi2_swap_estimator_matches_exact():
    ns = 8
    model = qb.TransverseFieldIsing(qb.SquareLattice(1, ns, 1, bc="pbc"), j=1.0, hx=1.0, hz=0.0)
    nqs = qb.NQS("rbm", model, alpha=1, dtype="complex64", seed=3, s_upd_fun="LOCAL", s_numchains=1024,
                 s_numsamples=16, s_sweep_steps=8, s_therm_steps=20, init_scale=0.5)
    psi = _exact_psi(nqs.net, ns).reshape(1 << (ns // 2), 1 << (ns // 2))   # sites 0..3 = most significant bits
    rho = psi @ psi.conj().T
    s2_exact = -np.log(np.real(np.trace(rho @ rho)))
    s2, err = qb.NQS.compute_renyi2(nqs, region=np.arange(ns // 2), return_error=True)
    assert abs(s2 - s2_exact) < 5 * err + 0.02, (s2, s2_exact, err)


def test_overlap_of_identical_and_different_states():
    ns = 8
    model = qb.TransverseFieldIsing(qb.SquareLattice(1, ns, 1, bc="pbc"), j=1.0, hx=1.0, hz=0.0)
    kw = dict(alpha=1, dtype="complex64", s_upd_fun="LOCAL", s_numchains=1024, s_numsamples=8, s_sweep_steps=8,
              s_therm_steps=20, init_scale=0.4)
    a = qb.NQS("rbm", model, seed=4, **kw)
    a2 = qb.NQS("rbm", model, seed=4, **kw)
    assert qb.NQS.compute_overlap(a, a2, num_samples=8) == pytest.approx(1.0, abs=1e-4)
    b = qb.NQS("rbm", model, seed=5, **kw)
    f_exact = abs(np.vdot(_exact_psi(a.net, ns), _exact_psi(b.net, ns))) ** 2
    f = qb.NQS.compute_overlap(a, b, num_samples=8)
    assert abs(f - f_exact) < 0.05, (f, f_exact)


def test_tilings_agree_and_graphs_follow_tiling_changes(sr_impl):
    """The O^H u tilings give the same solution, and a CG graph captured under one tiling is not
    replayed under another."""
    ns, nh, n = 36, 144, 4096
    model = qb.XXZ(qb.SquareLattice(2, 6, 6), jxy=-1.0, jz=-1.0)
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=71, init_scale=0.1)
    bits = dv.init_chains(_lib.INIT_RND_FIXED, n, ns, seed=7, n_up=18)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    xs = []
    try:
        for st in [(0, 0, 0), (2, 64, 296), (2, 128, 148), (2, 0, 148), (0, 0, 0)]:
            _lib.call("qes_sr_set_tiling", *st)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=400,
                                     check_every=8)
            assert info["iterations"] > 8
            xs.append(x.cpu().numpy())
    finally:
        _lib.call("qes_sr_set_tiling", 0, 0, 0)
    # float32 products summed in a different order; CG carries that through the conditioning of S: with
    # P > Ns, S + shift has many eigenvalues equal to the shift, so the solutions are compared in the
    # (S + shift)-norm, the error norm CG minimises, not entry by entry
    assert rel_err(xs[-1], xs[0]) < 1e-12          # same tiling again (graph replay): identical
    x0 = torch.as_tensor(xs[0]).cuda()
    a0 = torch.vdot(x0, dv.sr_matvec(net.flat, ns, nh, bits, tn, x0, shift=1e-2)).real.item()
    for x in xs[1:-1]:
        e = torch.as_tensor(x).cuda() - x0
        ae = torch.vdot(e, dv.sr_matvec(net.flat, ns, nh, bits, tn, e, shift=1e-2)).real.item()
        assert np.sqrt(max(ae, 0.0) / a0) < 1e-3


@pytest.mark.parametrize("cplx,ns,nh,n", [(False, 16, 16, 300), (True, 100, 200, 1000), (True, 36, 144, 700),
                                           (False, 400, 1600, 300), (False, 10, 600, 257), (True, 10, 300, 129)])
def test_forward_tensor_cores_match_cuda_cores_and_oracle(cplx, ns, nh, n):
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=81, init_scale=0.1)
    st = rand_states(n, ns, seed=82)
    bits = dv.pack_states(st)
    th0, tn0, lp0 = dv.rbm_forward(net.flat, ns, nh, bits, theta=True)
    th1, tn1, lp1 = dv.rbm_forward(net.flat, ns, nh, bits, theta=True, tensor_cores=True)
    assert rel_err(th1.cpu().numpy(), th0.cpu().numpy()) < 1e-5
    # tanh of a complex theta near a pole amplifies the 1e-7 theta difference of the two summation
    # orders, so tanh is checked against float64 tanh of the path's own theta
    t1 = th1.cpu().numpy().astype(np.complex128 if cplx else np.float64)
    assert rel_err(tn1.cpu().numpy(), np.tanh(t1)) < 1e-5
    wrap_close(lp1.cpu().numpy(), lp0.cpu().numpy())
    p = oracle_params(net)
    wrap_close(lp1.cpu().numpy(), orbm.log_psi(p, orbm.to_sigma(st)))


# ------------------------------------------------------------------------- bulk-copy split reduction
@pytest.mark.parametrize("cplx,ns,nh,n", [(True, 100, 200, 4000), (False, 36, 144, 3000), (True, 24, 48, 777)])
def test_bulk_split_reduction_is_bit_identical(sr_impl, cplx, ns, nh, n):
    """qes_set_reduce_bulk(1) (the split-K partials moved into shared memory by bulk copies) against
    the register-load reduction (0, the default): the same sums in the same order, so the S v of
    the tensor-core and CUDA-core forms and a CG solve agree bit for bit."""
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=31, init_scale=0.1)
    st = rand_states(n, ns, seed=32)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    rng = np.random.default_rng(33)
    P = dv.n_params(ns, nh)
    v = torch.as_tensor(rng.normal(size=P) + (1j * rng.normal(size=P) if cplx else 0)).cuda()
    eloc = torch.as_tensor((rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex64)).cuda()
    out = {}
    try:
        for impl in (_lib.SR_IMPL_TENSOR_CORES, _lib.SR_IMPL_CUDA_CORES):
            sr_impl(impl)
            for bulk in (1, 0):
                _lib.call("qes_set_reduce_bulk", bulk)
                y = dv.sr_matvec(net.flat, ns, nh, bits, tn, v, shift=1e-3).cpu().numpy()
                x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-8, maxiter=500,
                                         check_every=16)
                out[impl, bulk] = (y, x.cpu().numpy(), info["iterations"])
    finally:
        _lib.call("qes_set_reduce_bulk", 0)
    for impl in (_lib.SR_IMPL_TENSOR_CORES, _lib.SR_IMPL_CUDA_CORES):
        (y1, x1, i1), (y0, x0, i0) = out[impl, 1], out[impl, 0]
        assert np.array_equal(y1, y0), impl
        assert np.array_equal(x1, x0) and i1 == i0, impl


@pytest.mark.parametrize("impl", [_lib.SR_IMPL_TENSOR_CORES, _lib.SR_IMPL_CUDA_CORES])
@pytest.mark.parametrize("cplx,precond", [(True, None), (True, "jacobi"), (False, None)])
def test_cg_xrp_kernel_is_bit_identical(sr_impl, impl, cplx, precond):
    """qes_set_cg_xrp(1) (the default: the x/r and direction updates in one launch with a grid
    barrier) against cg_xr + cg_p (0): the same per-block partials summed in the same order, so the
    solutions, iteration counts and residuals agree bit for bit, through the device loop's graph."""
    ns, nh, n = 30, 60, 3000                     # P = 1,890: a multi-block vector grid
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=41, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=42))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(impl)
    out = {}
    try:
        _lib.call("qes_set_cg_fused", 0)
        for on in (1, 0):
            _lib.call("qes_set_cg_xrp", on)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=2000,
                                     check_every=8, precond=precond)
            out[on] = (x.cpu().numpy(), info["iterations"], info["residual"], info["converged"])
    finally:
        _lib.call("qes_set_cg_xrp", 1)
        _lib.call("qes_set_cg_fused", 1)
    assert out[1][3] and out[0][3] and out[1][1] > 16
    assert out[1][1] == out[0][1] and out[1][2] == out[0][2]
    assert np.array_equal(out[1][0], out[0][0])


def test_ovz_l2_prefetch_changes_nothing(sr_impl):
    """qes_sr_set_prefetch(1) only adds an L2 prefetch of the z-form O v kernel's T tile: S v and a CG
    solve through the device loop are bit-identical with and without it."""
    ns, nh, n = 100, 200, 2000
    net = RBM((ns,), n_hidden=nh, dtype="complex64", seed=51, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=52))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    assert _lib.sr_tc_plan(_lib.DTYPE_C64, ns, nh, n)["ovz"] == 1
    rng = np.random.default_rng(53)
    P = dv.n_params(ns, nh)
    v = torch.as_tensor(rng.normal(size=P) + 1j * rng.normal(size=P)).cuda()
    eloc = torch.as_tensor((rng.normal(size=n) + 1j * rng.normal(size=n)).astype(np.complex64)).cuda()
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    out = {}
    try:
        for on in (1, 0):
            _lib.call("qes_sr_set_prefetch", on)
            y = dv.sr_matvec(net.flat, ns, nh, bits, tn, v, shift=1e-3).cpu().numpy()
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-8, maxiter=300,
                                     check_every=8)
            out[on] = (y, x.cpu().numpy(), info["iterations"])
    finally:
        _lib.call("qes_sr_set_prefetch", 0)
    assert np.array_equal(out[1][0], out[0][0])
    assert np.array_equal(out[1][1], out[0][1]) and out[1][2] == out[0][2]


@pytest.mark.parametrize("cplx", [True, False])
def test_fused_vector_kernel_pdl_launch_is_bit_identical(sr_impl, cplx):
    """qes_set_cg_fused_pdl(1) (the default: the fused vector kernel launched by programmatic dependent
    launch) against the cooperative launch (0): the same kernel and sums, so the CG solutions,
    iteration counts and residuals agree bit for bit."""
    ns, nh, n = 16, 32, 2048
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=61, init_scale=0.1)
    bits = dv.pack_states(rand_states(n, ns, seed=62))
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(qb.XXZ(qb.SquareLattice(1, ns), jxy=-1.0, jz=-1.0, hx=0.3).lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    sr_impl(_lib.SR_IMPL_TENSOR_CORES)
    out = {}
    try:
        _lib.call("qes_set_cg_fused", 2)
        for on in (1, 0):
            _lib.call("qes_set_cg_fused_pdl", on)
            x, info = dv.sr_solve_cg(net.flat, ns, nh, bits, tn, eloc, shift=1e-2, rtol=1e-9, maxiter=2000,
                                     check_every=8)
            out[on] = (x.cpu().numpy(), info["iterations"], info["residual"], info["converged"])
    finally:
        _lib.call("qes_set_cg_fused_pdl", 1)
        _lib.call("qes_set_cg_fused", 1)
    assert out[1][3] and out[0][3]
    assert out[1][1] == out[0][1] and out[1][2] == out[0][2]
    assert np.array_equal(out[1][0], out[0][0])
