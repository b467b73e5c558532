"""The CPU oracle against the reference's own known-answer fixtures (no GPU)."""

import json
import os

import numpy as np
import pytest

from oracle import philox, lattice, hamiltonian as H, rbm, estimator, sampler as osm, sr, ed

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.json")))


def _c(x):
    a = np.asarray(x, dtype=np.float64)
    return a[..., 0] + 1j * a[..., 1]


# ---------------------------------------------------------------- Philox (published KAT vectors)
@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox_known_answers(ctr, key, expect):
    out = philox.philox4x32_10(*ctr, *key)
    assert tuple(int(v) for v in out) == expect


def test_uniform_open_is_float32_exact_and_open():
    r = np.array([0, 1, 2 ** 32 - 1, 12345678], dtype=np.uint64)
    u = philox.uniform_open(r)
    assert np.all(u > 0) and np.all(u < 1)
    assert np.array_equal(u.astype(np.float32).astype(np.float64), u)


# ---------------------------------------------------------------- SR normalisation fixtures
def test_sr_gram_fixture_matches_dense_solve():
    g = GOLDEN["sr"]
    O, loss, shift = _c(g["O"]), _c(g["loss"]), g["shift_gram"]
    n = O.shape[0]
    b = O.conj().T @ loss / n
    expected = np.linalg.solve(O.conj().T @ O / n + shift * np.eye(O.shape[1]), b)
    x, it, res, conv = sr.cg(lambda v: O.conj().T @ (O @ v) / n + shift * v, b, rtol=1e-12, maxiter=200)
    assert conv
    np.testing.assert_allclose(x, expected, rtol=g["rtol"], atol=2e-6)


def test_sr_minsr_fixture_matches_push_through():
    g = GOLDEN["sr"]
    O, loss, shift = _c(g["O"]), _c(g["loss"]), g["shift_minsr_solvers"]
    n = O.shape[0]
    # MinSR system of the reference test: (O O^H / n + shift) y = loss / n
    y = np.linalg.solve(O @ O.conj().T / n + shift * np.eye(n), loss / n)
    # The push-through identity: O^H y equals the parameter-space SR solution of the same data
    x_param = np.linalg.solve(O.conj().T @ O / n + shift * np.eye(O.shape[1]), O.conj().T @ loss / n)
    np.testing.assert_allclose(O.conj().T @ y, x_param, rtol=1e-10, atol=1e-12)


def test_sr_solver_centres_and_applies_prefactor():
    g = GOLDEN["sr"]
    O, loss = _c(g["O"]), _c(g["loss"])
    x, info = sr.solve_sr(loss, O, shift=0.2, method="dense", rhs_prefactor=-1.0)
    Oc = O - O.mean(0)
    ec = loss - loss.mean()
    n = O.shape[0]
    ref = np.linalg.solve(Oc.conj().T @ Oc / n + 0.2 * np.eye(O.shape[1]), Oc.conj().T @ ec / n)
    np.testing.assert_allclose(x, -ref, rtol=1e-12, atol=1e-14)
    xc, infoc = sr.solve_sr(loss, O, shift=0.2, method="cg", rtol=1e-12)
    np.testing.assert_allclose(xc, x, rtol=1e-9, atol=1e-12)


# ---------------------------------------------------------------- estimator orientation / reweighting
def test_sigma_y_orientation_fixture():
    g = GOLDEN["sigma_y_orientation"]
    psi = _c(g["psi"])
    matrix = _c(g["matrix"])
    probs = np.abs(psi) ** 2 / np.vdot(psi, psi).real
    states = np.array([[-0.5], [0.5]])
    logv = np.log(psi)

    def local(s):
        bit = s[0] > 0
        return np.array([[-0.5 if bit else 0.5]]), np.array([0.5j if bit else -0.5j])

    def logpsi(q):
        return logv[(q[:, 0] > 0).astype(int)]

    el = estimator.local_energy_generic(local, logpsi, states, logv)
    mean, _ = estimator.loss_stats(el, 2.0 * probs)
    expected = np.vdot(psi, matrix @ psi) / np.vdot(psi, psi)
    np.testing.assert_allclose(mean, expected, rtol=1e-12, atol=1e-12)


def test_reweighting_fixture():
    g = GOLDEN["reweighting"]
    la = _c(g["log_ansatz"])
    got = estimator.sample_probs(la, la.shape[0], g["exponent"])
    lu = g["exponent"] * la.real
    exp = np.exp(lu - lu.max())
    exp = exp / exp.sum() * la.shape[0]
    np.testing.assert_allclose(got, exp, rtol=1e-14)
    gb = GOLDEN["reweighting_beta"]
    expo = 1.0 / gb["logprob_fact"] - gb["mu"] * gb["beta"]
    lp = np.asarray(gb["states"])[:, 0]
    got = estimator.sample_probs(lp, 3, expo)
    e = np.exp(expo * lp)
    np.testing.assert_allclose(got, e / e.sum() * 3, rtol=1e-14)


def test_chunking_fixture_linear_logpsi():
    g = GOLDEN["chunking"]
    params = np.asarray(g["params"])
    states = np.asarray(g["states"])

    def local(s):
        shifts = np.arange(5).reshape(5, 1)
        return s[None, :] + shifts, np.arange(1, 6, dtype=np.float64)

    lp_fn = lambda q: q @ params
    full = estimator.local_energy_generic(local, lp_fn, states, lp_fn(states))
    part = np.concatenate([estimator.local_energy_generic(local, lp_fn, states[i:i + 1], lp_fn(states[i:i + 1]))
                           for i in range(2)])
    np.testing.assert_allclose(full, part)


# ---------------------------------------------------------------- RBM fast update contract
def test_rbm_fast_update_fixture_masked_and_repeated_flips():
    g = GOLDEN["rbm_fast_update"]
    states = np.asarray(g["states"], dtype=np.float64)
    idx = np.asarray(g["indices"])
    mask = np.asarray(g["valid_mask"])
    p = rbm.random_params(states.shape[1], g["n_hidden"], complex_=True, scale=0.3, seed=7)
    flips = [[int(i) for i, ok in zip(idx[r], mask[r]) if ok] for r in range(len(states))]
    delta, new_theta = rbm.log_psi_delta_flips(p, states, flips)
    proposed = states.copy()
    for r, fl in enumerate(flips):
        for i in fl:
            proposed[r, i] = -proposed[r, i]
    direct = rbm.log_psi(p, proposed) - rbm.log_psi(p, states)
    np.testing.assert_allclose(np.exp(delta), np.exp(direct), rtol=1e-12)
    np.testing.assert_allclose(new_theta, rbm.theta(p, proposed), rtol=1e-12, atol=1e-14)


def test_rbm_single_flip_fixture():
    g = GOLDEN["rbm_single_flip"]
    s = np.asarray(g["state"], dtype=np.float64)
    p = rbm.random_params(6, 4, complex_=False, scale=0.5, seed=123)
    d, _ = rbm.log_psi_delta_flips(p, s[None, :], [[g["flip"]]])
    s2 = s.copy()
    s2[g["flip"]] *= -1
    np.testing.assert_allclose(d[0], rbm.log_psi(p, s2) - rbm.log_psi(p, s), rtol=1e-12)


def test_log_derivatives_match_central_differences():
    p = rbm.random_params(5, 3, complex_=True, scale=0.4, seed=2)
    sig = np.array([[1, -1, 1, 1, -1], [-1, -1, 1, -1, 1]], dtype=np.float64)
    O = rbm.log_derivatives(p, sig)
    flat = p.flat()
    h = 1e-5
    for k in range(flat.size):
        e = np.zeros_like(flat)
        e[k] = h
        lp = rbm.log_psi(rbm.RBMParams.from_flat(flat + e, 5, 3), sig)
        lm = rbm.log_psi(rbm.RBMParams.from_flat(flat - e, 5, 3), sig)
        np.testing.assert_allclose((lp - lm) / (2 * h), O[:, k], rtol=1e-7, atol=1e-8)


# ---------------------------------------------------------------- operator encoding
def test_integer_operator_fixtures():
    cases = GOLDEN["int_operators"]["cases"]
    for name, c in cases.items():
        state_int, ns, sites = c["args"]
        state = H.int_to_state(state_int, ns)
        op = "x" if c["op"].startswith("sigma_x") else "z"
        new, coeff = H.apply_term(H.Term(op, tuple(sites), 1.0), state)
        assert H.state_to_int(new) == c["states"][0]
        assert coeff == pytest.approx(c["coeffs"][0])


def test_two_site_sigma_x_coefficient_fixture():
    state = np.array([-0.5, 0.5, -0.5, 0.5])
    _, c = H.apply_term(H.Term("x", (1, 2), 1.0), state)
    assert c == pytest.approx(GOLDEN["sigma_x_two_site"]["coeff"])


def test_sigma_y_spin_half_convention():
    for s, expect in [(-0.5, -0.5j), (0.5, 0.5j)]:
        new, c = H.apply_term(H.Term("y", (0,), 1.0), np.array([s]))
        assert new[0] == -s and c == pytest.approx(expect)


# ---------------------------------------------------------------- estimator vs exact expectation, ED
@pytest.mark.parametrize("model", ["tfim", "xxz", "j1j2"])
def test_estimator_exact_expectation(model):
    if model == "tfim":
        lat = lattice.SquareLattice(1, 8, bc="pbc")
        terms = H.tfim_terms(lat, j=1.0, hx=0.7, hz=0.2)
    elif model == "xxz":
        lat = lattice.SquareLattice(2, 3, 3, bc="pbc")
        terms = H.xxz_terms(lat, jxy=-1.0, jz=-0.6, hx=0.3)
    else:
        lat = lattice.SquareLattice(2, 3, 3, bc="pbc")
        terms = H.j1j2_terms(lat, J1=-1.0, J2=-0.5, hy=0.2)
    ns = lat.ns
    p = rbm.random_params(ns, 2 * ns, complex_=True, scale=0.2, seed=3)
    allb = np.arange(1 << ns)
    st = np.stack([H.int_to_state(b, ns) for b in allb])
    psi = np.exp(rbm.log_psi(p, rbm.to_sigma(st)))
    Hm, _ = H.sparse_hamiltonian(terms, ns)
    exact = np.vdot(psi, Hm @ psi) / np.vdot(psi, psi)
    el = estimator.local_energy_full(p, terms, st)
    w = np.abs(psi) ** 2
    w /= w.sum()
    np.testing.assert_allclose(np.sum(w * el), exact, rtol=1e-10, atol=1e-12)


def test_ed_matches_dense_diagonalisation():
    lat = lattice.SquareLattice(1, 10, bc="pbc")
    terms = H.tfim_terms(lat, j=1.0, hx=1.0, hz=0.0)
    Hm, _ = H.sparse_hamiltonian(terms, 10)
    assert abs(Hm - Hm.getH()).max() < 1e-14
    e_dense = np.linalg.eigvalsh(Hm.toarray())[0]
    assert ed.ground_energy(terms, 10) == pytest.approx(e_dense, rel=1e-10)
    lat2 = lattice.SquareLattice(2, 4, 3, bc="pbc")
    t2 = H.xxz_terms(lat2, jxy=-1.0, jz=-1.0)
    H2, _ = H.sparse_hamiltonian(t2, 12, n_up=6)
    assert ed.ground_energy(t2, 12, n_up=6) == pytest.approx(np.linalg.eigvalsh(H2.toarray())[0], rel=1e-10)


def test_connected_raw_slot_layout_xxz():
    lat = lattice.SquareLattice(2, 3, 3, bc="pbc")
    terms = H.xxz_terms(lat, jxy=-1.0, jz=-1.0, hx=0.5)
    s = H.int_to_state(0b101010101, 9)
    st, co = H.connected_raw(terms, s)
    nb = len(lat.nn_bonds())
    assert st.shape == (1 + 9 + 2 * nb, 9)
    # group order: Sx singles, then XX of every bond, then YY of every bond
    for k, (i, j) in enumerate(lat.nn_bonds()):
        xx, yy = co[1 + 9 + k], co[1 + 9 + nb + k]
        assert xx == pytest.approx(0.25)          # mult = -jxy = +1
        si, sj = np.sign(s[i]), np.sign(s[j])
        assert yy == pytest.approx(1.0 * (1j * 0.5 * si) * (1j * 0.5 * sj))


def test_sampler_oracle_init_fixed_conserves():
    st = osm.init_states("RND_FIXED", 16, 36, seed=5, n_up=18)
    assert np.all((st > 0).sum(1) == 18)
    st2 = osm.init_states("RND_FIXED", 16, 36, seed=5, n_up=18)
    assert np.array_equal(st, st2)


def test_oracle_sampler_matches_exact_distribution():
    lat = lattice.SquareLattice(1, 6, bc="pbc")
    p = rbm.random_params(6, 6, complex_=True, scale=0.4, seed=11)
    smp = osm.MetropolisSampler(6, 256, rule="LOCAL", seed=3, therm_steps=4, sweep_steps=6)
    cfg, _, _ = smp.sample(p, 40)
    ints = ((cfg > 0).astype(int) * (1 << np.arange(5, -1, -1))).sum(1)
    basis, w = osm.exact_distribution(p, 6)
    hist = np.bincount(ints, minlength=64) / len(ints)
    tv = 0.5 * np.abs(hist - w).sum()
    assert tv < 0.05


def test_oracle_parallel_tempering_samples_physical_distribution():
    """Replica exchange keeps detailed balance: physical-slot samples follow |psi|^2."""
    p = rbm.random_params(6, 6, complex_=True, scale=0.6, seed=13)
    pt = osm.ParallelTemperingSampler(6, 256, [1.0, 0.5, 0.2], rule="LOCAL", seed=4, therm_steps=4, sweep_steps=6)
    cfg, lp, probs = pt.sample(p, 40)
    assert probs is None                               # 1/lpf - mu*beta_phys = 0 at beta = 1
    assert cfg.shape == (40 * 256, 6)
    assert pt.swaps.sum() > 0
    ints = ((cfg > 0).astype(int) * (1 << np.arange(5, -1, -1))).sum(1)
    basis, w = osm.exact_distribution(p, 6)
    hist = np.bincount(ints, minlength=64) / len(ints)
    assert 0.5 * np.abs(hist - w).sum() < 0.05
    # every column holds each ladder value exactly once (labels are permuted, never lost)
    assert np.all(np.sort(pt.betas, axis=0) == np.sort(pt.pt_betas)[:, None])
