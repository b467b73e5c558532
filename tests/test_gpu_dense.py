"""The formed SR matrix (qes_sr_gram: tcgen05 Gram of the centred, weighted O) and its float64
Cholesky solve (qes_sr_solve_dense) against the oracle, on the workloads the dense form is meant
for: the 16-site TFIM chain (real RBM alpha = 1, P = 288, Ns > P) and the 6x6 J1-J2 model (complex
RBM alpha = 4, P = 5,364).  The oracle forms O from the network's own float32 tanh(theta) rows
(what the reference's SR receives after promoting the float32 network's O to float64).

Bars: S to 1e-4 of max|S| (BF16 hi/lo split with FP32 accumulation: the dropped lo*lo term and
the BF16 rounding of lo are each ~2^-18 of a product; measured 1-3e-5); the full-rank solve (Ns > P)
entrywise to 1e-2 (condition number ~1e3 times the Gram's rounding); the rank-deficient one (Ns < P, condition ~1e5) by its backward error (true
residual in the oracle's float64 operator below 1e-4, (S + shift)-norm error below 1e-2).
"""

import numpy as np
import pytest
import torch

from oracle import rbm as orbm, sampler as osm, sr as osr
import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.rbm import RBM
from pyqusolver_b200.tdvp import TDVP

pytestmark = pytest.mark.gpu


def _case(name, n, seed=3):
    if name == "tfim16":
        model = qb.TransverseFieldIsing(qb.SquareLattice(1, 16), j=1.0, hx=1.0)
        net = RBM((16,), alpha=1, dtype="float32", seed=seed, init_scale=0.1)
        st = np.where(np.random.default_rng(seed).random((n, 16)) < 0.5, 0.5, -0.5)
    else:
        model = qb.J1J2Model(qb.SquareLattice(2, 6, 6), J1=-1.0, J2=-0.5)
        net = RBM((36,), alpha=4, dtype="complex64", seed=seed, init_scale=0.05)
        st = osm.init_states("RND_FIXED", n, 36, seed=seed, n_up=18) * 0.5
    bits = dv.pack_states(st)
    _, tn, lp = dv.rbm_forward(net.flat, net.ns, net.nh, bits, tanh=True, logpsi=True)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, net.ns, net.nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, net.ns, net.nh, bits, tn, h, tables)
    return net, st, bits, tn, lp, eloc


def _oracle(st, tn, eloc, cplx, probs=None):
    O = osr.o_rows(None, orbm.to_sigma(st), tanh=tn.cpu().numpy())
    e = eloc.cpu().numpy().astype(np.complex128)
    if not cplx:
        e = e.real
    w = None if probs is None else probs / probs.sum() * len(probs)
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    return osr.s_matrix(Oc, w_), osr.force(Oc, ec, w_)


@pytest.mark.parametrize("name,n,weighted", [("tfim16", 1024, False), ("tfim16", 1000, True),
                                             ("j1j2_6x6", 512, False), ("j1j2_6x6", 700, True)])
def test_gram_matches_oracle(name, n, weighted):
    net, st, bits, tn, lp, eloc = _case(name, n)
    probs = None
    if weighted:
        lu = lp.real.double()
        probs = torch.exp(lu - lu.max()).float()
    S = dv.sr_gram(net.flat, net.ns, net.nh, bits, tn, probs=probs).cpu().numpy()
    S_ref, _ = _oracle(st, tn, eloc, net.is_complex, None if probs is None else probs.double().cpu().numpy())
    assert np.max(np.abs(S - S_ref)) <= 1e-4 * np.max(np.abs(S_ref))
    assert np.allclose(S, np.conj(S.T), rtol=0, atol=1e-12 * np.max(np.abs(S)))


@pytest.mark.parametrize("name,n,shift", [("tfim16", 1024, 1e-3), ("j1j2_6x6", 512, 1e-3)])
def test_dense_solve_matches_oracle(name, n, shift):
    net, st, bits, tn, lp, eloc = _case(name, n)
    x, info, _ = dv.sr_solve_dense(net.flat, net.ns, net.nh, bits, tn, eloc, shift=shift, rhs_prefactor=-1.0)
    assert info["converged"] and info["iterations"] == 0
    S, F = _oracle(st, tn, eloc, net.is_complex)
    A = S + shift * np.eye(S.shape[0])
    xr = -np.linalg.solve(A, F)
    xg = x.cpu().numpy()
    resid = np.linalg.norm(A @ (-xg) - F) / np.linalg.norm(F)
    assert resid < 1e-4 and 0.0 <= info["true_residual"] < 1e-6
    if n > S.shape[0]:
        # full rank: entrywise, at the conditioning of S + shift times the 1e-6 - 1e-5 error of the
        # BF16-split Gram
        assert np.max(np.abs(xg - xr)) <= 1e-2 * np.max(np.abs(xr))
    else:
        err = xg - xr
        assert np.sqrt(abs(np.vdot(err, A @ err)) / abs(np.vdot(xr, A @ xr))) < 1e-2
    # the CG on the same data reaches the same solution in the same backward sense
    xc, ic = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=shift, rtol=1e-10, maxiter=4000)
    rc = np.linalg.norm(A @ (-xc.cpu().numpy()) - F) / np.linalg.norm(F)
    assert rc < 1e-4


def test_tdvp_form_matrix_uses_the_dense_path_and_nqs_trains():
    model = qb.TransverseFieldIsing(qb.SquareLattice(1, 8), j=1.0, hx=1.0, hz=0.0)
    nqs = qb.NQS("rbm", model, alpha=1.0, dtype="float32", seed=1, s_numchains=256, s_numsamples=8,
                 s_therm_steps=10, s_sweep_steps=8)
    stats = nqs.train(n_epochs=120, lr=0.05, diag_shift=1e-3, lin_force_mat=True, lin_solver="cholesky")
    assert nqs._tdvp.form_matrix
    from oracle import lattice as olat, hamiltonian as oH, ed as oed
    e0 = oed.ground_energy(oH.tfim_terms(olat.SquareLattice(1, 8), 1.0, 1.0, 0.0), 8)
    tail = np.mean([h.real for h in stats.history[-10:]])
    assert abs(tail - e0) / abs(e0) < 5e-3, (tail, e0)
    with pytest.raises(ValueError):
        TDVP(sr_lin_solver="cholesky")                      # a direct solve needs the formed matrix


def test_dense_refuses_oversized_systems():
    import ctypes as C
    out = C.c_size_t(0)
    rc = _lib.call("qes_sr_dense_workspace_bytes", _lib.DTYPE_F32, 400, 1600, 16384, 0, C.byref(out),
                   allow=(_lib.QES_ERR_SIZE,))
    assert rc == _lib.QES_ERR_SIZE and out.value > (100 << 30)
