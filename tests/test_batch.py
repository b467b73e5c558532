"""Batched problems of uneven size against the single-problem path (and the oracle).

Problem b of an ``NQSBatch`` must behave exactly like an ``NQS`` built with
seed = s_seed = seeds[b]: bit-identical sampler trajectories and acceptance
counters, identical tanh(theta) / E_loc (same kernels on the same inputs),
and an SR solution within the float32 SR bar (1e-4 relative) of the
single-problem CUDA-core solve: the batched matvec kernels sum the same
float32 products in a different order, and CG amplifies that rounding by
the condition number of S + shift.
"""

import numpy as np
import pytest
import torch

from oracle import lattice as olat, hamiltonian as oH, rbm as orbm, estimator as oest
import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.batch import NQSBatch

pytestmark = pytest.mark.gpu


def tfim_chain(L, hx):
    return qb.TransverseFieldIsing(qb.SquareLattice(1, L, 1, bc="pbc"), j=1.0, hx=hx, hz=0.0)


def single(model, seed, dtype, chains, nsamp, alpha):
    ns = model.ns
    return qb.NQS("rbm", model, alpha=alpha, dtype=dtype, seed=seed, s_seed=seed, s_upd_fun="LOCAL",
                  s_numchains=chains, s_numsamples=nsamp, s_sweep_steps=ns, s_therm_steps=1, init_scale=0.01)


@pytest.mark.parametrize("dtype", ["float32", "complex64"])
def test_batch_matches_single_problem_path(dtype):
    Ls, hxs, seeds = [6, 13, 33, 20], [0.7, 1.0, 1.3, 0.9], [11, 5, 7, 3]
    models = [tfim_chain(L, h) for L, h in zip(Ls, hxs)]
    if dtype == "complex64":
        models[1] = qb.XXZ(qb.SquareLattice(1, 13, 1, bc="pbc"), jxy=-1.0, jz=-0.5)
    chains, nsamp, alpha = 40, 3, 2
    B = NQSBatch(models, alpha=alpha, dtype=dtype, seeds=seeds, s_numchains=chains, s_numsamples=nsamp,
                 s_therm_steps=1, autotune=False, warps_per_block=4, blocks_per_sm=2)
    _lib.set_sr_impl(_lib.SR_IMPL_CUDA_CORES)
    try:
        B.sample()
        B.forward()
        B.local_energy()
        st = B.loss_stats().cpu().numpy()
        x, res = B.sr_solve(shift=1e-3, rtol=1e-8, maxiter=500)
        xs = x.cpu().numpy()
        acc = B.acceptance()
        for b, m in enumerate(models):
            q = single(m, seeds[b], dtype, chains, nsamp, alpha)
            assert torch.equal(q.net.master.cpu(), B.params(b).cpu())
            bits, lp = q.sampler.sample_bits()
            bb, blp = B.samples(b)
            assert torch.equal(bits.cpu(), bb.cpu()), f"problem {b}: samples differ"
            assert torch.equal(lp.cpu(), blp.cpu())
            o = int(B.chain_off[b])
            assert torch.equal(B.accepted[o:o + chains].cpu(), q.sampler.accepted.cpu())
            assert torch.equal(B.proposed[o:o + chains].cpu(), q.sampler.proposed.cpu())
            assert acc[b] == pytest.approx(q.sampler.accepted_ratio.mean().item(), rel=1e-12)
            _, tn, _ = dv.rbm_forward(q.net.flat, q.net.ns, q.net.nh, bits, theta=False, tanh=True, logpsi=False)
            assert torch.equal(tn.cpu(), B.tanh_theta(b).cpu())
            e = q.local_energy_bits(bits, tn)
            assert torch.equal(e.cpu(), B.local_energies(b).cpu())
            s1 = dv.loss_stats(e).cpu().numpy()
            assert st[b, 0] == pytest.approx(s1[0], rel=1e-12, abs=1e-12)
            assert st[b, 3] == pytest.approx(s1[3], rel=1e-9)
            x1, info = dv.sr_solve_cg(q.net.flat, q.net.ns, q.net.nh, bits, tn, e, shift=1e-3, rtol=1e-8,
                                      maxiter=500)
            o = int(B.param_off[b])
            xb = xs[o:o + int(B.P[b])]
            x1 = x1.cpu().numpy()
            assert np.max(np.abs(xb - x1)) <= 1e-4 * np.max(np.abs(x1)), f"problem {b}: SR solution differs"
            assert res[b].converged == int(info["converged"])
            assert abs(res[b].iterations - info["iterations"]) <= max(3, 0.05 * info["iterations"])
    finally:
        _lib.set_sr_impl(_lib.SR_IMPL_AUTO)


def test_batch_local_energy_matches_oracle():
    Ls, seeds = [8, 17, 30], [1, 2, 3]
    models = [tfim_chain(L, 0.5 + 0.3 * q) for q, L in enumerate(Ls)]
    B = NQSBatch(models, alpha=2, dtype="float32", seeds=seeds, s_numchains=16, s_numsamples=2,
                 autotune=False, warps_per_block=2, blocks_per_sm=4)
    B.sample()
    B.forward()
    B.local_energy()
    for b, L in enumerate(Ls):
        bits, _ = B.samples(b)
        states = dv.unpack_states(bits, L).cpu().numpy()
        flat = B.params(b).cpu().numpy()
        prm = orbm.RBMParams.from_flat(flat.astype(np.float32).astype(np.float64), L, 2 * L)
        terms = oH.tfim_terms(olat.SquareLattice(1, L, 1, "pbc"), 1.0, 0.5 + 0.3 * b, 0.0)
        ref = oest.local_energy_full(prm, terms, states)
        got = B.local_energies(b).cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-5 * max(1.0, np.max(np.abs(ref)))


def test_batch_training_step_updates_each_problem_like_single():
    Ls, seeds = [10, 24], [4, 9]
    models = [tfim_chain(L, 1.0) for L in Ls]
    B = NQSBatch(models, alpha=2, dtype="float32", seeds=seeds, s_numchains=32, s_numsamples=4,
                 autotune=False, warps_per_block=4, blocks_per_sm=2)
    _lib.set_sr_impl(_lib.SR_IMPL_CUDA_CORES)
    try:
        before = [B.params(b).clone() for b in range(len(models))]
        info = B.train_step(lr=0.02, diag_shift=1e-3)
        from pyqusolver_b200.tdvp import TDVP
        for b, m in enumerate(models):
            q = single(m, seeds[b], "float32", 32, 4, 2)
            assert torch.equal(q.net.master, before[b])
            i1 = q.train_step(lr=0.02, tdvp=TDVP(rhs_prefactor=-1.0, sr_diag_shift=1e-3))
            assert info["mean"][b] == pytest.approx(i1["mean"], rel=1e-12)
            d_batch = B.params(b) - before[b]
            d_single = q.net.master - before[b]
            assert (d_batch - d_single).abs().max().item() <= 1e-4 * d_single.abs().max().item()
    finally:
        _lib.set_sr_impl(_lib.SR_IMPL_AUTO)


def test_batch_autotune_persists_choice(tmp_path):
    models = [tfim_chain(L, 1.0) for L in (12, 20, 31)]
    B = NQSBatch(models, alpha=2, dtype="float32", s_numchains=64, s_numsamples=2, autotune=False,
                 warps_per_block=4, blocks_per_sm=4)
    cache = tmp_path / "tune.json"
    before = B.chain_bits.clone()
    best = B.autotune_sampler(candidates=((2, 4), (4, 4), (8, 2)), repeats=1, cache=str(cache))
    assert torch.equal(before, B.chain_bits)           # tuning ran on scratch chains
    assert cache.exists()
    B2 = NQSBatch(models, alpha=2, dtype="float32", s_numchains=64, s_numsamples=2, autotune=False,
                  warps_per_block=1, blocks_per_sm=1)
    assert B2.autotune_sampler(cache=str(cache)) == tuple(best)
