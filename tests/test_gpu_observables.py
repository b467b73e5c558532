"""Observables through the ratio kernel (NQS.compute_observable / measure / expectation): local
values of lowered spin operators against the oracle's full re-evaluation estimator on identical
configurations (1e-5), and the Monte Carlo expectation against the exact one of the RBM state."""

import numpy as np
import pytest
import torch

from oracle import hamiltonian as oH, rbm as orbm, estimator as oest, sampler as osm
import pyqusolver_b200 as qb
from pyqusolver_b200.nqs import NQSObservable

pytestmark = pytest.mark.gpu


def _oracle_terms(op):
    return [oH.Term(t.op, t.sites, t.mult) for t in op.terms]


def _params(nqs):
    net = nqs.net
    flat = net.flat.detach().cpu().numpy().astype(np.complex128 if net.is_complex else np.float64)
    return orbm.RBMParams.from_flat(flat, net.ns, net.nh)


def _ops(L):
    return [qb.SpinOperator.magnetization(L, "z"), qb.SpinOperator.correlation(L, 0, 5, "z"),
            qb.SpinOperator.exchange(L, 0, 1), qb.SpinOperator.sigma(L, "x", 3),
            qb.SpinOperator.sigma(L, "y", 2), qb.SpinOperator.correlation(L, 2, 7, "x")]


@pytest.mark.parametrize("cplx", [True, False])
def test_local_values_match_oracle(cplx):
    L = qb.SquareLattice(2, 4, 4)
    model = qb.XXZ(L, jxy=-1.0, jz=-1.0)
    nqs = qb.NQS("rbm", model, alpha=1, dtype="complex64" if cplx else "float32", seed=3, init_scale=0.3,
                 s_numchains=64, s_numsamples=2)
    st = osm.init_states("RND", 300, 16, seed=5) * 0.5
    ops = _ops(L)
    res = nqs.compute_observable(states=st, functions=ops)
    p = _params(nqs)
    for op, r in zip(ops, res):
        ref = oest.local_energy_full(p, _oracle_terms(op), st)
        got = r.values.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-5 * max(1.0, np.max(np.abs(ref))), op.name
        assert r.mean == pytest.approx(np.mean(ref), rel=1e-5, abs=1e-6)
        assert r.n_samples == 300 and r.observable_name == op.name
    vals = nqs.compute_observable(states=st, functions=ops[:2], return_values=True)
    assert len(vals) == 2 and torch.equal(vals[0], res[0].values)
    with pytest.raises(TypeError):
        nqs.compute_observable(states=st, functions=lambda s: s)


def test_monte_carlo_expectation_matches_exact():
    L = qb.SquareLattice(1, 10)
    model = qb.TransverseFieldIsing(L, j=1.0, hx=0.8)
    nqs = qb.NQS("rbm", model, alpha=1, dtype="complex64", seed=12, init_scale=0.25, s_numchains=2048,
                 s_numsamples=20, s_therm_steps=20, s_sweep_steps=20)
    ops = {"Mz": qb.SpinOperator.magnetization(L, "z"), "SxSx": qb.SpinOperator.correlation(L, 0, 1, "x"),
           "SS": qb.SpinOperator.exchange(L, 4, 5), "H": model}
    res = nqs.measure(ops)
    assert set(res) == set(ops) and all(isinstance(r, NQSObservable) for r in res.values())
    p = _params(nqs)
    basis, w = osm.exact_distribution(p, 10)
    allst = ((basis[:, None] >> np.arange(9, -1, -1)) & 1) - 0.5
    for name, op in ops.items():
        terms = _oracle_terms(op)
        exact = np.sum(w * oest.local_energy_full(p, terms, allst)).real
        r = res[name]
        assert abs(r.mean.real - exact) <= 5 * r.error_of_mean + 1e-3, (name, r.mean, exact, r.error_of_mean)
