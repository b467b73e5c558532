"""Local energy by full re-evaluation of every connected state (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Restates the contract of ``net_utils_jax.apply_callable_batched_jax`` (empty
submodule; called from ``QES/NQS/src/nqs_kernels.py:87-145`` and pinned by
``Python/tests/nqs/test_nqs_generic_config_and_learning.py:282-371``):

    E_loc(s) = sum_k conj(c_k(s)) * exp(log psi(s'_k) - log psi(s))

where (s'_k, c_k) is the slot list of ``local_energy_jax_wrap`` and c_k is the
matrix element <s'_k|H|s>; the conjugate is what makes the sample mean equal
<psi|H|psi>/<psi|psi> for a complex operator (the sigma^y orientation test,
``test_nqs_generic_config_and_learning.py:337-371``).  The weighted mean is
sum_s w_s E_s / Ns with weights normalised to sum Ns (``vmc.py:1173-1184``),
or the plain mean when the sampler reports uniform weights (probs is None).
"""

from __future__ import annotations

import numpy as np

from . import rbm as rbm_mod
from .hamiltonian import connected_raw


def local_energy_full(params, terms, states_pm, chunk=4096):
    """E_loc for every row of ``states_pm`` (+-0.5), evaluating log psi on every slot."""
    states_pm = np.atleast_2d(np.asarray(states_pm, dtype=np.float64))
    out = np.zeros(states_pm.shape[0], dtype=np.complex128)
    for r0 in range(0, states_pm.shape[0], chunk):
        blk = states_pm[r0:r0 + chunk]
        all_states, all_coeffs = [], []
        for s in blk:
            st, co = connected_raw(terms, s)
            all_states.append(st)
            all_coeffs.append(co)
        K = all_states[0].shape[0]
        st = np.concatenate(all_states)
        co = np.concatenate(all_coeffs).reshape(len(blk), K)
        lp_conn = rbm_mod.log_psi(params, rbm_mod.to_sigma(st)).reshape(len(blk), K)
        lp_in = rbm_mod.log_psi(params, rbm_mod.to_sigma(blk))
        out[r0:r0 + len(blk)] = np.sum(np.conj(co) * np.exp(lp_conn - lp_in[:, None]), axis=1)
    return out


def local_energy_generic(local_fn, logpsi_fn, states, logpsi_in):
    """Generic form: ``local_fn(s) -> (states, coeffs)``, ``logpsi_fn(states) -> log psi``."""
    out = []
    for s, lp in zip(states, logpsi_in):
        st, co = local_fn(s)
        out.append(np.sum(np.conj(co) * np.exp(logpsi_fn(st) - lp)))
    return np.asarray(out)


def loss_stats(e_loc, probs=None):
    """(mean, std) of E_loc; weighted by ``probs`` normalised to sum Ns when given."""
    e_loc = np.asarray(e_loc)
    n = e_loc.shape[0]
    if probs is None:
        mean = np.mean(e_loc)
        std = np.std(e_loc)
    else:
        w = np.asarray(probs, dtype=np.float64).reshape(-1)
        mean = np.sum(w * e_loc) / n
        std = np.sqrt(np.sum(w * np.abs(e_loc - mean) ** 2) / n)
    return mean, std


def step_rhat(e_loc, num_chains=1):
    """Gelman-Rubin R-hat of Re E_loc (``QES/NQS/src/tdvp.py:1487-1518``).

    The flattened batch is reshaped to (num_chains, chain_len) literally, as the
    reference does; NaN for an invalid split.
    """
    vals = np.real(np.asarray(e_loc)).reshape(-1).astype(np.float64)
    nch = max(int(num_chains), 1)
    n_tot = vals.shape[0]
    if nch <= 1 or n_tot <= nch or n_tot % nch != 0 or n_tot // nch <= 1:
        return float("nan")
    L = n_tot // nch
    chains = vals.reshape(nch, L)
    w = np.mean(np.var(chains, axis=1, ddof=1))
    b = L * np.var(np.mean(chains, axis=1), ddof=1)
    var_hat = ((L - 1.0) / L) * w + b / L
    return float(np.sqrt(var_hat / max(w, 1e-12)))


def step_sigma2(e_loc):
    """sigma^2 = var(Re E_loc), uniform, ddof 0 (``QES/NQS/src/tdvp.py:1642``)."""
    return float(np.var(np.real(np.asarray(e_loc)).astype(np.float64)))


def sample_probs(log_ansatz, total_samples, exponent):
    """Reweighting factors (``vmc.py:1173-1184``)."""
    lu = exponent * np.real(np.asarray(log_ansatz))
    pr = np.exp(lu - np.max(lu))
    return pr / max(np.sum(pr), 1e-10) * total_samples
