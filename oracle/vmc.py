"""One whole VMC step, restated from the reference (oracle side and CPU baseline).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  ``bench.py`` times it
as the CPU baseline; it is never on the product path.

One training epoch of ``NQSTrainer.train`` (``QES/NQS/src/nqs_train.py:1460-1619``):
sample (``VMCSampler.sample``), local energy with full re-evaluation of every
connected state, per-sample log-derivatives, SR solve (CG, float64), Euler/SGD
update.  The local energy is vectorised over a block of samples: every slot
of every sample is a full RBM evaluation, as in the reference estimator.
"""

from __future__ import annotations

import numpy as np

from . import rbm as rbm_mod
from . import sr as sr_mod
from .hamiltonian import connected_raw_batch
from .estimator import loss_stats


def local_energy_batched(params, terms, configs_pm, block=256):
    configs_pm = np.atleast_2d(configs_pm)
    out = np.empty(configs_pm.shape[0], dtype=np.complex128)
    for r0 in range(0, configs_pm.shape[0], block):
        blk = configs_pm[r0:r0 + block]
        st, co = connected_raw_batch(terms, blk)
        B, K, N = st.shape
        lp = rbm_mod.log_psi(params, rbm_mod.to_sigma(st.reshape(B * K, N))).reshape(B, K)
        out[r0:r0 + B] = np.sum(np.conj(co) * np.exp(lp - lp[:, :1]), axis=1)
    return out


def vmc_step(params: rbm_mod.RBMParams, terms, sampler, num_samples, *, lr=0.01,
             shift=1e-3, rtol=1e-8, maxiter=1000, rhs_prefactor=-1.0):
    """Returns (new_params, stats dict)."""
    configs, logpsi, probs = sampler.sample(params, num_samples)
    e_loc = local_energy_batched(params, terms, configs * 0.5)
    O = rbm_mod.log_derivatives(params, configs)
    x, info = sr_mod.solve_sr(e_loc, O, shift=shift, probs=probs, method="cg",
                              rtol=rtol, maxiter=maxiter, rhs_prefactor=rhs_prefactor)
    n, m = params.n_visible, params.n_hidden
    flat = params.flat()
    if not np.iscomplexobj(flat):
        x = np.real(x)
    new = rbm_mod.RBMParams.from_flat(flat + lr * x, n, m)
    mean, std = loss_stats(e_loc, probs)
    return new, {"mean": mean, "std": std, "cg_iters": info.get("iterations"),
                 "accept": float(np.mean(sampler.accepted / np.maximum(sampler.proposed, 1)))}
