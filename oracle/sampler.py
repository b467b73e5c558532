"""Metropolis VMC sampler restated from the reference (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``VMCSampler`` (``QES/Solver/MonteCarlo/vmc.py``):

* one step for all chains (``_sweep_chain_jax_step_inner``, ``:1016-1097``):
  propose, Delta = log psi(s') - log psi(s), log_acc = min(beta*mu*Re Delta, 0),
  accept iff log u < log_acc, masked select, proposed += 1, accepted += keep;
* proposals: single flip of a uniform site (``updates/spin_jax.py:51-91``);
  exchange of a uniform site i with a uniform slot of its neighbour-table row,
  swapped only when the slot is valid and sigma_i != sigma_j -- otherwise the
  proposal is the unchanged state, Delta = 0, and it is counted as accepted
  (``spin_jax.py:97-158`` with the full re-evaluation branch ``vmc.py:1050-1054``);
* schedule (``vmc.py:324-329,1718-1719``): the first call after a reset runs
  therm_steps * sweep_steps * N thermalisation proposals, every later call none;
  each recorded sample is preceded by sweep_steps proposals;
* outputs are sample-major: row = sample * n_chains + chain (``lax.scan`` stacking,
  ``vmc.py:1265-1270``); probs are None when 1/logprob_fact - mu*beta == 0.

The random numbers come from the Philox streams of ``oracle.philox`` instead
of JAX keys, so the GPU chains can be compared with these step by step.
"""

from __future__ import annotations

import numpy as np

from . import philox
from . import rbm as rbm_mod
from .estimator import sample_probs


def init_states(kind, n_chains, ns, seed, n_up=None, chain_offset=0):
    """Initial +-1 chains: 'RND' (independent bits) or 'RND_FIXED' (n_up up spins, shuffled)."""
    k0, k1 = philox.seed_key(seed)
    chains = np.arange(chain_offset, chain_offset + n_chains, dtype=np.uint64)
    out = np.empty((n_chains, ns), dtype=np.float64)
    kind = str(kind).upper()
    if kind in ("RND", "RANDOM", "NONE"):
        nwords = (ns + 31) // 32
        for w in range(nwords):
            r = philox.philox4x32_10(chains, w, 0, philox.STREAM_INIT_RND, k0, k1)[0]
            for b in range(32):
                i = 32 * w + b
                if i >= ns:
                    break
                out[:, i] = np.where((r >> np.uint32(b)) & np.uint32(1), 1.0, -1.0)
        return out
    if kind in ("RND_FIXED", "FIXED", "CONSERVED"):
        nu = ns // 2 if n_up is None else int(n_up)
        base = np.concatenate([np.ones(nu), -np.ones(ns - nu)])
        out[:] = base
        for pos in range(ns - 1, 0, -1):
            r = philox.philox4x32_10(chains, pos, 0, philox.STREAM_INIT_FIXED, k0, k1)[0]
            j = philox.bounded(r, pos + 1)
            rows = np.arange(n_chains)
            tmp = out[rows, pos].copy()
            out[rows, pos] = out[rows, j]
            out[rows, j] = tmp
        return out
    if kind == "UP":
        out[:] = 1.0
        return out
    if kind == "DOWN":
        out[:] = -1.0
        return out
    raise ValueError(f"unknown initial state {kind}")


class MetropolisSampler:
    def __init__(self, ns, n_chains, *, rule="LOCAL", neighbor_table=None, seed=0,
                 mu=2.0, beta=1.0, therm_steps=1, sweep_steps=1, logprob_fact=0.5,
                 init="RND", n_up=None, chain_offset=0):
        self.ns = ns
        self.n_chains = n_chains
        self.rule = rule.upper()
        if self.rule == "EXCHANGE":
            if neighbor_table is None:
                raise ValueError("EXCHANGE needs a neighbour table")
            self.nt = np.asarray(neighbor_table, dtype=np.int64)
        elif self.rule != "LOCAL":
            raise ValueError(f"rule {rule} not supported")
        self.seed = seed
        self.mu, self.beta = float(mu), float(beta)
        self.therm_steps = max(1, int(therm_steps))
        self.sweep_steps = max(1, int(sweep_steps))
        self.logprob_fact = logprob_fact
        self.chain_ids = np.arange(chain_offset, chain_offset + n_chains, dtype=np.uint64)
        self.states = init_states(init, n_chains, ns, seed, n_up=n_up, chain_offset=chain_offset)
        self.step = 0
        self.proposed = np.zeros(n_chains, dtype=np.int64)
        self.accepted = np.zeros(n_chains, dtype=np.int64)
        # smallest |log u - log_acc| met by each chain's decisions: a float32 implementation can take
        # the other branch only where this margin is within its rounding of Delta log psi
        self.min_margin = np.full(n_chains, np.inf)
        self.needs_therm = True

    def _propose(self, r0, r1):
        n = self.n_chains
        rows = np.arange(n)
        new = self.states.copy()
        i = philox.bounded(r0, self.ns)
        if self.rule == "LOCAL":
            new[rows, i] = -new[rows, i]
            moved = np.ones(n, dtype=bool)
        else:
            deg = self.nt.shape[1]
            k = philox.bounded(r1, deg)
            j = self.nt[i, k]
            valid = j >= 0
            jj = np.where(valid, j, i)
            si, sj = self.states[rows, i], self.states[rows, jj]
            moved = valid & (si != sj)
            new[rows[moved], i[moved]] = sj[moved]
            new[rows[moved], jj[moved]] = si[moved]
        return new, moved

    def run_steps(self, params, steps):
        lp = rbm_mod.log_psi(params, self.states)
        for _ in range(steps):
            r0, r1, r2, _r3 = philox.proposal_draws(self.seed, self.chain_ids, self.step)
            new, moved = self._propose(r0, r1)
            lp_new = lp.copy()
            if np.any(moved):
                lp_new[moved] = rbm_mod.log_psi(params, new[moved])
            delta = np.real(lp_new - lp)
            log_acc = np.minimum(self.beta * self.mu * delta, 0.0)
            logu = np.log(philox.uniform_open(r2))
            keep = logu < log_acc
            self.min_margin = np.minimum(self.min_margin, np.abs(logu - log_acc))
            self.states = np.where(keep[:, None], new, self.states)
            lp = np.where(keep, lp_new, lp)
            self.proposed += 1
            self.accepted += keep
            self.step += 1
        return lp

    def sample(self, params, num_samples):
        if self.needs_therm:
            self.run_steps(params, self.therm_steps * self.sweep_steps * self.ns)
            self.needs_therm = False
        cfg, lps = [], []
        for _ in range(num_samples):
            lp = self.run_steps(params, self.sweep_steps)
            cfg.append(self.states.copy())
            lps.append(lp.copy())
        configs = np.concatenate(cfg)
        logpsi = np.concatenate(lps)
        exponent = 1.0 / self.logprob_fact - self.mu * self.beta
        probs = None if exponent == 0.0 else sample_probs(logpsi, configs.shape[0], exponent)
        return configs, logpsi, probs


class ParallelTemperingSampler:
    """Replica exchange of beta labels (``QES/Solver/MonteCarlo/vmc.py:1289-1507``).

    Slots r = 0..R-1 hold n_chains chains each (chain id r * n_chains + c, the ids of one
    ``MetropolisSampler`` over R * n_chains chains).  One round = ``sweep_steps`` Metropolis
    steps of every chain at its current beta (``_run_pt_round_jax``), then a swap of beta
    labels between adjacent slots of one parity (``_replica_exchange_kernel_jax_betas``):
    accept iff log u < min((b_r - b_r+1) mu (Re lpsi_r+1 - Re lpsi_r), 0).  Thermalisation
    runs max(1, ceil(therm_updates / sweep_steps)) rounds on every call, with therm_updates
    = therm_steps * sweep_steps * N on the first call and 0 afterwards (``:1439``, ``:1585``).
    After each sampling round the physical slot (beta == pt_betas[0]) of every chain is
    recorded (``_collect_pt_physical_samples_jax``).  Random draws: the phase is Philox counter
    (round, 0, 0, STREAM_PT_PHASE) word 0 & 1; the swap uniform of pair r in chain c is
    counter (c, round, r, STREAM_PT_SWAP) word 0 (the reference uses JAX keys).  Betas are
    float32 values, as the device stores them.
    """

    def __init__(self, ns, n_chains, pt_betas, **kw):
        self.pt_betas = np.asarray(pt_betas, dtype=np.float32).astype(np.float64)
        self.R = len(self.pt_betas)
        self.C = int(n_chains)
        self.base = MetropolisSampler(ns, self.R * self.C, **kw)
        # every slot starts from the same base states (``vmc.py:397-405``)
        base = init_states(kw.get("init", "RND"), self.C, ns, kw.get("seed", 0), n_up=kw.get("n_up"),
                           chain_offset=kw.get("chain_offset", 0))
        self.base.states = np.tile(base, (self.R, 1))
        self.betas = np.repeat(self.pt_betas[:, None], self.C, axis=1)
        self.round = 0
        self.swaps = np.zeros(max(self.R - 1, 1), dtype=np.int64)
        self.swap_margin = np.full(self.C, np.inf)     # as MetropolisSampler.min_margin, for the swaps

    def _round(self, params):
        b = self.base
        b.beta = self.betas.reshape(-1)
        lp = b.run_steps(params, b.sweep_steps).reshape(self.R, self.C)
        k0, k1 = philox.seed_key(b.seed)
        rnd = np.uint64(self.round)
        ph = philox.philox4x32_10(rnd & np.uint64(0xFFFFFFFF), rnd >> np.uint64(32), 0,
                                  philox.STREAM_PT_PHASE, k0, k1)[0]
        phase = int(ph) & 1
        cols = np.arange(self.C, dtype=np.uint64)
        for r in range(phase, self.R - 1, 2):
            bi, bj = self.betas[r].copy(), self.betas[r + 1].copy()
            log_acc = (bi - bj) * b.mu * (np.real(lp[r + 1]) - np.real(lp[r]))
            u = philox.uniform_open(philox.philox4x32_10(cols, self.round, r, philox.STREAM_PT_SWAP, k0, k1)[0])
            acc = np.log(u) < np.minimum(log_acc, 0.0)
            self.swap_margin = np.minimum(self.swap_margin, np.abs(np.log(u) - np.minimum(log_acc, 0.0)))
            self.betas[r] = np.where(acc, bj, bi)
            self.betas[r + 1] = np.where(acc, bi, bj)
            self.swaps[r] += int(acc.sum())
        self.round += 1
        return lp

    @property
    def min_margin(self):
        """Per chain column: the smallest decision margin of its R slots' Metropolis steps and swaps."""
        return np.minimum(self.base.min_margin.reshape(self.R, self.C).min(axis=0), self.swap_margin)

    def sample(self, params, num_samples):
        b = self.base
        therm_updates = b.therm_steps * b.sweep_steps * b.ns if b.needs_therm else 0
        for _ in range(max(1, -(-therm_updates // b.sweep_steps))):
            self._round(params)
        b.needs_therm = False
        cfg, lps = [], []
        states = lambda: b.states.reshape(self.R, self.C, b.ns)
        for _ in range(num_samples):
            lp = self._round(params)
            phys = np.abs(self.betas - self.pt_betas[0]) < 1e-5
            slot = np.argmax(phys, axis=0)
            cols = np.arange(self.C)
            cfg.append(states()[slot, cols].copy())
            lps.append(lp[slot, cols].copy())
        configs = np.concatenate(cfg)
        logpsi = np.concatenate(lps)
        exponent = 1.0 / b.logprob_fact - b.mu * self.pt_betas[0]
        probs = None if exponent == 0.0 else sample_probs(logpsi, configs.shape[0], exponent)
        return configs, logpsi, probs


def exact_distribution(params, ns, n_up=None):
    """|psi|^2 over the full (or fixed-n_up) basis, in the big-endian integer order."""
    allb = np.arange(1 << ns, dtype=np.int64)
    if n_up is not None:
        allb = allb[np.bitwise_count(allb) == n_up]
    shifts = np.arange(ns - 1, -1, -1, dtype=np.int64)
    sig = np.where(((allb[:, None] >> shifts[None, :]) & 1) == 1, 1.0, -1.0)
    lp = rbm_mod.log_psi(params, sig)
    w = np.exp(2.0 * (np.real(lp) - np.max(np.real(lp))))
    return allb, w / np.sum(w)
