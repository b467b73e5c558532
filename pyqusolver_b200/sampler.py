"""``VMCSampler`` with the reference's interface, backed by the persistent GPU sampler.

Mirrors ``QES/Solver/MonteCarlo/vmc.py`` (``VMCSampler.__init__`` ``:136-320``,
``sample`` ``:1548-1623``, schedule ``:324-329,1718-1719``):

* the first ``sample`` after construction / ``reset`` thermalises with
  therm_steps * sweep_steps * N proposals, later calls continue the chains;
* each recorded sample is preceded by ``sweep_steps`` proposals;
* ``sample`` returns ((last_states, last_logpsi), (states, logpsi), probs) with
  sample-major rows (row = sample * n_chains + chain) and probs = None when
  1/logprob_fact - mu*beta == 0 (``vmc.py:1173-1184,1995-2008``);
* ``upd_fun`` accepts "LOCAL" (single flip) and "EXCHANGE" (neighbour swap,
  neighbour table from ``get_neighbor_table``, ``sampler.py:991-1023``);
* ``initstate`` accepts None/"RND" and "RND_FIXED" (with ``n_particles`` up
  spins, ``initialization/states.py:242-297``).

The Metropolis work runs in ``qes_sampler_run``; random numbers come from
Philox streams addressed by (chain, step), so a run is reproducible from the
seed alone.  States are returned as float32 +-0.5 tensors on the GPU and the
packed words stay available as ``last_sample_bits`` for the estimator.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from . import device as dv
from .lattice import get_neighbor_table


class VMCSampler:
    def __init__(self, net, shape, *, rng=None, rng_k=None, upd_fun=None, mu=2.0, beta=1.0, therm_steps=None,
                 sweep_steps=None, seed=None, hilbert=None, numsamples=1, numchains=1, numupd=1, initstate=None,
                 backend="default", logprob_fact=0.5, statetype=np.float32, n_particles=None, lattice=None,
                 recompute_every=None, exchange_order=1, chain_offset=0, **kwargs):
        if net is None:
            raise ValueError("A network (or callable) must be provided for evaluation.")
        if not hasattr(net, "flat") or not hasattr(net, "nh"):
            raise TypeError("the GPU sampler needs the RBM ansatz of this package")
        self._net = net
        self._shape = tuple(shape) if not np.isscalar(shape) else (int(shape),)
        self._size = int(np.prod(self._shape))
        if self._size != net.ns:
            raise ValueError("sampler shape does not match the network input size")
        if mu < 0.0 or mu > 2.0:
            raise ValueError("mu must be in [0, 2]")
        self._mu, self._beta = float(mu), float(beta)
        if therm_steps is None or sweep_steps is None:
            # the reference's GPU-backend defaults (vmc.py:216-236)
            therm_steps = 8 if therm_steps is None else therm_steps
            sweep_steps = 480 if sweep_steps is None else sweep_steps
        self._therm_steps = max(1, int(therm_steps))
        self._sweep_steps = max(1, int(sweep_steps))
        self._numsamples = int(numsamples)
        self._numchains = int(numchains)
        self._logprob_fact = float(logprob_fact)
        self._seed = int(seed if seed is not None else (rng_k if isinstance(rng_k, int) else 0))
        self._chain_offset = int(chain_offset)
        self._recompute_every = int(recompute_every) if recompute_every else 0
        name = "LOCAL" if upd_fun is None else str(getattr(upd_fun, "name", upd_fun)).upper()
        if name not in ("LOCAL", "EXCHANGE"):
            raise ValueError(f"update rule {upd_fun!r} is not supported by the GPU sampler (LOCAL, EXCHANGE)")
        self._rule = _lib.RULE_LOCAL if name == "LOCAL" else _lib.RULE_EXCHANGE
        self._upd_rule_name = name
        self._hilbert = hilbert
        lat = lattice if lattice is not None else getattr(hilbert, "lattice", None)
        self._exch_static = None
        if self._rule == _lib.RULE_EXCHANGE:
            if lat is None:
                raise ValueError("EXCHANGE needs a lattice (pass hilbert= or lattice=)")
            self._build_exchange(get_neighbor_table(lat, order=exchange_order))
        init = "RND" if initstate is None else str(initstate).upper()
        if init in ("RND", "RANDOM"):
            self._init_kind, self._n_up = _lib.INIT_RND, 0
        elif init in ("RND_FIXED", "RANDOM_FIXED", "FIXED_N", "CONSERVED"):
            self._init_kind = _lib.INIT_RND_FIXED
            self._n_up = self._size // 2 if n_particles is None else int(n_particles)
        elif init == "UP":
            self._init_kind, self._n_up = _lib.INIT_UP, 0
        elif init == "DOWN":
            self._init_kind, self._n_up = _lib.INIT_DOWN, 0
        else:
            raise ValueError(f"initial state {initstate!r} is not supported")
        self._tables = None
        self._tables_version = -1
        self.reset()

    # ------------------------------------------------------------------ state
    def _build_exchange(self, nt):
        ns, deg = nt.shape
        pairs = {}
        pi, pj = [], []
        nbr_pair = np.full(nt.shape, -1, dtype=np.int32)
        for i in range(ns):
            for k in range(deg):
                j = int(nt[i, k])
                if j < 0:
                    continue
                key = (min(i, j), max(i, j))
                if key not in pairs:
                    pairs[key] = len(pi)
                    pi.append(key[0])
                    pj.append(key[1])
                nbr_pair[i, k] = pairs[key]
        dev = self._net.device
        self._deg = deg
        self._nbr = torch.as_tensor(nt.reshape(-1), dtype=torch.int32, device=dev)
        self._nbr_pair = torch.as_tensor(nbr_pair.reshape(-1), dtype=torch.int32, device=dev)
        self._pair_i = torch.as_tensor(np.asarray(pi, dtype=np.int32), device=dev)
        self._pair_j = torch.as_tensor(np.asarray(pj, dtype=np.int32), device=dev)
        self._pair_kind = torch.full((len(pi),), _lib.MOVE_PAIR_ANTI, dtype=torch.int32, device=dev)
        self.neighbor_table = nt

    def reset(self):
        net = self._net
        self._states = dv.init_chains(self._init_kind, self._numchains, net.ns, self._seed, self._n_up,
                                      self._chain_offset, net.device)
        self._step = torch.zeros((self._numchains,), dtype=torch.int64, device=net.device)
        self._num_proposed = torch.zeros((self._numchains,), dtype=torch.int32, device=net.device)
        self._num_accepted = torch.zeros((self._numchains,), dtype=torch.int32, device=net.device)
        self._logprobas = None
        self._needs_thermalization = True

    def _sampler_tables(self):
        net = self._net
        if self._tables is not None and self._tables_version == net.version:
            return self._tables
        if self._rule == _lib.RULE_LOCAL:
            sites = torch.arange(net.ns, dtype=torch.int32, device=net.device)
            kinds = torch.full((net.ns,), _lib.MOVE_FLIP1, dtype=torch.int32, device=net.device)
            fC, fS, _ = dv.move_tables(net.flat, net.ns, net.nh, sites, sites, kinds, move_major=True)
            self._tables = ((fC, fS), None)
        else:
            pC, pS, _ = dv.move_tables(net.flat, net.ns, net.nh, self._pair_i, self._pair_j, self._pair_kind,
                                       move_major=True)
            self._tables = (None, (self._nbr, self._nbr_pair, self._pair_i, self._pair_j, pC, pS))
        self._tables_version = net.version
        return self._tables

    # ------------------------------------------------------------------ properties
    @property
    def numsamples(self):
        return self._numsamples

    @property
    def numchains(self):
        return self._numchains

    @property
    def states(self):
        return dv.unpack_states(self._states, self._net.ns)

    @property
    def proposed(self):
        return self._num_proposed

    @property
    def accepted(self):
        return self._num_accepted

    @property
    def accepted_ratio(self):
        p = self._num_proposed.to(torch.float64)
        return (self._num_accepted.to(torch.float64) / torch.clamp(p, min=1.0))

    @property
    def has_uniform_weights(self):
        return (1.0 / self._logprob_fact - self._mu * self._beta) == 0.0

    def set_numchains(self, n):
        if int(n) != self._numchains:
            self._numchains = int(n)
            self.reset()

    def set_numsamples(self, n):
        self._numsamples = int(n)

    # ------------------------------------------------------------------ sampling
    def sample_bits(self, num_samples=None, num_therm=None):
        """Run the chains; returns (sample_bits (Ns, nw) int32, sample_logpsi (Ns,))."""
        net = self._net
        ns_ = self._numsamples if num_samples is None else int(num_samples)
        therm = self._therm_steps if num_therm is None else int(num_therm)
        therm_total = therm * self._sweep_steps * net.ns if self._needs_thermalization else 0
        nc = self._numchains
        nw = dv.n_words(net.ns)
        sample_bits = torch.empty((ns_ * nc, nw), dtype=torch.int32, device=net.device)
        sample_lp = torch.empty((ns_ * nc,), dtype=net.dtype, device=net.device)
        last_lp = torch.empty((nc,), dtype=net.dtype, device=net.device)
        flip, exch = self._sampler_tables()
        cfg = _lib.SamplerConfig(self._rule, net.ns, net.nh, nc, self._chain_offset, ns_, therm_total,
                                 self._sweep_steps, self._recompute_every, self._mu, self._beta,
                                 self._seed & (2 ** 64 - 1), self._deg if exch is not None else 0)
        dv.sampler_run(net.flat, net.ns, net.nh, cfg, flip, exch, self._states, self._step, self._num_proposed,
                       self._num_accepted, sample_bits, sample_lp, last_lp)
        self._needs_thermalization = False
        self._logprobas = last_lp
        self.last_sample_bits = sample_bits
        self.last_sample_logpsi = sample_lp
        return sample_bits, sample_lp

    def sample(self, parameters=None, num_samples=None, *, num_chains=None, num_therm=None, betas=None):
        if betas is not None:
            raise NotImplementedError("parallel tempering is not part of the GPU sampler")
        if parameters is not None:
            self._net.set_params(parameters)
        if num_chains is not None:
            self.set_numchains(num_chains)
        bits, lp = self.sample_bits(num_samples, num_therm)
        states = dv.unpack_states(bits, self._net.ns)
        probs = None
        if not self.has_uniform_weights:
            exponent = 1.0 / self._logprob_fact - self._mu * self._beta
            lu = exponent * lp.real.to(torch.float64)
            pr = torch.exp(lu - lu.max())
            probs = (pr / torch.clamp(pr.sum(), min=1e-10) * lp.shape[0]).to(torch.float32)
        last = (dv.unpack_states(self._states, self._net.ns), self._logprobas)
        return last, (states, lp), probs
