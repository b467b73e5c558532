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
                 recompute_every=None, exchange_order=1, chain_offset=0, pt_betas=None, pt_replicas=None,
                 **kwargs):
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
        self._pt_betas = None
        self._n_replicas = 1
        self._pt_round = 0
        if pt_betas is not None or (pt_replicas is not None and int(pt_replicas) > 1):
            self.set_replicas(pt_betas, pt_replicas)
        else:
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
        R, nc = self._n_replicas, self._numchains
        base = dv.init_chains(self._init_kind, nc, net.ns, self._seed, self._n_up, self._chain_offset, net.device)
        # parallel tempering: every replica slot starts from the same base states (vmc.py:397-405)
        self._states = base.repeat(R, 1).contiguous() if R > 1 else base
        self._step = torch.zeros((R * nc,), dtype=torch.int64, device=net.device)
        self._num_proposed = torch.zeros((R * nc,), dtype=torch.int32, device=net.device)
        self._num_accepted = torch.zeros((R * nc,), dtype=torch.int32, device=net.device)
        if R > 1:
            b = torch.as_tensor(np.asarray(self._pt_betas, dtype=np.float32), device=net.device)
            self._chain_beta = b[:, None].repeat(1, nc).reshape(-1).contiguous()
            self._pt_swaps = torch.zeros((R,), dtype=torch.int32, device=net.device)
        self._pt_round = 0
        self._logprobas = None
        self._needs_thermalization = True

    # ------------------------------------------------------------------ parallel tempering
    def set_replicas(self, betas=None, n_replicas=None, min_beta=None):
        """Beta ladder of parallel tempering (``vmc.py:1880-1911``): an explicit descending ladder, or
        ``n_replicas`` log-spaced values from the sampler's beta down to ``min_beta`` (beta / 10)."""
        if betas is None and n_replicas is not None and int(n_replicas) > 1:
            max_beta = float(self._beta)
            min_beta = float(min_beta if min_beta is not None else max_beta / 10.0)
            if max_beta <= 0.0 or min_beta <= 0.0:
                raise ValueError("PT beta ladder values must be positive.")
            betas = np.logspace(np.log10(max_beta), np.log10(min_beta), int(n_replicas))
        elif betas is not None:
            betas = np.asarray(betas, dtype=np.float64)
            if betas.ndim != 1:
                raise ValueError("PT beta ladder must be a one-dimensional array.")
            if np.any(betas <= 0.0):
                raise ValueError("PT beta ladder values must be positive.")
            if betas.shape[0] <= 1:
                betas = None
        cur = self._pt_betas
        if (cur is None and betas is None) or (cur is not None and betas is not None and len(cur) == len(betas)
                                                and np.allclose(cur, betas)):
            if not hasattr(self, "_states"):
                self.reset()
            return
        self._pt_betas = betas
        self._n_replicas = len(betas) if betas is not None else 1
        self.reset()

    set_pt_betas = set_replicas

    @property
    def is_pt(self):
        return self._pt_betas is not None

    @property
    def n_replicas(self):
        return self._n_replicas

    @property
    def pt_betas(self):
        return None if self._pt_betas is None else np.asarray(self._pt_betas, dtype=np.float32)

    @property
    def chain_betas(self):
        """Current beta label of every (slot, chain), shape (n_replicas, numchains)."""
        if not self.is_pt:
            return None
        return self._chain_beta.view(self._n_replicas, self._numchains)

    def _sample_bits_pt(self, num_samples, therm_steps):
        net = self._net
        R, nc = self._n_replicas, self._numchains
        nw = dv.n_words(net.ns)
        therm_updates = therm_steps * self._sweep_steps * net.ns if self._needs_thermalization else 0
        n_therm = max(1, -(-therm_updates // self._sweep_steps))
        flip, exch = self._sampler_tables()
        cfg = _lib.SamplerConfig(self._rule, net.ns, net.nh, R * nc, self._chain_offset, 0, self._sweep_steps,
                                 self._sweep_steps, self._recompute_every, self._mu, self._beta,
                                 self._seed & (2 ** 64 - 1), self._deg if exch is not None else 0)
        last_lp = torch.empty((R * nc,), dtype=net.dtype, device=net.device)
        sample_bits = torch.empty((num_samples * nc, nw), dtype=torch.int32, device=net.device)
        sample_lp = torch.empty((num_samples * nc,), dtype=net.dtype, device=net.device)
        dc = dv.dtype_code(net.flat)
        target = float(np.float32(self._pt_betas[0]))

        def one_round():
            dv.sampler_run(net.flat, net.ns, net.nh, cfg, flip, exch, self._states, self._step, self._num_proposed,
                           self._num_accepted, None, None, last_lp, chain_beta=self._chain_beta)
            _lib.call("qes_pt_swap", dc, R, nc, _lib.ptr(last_lp), _lib.ptr(self._chain_beta), float(self._mu),
                      _lib.C.c_uint64(self._seed & (2 ** 64 - 1)), int(self._pt_round), _lib.ptr(self._pt_swaps),
                      _lib.stream_ptr())
            self._pt_round += 1

        for _ in range(n_therm):
            one_round()
        for k in range(num_samples):
            one_round()
            _lib.call("qes_pt_collect", dc, R, nc, net.ns, _lib.ptr(self._chain_beta), target, _lib.ptr(self._states),
                      _lib.ptr(last_lp), _lib.ptr(sample_bits[k * nc:(k + 1) * nc]),
                      _lib.ptr(sample_lp[k * nc:(k + 1) * nc]), _lib.stream_ptr())
        self._needs_thermalization = False
        self._logprobas = last_lp
        self.last_sample_bits = sample_bits
        self.last_sample_logpsi = sample_lp
        return sample_bits, sample_lp

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
    def _phys_beta(self):
        return float(self._pt_betas[0]) if self._pt_betas is not None else self._beta

    @property
    def has_uniform_weights(self):
        return (1.0 / self._logprob_fact - self._mu * self._phys_beta) == 0.0

    def sample_probs(self, logpsi):
        """Reweighting factors of a batch (``vmc.py:1173-1184``): exp((1/logprob_fact - mu beta) Re log psi)
        normalised to sum Ns, or None when the sampler draws |psi|^2 itself (uniform weights)."""
        if self.has_uniform_weights:
            return None
        exponent = 1.0 / self._logprob_fact - self._mu * self._phys_beta
        lu = exponent * logpsi.real.to(torch.float64)
        pr = torch.exp(lu - lu.max())
        return (pr / torch.clamp(pr.sum(), min=1e-10) * logpsi.shape[0]).to(torch.float32)

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
        if self.is_pt:
            return self._sample_bits_pt(ns_, therm)
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
            self.set_replicas(betas)
        if parameters is not None:
            self._net.set_params(parameters)
        if num_chains is not None:
            self.set_numchains(num_chains)
        bits, lp = self.sample_bits(num_samples, num_therm)
        states = dv.unpack_states(bits, self._net.ns)
        probs = self.sample_probs(lp)
        last_states = dv.unpack_states(self._states, self._net.ns)
        if self.is_pt:
            last_states = last_states.view(self._n_replicas, self._numchains, self._net.ns)
        last = (last_states, self._logprobas)
        return last, (states, lp), probs
