"""Many independent RBM-VMC problems of uneven size, advanced together on one GPU.

The reference trains one ``NQS`` per Hamiltonian (``QES/NQS/nqs.py:241``); a
study over many instances (system sizes, couplings) is a Python loop over
such objects.  ``NQSBatch`` keeps each problem's semantics -- its own RBM
initialisation (identical to ``RBM(..., seed=seed_b)``), its own sampler key
(identical to ``VMCSampler(..., seed=s_seed_b)``), its own SR solve -- but
runs every phase of the VMC epoch as ONE launch over all problems:

* the sampler is a persistent kernel whose warps take (problem, chain) work
  items from a device queue, heaviest problems first;
* forward, local energy and the SR matvec halves run over work lists of
  (problem, tile) items;
* the CG of every problem advances in lockstep launches, each problem frozen
  at its own convergence.

Buffers are the concatenation of the per-problem buffers; the layout is the
``qes_batch_instance`` descriptor of ``include/qes_b200.h``.
"""

from __future__ import annotations

import ctypes as C
import json
import os
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import device as dv
from ._lib import call, ptr, stream_ptr
from .hamiltonian import SpinHamiltonian

OHU_SPLIT = 256                             # samples per split of the O^H u partials (sr.cu)
OV_ROWS, FWD_SB, ELOC_SB, RED_SB = 64, 16, 32, 256


def _ceil(a, b):
    return (a + b - 1) // b


@dataclass
class NQSBatchStats:
    """Per-epoch history of every problem (rows = epochs, columns = problems)."""
    history: List[np.ndarray] = field(default_factory=list)
    history_std: List[np.ndarray] = field(default_factory=list)
    cg_iterations: List[np.ndarray] = field(default_factory=list)
    acceptance: List[np.ndarray] = field(default_factory=list)
    timings: List[float] = field(default_factory=list)

    def energies(self):
        return np.array(self.history)


class NQSBatch:
    def __init__(self, models: Sequence[SpinHamiltonian], *, alpha=2.0, dtype="float32", seeds=None,
                 s_numchains=256, s_numsamples=8, s_sweep_steps=None, s_therm_steps=1, s_mu=2.0, s_beta=1.0,
                 s_initstate=None, init_scale=0.01, recompute_every=0, device=None, autotune=True,
                 warps_per_block=None, blocks_per_sm=None):
        if not models:
            raise ValueError("NQSBatch needs at least one model")
        for m in models:
            if not isinstance(m, SpinHamiltonian):
                raise TypeError("NQSBatch takes TransverseFieldIsing / XXZ / J1J2Model instances")
        self.models = list(models)
        self.n_inst = len(self.models)
        self.device = torch.device("cuda") if device is None else torch.device(device)
        self.is_complex = str(dtype).lower() in ("complex64", "complex", "c64") or dtype in (np.complex64, torch.complex64)
        self.dtype = torch.complex64 if self.is_complex else torch.float32
        self.master_dtype = torch.complex128 if self.is_complex else torch.float64
        self.dtype_code = _lib.DTYPE_C64 if self.is_complex else _lib.DTYPE_F32
        seeds = list(range(self.n_inst)) if seeds is None else [int(s) for s in seeds]
        if len(seeds) != self.n_inst:
            raise ValueError("one seed per model")
        self.seeds = seeds
        self.mu, self.beta = float(s_mu), float(s_beta)
        self.recompute_every = int(recompute_every)
        init = "RND" if s_initstate is None else str(s_initstate).upper()
        if init not in ("RND", "RANDOM"):
            raise ValueError("the batched sampler starts from RND states (single-flip moves)")

        ns = np.array([m.ns for m in self.models], dtype=np.int64)
        nh = np.array([int(round(alpha * n)) for n in ns], dtype=np.int64)
        if ns.max() > 2048 or nh.max() > (512 if self.is_complex else 2048):
            raise ValueError("the batched sampler holds ns <= 2048 spins and nh <= 2048 (real) / 512 (complex) "
                             "hidden units per chain")
        chains = np.full(self.n_inst, int(s_numchains), dtype=np.int64)
        nsamp = np.full(self.n_inst, int(s_numsamples), dtype=np.int64)
        sweep = ns.copy() if s_sweep_steps is None else np.full(self.n_inst, int(s_sweep_steps), dtype=np.int64)
        therm = int(s_therm_steps) * sweep * ns
        nw = (ns + 31) // 32
        rows = chains * nsamp
        P = ns + nh + ns * nh
        lowered = [m.lower() for m in self.models]
        K = np.array([lw.n_moves for lw in lowered], dtype=np.int64)
        nzz = np.array([len(lw.zz_i) for lw in lowered], dtype=np.int64)
        nzf = np.array([len(lw.zf_site) for lw in lowered], dtype=np.int64)
        excl = lambda v: np.concatenate([[0], np.cumsum(v)[:-1]]).astype(np.int64)
        self.ns, self.nh, self.P, self.rows, self.chains = ns, nh, P, rows, chains
        self.sweep = sweep
        self.param_off = excl(P)
        self.sample_off = excl(rows)
        self.chain_off = excl(chains)
        self.n_params_total = int(P.sum())
        self.n_samples_total = int(rows.sum())
        self.n_chains_total = int(chains.sum())
        nsplit = _ceil(rows, OHU_SPLIT)
        self.sr_part_total = int((nsplit * P).sum())
        arr = (_lib.BatchInstance * self.n_inst)()
        offs = dict(param_off=excl(P), chain_off=excl(chains), chain_word_off=excl(chains * nw),
                    sample_off=excl(rows), sample_word_off=excl(rows * nw), tanh_off=excl(rows * nh),
                    flip_off=excl(ns * nh), move_table_off=excl(nh * K), move_off=excl(K), zz_off=excl(nzz),
                    zf_off=excl(nzf), eloc_part_off=excl(_ceil(K, 32) * rows), sr_part_off=excl(nsplit * P))
        for b in range(self.n_inst):
            d = arr[b]
            d.ns, d.nh, d.n_moves, d.n_zz, d.n_zfield = int(ns[b]), int(nh[b]), int(K[b]), int(nzz[b]), int(nzf[b])
            d.n_chains, d.num_samples, d.sweep_steps = int(chains[b]), int(nsamp[b]), int(sweep[b])
            d.therm_steps_total = int(therm[b])
            d.seed = seeds[b] & (2 ** 64 - 1)
            for k, v in offs.items():
                setattr(d, k, int(v[b]))
        self._host_inst = arr
        raw = np.frombuffer(bytes(arr), dtype=np.uint8)
        self.inst = torch.as_tensor(raw.copy(), device=self.device)

        # parameters: problem b is initialised exactly like RBM((ns_b,), nh_b, seed=seeds[b])
        master = []
        for b in range(self.n_inst):
            rng = np.random.default_rng(seeds[b])
            x = rng.normal(0.0, init_scale, size=int(P[b]))
            if self.is_complex:
                x = x + 1j * rng.normal(0.0, init_scale, size=int(P[b]))
            master.append(x)
        self.master = torch.as_tensor(np.concatenate(master), dtype=self.master_dtype, device=self.device)
        self.flat = self.master.to(self.dtype).contiguous()

        # Hamiltonians
        cat = lambda key, dt: torch.as_tensor(
            np.concatenate([np.asarray(getattr(lw, key)).reshape(-1) for lw in lowered] + [np.zeros(0)]).astype(dt),
            device=self.device)
        self.move_i, self.move_j = cat("move_i", np.int32), cat("move_j", np.int32)
        self.move_kind = cat("move_kind", np.int32)
        self.move_coef = cat("move_coef", np.float32)
        self.zf_site, self.zf_h = cat("zf_site", np.int32), cat("zf_h", np.float32)
        self.zz_i, self.zz_j, self.zz_J = cat("zz_i", np.int32), cat("zz_j", np.int32), cat("zz_J", np.float32)
        self.n_moves = K

        # chains and sampler state
        dev = self.device
        self.chain_bits = torch.empty((int((chains * nw).sum()),), dtype=torch.int32, device=dev)
        for b in range(self.n_inst):
            o, n = int(offs["chain_word_off"][b]), int(chains[b] * nw[b])
            call("qes_init_chains", _lib.INIT_RND, 0, C.c_uint64(seeds[b] & (2 ** 64 - 1)), 0, int(chains[b]),
                 int(ns[b]), ptr(self.chain_bits[o:o + n]), stream_ptr())
        self.chain_step = torch.zeros((self.n_chains_total,), dtype=torch.int64, device=dev)
        self.proposed = torch.zeros((self.n_chains_total,), dtype=torch.int32, device=dev)
        self.accepted = torch.zeros((self.n_chains_total,), dtype=torch.int32, device=dev)
        self.last_logpsi = torch.empty((self.n_chains_total,), dtype=self.dtype, device=dev)
        self.sample_bits = torch.empty((int((rows * nw).sum()),), dtype=torch.int32, device=dev)
        self.sample_logpsi = torch.empty((self.n_samples_total,), dtype=self.dtype, device=dev)
        self.tanh = torch.empty((int((rows * nh).sum()),), dtype=self.dtype, device=dev)
        self.eloc = torch.empty((self.n_samples_total,), dtype=torch.complex64, device=dev)
        self.flipC = torch.empty((int((ns * nh).sum()),), dtype=self.dtype, device=dev)
        self.flipS = torch.empty_like(self.flipC)
        nmt = max(int((nh * K).sum()), 1)
        self.Ct = torch.empty((nmt,), dtype=self.dtype, device=dev)
        self.St = torch.empty_like(self.Ct)
        self.A = torch.empty((max(int(K.sum()), 1),), dtype=self.dtype, device=dev)
        self.eloc_part = torch.empty((max(int((_ceil(K, 32) * rows).sum()), 1),), dtype=torch.complex64, device=dev)
        self.counter = torch.zeros((64,), dtype=torch.int32, device=dev)
        self.stats_out = torch.empty((self.n_inst, 4), dtype=torch.float64, device=dev)
        self.x = torch.empty((self.n_params_total,), dtype=self.master_dtype, device=dev)
        nb = C.c_size_t(0)
        call("qes_batch_sr_workspace_bytes", self.dtype_code, self.n_inst, self.n_params_total, self.n_samples_total,
             self.sr_part_total, C.byref(nb))
        self.sr_ws = torch.empty((int(nb.value),), dtype=torch.uint8, device=dev)
        self._thermalize = True
        self._tables_dirty = True

        # work lists, heaviest problems first
        order = np.argsort(-(ns * nh), kind="stable")
        samp_cost = (nsamp * sweep + therm) * nh
        sorder = np.argsort(-samp_cost, kind="stable")
        L = lambda items: torch.as_tensor(np.asarray(items, dtype=np.int32).reshape(-1, 4), device=dev)
        self.items_flip = L([(b, q, 0, 0) for b in order for q in range(_ceil(int(ns[b] * nh[b]), 256))])
        self.items_moves_tab = L([(b, q, 0, 0) for b in order for q in range(_ceil(int(nh[b] * K[b]), 256))]
                                 or [(0, 0, 0, 0)])
        self.n_items_moves_tab = int(sum(_ceil(int(nh[b] * K[b]), 256) for b in range(self.n_inst)))
        self.items_chains = L([(b, c, 0, 0) for b in sorder for c in range(int(chains[b]))])
        self.items_fwd = L([(b, q, 0, 0) for b in order for q in range(_ceil(int(rows[b]), FWD_SB))])
        eloc_items = [(b, kb, sb, 0) for b in order for kb in range(_ceil(int(K[b]), 32))
                      for sb in range(_ceil(int(rows[b]), ELOC_SB))]
        self.n_items_eloc = len(eloc_items)
        self.items_eloc = L(eloc_items or [(0, 0, 0, 0)])
        self.items_red = L([(b, q, 0, 0) for b in order for q in range(_ceil(int(rows[b]), RED_SB))])
        self.items_ov = L([(b, r0, min(OV_ROWS, int(rows[b]) - r0), 0) for b in order
                           for r0 in range(0, int(rows[b]), OV_ROWS)])
        self.items_ohu = L([(b, z, 0, 0) for b in order for z in range(int(nsplit[b]))])
        self.max_nh = int(nh.max())
        props = torch.cuda.get_device_properties(self.device)
        self.n_sm = props.multi_processor_count
        self.warps_per_block = warps_per_block
        self.blocks_per_sm = blocks_per_sm
        if self.warps_per_block is None or self.blocks_per_sm is None:
            if autotune:
                self.autotune_sampler()
            else:
                self.warps_per_block, self.blocks_per_sm = 4, 8

    # ------------------------------------------------------------------ parameters
    def params(self, b):
        """float64 / complex128 master parameters [a, b, W] of problem b (a view)."""
        o = int(self.param_off[b])
        return self.master[o:o + int(self.P[b])]

    def set_params(self, b, x):
        o = int(self.param_off[b])
        self.master[o:o + int(self.P[b])] = torch.as_tensor(x, dtype=self.master_dtype, device=self.device)
        self.flat = self.master.to(self.dtype).contiguous()
        self._tables_dirty = True

    def samples(self, b):
        """(sample_bits (rows, nw) int32, log psi (rows,)) of problem b from the last sampling call."""
        nw = (int(self.ns[b]) + 31) // 32
        wo = int(sum(int(self.rows[q]) * ((int(self.ns[q]) + 31) // 32) for q in range(b)))
        r, o = int(self.rows[b]), int(self.sample_off[b])
        return self.sample_bits[wo:wo + r * nw].view(r, nw), self.sample_logpsi[o:o + r]

    def local_energies(self, b):
        o = int(self.sample_off[b])
        return self.eloc[o:o + int(self.rows[b])]

    def tanh_theta(self, b):
        to = int(sum(int(self.rows[q] * self.nh[q]) for q in range(b)))
        r, m = int(self.rows[b]), int(self.nh[b])
        return self.tanh[to:to + r * m].view(r, m)

    def acceptance(self):
        p = self.proposed.to(torch.float64).clamp(min=1.0)
        acc = (self.accepted.to(torch.float64) / p).cpu().numpy()
        return np.array([acc[int(self.chain_off[b]):int(self.chain_off[b] + self.chains[b])].mean()
                         for b in range(self.n_inst)])

    # ------------------------------------------------------------------ phases
    def build_tables(self):
        call("qes_batch_move_tables", self.dtype_code, self.n_inst, ptr(self.inst), 0, int(self.items_flip.shape[0]),
             ptr(self.items_flip), ptr(self.flat), None, None, None, ptr(self.flipC), ptr(self.flipS), None,
             stream_ptr())
        if self.n_items_moves_tab:
            call("qes_batch_move_tables", self.dtype_code, self.n_inst, ptr(self.inst), 1, self.n_items_moves_tab,
                 ptr(self.items_moves_tab), ptr(self.flat), ptr(self.move_i), ptr(self.move_j), ptr(self.move_kind),
                 ptr(self.Ct), ptr(self.St), ptr(self.A), stream_ptr())
        self._tables_dirty = False

    def _run_sampler(self, warps, bps, thermalize, chain_bits=None, chain_step=None, proposed=None, accepted=None):
        call("qes_batch_sampler_run", self.dtype_code, self.n_inst, ptr(self.inst), self.max_nh,
             int(self.items_chains.shape[0]), ptr(self.items_chains), int(warps), int(bps * self.n_sm),
             1 if thermalize else 0, self.mu, self.beta, self.recompute_every, ptr(self.flat), ptr(self.flipC),
             ptr(self.flipS), ptr(self.chain_bits if chain_bits is None else chain_bits),
             ptr(self.chain_step if chain_step is None else chain_step),
             ptr(self.proposed if proposed is None else proposed), ptr(self.accepted if accepted is None else accepted),
             ptr(self.sample_bits), ptr(self.sample_logpsi), ptr(self.last_logpsi), ptr(self.counter), stream_ptr())

    def sample(self):
        if self._tables_dirty:
            self.build_tables()
        self._run_sampler(self.warps_per_block, self.blocks_per_sm, self._thermalize)
        self._thermalize = False

    def forward(self):
        call("qes_batch_rbm_forward", self.dtype_code, self.n_inst, ptr(self.inst), int(self.items_fwd.shape[0]),
             ptr(self.items_fwd), ptr(self.flat), ptr(self.sample_bits), ptr(self.tanh), None, stream_ptr())

    def local_energy(self):
        call("qes_batch_local_energy", self.dtype_code, self.n_inst, ptr(self.inst), self.n_items_eloc,
             ptr(self.items_eloc), int(self.items_red.shape[0]), ptr(self.items_red), ptr(self.sample_bits),
             ptr(self.tanh), ptr(self.move_i), ptr(self.move_j), ptr(self.move_kind), ptr(self.move_coef),
             ptr(self.Ct), ptr(self.St), ptr(self.A), ptr(self.zf_site), ptr(self.zf_h), ptr(self.zz_i),
             ptr(self.zz_j), ptr(self.zz_J), ptr(self.eloc_part), ptr(self.eloc), stream_ptr())

    def loss_stats(self):
        call("qes_batch_loss_stats", self.n_inst, ptr(self.inst), ptr(self.eloc), ptr(self.stats_out), stream_ptr())
        return self.stats_out

    def sr_solve(self, shift=1e-3, rtol=1e-8, atol=0.0, maxiter=1000, check_every=16, rhs_prefactor=-1.0):
        opts = _lib.SROptions(float(shift), float(rtol), float(atol), int(maxiter), int(check_every),
                              float(rhs_prefactor))
        res = (_lib.SRResult * self.n_inst)()
        call("qes_batch_sr_solve_cg", self.dtype_code, self.n_inst, ptr(self.inst), int(self.items_ov.shape[0]),
             ptr(self.items_ov), int(self.items_ohu.shape[0]), ptr(self.items_ohu), self.n_params_total,
             self.n_samples_total, self.sr_part_total, ptr(self.sample_bits), ptr(self.tanh), ptr(self.eloc),
             C.byref(opts), ptr(self.x), C.cast(res, C.c_void_p), ptr(self.sr_ws), int(self.sr_ws.numel()),
             stream_ptr(), allow=(_lib.QES_ERR_NOT_CONVERGED,))
        self.last_sr = res
        return self.x, res

    def update(self, lr):
        call("qes_param_update", self.dtype_code, self.n_params_total, float(lr), ptr(self.x), ptr(self.master),
             ptr(self.flat), stream_ptr())
        self._tables_dirty = True

    # ------------------------------------------------------------------ epochs
    def train_step(self, lr=1e-2, diag_shift=1e-3, sr_tol=1e-8, sr_maxiter=1000, check_every=16):
        """One VMC epoch of every problem; returns per-problem host statistics."""
        self.sample()
        self.forward()
        self.local_energy()
        st = self.loss_stats()
        _, res = self.sr_solve(shift=diag_shift, rtol=sr_tol, maxiter=sr_maxiter, check_every=check_every)
        self.update(lr)
        s = st.cpu().numpy()
        return {"mean": s[:, 0] + 1j * s[:, 1], "var": s[:, 2], "std": s[:, 3],
                "cg_iterations": np.array([r.iterations for r in res]),
                "cg_converged": np.array([bool(r.converged) for r in res])}

    def train(self, n_epochs=300, lr=1e-2, diag_shift=1e-3, sr_tol=1e-8, sr_maxiter=1000, callback=None):
        stats = NQSBatchStats()
        for ep in range(int(n_epochs)):
            t0 = time.perf_counter()
            info = self.train_step(lr=lr, diag_shift=diag_shift, sr_tol=sr_tol, sr_maxiter=sr_maxiter)
            stats.timings.append(time.perf_counter() - t0)
            stats.history.append(info["mean"])
            stats.history_std.append(info["std"])
            stats.cg_iterations.append(info["cg_iterations"])
            if callback is not None:
                callback(ep, info)
        return stats

    # ------------------------------------------------------------------ autotuning
    def _signature(self):
        name = torch.cuda.get_device_name(self.device)
        return (f"{name}|{'c64' if self.is_complex else 'f32'}|inst={self.n_inst}|chains={self.n_chains_total}"
                f"|maxnh={self.max_nh}|work={int(((self.rows // np.maximum(self.chains, 1)) * self.sweep * self.nh * self.chains).sum())}")

    def autotune_sampler(self, candidates=((1, 8), (2, 8), (4, 4), (4, 8), (4, 16), (8, 4), (8, 8), (16, 2)),
                         repeats=2, cache=None):
        """Pick (warps per block, blocks per SM) of the persistent sampler by timing each candidate.

        The timing runs advance scratch copies of the chains, so the trajectories do not depend on the
        choice (each chain's proposals are keyed by its own counter).  Results persist in a JSON cache
        (``$QES_B200_AUTOTUNE`` or ``~/.cache/pyqusolver_b200/autotune.json``) keyed by device and workload.
        """
        path = cache or os.environ.get("QES_B200_AUTOTUNE",
                                       os.path.join(os.path.expanduser("~"), ".cache", "pyqusolver_b200",
                                                    "autotune.json"))
        key = self._signature()
        table = {}
        try:
            with open(path) as f:
                table = json.load(f)
        except (OSError, ValueError):
            table = {}
        if key in table:
            self.warps_per_block, self.blocks_per_sm = table[key]
            return tuple(table[key])
        if self._tables_dirty:
            self.build_tables()
        cb, cs = self.chain_bits.clone(), self.chain_step.clone()
        pp, aa = self.proposed.clone(), self.accepted.clone()
        best, best_t = None, float("inf")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for (w, bps) in candidates:
            ts = []
            for _ in range(repeats + 1):
                ev0.record()
                try:
                    self._run_sampler(w, bps, False, cb, cs, pp, aa)
                except _lib.QESError as e:
                    if e.code != _lib.QES_ERR_ARG:
                        raise
                    ts = []
                    break                      # block size beyond the kernel's register budget
                ev1.record()
                torch.cuda.synchronize()
                ts.append(ev0.elapsed_time(ev1))
            if len(ts) < 2:
                continue
            t = min(ts[1:])
            if t < best_t:
                best, best_t = (w, bps), t
        self.warps_per_block, self.blocks_per_sm = best
        table[key] = list(best)
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(table, f, indent=1)
        except OSError:
            pass
        self.autotune_ms = best_t
        return best
