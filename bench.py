"""Benchmark of one RBM-VMC step (sample -> E_loc -> SR -> update) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config heis10x10] [--impl ours|reference]

Workload (default): Heisenberg XXX on the 10x10 periodic square lattice in
the Sz = 0 sector (XXZ with jxy = jz = -1 in QES's literal sign convention,
i.e. the antiferromagnet), complex64 RBM with alpha = 2 (M = 200, P = 20,300),
init N(0, 0.01), 4096 chains x 4 samples = 16,384 samples per step, exchange
moves, sweep_steps = N = 100 proposals between samples, SR with diagonal
shift 1e-3 solved by CG (rtol 1e-8, maxiter 1000), Euler/SGD lr 0.01.
One step = one VMC epoch: persistent sampler kernel, theta/tanh forward,
fused local energy, float64 statistics, structured SR CG, float64 update.
Synthetic data: random-init parameters and random Sz = 0 starting chains.

value = samples/s of the whole job (N GPUs x 16,384 samples per step / time);
vmc_steps_per_s is reported beside it.  With --gpus N > 1 every rank runs its
own independent VMC (replicas, weak scaling, no collective on the data path).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "VMC steps/s & samples/s: mixed+batched vs plain FP32 on B200 at equal ΔE vs ED"

CONFIGS = {
    # name: (dim, lx, ly, model, coupling kwargs, alpha, dtype, chains, samples, rule, sweep, shift, lr, cg rtol)
    "heis10x10": dict(name="heis10x10", dim=2, lx=10, ly=10, model="xxz", kw=dict(jxy=-1.0, jz=-1.0), alpha=2, dtype="complex64",
                      chains=4096, samples=4, rule="EXCHANGE", sweep=100, shift=1e-3, lr=0.01, rtol=1e-8,
                      maxiter=1000, init="RND_FIXED"),
    "tfim16": dict(name="tfim16", dim=1, lx=16, ly=1, model="tfim", kw=dict(j=1.0, hx=1.0, hz=0.0), alpha=1, dtype="float32",
                   chains=16, samples=64, rule="LOCAL", sweep=16, shift=1e-3, lr=0.01, rtol=1e-8, maxiter=1000,
                   init="RND"),
    "j1j2_6x6": dict(name="j1j2_6x6", dim=2, lx=6, ly=6, model="j1j2", kw=dict(J1=-1.0, J2=-0.5), alpha=4, dtype="complex64",
                     chains=2048, samples=4, rule="EXCHANGE", sweep=36, shift=1e-3, lr=0.01, rtol=1e-8,
                     maxiter=1000, init="RND_FIXED"),
    # 64 independent TFIM chains, L ~ U{12..64}, hx ~ U[0.5, 1.5], J = 1, PBC; real RBM alpha = 2 each;
    # 256 chains x 8 samples per problem; single flips; one launch per phase over all problems
    "tfim_batch64": dict(name="tfim_batch64", batch=True, n_inst=64, L_lo=12, L_hi=64, hx_lo=0.5, hx_hi=1.5,
                         draw_seed=2024, alpha=2, dtype="float32", chains=256, samples=8, rule="LOCAL",
                         shift=1e-3, lr=0.02, rtol=1e-8, maxiter=1000, model="tfim", kw=dict(j=1.0)),
    "tfim20x20": dict(name="tfim20x20", dim=2, lx=20, ly=20, model="tfim", kw=dict(j=1.0, hx=3.04, hz=0.0), alpha=4, dtype="float32",
                      chains=4096, samples=4, rule="LOCAL", sweep=400, shift=1e-4, lr=0.01, rtol=1e-8, maxiter=1000,
                      init="RND"),
}


def env_rank():
    from pyqusolver_b200.replicas import rank_env
    return rank_env()


# ---------------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------------------- our arm
def build_nqs(cfg, seed, sampler_seed=None):
    import pyqusolver_b200 as qb
    L = qb.SquareLattice(cfg["dim"], cfg["lx"], cfg["ly"], bc="pbc")
    if cfg["model"] == "xxz":
        model = qb.XXZ(L, **cfg["kw"])
    elif cfg["model"] == "j1j2":
        model = qb.J1J2Model(L, **cfg["kw"])
    else:
        model = qb.TransverseFieldIsing(L, **cfg["kw"])
    nqs = qb.NQS("rbm", model, alpha=cfg["alpha"], dtype=cfg["dtype"], seed=seed, s_upd_fun=cfg["rule"],
                 s_initstate=cfg["init"], nparticles=L.ns // 2, s_numchains=cfg["chains"],
                 s_numsamples=cfg["samples"], s_therm_steps=1, s_sweep_steps=cfg["sweep"],
                 s_seed=seed if sampler_seed is None else sampler_seed, init_scale=0.01)
    from pyqusolver_b200.tdvp import TDVP
    # CG chunks of 16 iterations: the device loop tests convergence once per chunk, and the launches of
    # a chunk after the converging iteration return at once (heis10x10 solve: 7.07 ms with chunks of
    # 32, 7.01 ms with 16, 7.03 ms with 8)
    tdvp = TDVP(rhs_prefactor=-1.0, sr_diag_shift=cfg["shift"], sr_tol=cfg["rtol"], sr_maxiter=cfg["maxiter"], check_every=16)
    return nqs, tdvp


def timed_step(nqs, tdvp, cfg, ev):
    """One VMC step with CUDA events between the phases (all on the current stream)."""
    import torch
    from pyqusolver_b200 import device as dv
    net = nqs.net
    ev[0].record()
    bits, _ = nqs.sampler.sample_bits()
    ev[1].record()
    _, tn, _ = dv.rbm_forward_step(net.flat, net.ns, net.nh, bits, theta=False, tanh=True, logpsi=False)
    ev[2].record()
    eloc = nqs.local_energy_bits(bits, tn)
    ev[3].record()
    st = dv.loss_stats(eloc)
    ev[4].record()
    x = tdvp.solve(net, bits, tn, eloc)
    ev[5].record()
    dv.param_update(net.flat, net.master, x, cfg["lr"])
    net.bump()
    ev[6].record()
    return st, tdvp.last_info


PHASES = ["sample", "forward", "local_energy", "stats", "sr_solve", "update"]


def timed_loop(nqs, tdvp, cfg, steps, flush, profile=False):
    import torch
    from pyqusolver_b200 import _lib
    mk = lambda: [torch.cuda.Event(enable_timing=True) for _ in range(7)]
    if profile:
        _lib.profile_read(reset=True)
        _lib.profile_enable(True)
    _lib.launch_count(reset=True)
    step_ms, phase_ms, cg_iters = [], {p: [] for p in PHASES}, []
    for _ in range(steps):
        flush.fill_(1.0)
        ev = mk()
        timed_step(nqs, tdvp, cfg, ev)
        torch.cuda.synchronize()
        step_ms.append(ev[0].elapsed_time(ev[6]))
        for k, p in enumerate(PHASES):
            phase_ms[p].append(ev[k].elapsed_time(ev[k + 1]))
        cg_iters.append(tdvp.last_info.get("iterations", 0))
    launches = _lib.launch_count(reset=True)
    prof = None
    if profile:
        prof = _lib.profile_read(reset=True)
        _lib.profile_enable(False)
    return step_ms, phase_ms, cg_iters, launches, prof


def accuracy_check(epochs, name="tfim16"):
    """Equal-Delta-E evidence: train the ED-checkable workload in both forms from the same start and
    compare the final energies with the exact ground energy (GPU Lanczos, ``qes_ed_lanczos``)."""
    import torch
    from pyqusolver_b200 import _lib
    cfg = CONFIGS[name]
    out = {"workload": name, "epochs": int(epochs), "lr": cfg["lr"], "shift": cfg["shift"],
           "exact_method": "GPU Lanczos over the full 2^N basis (qes_ed_lanczos)"}
    e_exact = None
    for form, impl in (("plain_fp32", _lib.SR_IMPL_CUDA_CORES), ("mixed", _lib.SR_IMPL_AUTO)):
        _lib.set_sr_impl(impl)
        nqs, tdvp = build_nqs(cfg, seed=1)
        if e_exact is None:
            e_exact = float(nqs.model.diagonalize(method="lanczos")[0])
        hist = []
        t0 = time.perf_counter()
        for _ in range(int(epochs)):
            info = nqs.train_step(lr=cfg["lr"], tdvp=tdvp)
            hist.append(info["mean"].real)
        torch.cuda.synchronize()
        tail = np.array(hist[-30:])
        e = float(tail.mean())
        out[form] = {"energy": e, "stderr": float(tail.std() / np.sqrt(len(tail))),
                     "rel_err": abs(e - e_exact) / abs(e_exact), "seconds": time.perf_counter() - t0}
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    out["e_exact"] = e_exact
    out["equal_dE_1e-4"] = bool(out["mixed"]["rel_err"] <= 1e-4 and out["plain_fp32"]["rel_err"] <= 1e-4)
    return out


def ed_energy_check(epochs, name="j1j2_6x6"):
    """Energy against ED on the 6x6 J1-J2 workload: train it (mixed form) and compare the mean
    energy of the last 50 epochs with the exact ground energy of the committed fixture
    ``tests/golden/ed_j1j2_6x6.json`` (GPU Lanczos in the k = 0, even-flip sector,
    ``qes_ed_lanczos_symm``; regenerate with ``python tests/golden/make_ed_j1j2_6x6.py``)."""
    import torch
    from pyqusolver_b200 import _lib
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "ed_j1j2_6x6.json")) as f:
        e_exact = float(json.load(f)["e0_j2_0.5"])
    cfg = CONFIGS[name]
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    nqs, tdvp = build_nqs(cfg, seed=1)
    hist = []
    t0 = time.perf_counter()
    for _ in range(int(epochs)):
        info = nqs.train_step(lr=cfg["lr"], tdvp=tdvp)
        hist.append(info["mean"].real)
    torch.cuda.synchronize()
    tail = np.array(hist[-50:])
    e = float(tail.mean())
    return {"workload": name, "epochs": int(epochs), "lr": cfg["lr"], "shift": cfg["shift"],
            "exact_method": "GPU Lanczos, 6x6 k=0 even-flip sector (qes_ed_lanczos_symm), committed fixture",
            "e_exact": e_exact, "energy": e, "stderr": float(tail.std() / np.sqrt(len(tail))),
            "rel_err": abs(e - e_exact) / abs(e_exact), "energy_by_100_epochs": [float(np.mean(hist[i:i + 100]))
                                                                                 for i in range(0, len(hist), 100)],
            "seconds": time.perf_counter() - t0}


def matched_energy_check(epochs, every, name="heis10x10"):
    """Equal-Delta-E on the benchmarked workload, where no ED exists.  Independent VMC runs cannot
    resolve 1e-4 here: the Markov chains of two runs decorrelate within a few epochs in any
    precision, and the final energies of two float64 runs that differ only in their sampler seeds
    differ by ~1e-2 after a few hundred epochs.  So the forms are compared on the same batches: the
    mixed form drives the training run, and every `every` epochs the batch it has just drawn is also
    solved by the float64 form (SR contractions in float64 on CUDA cores, the reference's SR
    precision) and by the plain-FP32 form.  Per checked epoch: the first-order energy change of the
    update, dE = 2 lr Re(F^H x) (the SR step minimises it), for each form against the float64 one,
    the error of x in the (S + shift)-norm of the float64 operator, and each solve's true residual."""
    import torch
    from pyqusolver_b200 import _lib, device as dv
    from pyqusolver_b200.tdvp import TDVP
    cfg = CONFIGS[name]
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    nqs, tdvp = build_nqs(cfg, seed=1)
    net = nqs.net
    forms = {"fp64": _lib.SR_IMPL_FP64, "mixed": _lib.SR_IMPL_AUTO, "plain_fp32": _lib.SR_IMPL_CUDA_CORES}
    rows, energies = [], []
    t0 = time.perf_counter()
    for ep in range(int(epochs)):
        info = nqs.train_step(lr=cfg["lr"], tdvp=tdvp)
        energies.append(info["mean"].real)
        if (ep + 1) % int(every):
            continue
        # the next batch, solved by every form (then used by the mixed form's training step)
        bits, _ = nqs.sampler.sample_bits()
        _, tn, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, tanh=True, logpsi=False)
        eloc = nqs.local_energy_bits(bits, tn)
        xs, res = {}, {}
        for form, impl in forms.items():
            _lib.set_sr_impl(impl)
            x, inf = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=cfg["shift"], rtol=cfg["rtol"],
                                    maxiter=4 * cfg["maxiter"], check_every=32)
            xs[form], res[form] = x, inf
        _lib.set_sr_impl(_lib.SR_IMPL_FP64)
        F = dv.sr_force(net.flat, net.ns, net.nh, bits, tn, eloc)
        Ax = lambda v: dv.sr_matvec(net.flat, net.ns, net.nh, bits, tn, v, shift=cfg["shift"])
        _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
        x64 = xs["fp64"]
        dE64 = 2 * cfg["lr"] * torch.vdot(F, x64).real.item()
        nA64 = torch.vdot(x64, Ax(x64)).real.item()
        row = {"epoch": ep + 1, "dE_fp64": dE64, "cg_iterations": {f: res[f]["iterations"] for f in forms},
               "true_residual": {f: res[f]["true_residual"] for f in forms}}
        for form in ("mixed", "plain_fp32"):
            dE = 2 * cfg["lr"] * torch.vdot(F, xs[form]).real.item()
            e = xs[form] - x64
            row[form] = {"dE_rel_diff": abs(dE - dE64) / abs(dE64),
                         "x_err_A_norm": float(np.sqrt(max(torch.vdot(e, Ax(e)).real.item(), 0.0) / nA64))}
        rows.append(row)
        # the mixed form's step on this batch (the same update the training run would make)
        x = tdvp.solve(net, bits, tn, eloc)
        dv.param_update(net.flat, net.master, x, cfg["lr"])
        net.bump()
    torch.cuda.synchronize()
    E = np.array(energies)
    out = {"workload": name, "epochs": int(epochs), "checked_every": int(every), "checked_epochs": len(rows),
           "lr": cfg["lr"], "shift": cfg["shift"], "driver_form": "mixed", "seconds": time.perf_counter() - t0,
           "reference": "float64 form (impl 3): float64 SR contractions of the float32 T",
           "energy_first": float(E[0]), "energy_last10_mean": float(E[-10:].mean())}
    for form in ("mixed", "plain_fp32"):
        d = np.array([r[form]["dE_rel_diff"] for r in rows])
        a = np.array([r[form]["x_err_A_norm"] for r in rows])
        out[form] = {"dE_rel_diff_max": float(d.max()), "dE_rel_diff_median": float(np.median(d)),
                     "x_err_A_norm_max": float(a.max()), "x_err_A_norm_median": float(np.median(a)),
                     "true_residual_max": float(max(r["true_residual"][form] for r in rows))}
    out["fp64_true_residual_max"] = float(max(r["true_residual"]["fp64"] for r in rows))
    out["equal_dE_1e-4"] = bool(out["mixed"]["dE_rel_diff_max"] <= 1e-4 and out["plain_fp32"]["dE_rel_diff_max"] <= 1e-4)
    out["per_epoch"] = rows
    return out


def build_batch(cfg, seed):
    import pyqusolver_b200 as qb
    from pyqusolver_b200.batch import NQSBatch
    rng = np.random.default_rng(cfg["draw_seed"])
    Ls = rng.integers(cfg["L_lo"], cfg["L_hi"] + 1, size=cfg["n_inst"])
    hx = rng.uniform(cfg["hx_lo"], cfg["hx_hi"], size=cfg["n_inst"])
    models = [qb.TransverseFieldIsing(qb.SquareLattice(1, int(L), 1, bc="pbc"), j=1.0, hx=float(h), hz=0.0)
              for L, h in zip(Ls, hx)]
    B = NQSBatch(models, alpha=cfg["alpha"], dtype=cfg["dtype"], seeds=[seed * 1000 + b for b in range(len(models))],
                 s_numchains=cfg["chains"], s_numsamples=cfg["samples"], autotune=True)
    return B, Ls, hx


BATCH_PHASES = ["sample", "forward", "local_energy", "stats", "sr_solve", "update"]


def run_batch(args, cfg, rank, world, local_rank):
    """Batched uneven problems (one launch per phase over all problems); one form (float32 CUDA cores)."""
    import torch
    from pyqusolver_b200 import _lib
    from pyqusolver_b200 import replicas
    torch.cuda.set_device(local_rank)
    dist = replicas.init_group(world)
    B, Ls, hx = build_batch(cfg, seed=replicas.replica_seed(1, rank))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    kw = dict(shift=cfg["shift"], rtol=cfg["rtol"], maxiter=cfg["maxiter"], check_every=32)

    def step(ev):
        ev[0].record(); B.sample()
        ev[1].record(); B.forward()
        ev[2].record(); B.local_energy()
        ev[3].record(); st = B.loss_stats()
        ev[4].record(); _, res = B.sr_solve(**kw)
        ev[5].record(); B.update(cfg["lr"])
        ev[6].record()
        return st, res

    mk = lambda: [torch.cuda.Event(enable_timing=True) for _ in range(7)]
    for _ in range(args.warmup):
        step(mk())
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    _lib.launch_count(reset=True)
    step_ms, phase_ms, cg = [], {p: [] for p in BATCH_PHASES}, []
    for _ in range(args.steps):
        flush.fill_(1.0)
        ev = mk()
        st, res = step(ev)
        torch.cuda.synchronize()
        step_ms.append(ev[0].elapsed_time(ev[6]))
        for k, p in enumerate(BATCH_PHASES):
            phase_ms[p].append(ev[k].elapsed_time(ev[k + 1]))
        cg.append(max(r.iterations for r in res))
    launches = _lib.launch_count(reset=True)
    clk = clocks.stop()
    # per-kernel CUDA-event timing for the roofline, in separate steps
    _lib.profile_read(reset=True)
    _lib.profile_enable(True)
    prof_total = 0.0
    for _ in range(min(args.steps, 3)):
        flush.fill_(1.0)
        ev = mk()
        step(ev)
        torch.cuda.synchronize()
        prof_total += ev[0].elapsed_time(ev[6])
    prof = _lib.profile_read(reset=True)
    _lib.profile_enable(False)
    total = replicas.max_over_ranks(float(np.sum(step_ms)), dist)
    n_step = B.n_samples_total
    value = replicas.job_throughput(n_step, args.steps, total, world)
    ms = total / args.steps

    # end to end: the same training run once more through the public API (a fresh batch built like
    # the timed one), host-driven: parameters in from pinned host memory, statistics and parameters
    # back every step, the downloaded parameters uploaded by the next step
    smp_shape = (B.warps_per_block, B.blocks_per_sm)
    del B
    B, _, _ = build_batch(cfg, seed=1 + rank)
    host_in = torch.empty_like(B.master, device="cpu").pin_memory()
    host_in.copy_(B.master.cpu())
    host_out = torch.empty_like(host_in).pin_memory()
    times = []
    for k in range(args.warmup + args.steps):                 # warm-up steps untimed, as above
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        B.master.copy_(host_in, non_blocking=True)
        B.flat.copy_(B.master)
        B._tables_dirty = True
        B.train_step(lr=cfg["lr"], diag_shift=cfg["shift"], sr_tol=cfg["rtol"], sr_maxiter=cfg["maxiter"])
        host_out.copy_(B.master, non_blocking=True)
        s1.record()
        torch.cuda.synchronize()
        if k >= args.warmup:
            times.append(s0.elapsed_time(s1))
        host_in, host_out = host_out, host_in
    e2e_total = float(np.sum(times))
    nb = host_in.numel() * host_in.element_size()
    e2e = {"value": world * n_step * args.steps / (e2e_total / 1e3), "unit": "samples/s",
           "h2d_bytes_per_step": int(nb), "d2h_bytes_per_step": int(nb + 32 * B.n_inst),
           "ms_per_step": e2e_total / args.steps}

    # roofline: dominant profiled kernel class (batched ov / ohu / CG update) or phase
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    rows, ns, nh, P = B.rows, B.ns, B.nh, B.P
    nw = (ns + 31) // 32
    # algorithmic bytes (operands once, outputs once; no split partials), as kernel_bytes()
    algo = {"ov": int((rows * nh * 4 + rows * nw * 4 + P * 8 + rows * 8).sum()),
            "ohu": int((rows * nh * 4 + rows * nw * 4 + rows * 8 + P * 8).sum()),
            "reduce": int((5 * P * 8).sum())}
    names = {"ov": "batch_ov_tile_kernel", "ohu": "batch_ohu_tile_kernel", "reduce": "batch_cg_update_kernel"}
    cands = {k: v for k, v in prof.items() if v[1]}
    dom = max(cands, key=lambda k: cands[k][0])
    avg_s = cands[dom][0] / cands[dom][1] / 1e3
    ach = algo[dom] / avg_s / 1e9
    roof = {"kernel": names[dom], "launches_timed": cands[dom][1], "avg_launch_us": avg_s * 1e6,
            "share_of_timed_region": cands[dom][0] / prof_total, "bound": "hbm", "achieved": ach, "peak": hbm,
            "unit": "GB/s", "frac": ach / hbm, "algorithmic_bytes_per_launch": algo[dom],
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "traffic": json.load(open(os.path.join(ROOT, "profiles", "dram_traffic_per_launch.json"))).get(
                cfg["name"], {}).get(dom) if os.path.exists(os.path.join(ROOT, "profiles",
                                                                          "dram_traffic_per_launch.json")) else None}
    line = {
        "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "vmc_steps_per_s": 1e3 / ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (random-init RBMs, random chains)",
        "config": {"workload": args.config, "problems": int(B.n_inst), "L_range": [int(Ls.min()), int(Ls.max())],
                   "hx_range": [float(hx.min()), float(hx.max())], "alpha": cfg["alpha"],
                   "chains_per_problem": cfg["chains"], "samples_per_chain": cfg["samples"],
                   "samples_per_step": int(n_step), "n_params_total": int(B.n_params_total),
                   "sampler_warps_per_block": smp_shape[0], "sampler_blocks_per_sm": smp_shape[1],
                   "sr": f"per-problem structured CG fp64 in lockstep, shift {cfg['shift']}, rtol {cfg['rtol']}",
                   "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "phase_ms": {p: float(np.mean(v)) for p, v in phase_ms.items()},
        "cg_iterations_max_mean": float(np.mean(cg)),
        "gpu_launches": int(launches), "clocks": clk, "e2e": e2e, "roofline": roof,
    }
    if rank == 0 and args.accuracy_epochs > 0:
        line["accuracy"] = batch_accuracy(B, cfg, args.accuracy_epochs, Ls)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, budget_s=args.cpu_budget)
    replicas.finish(dist)
    if rank == 0:
        print(json.dumps(line))


def batch_accuracy(B, cfg, epochs, Ls):
    """Train every problem for `epochs` more epochs; energy error per problem against the GPU Lanczos
    ground energy for L <= 20."""
    hist = []
    for _ in range(int(epochs)):
        info = B.train_step(lr=cfg["lr"], diag_shift=cfg["shift"], sr_tol=cfg["rtol"], sr_maxiter=cfg["maxiter"])
        hist.append(info["mean"].real)
    tail = np.array(hist[-20:]).mean(axis=0)
    rows = []
    for b, m in enumerate(B.models):
        if m.ns <= 20:
            e0 = float(m.diagonalize(method="lanczos")[0])
            rows.append({"problem": b, "L": int(m.ns), "e_exact": e0, "energy": float(tail[b]),
                         "rel_err": abs(float(tail[b]) - e0) / abs(e0)})
    return {"epochs": int(epochs), "checked_problems": len(rows),
            "max_rel_err": max((r["rel_err"] for r in rows), default=None), "problems": rows}


def run_ours(args, cfg, rank, world, local_rank):
    import torch
    from pyqusolver_b200 import _lib
    from pyqusolver_b200 import replicas
    torch.cuda.set_device(local_rank)
    dist = replicas.init_group(world)
    ns_per_step = cfg["chains"] * cfg["samples"]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist)

    forms = {}
    tuned = None
    # plain FP32 form: every SR contraction on CUDA cores in float32 (float64 CG vectors)
    # mixed form: SR contractions on tcgen05 tensor cores (BF16 hi/lo split, FP32 accumulate)
    wanted = [f.strip() for f in args.forms.split(",") if f.strip()]
    for form, impl in (("plain_fp32", _lib.SR_IMPL_CUDA_CORES), ("mixed", _lib.SR_IMPL_AUTO)):
        if form not in wanted:
            continue
        _lib.set_sr_impl(impl)
        nqs, tdvp = build_nqs(cfg, seed=replicas.replica_seed(1234, rank))
        for _ in range(args.warmup):                        # the first call thermalises the chains
            timed_step(nqs, tdvp, cfg, [torch.cuda.Event(enable_timing=True) for _ in range(7)])
        torch.cuda.synchronize()
        if form == "mixed" and args.autotune:
            # tensor-core SR tiling picked by timing the candidates on the current batch (autotune.py)
            from pyqusolver_b200.autotune import tune_sr_tiling
            from pyqusolver_b200 import device as dv
            net = nqs.net
            bits, _ = nqs.sampler.sample_bits()
            _, tn, _ = dv.rbm_forward_step(net.flat, net.ns, net.nh, bits, tanh=True, logpsi=False)
            tuned = tune_sr_tiling(net, bits, tn)
            for _ in range(2):
                timed_step(nqs, tdvp, cfg, [torch.cuda.Event(enable_timing=True) for _ in range(7)])
            torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        clocks = ClockSampler(local_rank) if form == "mixed" else None
        if clocks:
            clocks.start()
        step_ms, phase_ms, cg_iters, launches, _ = timed_loop(nqs, tdvp, cfg, args.steps, flush, profile=False)
        clk = clocks.stop() if clocks else None
        total_ms = max_over_ranks(float(np.sum(step_ms)))
        prof = prof_phases = prof_iters = None
        if form == "mixed":
            # per-kernel CUDA-event timing (roofline) in separate steps: the event pairs and the graph-less CG
            # they need would otherwise slow the timed steps
            ce = tdvp.check_every
            tdvp.check_every = 1          # no launch after convergence: every bracketed launch did work
            _, prof_phases, prof_iters, _, prof = timed_loop(nqs, tdvp, cfg, min(args.steps, 5), flush, profile=True)
            tdvp.check_every = ce
        forms[form] = {"nqs": nqs, "tdvp": tdvp, "total_ms": total_ms, "phase_ms": phase_ms, "cg_iters": cg_iters,
                       "launches": launches, "prof": prof, "prof_phase_ms": prof_phases, "prof_cg_iters": prof_iters,
                       "clocks": clk, "energy": float(nqs_energy(tdvp.last_info))}
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    mixed = forms["mixed"]
    plain = forms.get("plain_fp32")
    value = replicas.job_throughput(ns_per_step, args.steps, mixed["total_ms"], world)
    ms_step = mixed["total_ms"] / args.steps
    nqs, tdvp = mixed["nqs"], mixed["tdvp"]

    # --- end to end through the public API with host buffers (params in, stats + params out)
    e2e = run_e2e(cfg, args, dist, world, seed=replicas.replica_seed(1234, rank))

    # --- roofline of the dominant kernel (measured live over the timed steps)
    roof = roofline(cfg, nqs, mixed)

    def form_summary(f):
        ms = f["total_ms"] / args.steps
        return {"ms_per_step": ms, "vmc_steps_per_s": 1e3 / ms,
                "samples_per_s": world * ns_per_step * 1e3 / ms,
                "phase_ms": {p: float(np.mean(v)) for p, v in f["phase_ms"].items()},
                "cg_iterations_mean": float(np.mean(f["cg_iters"])), "energy_mean_last": f["energy"]}

    line = {
        "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "vmc_steps_per_s": 1e3 / ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64",
        "data": "synthetic (random-init RBM, random Sz=0 chains)",
        "config": {"workload": args.config, "lattice": f"{cfg['lx']}x{cfg['ly']} pbc", "model": cfg["model"],
                   "couplings": cfg["kw"], "alpha": cfg["alpha"], "param_dtype": cfg["dtype"],
                   "n_params": nqs.net.n_params, "chains": cfg["chains"], "samples_per_chain": cfg["samples"],
                   "samples_per_step": ns_per_step, "update": cfg["rule"], "sweep_steps": cfg["sweep"],
                   "sr": f"structured CG fp64, shift {cfg['shift']}, rtol {cfg['rtol']}, maxiter {cfg['maxiter']}",
                   "lr": cfg["lr"], "l2": "flushed (256 MB write) between timed steps",
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
        "phase_ms": {p: float(np.mean(v)) for p, v in mixed["phase_ms"].items()},
        "cg_iterations_mean": float(np.mean(mixed["cg_iters"])),
        "energy_mean_last": mixed["energy"],
        "forms": ({"mixed": form_summary(mixed), "plain_fp32": form_summary(plain),
                   "mixed_over_plain_steps_per_s": plain["total_ms"] / mixed["total_ms"]}
                  if plain else {"mixed": form_summary(mixed)}),
        "gpu_launches": int(mixed["launches"]),
        "clocks": mixed["clocks"],
        "e2e": e2e,
        "roofline": roof,
        "issue_rooflines": issue_rooflines(cfg, nqs, mixed, mixed["clocks"]),
        "sr_tiling": ({"choice (mode, nc, ctas, pairs, fused_sv, ov_split, ovz)": tuned["choice"], "cg_iteration_ms": tuned["ms"],
                       "candidates_ms": tuned["timings"], "cached": tuned["cached"]} if tuned else "automatic"),
    }
    if tuned:
        # the tuned tiling is process-wide: the other workloads below run the automatic one
        from pyqusolver_b200.autotune import apply_tiling
        apply_tiling(0, 0, 0, 0, 0, 0)
    if rank == 0 and args.accuracy_epochs > 0:
        line["accuracy"] = accuracy_check(args.accuracy_epochs)
    if rank == 0 and world == 1 and args.ed_epochs > 0:
        line["accuracy_ed_j1j2_6x6"] = ed_energy_check(args.ed_epochs)
    if rank == 0 and args.matched_epochs > 0 and args.config == "heis10x10":
        line["accuracy_matched_fp64"] = matched_energy_check(args.matched_epochs, args.matched_every)
    if rank == 0 and world == 1 and args.matched_other_epochs > 0:
        # the same common-batch float64 comparison on the other single-problem workloads (C1, C3, C5)
        mo = {}
        for name in [n.strip() for n in args.matched_configs.split(",") if n.strip()]:
            if name == args.config or name not in CONFIGS or CONFIGS[name].get("batch"):
                continue
            r = matched_energy_check(args.matched_other_epochs, max(1, args.matched_other_epochs // 5), name=name)
            r.pop("per_epoch", None)
            mo[name] = r
        line["accuracy_matched_fp64_other"] = mo
    if rank == 0 and world == 1 and not args.no_other_configs:
        oc = {}
        for name in ("tfim16", "j1j2_6x6", "tfim20x20"):
            if name != args.config:
                oc[name] = config_summary(name, args.other_steps, 3, flush)
        oc["tfim_batch64"] = batch_summary(args.other_steps, 3, flush)
        line["other_configs"] = oc
    if rank == 0 and world == 1 and not args.no_dense:
        line["dense_sr"] = dense_summary(flush, names=[n.strip() for n in args.dense_configs.split(",") if n.strip()])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, budget_s=args.cpu_budget)
    replicas.finish(dist)
    if rank == 0:
        print(json.dumps(line))


def config_summary(name, steps, warmup, flush):
    """Both forms of another single-problem workload (fewer steps than the headline), with the live
    roofline of its dominant kernel from separately profiled steps."""
    import torch
    from pyqusolver_b200 import _lib
    cfg = CONFIGS[name]
    forms = {}
    for form, impl in (("plain_fp32", _lib.SR_IMPL_CUDA_CORES), ("mixed", _lib.SR_IMPL_AUTO)):
        _lib.set_sr_impl(impl)
        nqs, tdvp = build_nqs(cfg, seed=1234)
        for _ in range(warmup):
            timed_step(nqs, tdvp, cfg, [torch.cuda.Event(enable_timing=True) for _ in range(7)])
        torch.cuda.synchronize()
        step_ms, phase_ms, cg_iters, launches, _ = timed_loop(nqs, tdvp, cfg, steps, flush, profile=False)
        f = {"nqs": nqs, "total_ms": float(np.sum(step_ms)), "phase_ms": phase_ms, "cg_iters": cg_iters,
             "launches": launches, "prof": None}
        if form == "mixed":
            ce = tdvp.check_every
            tdvp.check_every = 1
            _, f["prof_phase_ms"], f["prof_cg_iters"], _, f["prof"] = timed_loop(nqs, tdvp, cfg, min(steps, 3), flush,
                                                                                profile=True)
            tdvp.check_every = ce
        forms[form] = f
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    n = cfg["chains"] * cfg["samples"]
    out = {"workload": name, "steps": steps, "warmup": warmup, "samples_per_step": n,
           "n_params": forms["mixed"]["nqs"].net.n_params}
    for form, f in forms.items():
        ms = f["total_ms"] / steps
        out[form] = {"ms_per_step": ms, "vmc_steps_per_s": 1e3 / ms, "samples_per_s": n * 1e3 / ms,
                     "phase_ms": {p: float(np.mean(v)) for p, v in f["phase_ms"].items()},
                     "cg_iterations_mean": float(np.mean(f["cg_iters"])), "gpu_launches": int(f["launches"])}
    out["mixed_over_plain_steps_per_s"] = forms["plain_fp32"]["total_ms"] / forms["mixed"]["total_ms"]
    out["roofline"] = roofline(cfg, forms["mixed"]["nqs"], forms["mixed"])
    out["issue_rooflines"] = issue_rooflines(cfg, forms["mixed"]["nqs"], forms["mixed"], None)
    return out


def dense_summary(flush, names=("tfim16", "j1j2_6x6", "heis10x10"), steps=3):
    """The formed-S path (TDVP sr_form_matrix=True): tensor-core Gram + float64 Cholesky.  Per workload,
    after a few matrix-free warm-up epochs: one profiled dense solve (Gram and Cholesky times from CUDA
    events on the launch stream, Gram TFLOP/s against the measured sustained BF16 peak) and, where a
    step takes under a second, the VMC steps/s of the dense form next to the matrix-free one."""
    import torch
    from pyqusolver_b200 import _lib, device as dv
    from pyqusolver_b200.tdvp import TDVP
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("bf16_tflops_sustained", 1400.0)
    out = {}
    _lib.set_sr_impl(_lib.SR_IMPL_AUTO)
    for name in names:
        cfg = CONFIGS[name]
        nqs, tdvp = build_nqs(cfg, seed=1234)
        for _ in range(3):
            nqs.train_step(lr=cfg["lr"], tdvp=tdvp)
        net = nqs.net
        bits, _ = nqs.sampler.sample_bits()
        _, tn, _ = dv.rbm_forward(net.flat, net.ns, net.nh, bits, tanh=True, logpsi=False)
        eloc = nqs.local_energy_bits(bits, tn)
        n, P = int(bits.shape[0]), net.n_params
        ws = dv.sr_dense_workspace(dv.dtype_code(net.flat), net.ns, net.nh, n, bits.device)
        dv.sr_solve_dense(net.flat, net.ns, net.nh, bits, tn, eloc, shift=cfg["shift"], workspace=ws)   # warm-up
        flush.fill_(1.0)
        _lib.profile_read(reset=True)
        _lib.profile_enable(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record()
        x, info, _ = dv.sr_solve_dense(net.flat, net.ns, net.nh, bits, tn, eloc, shift=cfg["shift"], workspace=ws)
        ev[1].record()
        torch.cuda.synchronize()
        prof = _lib.profile_read(reset=True)
        _lib.profile_enable(False)
        gram_ms, chol_ms = prof["gram"][0], prof["cholesky"][0]
        flops = (4.0 if net.is_complex else 1.0) * n * P * P          # Hermitian half of the Gram
        r = {"n_params": P, "samples": n, "solve_ms": ev[0].elapsed_time(ev[1]), "gram_ms": gram_ms,
             "cholesky_ms": chol_ms, "gram_algorithmic_flop": flops,
             "gram_tflops": flops / (gram_ms / 1e3) / 1e12 if gram_ms > 0 else None,
             "gram_frac_of_bf16_sustained": (flops / (gram_ms / 1e3) / 1e12) / peak if gram_ms > 0 else None,
             "peak_bf16_tflops_sustained": peak, "true_residual": info["true_residual"],
             "workspace_gb": ws.numel() / 1e9}
        if r["solve_ms"] < 1000.0:
            td = TDVP(rhs_prefactor=-1.0, sr_diag_shift=cfg["shift"], sr_form_matrix=True)
            for _ in range(2):
                nqs.train_step(lr=cfg["lr"], tdvp=td)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(steps):
                nqs.train_step(lr=cfg["lr"], tdvp=td)
            torch.cuda.synchronize()
            r["dense_vmc_steps_per_s"] = steps / (time.perf_counter() - t0)
            t0 = time.perf_counter()
            for _ in range(steps):
                nqs.train_step(lr=cfg["lr"], tdvp=tdvp)
            torch.cuda.synchronize()
            r["matrix_free_vmc_steps_per_s"] = steps / (time.perf_counter() - t0)
        del ws
        out[name] = r
    return out


def batch_summary(steps, warmup, flush):
    """The batched uneven workload (64 TFIM problems, one form): steps/s and the phase split."""
    import torch
    from pyqusolver_b200 import _lib
    cfg = CONFIGS["tfim_batch64"]
    B, Ls, hx = build_batch(cfg, seed=1)
    kw = dict(shift=cfg["shift"], rtol=cfg["rtol"], maxiter=cfg["maxiter"], check_every=32)
    mk = lambda: [torch.cuda.Event(enable_timing=True) for _ in range(7)]

    def step(ev):
        ev[0].record(); B.sample()
        ev[1].record(); B.forward()
        ev[2].record(); B.local_energy()
        ev[3].record(); B.loss_stats()
        ev[4].record(); B.sr_solve(**kw)
        ev[5].record(); B.update(cfg["lr"])
        ev[6].record()
    for _ in range(warmup):
        step(mk())
    torch.cuda.synchronize()
    _lib.launch_count(reset=True)
    tot, ph = [], {p: [] for p in BATCH_PHASES}
    for _ in range(steps):
        flush.fill_(1.0)
        ev = mk()
        step(ev)
        torch.cuda.synchronize()
        tot.append(ev[0].elapsed_time(ev[6]))
        for k, p in enumerate(BATCH_PHASES):
            ph[p].append(ev[k].elapsed_time(ev[k + 1]))
    ms = float(np.mean(tot))
    return {"workload": "tfim_batch64", "steps": steps, "warmup": warmup, "problems": int(B.n_inst),
            "samples_per_step": int(B.n_samples_total), "ms_per_step": ms, "vmc_steps_per_s": 1e3 / ms,
            "samples_per_s": B.n_samples_total * 1e3 / ms, "phase_ms": {p: float(np.mean(v)) for p, v in ph.items()},
            "gpu_launches": int(_lib.launch_count(reset=True))}


def nqs_energy(info):
    e = info.get("e_mean", 0.0) if isinstance(info, dict) else 0.0
    return np.real(e)


def run_e2e(cfg, args, dist, world, seed):
    """The mixed form's training run once more through the public API, now host-driven: a fresh NQS
    built like the timed one (same parameters, chains and trajectory), and every step uploads the
    parameters from pinned host memory, runs NQS.train_step (which reads the statistics back) and
    downloads the updated parameters, which the next step uploads again."""
    import torch
    nqs, _ = build_nqs(cfg, seed=seed)
    net = nqs.net
    host_in = torch.empty_like(net.master, device="cpu").pin_memory()
    host_in.copy_(net.master.cpu())
    host_out = torch.empty_like(host_in).pin_memory()
    from pyqusolver_b200.tdvp import TDVP
    tdvp = TDVP(rhs_prefactor=-1.0, sr_diag_shift=cfg["shift"], sr_tol=cfg["rtol"], sr_maxiter=cfg["maxiter"], check_every=16)
    times = []
    for k in range(args.warmup + args.steps):                 # warm-up steps untimed, as in the timed loop
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        net.master.copy_(host_in, non_blocking=True)          # H2D: the step's parameters
        net.flat.copy_(net.master)
        net.bump()
        nqs.train_step(lr=cfg["lr"], tdvp=tdvp)                # public API (reads the statistics back)
        host_out.copy_(net.master, non_blocking=True)          # D2H: updated parameters
        e.record()
        torch.cuda.synchronize()
        if k >= args.warmup:
            times.append(s.elapsed_time(e))
        host_in, host_out = host_out, host_in                  # the next step starts from them
    from pyqusolver_b200 import replicas
    total = replicas.max_over_ranks(float(np.sum(times)), dist)
    nbytes = host_in.numel() * host_in.element_size()
    return {"value": replicas.job_throughput(cfg["chains"] * cfg["samples"], args.steps, total, world),
            "unit": "samples/s",
            "h2d_bytes_per_step": int(nbytes), "d2h_bytes_per_step": int(nbytes + 32),
            "ms_per_step": total / args.steps}


def kernel_bytes(cfg, nqs, kind, tc):
    """Algorithmic bytes of one launch: the operands the contraction needs, read once, and its
    outputs, written once, at their unpadded sizes.  T (Ns x M) counts once at its float32 size
    (the BF16 hi + lo pair of the tensor-core form is the same number of bytes), the spins as packed
    words, u or w as one complex64 per sample, v or the output as one float64 / complex128 per
    parameter.  Split-K partial P-vectors, padded or expanded operand tiles and re-reads are not
    algorithmic: they are the kernels' own traffic (``traffic`` reports what DRAM saw)."""
    net = nqs.net
    ns, nh, n = net.ns, net.nh, cfg["chains"] * cfg["samples"]
    ts, vs = (8, 16) if net.is_complex else (4, 8)
    nw = (ns + 31) // 32
    P = ns + nh + ns * nh
    t_bytes, spins = n * nh * ts, n * nw * 4
    if kind == "ov":          # w = O v: T, spins and v in, w out
        return t_bytes + spins + P * vs + n * 8
    if kind == "ohu":         # O^H u: T, spins and u in, one P-vector out
        return t_bytes + spins + n * 8 + P * vs
    if kind == "sv":          # fused S v: T and spins once, v in, one P-vector out
        return t_bytes + spins + 2 * P * vs
    return 3 * P * vs         # split reduction: the P-vector out, p in, Ap out


def fp32_peak_tflops(clk):
    """Nominal FP32 FMA issue rate of the B200 (148 SMs x 128 lanes x 2 flops) at the median SM clock
    sampled during the timed steps (max clock when no sample)."""
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    return 148 * 128 * 2 * mhz * 1e6 / 1e12


def issue_rooflines(cfg, nqs, form, clk):
    """Sampler and local energy, bound by FP32 issue (their working sets live in shared memory and L2):
    achieved = algorithmic flops / phase time, against the nominal FP32 rate at the sampled clock.
    Work units (restated from the kernels' arithmetic): one ratio factor per hidden unit and
    proposal in the sampler (complex: (C + g t S) products, 14 flops; real: 3 flops), plus the
    accepted-move cache update it amortises; one (move, hidden unit) term per sample in the local
    energy (complex: one complex FMA and one complex multiply, 14 flops; real: 3 flops)."""
    net = nqs.net
    n = cfg["chains"] * cfg["samples"]
    f_unit = 14 if net.is_complex else 3
    proposals = cfg["chains"] * cfg["samples"] * cfg["sweep"]
    n_moves = nqs._dev_ham.n_moves
    peak = fp32_peak_tflops(clk)
    out = {}
    for phase, units, what in (("sample", proposals * net.nh, "proposal x hidden-unit ratio factors"),
                               ("local_energy", n * n_moves * net.nh, "sample x move x hidden-unit terms")):
        ms = float(np.mean(form["phase_ms"][phase]))
        tf = units * f_unit / (ms / 1e3) / 1e12
        out[phase] = {"kernel": "sampler_kernel" if phase == "sample" else "eloc_moves_kernel",
                      "bound": "fp32_issue", "work_units_per_launch": int(units), "unit_definition": what,
                      "flops_per_unit": f_unit, "avg_launch_us": ms * 1e3, "achieved": tf, "peak": peak,
                      "unit": "TFLOP/s", "frac": tf / peak,
                      "peak_source": "nominal FP32 FMA rate at the sampled SM clock (not a measured peak)"}
    return out


def roofline(cfg, nqs, form):
    """Roofline of the kernel with the largest share of the profiled steps (live CUDA-event times on the
    launching stream; the profiled CG checks convergence after every iteration, so every bracketed
    launch did work)."""
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic_db = {}
    try:
        traffic_db = json.load(open(os.path.join(ROOT, "profiles", "dram_traffic_per_launch.json")))
    except (OSError, ValueError):
        pass
    phases = form.get("prof_phase_ms") or form["phase_ms"]
    steps = len(form.get("prof_cg_iters") or form["cg_iters"])
    cands = {}
    for k, (ms, cnt) in (form["prof"] or {}).items():
        if cnt:
            cands[k] = (ms, cnt)
    for p in ("sample", "local_energy", "forward"):
        cands[p] = (float(np.sum(phases[p])), steps)
    dom = max(cands, key=lambda k: cands[k][0])
    total_ms, cnt = cands[dom]
    avg_s = total_ms / cnt / 1e3
    from pyqusolver_b200 import _lib, device as dv
    net = nqs.net
    tc = _lib.sr_uses_tensor_cores(dv.dtype_code(net.flat), net.ns, net.nh, cfg["chains"] * cfg["samples"])
    ovz = tc and _lib.sr_tc_plan(dv.dtype_code(net.flat), net.ns, net.nh, cfg["chains"] * cfg["samples"])["ovz"]
    names = {"ov": ("tc_ovz_kernel (O v through z = Sigma V, tcgen05)" if ovz else "tc_ov_kernel (O v, tcgen05)")
             if tc else "ov_kernel (O v, CUDA cores)",
             "ohu": "tc_ohu_kernel (O^H u, tcgen05)" if tc else "ohu_kernel (O^H u, CUDA cores)",
             "reduce": "reduce_splits_kernel / cg_fused_kernel", "sample": "sampler_kernel",
             "sv": "tc_sv_kernel (S v: O v and O^H u fused, tcgen05)",
             "local_energy": "eloc_moves_kernel",
             "forward": "theta_tc_kernel (tcgen05)" if dv.forward_uses_tensor_cores(
                 net.flat, net.ns, net.nh, cfg["chains"] * cfg["samples"]) else "rbm_forward_kernel"}
    out = {"kernel": names.get(dom, dom), "launches_timed": cnt, "avg_launch_us": avg_s * 1e6,
           "share_of_timed_region": total_ms / float(np.sum([np.sum(v) for v in phases.values()])),
           "bound": "hbm", "peak": hbm, "unit": "GB/s", "peak_source": src,
           # every profiled SR kernel class: launches and mean CUDA-event duration (the bracketing events
           # serialise the chain, so these are upper bounds of the live per-launch times)
           "sr_classes_us": {k: {"launches": int(c), "avg_us": float(ms) / c * 1e3}
                             for k, (ms, c) in (form["prof"] or {}).items() if c}}
    if dom in ("ov", "ohu", "reduce", "sv"):
        b = kernel_bytes(cfg, nqs, dom, tc=tc)
        tr = traffic_db.get(cfg.get("name", ""), {}).get(dom)
    elif dom in ("sample", "local_energy"):
        # working sets in shared memory and L2: bound by FP32 issue, not by HBM
        ir = issue_rooflines(cfg, nqs, {"phase_ms": phases}, None)[dom]
        ir["share_of_timed_region"] = out["share_of_timed_region"]
        return ir
    else:
        n = cfg["chains"] * cfg["samples"]
        b = n * net.nh * (8 if net.is_complex else 4) + n * ((net.ns + 31) // 32) * 4
        tr = None
    ach = b / avg_s / 1e9
    out.update({"achieved": ach, "frac": ach / hbm, "algorithmic_bytes_per_launch": int(b), "traffic": tr})
    return out


# ---------------------------------------------------------------------------------------- CPU (oracle)
def oracle_setup(cfg, n_chains, seed=0):
    from oracle import lattice as olat, hamiltonian as oH, rbm as orbm, sampler as osm
    L = olat.SquareLattice(cfg["dim"], cfg["lx"], cfg["ly"], bc="pbc")
    if cfg["model"] == "xxz":
        terms = oH.xxz_terms(L, **cfg["kw"])
    elif cfg["model"] == "j1j2":
        terms = oH.j1j2_terms(L, **cfg["kw"])
    else:
        terms = oH.tfim_terms(L, **cfg["kw"])
    ns = L.ns
    p = orbm.random_params(ns, cfg["alpha"] * ns, complex_=cfg["dtype"].startswith("complex"), scale=0.01, seed=seed)
    smp = osm.MetropolisSampler(ns, n_chains, rule=cfg["rule"], neighbor_table=olat.neighbor_table(L), seed=seed,
                                therm_steps=1, sweep_steps=cfg["sweep"],
                                init=cfg["init"], n_up=ns // 2)
    smp.needs_therm = False        # throughput only: thermalisation is not part of a steady-state step
    return p, terms, smp


def cpu_step(cfg, p, terms, smp):
    from oracle import vmc as ovmc
    return ovmc.vmc_step(p, terms, smp, cfg["samples"], lr=cfg["lr"], shift=cfg["shift"], rtol=cfg["rtol"],
                         maxiter=cfg["maxiter"])


def batch_problem_cfgs(cfg):
    """Per-problem single-workload configs of a batched workload (same draws as build_batch)."""
    rng = np.random.default_rng(cfg["draw_seed"])
    Ls = rng.integers(cfg["L_lo"], cfg["L_hi"] + 1, size=cfg["n_inst"])
    hx = rng.uniform(cfg["hx_lo"], cfg["hx_hi"], size=cfg["n_inst"])
    return [dict(name=f"{cfg['name']}[{b}]", dim=1, lx=int(L), ly=1, model="tfim", kw=dict(j=1.0, hx=float(h), hz=0.0),
                 alpha=cfg["alpha"], dtype=cfg["dtype"], chains=cfg["chains"], samples=cfg["samples"], rule="LOCAL",
                 sweep=int(L), shift=cfg["shift"], lr=cfg["lr"], rtol=cfg["rtol"], maxiter=cfg["maxiter"], init="RND")
            for b, (L, h) in enumerate(zip(Ls, hx))]


CPU_CHAINS = 64      # chains per timed CPU step (per-sample throughput is flat beyond a few dozen)


def cpu_port_threads():
    """Compile the oracle's multi-core log-cosh kernel (oracle/fast.py) before any timing; returns the
    host threads the port runs on (Numba's pool and OpenBLAS's, both sized to the host) and a label."""
    from oracle import fast
    on = fast.enable()
    if on:
        return max(fast.threads(), 1), "float64 NumPy/OpenBLAS + Numba prange (log cosh of the local energy)"
    return os.cpu_count() or 1, "float64 NumPy/OpenBLAS"


def cpu_baseline(cfg, budget_s=20.0):
    """The oracle (float64 NumPy restatement of the reference's algorithm) on the host cores."""
    threads, how = cpu_port_threads()
    if cfg.get("batch"):
        # bounded sample: one VMC step of 16 chains on successive problems until the budget is used
        t0 = time.perf_counter()
        samples, done = 0, 0
        for pc in batch_problem_cfgs(cfg):
            p, terms, smp = oracle_setup(pc, 16)
            cpu_step(pc, p, terms, smp)
            samples += 16 * pc["samples"]
            done += 1
            if time.perf_counter() - t0 > budget_s:
                break
        dt = time.perf_counter() - t0
        return {"value": samples / dt, "unit": "samples/s", "cores": threads, "kind": "port",
                "sample": f"one VMC step of 16 chains x {cfg['samples']} samples on each of the first {done} "
                          f"problems ({how}, problems one after another)"}
    n_chains = CPU_CHAINS
    p, terms, smp = oracle_setup(cfg, n_chains)
    t0 = time.perf_counter()
    steps = 0
    while True:
        p, _ = cpu_step(cfg, p, terms, smp)
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= 8:
            break
    dt = time.perf_counter() - t0
    samples = steps * n_chains * cfg["samples"]
    return {"value": samples / dt, "unit": "samples/s", "cores": threads, "kind": "port",
            "sample": f"{steps} steady-state VMC step(s) of {n_chains} chains x {cfg['samples']} samples (same "
                      f"per-sample algorithm as the reference: full RBM re-evaluation per connected state and per "
                      f"exchange proposal; {how}; thermalisation not timed)"}


def run_reference(args, cfg, rank, world):
    if rank != 0:
        return
    if cfg.get("batch"):
        cb = None
        t_all = []
        for _ in range(args.warmup + args.steps):
            cb = cpu_baseline(cfg, budget_s=min(args.cpu_budget, 10.0))
            t_all.append(cb["value"])
        v = float(np.mean(t_all[args.warmup:]))
        cb["value"] = v
        line = {"metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic", "config": {"workload": args.config}, "impl": "reference",
                "cpu_baseline": cb,
                "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    threads, how = cpu_port_threads()
    n_chains = CPU_CHAINS
    p, terms, smp = oracle_setup(cfg, n_chains)
    for _ in range(args.warmup):
        p, _ = cpu_step(cfg, p, terms, smp)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        p, _ = cpu_step(cfg, p, terms, smp)
    dt = time.perf_counter() - t0
    samples = args.steps * n_chains * cfg["samples"]
    v = samples / dt
    sample_desc = (f"each step {n_chains} chains x {cfg['samples']} samples of the {args.config} workload "
                   f"(bounded sample), oracle port of the reference algorithm ({how}) on {threads} host threads")
    line = {"metric": METRIC, "value": v, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": args.config, "samples_per_step": n_chains * cfg["samples"]},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "samples/s", "cores": threads, "kind": "port",
                             "sample": sample_desc},
            "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="heis10x10", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="plain_fp32,mixed", help="comma list of plain_fp32, mixed (mixed is required)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--ed-epochs", type=int, default=1500,
                    help="epochs of the 6x6 J1-J2 training compared with its exact energy (0: skip)")
    ap.add_argument("--accuracy-epochs", type=int, default=300,
                    help="epochs of the ED-checked mixed vs plain comparison on tfim16 (0 = skip)")
    ap.add_argument("--matched-epochs", type=int, default=300,
                    help="epochs of the float64 / mixed / plain comparison on heis10x10 (0 = skip)")
    ap.add_argument("--matched-configs", default="tfim16,j1j2_6x6,tfim20x20",
                    help="other workloads given the common-batch float64 comparison (summary only)")
    ap.add_argument("--matched-other-epochs", type=int, default=60,
                    help="training epochs of each of those comparisons (5 checked batches; 0 = skip)")
    ap.add_argument("--matched-every", type=int, default=15,
                    help="solve the batch of every n-th epoch in all three forms")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the per-workload summaries of tfim16, j1j2_6x6, tfim20x20 and tfim_batch64")
    ap.add_argument("--other-steps", type=int, default=8)
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the automatic tensor-core SR tiling instead of timing the candidates")
    ap.add_argument("--no-dense", action="store_true", help="skip the formed-S (Gram + Cholesky) summary")
    ap.add_argument("--dense-configs", default="tfim16,j1j2_6x6,heis10x10",
                    help="workloads of the formed-S summary")
    ap.add_argument("--chains", type=int, default=0,
                    help="override the workload's chain count (smaller cases for profiler captures; the "
                         "bench line of a workload uses its own count)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local_rank = env_rank()
    cfg = CONFIGS[args.config]
    if args.chains > 0:
        cfg = dict(cfg, chains=int(args.chains))
        CONFIGS[args.config] = cfg
    if args.impl == "reference":
        run_reference(args, cfg, rank, world)
    elif cfg.get("batch"):
        run_batch(args, cfg, rank, world, local_rank)
    else:
        run_ours(args, cfg, rank, world, local_rank)


if __name__ == "__main__":
    main()
