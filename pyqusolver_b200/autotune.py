"""Autotuner of the tensor-core SR matvec tiling.

The tcgen05 O^H u has two tilings (``qes_sr_tc_plan``): one 128-row M tile per sample chunk (small
problems) or an M/N-tiled kernel whose CTAs fold several sample chunks into TMEM (N chunks of NC
hidden units, a target CTA count); ``qes_sr_set_ohu_pairs`` runs the single-tile kernel as pairs
of CTAs that add their split-K partials through distributed shared memory, and
``qes_sr_set_fused_sv`` runs the single-tile matvec as one cooperative S v kernel (O v, the mean of
O v over a grid barrier and O^H u in the same CTAs).  ``tune_sr_tiling`` times
the SR matvec (``qes_sr_matvec``: O v, O^H u and the split reduction, the body of one CG iteration)
of a given batch for every candidate with CUDA events on the current stream, keeps the fastest,
applies it process-wide and persists it in a JSON cache keyed by device, dtype and shape
(``$QES_B200_AUTOTUNE`` or ``~/.cache/pyqusolver_b200/autotune.json``).  Candidates that the shapes
do not admit (QES_ERR_SIZE / QES_ERR_ARG) are skipped.  Every candidate computes the same matvec; the
choice changes only the order of the float32 partial sums.
"""

from __future__ import annotations

import json
import os

import torch

from . import _lib
from . import device as dv


def _cache_path(cache=None):
    return cache or os.environ.get("QES_B200_AUTOTUNE", os.path.join(os.path.expanduser("~"), ".cache",
                                                                      "pyqusolver_b200", "autotune.json"))


def _candidates(ns, nh, cplx):
    # (mode, nc, ctas, pairs, fused S v): automatic with the fused kernel, the kernel pair, the pair
    # with O^H u in CTA pairs, then the M/N-tiled O^H u
    out = [(0, 0, 0, 0, 1), (0, 0, 0, 0, 0), (0, 0, 0, 1, 0)]
    for nc in (256, 208, 128, 96, 64, 32):
        if nc > ((nh + 15) // 16) * 16:
            continue
        for ctas in (148, 296, 592):
            out.append((2, nc, ctas, 0, 0))
    return out


def tune_sr_tiling(net, bits, tanh_theta, *, repeats=5, cache=None, candidates=None):
    """Time the SR matvec of (net, bits, tanh_theta) under each tiling candidate (mode, nc, ctas, pairs, sv);
    apply and return the fastest as a dict with the timings.  A cached choice for the same device and
    shapes is applied without timing."""
    dc = dv.dtype_code(net.flat)
    n = int(bits.shape[0])
    dev = torch.cuda.get_device_name(bits.device)
    key = f"sr_tiling5|{dev}|{dc}|{net.ns}|{net.nh}|{n}"
    path = _cache_path(cache)
    table = {}
    try:
        with open(path) as f:
            table = json.load(f)
    except (OSError, ValueError):
        table = {}
    if key in table and candidates is None:
        apply_tiling(*table[key]["choice"])
        return dict(table[key], cached=True)
    cands = candidates or _candidates(net.ns, net.nh, net.is_complex)
    P = dv.n_params(net.ns, net.nh)
    v = torch.randn(P, dtype=dv.vec_dtype(net.flat.dtype), device=bits.device)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timings = {}
    best, best_t = None, float("inf")
    try:
        for cand in cands:
            apply_tiling(*cand)
            if not _lib.sr_uses_tensor_cores(dc, net.ns, net.nh, n):
                continue
            try:
                ws = dv.sr_workspace(dc, net.ns, net.nh, n, bits.device)
                dv.sr_matvec(net.flat, net.ns, net.nh, bits, tanh_theta, v, workspace=ws)   # warm-up
                torch.cuda.synchronize()
                ts = []
                for _ in range(repeats):
                    ev0.record()
                    dv.sr_matvec(net.flat, net.ns, net.nh, bits, tanh_theta, v, workspace=ws)
                    ev1.record()
                    torch.cuda.synchronize()
                    ts.append(ev0.elapsed_time(ev1))
            except _lib.QESError as e:
                if e.code not in (_lib.QES_ERR_SIZE, _lib.QES_ERR_ARG):
                    raise
                continue
            t = sorted(ts)[len(ts) // 2]
            timings[str(cand)] = t
            if t < best_t:
                best, best_t = cand, t
    finally:
        apply_tiling(*(best or (0, 0, 0, 0, 1)))
    if best is None:
        return {"choice": (0, 0, 0, 0, 1), "ms": None, "timings": timings, "cached": False}
    entry = {"choice": list(best), "ms": best_t, "timings": timings}
    table[key] = entry
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, path)
    except OSError:
        pass
    return dict(entry, cached=False)


def apply_tiling(mode, nc, ctas, pairs, sv=1):
    _lib.call("qes_sr_set_tiling", int(mode), int(nc), int(ctas))
    _lib.call("qes_sr_set_ohu_pairs", int(pairs))
    _lib.call("qes_sr_set_fused_sv", int(sv))
