"""Exact ground energies of the 6x6 J1-J2 workload (periodic 6x6 square lattice, J1 = 1,
J2 = 0.5, S^z = 0) and of the 6x6 Heisenberg model (J2 = 0), by the library's GPU Lanczos in the
translation + spin-flip reduced sectors (``qes_ed_lanczos_symm``).  The ground state lies in the
k = (0, 0), even-flip sector; the (pi, pi) and odd-flip sectors are computed as well and must lie
above it.  Writes ``ed_j1j2_6x6.json`` beside this script.

Needs a GPU (≈ 5 GB of device memory per sector):

    python tests/golden/make_ed_j1j2_6x6.py [--quick]

``--quick`` computes only the (0, 0) even-flip sector of J2 = 0.5.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import pyqusolver_b200 as qb  # noqa: E402


def sector_energy(j2, parity, momentum, tol=1e-12, maxiter=800):
    import torch
    model = qb.J1J2Model(qb.SquareLattice(2, 6, 6, bc="pbc"), J1=-1.0, J2=-j2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = float(model.diagonalize(n_up=18, spin_flip=parity, momentum=momentum, tol=tol, maxiter=maxiter)[0])
    torch.cuda.synchronize()
    return {"j1": 1.0, "j2": j2, "n_up": 18, "spin_flip": parity, "momentum": list(momentum),
            "e0": e0, "e0_per_site": e0 / 36.0, "sector_dim": model.sector_dim,
            "lanczos_iterations": model.lanczos_iterations, "seconds": round(time.perf_counter() - t0, 2)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true")
    ap.add_argument("--out", default=os.path.join(HERE, "ed_j1j2_6x6.json"))
    a = ap.parse_args()
    runs = [(0.5, 1, (0, 0))]
    if not a.quick:
        runs += [(0.5, -1, (0, 0)), (0.5, 1, (3, 3)), (0.0, 1, (0, 0))]
    out = {"lattice": "6x6 square, periodic", "units": "H = J1 sum S_i.S_j + J2 sum S_i.S_k, S = 1/2",
           "command": "python tests/golden/make_ed_j1j2_6x6.py" + (" --quick" if a.quick else ""),
           "sectors": []}
    for j2, parity, mom in runs:
        r = sector_energy(j2, parity, mom)
        print(json.dumps(r), flush=True)
        out["sectors"].append(r)
    gs = [r for r in out["sectors"] if r["j2"] == 0.5]
    out["e0_j2_0.5"] = min(r["e0"] for r in gs)
    with open(a.out, "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
