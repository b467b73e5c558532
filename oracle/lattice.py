"""Square / chain lattice restatement (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference's lattice class lives in the empty ``general_python`` submodule,
so its site order and forward-neighbour order are not pinned by any reference
file.  The convention written here (and mirrored by
``pyqusolver_b200/lattice.py``) is:

* site index      i = x + Lx * y
* nn forward      1D: (x+1);  2D: (x+1, y) then (x, y+1)   (PBC wraps, OBC drops)
* nnn forward     2D: (x+1, y+1) then (x-1, y+1)
* neighbour table row i = ascending ``flatnonzero`` of the NN adjacency row,
  padded with -1, as ``get_neighbor_table`` builds it
  (``QES/Solver/MonteCarlo/updates/utils.py:37-109``).
* bond boundary phase = 1 (no flux threaded), the value
  ``boundary_phase_from_winding`` gives for a plain periodic lattice.
"""

from __future__ import annotations

import numpy as np


class SquareLattice:
    def __init__(self, dim: int = 1, lx: int = 4, ly: int = 1, bc: str = "pbc"):
        if dim not in (1, 2):
            raise ValueError("dim must be 1 or 2")
        self.dim = dim
        self.lx = int(lx)
        self.ly = int(ly) if dim == 2 else 1
        self.bc = bc.lower()
        if self.bc not in ("pbc", "obc"):
            raise ValueError("bc must be 'pbc' or 'obc'")
        self.ns = self.lx * self.ly

    def site(self, x, y=0):
        return x + self.lx * y

    def coords(self, i):
        return i % self.lx, i // self.lx

    def _shift(self, i, dx, dy):
        x, y = self.coords(i)
        x2, y2 = x + dx, y + dy
        if self.bc == "pbc":
            x2 %= self.lx
            y2 %= self.ly
        elif not (0 <= x2 < self.lx and 0 <= y2 < self.ly):
            return -1
        return self.site(x2, y2)

    def nn_forward(self, i):
        shifts = [(1, 0)] if self.dim == 1 else [(1, 0), (0, 1)]
        out = []
        for dx, dy in shifts:
            j = self._shift(i, dx, dy)
            if j >= 0 and j != i:
                out.append(j)
        return out

    def nnn_forward(self, i):
        if self.dim == 1:
            return []
        out = []
        for dx, dy in [(1, 1), (-1, 1)]:
            j = self._shift(i, dx, dy)
            if j >= 0 and j != i:
                out.append(j)
        return out

    def nn_bonds(self):
        return [(i, j) for i in range(self.ns) for j in self.nn_forward(i)]

    def nnn_bonds(self):
        return [(i, j) for i in range(self.ns) for j in self.nnn_forward(i)]

    def adjacency(self):
        a = np.zeros((self.ns, self.ns), dtype=np.int64)
        for i, j in self.nn_bonds():
            a[i, j] = 1
            a[j, i] = 1
        return a


def neighbor_table(lat: SquareLattice, order: int = 1) -> np.ndarray:
    """Padded (-1) neighbour table, ascending per row (reference utils.py:37-109)."""
    adj = lat.adjacency()
    if order > 1:
        adj_b = adj != 0
        acc = adj_b.copy()
        cur = adj_b.copy()
        for _ in range(order - 1):
            cur = (cur.astype(np.int64) @ adj_b.astype(np.int64)) != 0
            acc = acc | cur
        np.fill_diagonal(acc, False)
        adj = acc.astype(np.int64)
    rows = [np.flatnonzero(adj[i]) for i in range(lat.ns)]
    deg = max((len(r) for r in rows), default=0)
    tab = np.full((lat.ns, deg), -1, dtype=np.int32)
    for i, r in enumerate(rows):
        tab[i, :len(r)] = r
    return tab
