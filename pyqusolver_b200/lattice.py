"""Square / chain lattice with the neighbour API the QES models and sampler call.

The reference's lattice (``general_python.lattices``) is not in the reference
snapshot; the methods kept here are the ones its callers use:
``get_nn_forward_num / get_nn_forward`` (model bond loops,
``QES/Algebra/Model/Interacting/Spin/transverse_ising.py:270-280``),
``get_nnn_forward_num / get_nnn_forward`` (``j1j2.py:261-291``),
``adjacency_matrix`` (``QES/Solver/MonteCarlo/updates/utils.py:61-64``),
``bond_winding`` / ``boundary_phase_from_winding`` and ``wrong_nei``.

Convention: site i = x + Lx*y; nn forward (x+1, y), (x, y+1); nnn forward
(x+1, y+1), (x-1, y+1); PBC wraps, OBC drops; boundary phase 1 (no flux).
"""

from __future__ import annotations

import numpy as np


class SquareLattice:
    def __init__(self, dim: int = 1, lx: int = 4, ly: int = 1, lz: int = 1, bc: str = "pbc", **_):
        if dim not in (1, 2):
            raise ValueError("SquareLattice: dim must be 1 or 2")
        self.dim = int(dim)
        self.lx = int(lx)
        self.ly = int(ly) if dim == 2 else 1
        self.bc = str(bc).lower()
        if self.bc not in ("pbc", "obc"):
            raise ValueError("SquareLattice: bc must be 'pbc' or 'obc'")
        if self.lx < 1 or self.ly < 1:
            raise ValueError("SquareLattice: sizes must be positive")
        self.ns = self.lx * self.ly
        self._nn = [self._fwd(i, [(1, 0)] if self.dim == 1 else [(1, 0), (0, 1)]) for i in range(self.ns)]
        self._nnn = [self._fwd(i, [] if self.dim == 1 else [(1, 1), (-1, 1)]) for i in range(self.ns)]

    @property
    def Ns(self):
        return self.ns

    def __len__(self):
        return self.ns

    def _shift(self, i, dx, dy):
        x, y = i % self.lx, i // self.lx
        x2, y2 = x + dx, y + dy
        if self.bc == "pbc":
            x2 %= self.lx
            y2 %= self.ly
        elif not (0 <= x2 < self.lx and 0 <= y2 < self.ly):
            return -1
        return x2 + self.lx * y2

    def _fwd(self, i, shifts):
        out = []
        for dx, dy in shifts:
            j = self._shift(i, dx, dy)
            if j >= 0 and j != i:
                out.append(j)
        return out

    # --- QES lattice API subset -------------------------------------------------
    def get_nn_forward_num(self, i):
        return len(self._nn[i])

    def get_nn_forward(self, i, num=0):
        return self._nn[i][num]

    def get_nnn_forward_num(self, i):
        return len(self._nnn[i])

    def get_nnn_forward(self, i, num=0):
        return self._nnn[i][num]

    @staticmethod
    def wrong_nei(j):
        return j is None or int(j) < 0

    def bond_winding(self, i, j):
        return 0, 0, 0

    def boundary_phase_from_winding(self, wx, wy, wz):
        return 1.0

    def nn_bonds(self):
        return [(i, j) for i in range(self.ns) for j in self._nn[i]]

    def nnn_bonds(self):
        return [(i, j) for i in range(self.ns) for j in self._nnn[i]]

    def adjacency_matrix(self, sparse=False):
        a = np.zeros((self.ns, self.ns), dtype=np.int64)
        for i, j in self.nn_bonds():
            a[i, j] = 1
            a[j, i] = 1
        if sparse:
            import scipy.sparse as sp
            return sp.csr_matrix(a)
        return a


def get_neighbor_table(lattice, max_neighbors=None, order: int = 1) -> np.ndarray:
    """Padded (-1) neighbour table, ascending per row (``updates/utils.py:37-109``)."""
    adj = np.asarray(lattice.adjacency_matrix(sparse=False))
    if order > 1:
        ab = adj != 0
        acc, cur = ab.copy(), ab.copy()
        for _ in range(order - 1):
            cur = (cur.astype(np.int64) @ ab.astype(np.int64)) != 0
            acc |= cur
        np.fill_diagonal(acc, False)
        adj = acc.astype(np.int64)
    rows = [np.flatnonzero(adj[i]) for i in range(adj.shape[0])]
    deg = max((len(r) for r in rows), default=0)
    if max_neighbors is not None:
        if deg > max_neighbors:
            raise ValueError(f"Lattice max degree {deg} exceeds requested max_neighbors {max_neighbors}")
        deg = max_neighbors
    tab = np.full((adj.shape[0], deg), -1, dtype=np.int32)
    for i, r in enumerate(rows):
        tab[i, :len(r)] = r
    return tab
