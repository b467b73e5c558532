"""Exact ground-state energy (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference diagonalises with ``model.diagonalize(method='lanczos')``
(``QES/Algebra/hamil.py:1809+`` -> ``QES/Algebra/Hamil/hamil_diag_engine.py:176-305``),
whose eigensolver is in the empty ``general_python`` submodule.  This
restatement builds the same sparse S^z-basis matrix from the oracle's term
list and calls SciPy's ARPACK Lanczos (``eigsh``, smallest algebraic).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as spla

from .hamiltonian import sparse_hamiltonian


def ground_energy(terms, ns, n_up=None, dense_below=64):
    H, _ = sparse_hamiltonian(terms, ns, n_up=n_up)
    if H.shape[0] <= dense_below:
        return float(np.min(np.linalg.eigvalsh(H.toarray())))
    Hr = H if np.abs(H.imag).max() > 0 else H.real
    vals = spla.eigsh(Hr, k=1, which="SA", tol=1e-12, return_eigenvectors=False)
    return float(np.real(vals[0]))


def symmetric_ground_energy(terms, lx, ly, n_up, parity=0, kx=0, ky=0):
    """Lowest eigenvalue of H in one momentum (0 or pi per axis) and spin-flip-parity sector.

    Built without representatives or orbit norms: with the group G of the lx*ly translations
    (times the spin flip when ``parity`` is +-1) and the character
    chi(T(a, b) F^f) = (-1)^(kx a + ky b) parity^f (``QES/Algebra/Symmetries/translation.py:470-519``
    with k = 0 or L/2), P = |G|^-1 sum_g chi(g) U_g is the orthogonal projector on the sector and
    commutes with H, so the lowest eigenvalue of H + lam (1 - P), lam above the spectral width, is
    the sector's ground energy.  Sites are x + lx*y; the oracle's integers carry site i at bit
    ns - 1 - i.
    """
    import scipy.sparse as sp

    ns = lx * ly
    H, basis = sparse_hamiltonian(terms, ns, n_up=n_up)
    nb = len(basis)
    pos = ns - 1 - np.arange(ns, dtype=np.int64)
    occ = (basis[:, None] >> pos[None, :]) & 1                     # occ[:, i]: site i up
    full = (1 << ns) - 1
    cols = np.arange(nb, dtype=np.int64)
    rows_all, cols_all, vals_all = [], [], []
    for b in range(ly):
        for a in range(lx):
            dest = np.array([(i % lx + a) % lx + lx * ((i // lx + b) % ly) for i in range(ns)], dtype=np.int64)
            moved = (occ << pos[dest][None, :]).sum(axis=1)           # site i's bit placed at site dest[i]
            chi = (-1.0) ** (kx * a + ky * b)
            images = [(moved, chi)]
            if parity:
                images.append((full ^ moved, chi * parity))
            for img, c in images:
                r = np.searchsorted(basis, img)
                assert np.all(basis[np.minimum(r, nb - 1)] == img)
                rows_all.append(r)
                cols_all.append(cols)
                vals_all.append(np.full(nb, c))
    m = lx * ly * (2 if parity else 1)
    P = sp.coo_matrix((np.concatenate(vals_all) / m, (np.concatenate(rows_all), np.concatenate(cols_all))),
                      shape=(nb, nb)).tocsr()
    Hr = H.real if np.abs(H.imag).max() == 0 else H
    lam = 2.0 * float(np.abs(Hr).sum(axis=1).max()) + 1.0
    Hs = Hr + lam * (sp.identity(nb, format="csr") - P)
    if nb <= 600:
        return float(np.min(np.linalg.eigvalsh(Hs.toarray())))
    vals = spla.eigsh(Hs, k=1, which="SA", tol=1e-12, return_eigenvectors=False)
    return float(np.real(vals[0]))


def symmetric_sector_dim(lx, ly, n_up, parity=0, kx=0, ky=0):
    """Dimension of the momentum / spin-flip sector: trace P = |G|^-1 sum_g chi(g) #{s : g s = s}
    over the S^z basis (the same group and characters as ``symmetric_ground_energy``)."""
    ns = lx * ly
    allb = np.arange(1 << ns, dtype=np.int64)
    basis = allb[np.bitwise_count(allb) == n_up]
    pos = ns - 1 - np.arange(ns, dtype=np.int64)
    occ = (basis[:, None] >> pos[None, :]) & 1
    full = (1 << ns) - 1
    tr = 0.0
    for b in range(ly):
        for a in range(lx):
            dest = np.array([(i % lx + a) % lx + lx * ((i // lx + b) % ly) for i in range(ns)], dtype=np.int64)
            moved = (occ << pos[dest][None, :]).sum(axis=1)
            chi = (-1.0) ** (kx * a + ky * b)
            tr += chi * np.count_nonzero(moved == basis)
            if parity:
                tr += chi * parity * np.count_nonzero((full ^ moved) == basis)
    m = lx * ly * (2 if parity else 1)
    return int(round(tr / m))


def symmetric_sector_dim_burnside(lx, ly, n_up, parity=0, kx=0, ky=0):
    """The same dimension without enumerating states (any size): trace P by counting fixed points.
    T(a, b) permutes the sites in ns / l cycles of length l = lcm(lx / gcd(a, lx), ly / gcd(b, ly));
    a state it fixes is constant on each cycle (C(ns / l, n_up / l) states when l divides n_up), and
    a state that F T(a, b) fixes alternates along each cycle (2^(ns / l) states when l is even)."""
    from math import comb, gcd

    ns = lx * ly
    tr = 0
    for b in range(ly):
        for a in range(lx):
            la, lb = lx // gcd(a, lx), ly // gcd(b, ly)
            cyc = la * lb // gcd(la, lb)
            c = ns // cyc
            chi = -1 if (kx * a + ky * b) % 2 else 1
            if n_up % cyc == 0:
                tr += chi * comb(c, n_up // cyc)
            if parity and cyc % 2 == 0 and 2 * n_up == ns:
                tr += chi * parity * 2 ** c
    m = lx * ly * (2 if parity else 1)
    assert tr % m == 0
    return tr // m
