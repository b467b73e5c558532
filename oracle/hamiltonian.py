"""Spin-1/2 lattice Hamiltonians and connected-state enumeration (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Term lists follow the reference's model builders term by term, in the same
insertion order, with the same signs and the same operator normalisation:

* TFIM  ``QES/Algebra/Model/Interacting/Spin/transverse_ising.py:192-300``:
  -hx_i Sx_i, -hz_i Sz_i, then -J_i * phase * Sz_i Sz_j on forward NN bonds.
* XXZ   ``QES/Algebra/Model/Interacting/Spin/xxz.py:278-433``:
  -hx Sx, -hz Sz, then per forward bond XX(-jxy), YY(-jxy), ZZ(-jz).
* J1-J2 ``QES/Algebra/Model/Interacting/Spin/j1j2.py:119-295``: local fields,
  then per NN bond XX, YY, ZZ with multiplier -phase*J1, then the same on NNN
  bonds with -phase*J2 (the code's literal sign, not its docstring's).

Operators act on +-0.5 vectors with the reference's coefficients
(``QES/Algebra/Operator/impl/jax/operators_spin.py:131-143,220-248,353-370``):
X on k sites flips them with coefficient 0.5**k; Y flips them with
prod(i * 0.5 * sigma_i) evaluated on the state before the flip; Z keeps the
state with prod(0.5 * sigma_i), sigma = sign(s).

``connected_raw`` reproduces the slot list of ``local_energy_jax_wrap``
(``QES/Algebra/Hamil/hamil_energy_jax.py:428-576``): slot 0 is the input
state with the summed diagonal, then one slot per modifying term, grouped by
(operator, arity) in order of first appearance and in insertion order inside
a group.  XX and YY of one bond are separate slots even when they cancel.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

import numpy as np
import scipy.sparse as sp

from .lattice import SquareLattice

SPIN_VALUE = 0.5


@dataclass(frozen=True)
class Term:
    op: str               # 'x', 'y' or 'z' (applied on every site in ``sites``)
    sites: tuple
    mult: complex

    @property
    def modifies(self):
        return self.op in ("x", "y")


def _per_site(v, ns):
    if v is None:
        return None
    if np.isscalar(v):
        return np.full(ns, float(v))
    v = np.asarray(v, dtype=float)
    if v.shape != (ns,):
        raise ValueError("site-resolved coupling must have length ns")
    return v


def _nz(v, i):
    return v is not None and not np.isclose(v[i], 0.0)


def tfim_terms(lat: SquareLattice, j=1.0, hx=1.0, hz=1.0) -> List[Term]:
    ns = lat.ns
    J, HX, HZ = _per_site(j, ns), _per_site(hx, ns), _per_site(hz, ns)
    terms = []
    for i in range(ns):
        if _nz(HX, i):
            terms.append(Term("x", (i,), -HX[i]))
    for i in range(ns):
        if _nz(HZ, i):
            terms.append(Term("z", (i,), -HZ[i]))
    for i in range(ns):
        for jn in lat.nn_forward(i):
            if not _nz(J, i):
                continue
            terms.append(Term("z", (i, jn), -J[i] * 1.0))
    return terms


def xxz_terms(lat: SquareLattice, jxy=1.0, jz=1.0, delta=None, hx=0.0, hz=0.0) -> List[Term]:
    ns = lat.ns
    JXY = _per_site(jxy, ns)
    JZ = _per_site(jz, ns)
    if delta is not None:
        JZ = JXY * _per_site(delta, ns)
    HX, HZ = _per_site(hx, ns), _per_site(hz, ns)
    terms = []
    for i in range(ns):
        if _nz(HX, i):
            terms.append(Term("x", (i,), -HX[i]))
    for i in range(ns):
        if _nz(HZ, i):
            terms.append(Term("z", (i,), -HZ[i]))
    for i in range(ns):
        for jn in lat.nn_forward(i):
            cxy = JXY[i] * 1.0
            if not np.isclose(cxy, 0.0):
                terms.append(Term("x", (i, jn), -cxy))
                terms.append(Term("y", (i, jn), -cxy))
            cz = JZ[i] * 1.0
            if not np.isclose(cz, 0.0):
                terms.append(Term("z", (i, jn), -cz))
    return terms


def j1j2_terms(lat: SquareLattice, J1=1.0, J2=0.0, hx=None, hy=None, hz=None) -> List[Term]:
    ns = lat.ns
    J1v, J2v = _per_site(J1, ns), _per_site(J2, ns)
    HX, HY, HZ = _per_site(hx, ns), _per_site(hy, ns), _per_site(hz, ns)
    terms = []
    for i in range(ns):
        if _nz(HX, i):
            terms.append(Term("x", (i,), -HX[i]))
        if _nz(HY, i):
            terms.append(Term("y", (i,), -HY[i]))
        if _nz(HZ, i):
            terms.append(Term("z", (i,), -HZ[i]))

    def exch(m, i, jn):
        if np.isclose(m, 0.0):
            return
        terms.append(Term("x", (i, jn), m))
        terms.append(Term("y", (i, jn), m))
        terms.append(Term("z", (i, jn), m))

    for i in range(ns):
        for jn in lat.nn_forward(i):
            exch(-1.0 * J1v[i], i, jn)
    for i in range(ns):
        for jn in lat.nnn_forward(i):
            exch(-1.0 * J2v[i], i, jn)
    return terms


# ---------------------------------------------------------------------------
# operator action on one +-0.5 state
# ---------------------------------------------------------------------------

def apply_term(term: Term, state: np.ndarray):
    """Return (new_state, coefficient) of one term on a +-0.5 vector (mult included)."""
    sites = list(term.sites)
    sig = np.sign(state[sites])
    if term.op == "x":
        new = state.copy()
        new[sites] = -new[sites]
        c = SPIN_VALUE ** len(sites)
    elif term.op == "y":
        new = state.copy()
        new[sites] = -new[sites]
        c = np.prod(1j * SPIN_VALUE * sig)
    elif term.op == "z":
        new = state
        c = np.prod(SPIN_VALUE * sig)
    else:
        raise ValueError(term.op)
    return new, complex(c) * complex(term.mult)


def connected_raw(terms: Sequence[Term], state: np.ndarray):
    """Slot list of ``local_energy_jax_wrap`` for one state: (states (K,N), coeffs (K,))."""
    state = np.asarray(state, dtype=np.float64)
    diag = 0.0 + 0.0j
    groups = {}
    order = []
    for t in terms:
        if t.modifies:
            key = (t.op, len(t.sites))
            if key not in groups:
                groups[key] = []
                order.append(key)
            groups[key].append(t)
        else:
            diag += apply_term(t, state)[1]
    states = [state.copy()]
    coeffs = [diag]
    for key in order:
        for t in groups[key]:
            s2, c = apply_term(t, state)
            states.append(s2)
            coeffs.append(c)
    return np.stack(states), np.asarray(coeffs, dtype=np.complex128)


def connected_raw_batch(terms: Sequence[Term], states: np.ndarray):
    """``connected_raw`` for a batch: states (B, N) -> (B, K, N), (B, K); same slot order."""
    states = np.atleast_2d(np.asarray(states, dtype=np.float64))
    B = states.shape[0]
    sig = np.sign(states)
    diag = np.zeros(B, dtype=np.complex128)
    groups, order = {}, []
    for t in terms:
        if t.modifies:
            key = (t.op, len(t.sites))
            if key not in groups:
                groups[key] = []
                order.append(key)
            groups[key].append(t)
        else:
            diag += t.mult * np.prod(SPIN_VALUE * sig[:, list(t.sites)], axis=1)
    mods = [t for key in order for t in groups[key]]
    K = 1 + len(mods)
    out_s = np.repeat(states[:, None, :], K, axis=1)
    out_c = np.zeros((B, K), dtype=np.complex128)
    out_c[:, 0] = diag
    for k, t in enumerate(mods, start=1):
        s = list(t.sites)
        out_s[:, k, s] = -out_s[:, k, s]
        if t.op == "x":
            out_c[:, k] = SPIN_VALUE ** len(s) * t.mult
        else:
            out_c[:, k] = np.prod(1j * SPIN_VALUE * sig[:, s], axis=1) * t.mult
    return out_s, out_c


def connected_merged(terms: Sequence[Term], state: np.ndarray, drop_zero=True):
    """Merged multiset {s' -> sum c}: the physical connected set (keys are +-1 tuples)."""
    st, co = connected_raw(terms, state)
    out = {}
    for s2, c in zip(st, co):
        key = tuple(np.sign(s2).astype(int).tolist())
        out[key] = out.get(key, 0.0) + c
    if drop_zero:
        out = {k: v for k, v in out.items() if abs(v) > 1e-14}
    return out


# ---------------------------------------------------------------------------
# integer basis (big-endian: site i <-> bit ns-1-i, bit 1 <-> +0.5)
# ---------------------------------------------------------------------------

def int_to_state(n: int, ns: int) -> np.ndarray:
    bits = [(n >> (ns - 1 - i)) & 1 for i in range(ns)]
    return np.where(np.asarray(bits) == 1, SPIN_VALUE, -SPIN_VALUE).astype(np.float64)


def state_to_int(state) -> int:
    ns = len(state)
    out = 0
    for i, s in enumerate(state):
        if s > 0:
            out |= 1 << (ns - 1 - i)
    return out


def sparse_hamiltonian(terms: Sequence[Term], ns: int, n_up=None):
    """Sparse H in the S^z basis, optionally restricted to a fixed number of up spins.

    Returns (H, basis_ints).  H[r, c] = <basis[r]| H |basis[c]>, built column by
    column from the same ``apply_term`` the local energy uses.
    """
    if n_up is None:
        basis = np.arange(1 << ns, dtype=np.int64)
    else:
        allb = np.arange(1 << ns, dtype=np.int64)
        basis = allb[np.bitwise_count(allb) == n_up]
    nb_ = len(basis)
    rows, cols, vals = [], [], []
    # vectorised over the basis: all states of the basis as +-1 arrays
    shifts = np.arange(ns - 1, -1, -1, dtype=np.int64)
    sig = np.where(((basis[:, None] >> shifts[None, :]) & 1) == 1, 1.0, -1.0)
    diag = np.zeros(nb_, dtype=np.complex128)
    col_all = np.arange(nb_, dtype=np.int64)
    for t in terms:
        s = list(t.sites)
        if t.op == "z":
            diag += t.mult * np.prod(SPIN_VALUE * sig[:, s], axis=1)
            continue
        mask = 0
        for site in s:
            mask |= 1 << (ns - 1 - site)
        new = basis ^ mask
        if t.op == "x":
            c = np.full(nb_, SPIN_VALUE ** len(s), dtype=np.complex128)
        else:
            c = np.prod(1j * SPIN_VALUE * sig[:, s], axis=1)
        c = c * t.mult
        r = np.searchsorted(basis, new)
        r = np.minimum(r, nb_ - 1)
        ok = basis[r] == new
        rows.append(r[ok])
        cols.append(col_all[ok])
        vals.append(c[ok])
    rows.append(col_all)
    cols.append(col_all)
    vals.append(diag)
    H = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nb_, nb_)).tocsr()
    return H, basis
