"""TFIM / XXZ / J1-J2 spin-1/2 models and their lowering to the GPU move table.

Each model builds the reference's operator term list with the same
insertion order, signs and spin-1/2 normalisation:

* ``TransverseFieldIsing``  ``QES/Algebra/Model/Interacting/Spin/transverse_ising.py:192-300``
  terms -hx_i Sx_i, -hz_i Sz_i, -J_i Sz_i Sz_j (forward NN bonds);
* ``XXZ``                   ``xxz.py:278-433``: -hx Sx, -hz Sz, per bond -jxy (SxSx + SySy), -jz SzSz;
* ``J1J2Model``             ``j1j2.py:119-295``: fields, then -J1 (S.S) on NN, -J2 (S.S) on NNN
  (the code's literal sign: J1 = +1 is ferromagnetic, J1 = -1 antiferromagnetic).

A term is (op, sites, mult) with op in x/y/z acting on every listed site:
X flips with coefficient 0.5**k, Y flips with prod(i 0.5 sigma) on the state
before the flip, Z keeps the state with prod(0.5 sigma)
(``QES/Algebra/Operator/impl/jax/operators_spin.py:131-143,220-248,353-370``).

``lower()`` merges the terms into the device description used by the local
energy kernel: diagonal z-fields and zz-bonds, and off-diagonal *moves*
(single flips and pair flips) whose coefficient already carries the
conjugate that the estimator needs (E_loc(s) = sum conj(<s'|H|s>) psi(s')/psi(s)).
XX and YY slots of one bond merge into one pair move: anti-parallel spins
get (mx + my)/4, parallel spins (mx - my)/4, which is zero for the
isotropic models and then dropped.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple

import numpy as np

from .hilbert import HilbertSpace
from .lattice import SquareLattice, get_neighbor_table
from . import _lib

SPIN_VALUE = 0.5


@dataclass(frozen=True)
class Term:
    op: str
    sites: tuple
    mult: complex

    @property
    def modifies(self):
        return self.op in ("x", "y")


@dataclass
class LoweredHamiltonian:
    """Host arrays of the C struct ``qes_hamiltonian``."""
    ns: int
    move_i: np.ndarray
    move_j: np.ndarray
    move_kind: np.ndarray
    move_coef: np.ndarray          # (K, 4) float32: coefA re, im, coefB re, im
    zf_site: np.ndarray
    zf_h: np.ndarray
    zz_i: np.ndarray
    zz_j: np.ndarray
    zz_J: np.ndarray
    is_real: bool = True

    @property
    def n_moves(self):
        return int(self.move_i.shape[0])


def _coupling(v, ns):
    if v is None:
        return None
    if np.isscalar(v):
        return np.full(ns, float(np.real(v)))
    v = np.asarray(v, dtype=float)
    if v.shape != (ns,):
        raise ValueError("site-resolved couplings must have length ns")
    return v


def _nz(v, i):
    return v is not None and not np.isclose(v[i], 0.0)


class SpinHamiltonian:
    """Base: holds the lattice, Hilbert space and the ordered term list."""

    def __init__(self, lattice, hilbert_space=None, dtype=np.float64, backend="default", **kwargs):
        if lattice is None:
            raise ValueError(f"{type(self).__name__} requires a lattice")
        self.lattice = lattice
        self._lattice = lattice
        self.hilbert_space = hilbert_space if hilbert_space is not None else HilbertSpace(lattice=lattice)
        self.ns = lattice.ns
        self._dtype = dtype
        self.terms: List[Term] = []

    @property
    def hilbert(self):
        return self.hilbert_space

    def add(self, op, mult, sites):
        self.terms.append(Term(op, tuple(int(s) for s in sites), complex(mult)))

    # -- connected states of one +-0.5 state, in the reference slot order ----------------
    def connected(self, state):
        """(states (K, ns), coeffs (K,)) with the slot order of ``local_energy_jax_wrap``
        (``QES/Algebra/Hamil/hamil_energy_jax.py:428-576``): diagonal first, then the
        modifying terms grouped by (operator, arity) in order of first appearance."""
        state = np.asarray(state, dtype=np.float64)
        sig = np.where(state > 0, 1.0, -1.0)
        diag = 0j
        groups: Dict[Tuple[str, int], List[Term]] = {}
        for t in self.terms:
            if t.modifies:
                groups.setdefault((t.op, len(t.sites)), []).append(t)
            else:
                diag += t.mult * np.prod(SPIN_VALUE * sig[list(t.sites)])
        states, coeffs = [state.copy()], [diag]
        for key in groups:
            for t in groups[key]:
                s = list(t.sites)
                new = state.copy()
                new[s] = -new[s]
                c = SPIN_VALUE ** len(s) if t.op == "x" else np.prod(1j * SPIN_VALUE * sig[s])
                states.append(new)
                coeffs.append(c * t.mult)
        return np.stack(states), np.asarray(coeffs, dtype=np.complex128)

    def get_loc_energy_fun(self):
        return self.connected

    # -- exact ground energy -------------------------------------------------------------
    def diagonalize(self, method: str = "lanczos", k: int = 1, tol: float = 1e-12, maxiter: int = 600,
                    seed: int = 7, n_up=None, spin_flip=None, momentum=None, **kwargs):
        """Ground energy by Lanczos on the GPU (``qes_ed_lanczos``: the full 2^ns basis; with ``n_up``,
        ``qes_ed_lanczos_sector``: the S^z sector of n_up up spins, and with ``spin_flip`` = +1 / -1
        also one spin-flip parity, for S^z-conserving models without a field).  With ``momentum``
        (the translation sector index per axis, ``n`` or ``(nx, ny)``, each 0 or L/2 as in
        ``QES/Algebra/Symmetries/translation.py:196-262``; periodic lattices only),
        ``qes_ed_lanczos_symm``: the sector reduced by the lattice translations as well; the sector
        dimension is stored in ``sector_dim``.

        Mirrors ``model.diagonalize(method='lanczos')`` (``QES/Algebra/hamil.py:1809``) for the
        lowest eigenvalue: the result is stored in ``eig_val`` (ascending, length 1).
        """
        if str(method).lower() not in ("lanczos", "auto", "exact"):
            raise NotImplementedError(f"diagonalize(method={method!r}): the GPU path implements Lanczos")
        if int(k) != 1:
            raise NotImplementedError("the GPU Lanczos returns the ground energy only (k=1)")
        import ctypes as C
        import torch
        from . import _lib, device as dv
        dh = dv.DeviceHamiltonian(self.lower())
        if momentum is not None:
            return self._diagonalize_symm(dh, n_up, spin_flip, momentum, maxiter, tol, seed)
        if n_up is not None or spin_flip is not None:
            n_up = self.ns // 2 if n_up is None else int(n_up)
            parity = 0 if spin_flip in (None, 0) else (1 if int(spin_flip) > 0 else -1)
            nb = C.c_size_t(0)
            _lib.call("qes_ed_sector_workspace_bytes", self.ns, n_up, parity, C.byref(nb))
            ws = torch.empty((int(nb.value),), dtype=torch.uint8, device="cuda")
            e0, its = C.c_double(0.0), C.c_int(0)
            _lib.call("qes_ed_lanczos_sector", self.ns, n_up, parity, C.byref(dh.struct), int(maxiter), float(tol),
                      C.c_uint64(int(seed)), C.byref(e0), C.byref(its), _lib.ptr(ws), int(ws.numel()),
                      _lib.stream_ptr())
            del ws
            self._eig_val = np.array([e0.value])
            self.lanczos_iterations = its.value
            return self._eig_val
        nb = C.c_size_t(0)
        _lib.call("qes_ed_workspace_bytes", self.ns, C.byref(nb))
        ws = torch.empty((int(nb.value),), dtype=torch.uint8, device="cuda")
        e0, its = C.c_double(0.0), C.c_int(0)
        _lib.call("qes_ed_lanczos", self.ns, C.byref(dh.struct), int(maxiter), float(tol),
                  C.c_uint64(int(seed)), C.byref(e0), C.byref(its), _lib.ptr(ws), int(ws.numel()),
                  _lib.stream_ptr())
        self._eig_val = np.array([e0.value])
        self.lanczos_iterations = its.value
        return self._eig_val

    def _diagonalize_symm(self, dh, n_up, spin_flip, momentum, maxiter, tol, seed):
        import ctypes as C
        import torch
        from . import _lib
        lat = self.lattice
        lx, ly = int(getattr(lat, "lx", self.ns)), int(getattr(lat, "ly", 1))
        if lx * ly != self.ns or str(getattr(lat, "bc", "pbc")).lower() != "pbc":
            raise ValueError("diagonalize(momentum=...): needs a periodic lx x ly lattice")
        mom = (momentum,) if np.isscalar(momentum) else tuple(momentum)
        mom = tuple(int(m) for m in mom) + (0,) * (2 - len(mom))
        k = []
        for n, size in zip(mom, (lx, ly)):
            n %= size
            if n == 0:
                k.append(0)
            elif 2 * n == size:
                k.append(1)
            else:
                raise NotImplementedError("diagonalize(momentum=...): sector index 0 or L/2 per axis "
                                          "(the real characters)")
        n_up = self.ns // 2 if n_up is None else int(n_up)
        parity = 0 if spin_flip in (None, 0) else (1 if int(spin_flip) > 0 else -1)
        args = (lx, ly, n_up, parity, k[0], k[1])
        nb = C.c_size_t(0)
        _lib.call("qes_ed_symm_workspace_bytes", *args, C.c_uint64(0), C.byref(nb))
        ws = torch.empty((int(nb.value),), dtype=torch.uint8, device="cuda")
        dim = C.c_uint64(0)
        _lib.call("qes_ed_symm_dim", *args, C.byref(dim), _lib.ptr(ws), int(ws.numel()), _lib.stream_ptr())
        if dim.value == 0:
            raise ValueError(f"diagonalize: the sector {dict(n_up=n_up, spin_flip=parity, momentum=mom)} is empty")
        _lib.call("qes_ed_symm_workspace_bytes", *args, C.c_uint64(dim.value), C.byref(nb))
        del ws
        ws = torch.empty((int(nb.value),), dtype=torch.uint8, device="cuda")
        e0, its, d2 = C.c_double(0.0), C.c_int(0), C.c_uint64(0)
        _lib.call("qes_ed_lanczos_symm", *args, C.byref(dh.struct), int(maxiter), float(tol), C.c_uint64(int(seed)),
                  C.byref(e0), C.byref(its), C.byref(d2), _lib.ptr(ws), int(ws.numel()), _lib.stream_ptr())
        del ws
        self._eig_val = np.array([e0.value])
        self.lanczos_iterations = its.value
        self.sector_dim = int(d2.value)
        return self._eig_val

    @property
    def eig_val(self):
        return getattr(self, "_eig_val", None)

    # -- lowering -----------------------------------------------------------------------
    def lower(self) -> LoweredHamiltonian:
        zf: Dict[int, complex] = {}
        zz: Dict[Tuple[int, int], complex] = {}
        flips: Dict[int, List[complex]] = {}
        pairs: Dict[Tuple[int, int], List[complex]] = {}
        order: List[Tuple[str, object]] = []
        for t in self.terms:
            s = t.sites
            if t.op == "z":
                if len(s) == 1:
                    zf[s[0]] = zf.get(s[0], 0j) + t.mult * SPIN_VALUE
                elif len(s) == 2:
                    zz[s] = zz.get(s, 0j) + t.mult * SPIN_VALUE ** 2
                else:
                    raise NotImplementedError("z terms on more than two sites are not lowered")
                continue
            if len(s) == 1:
                if s[0] not in flips:
                    flips[s[0]] = [0j, 0j]
                    order.append(("f", s[0]))
                flips[s[0]][0 if t.op == "x" else 1] += t.mult
            elif len(s) == 2:
                if s[0] == s[1]:
                    raise ValueError("pair term on one site")
                if s not in pairs:
                    pairs[s] = [0j, 0j]
                    order.append(("p", s))
                pairs[s][0 if t.op == "x" else 1] += t.mult
            else:
                raise NotImplementedError("flip terms on more than two sites are not lowered")
        mi, mj, mk, mc = [], [], [], []
        for kind, key in order:
            if kind == "f":
                mx, my = flips[key]
                cA = np.conj(mx) * SPIN_VALUE
                cB = -1j * np.conj(my) * SPIN_VALUE
                if abs(cA) == 0 and abs(cB) == 0:
                    continue
                mi.append(key); mj.append(-1); mk.append(_lib.MOVE_FLIP1)
                mc.append([cA.real, cA.imag, cB.real, cB.imag])
            else:
                mx, my = pairs[key]
                anti = np.conj(mx + my) * SPIN_VALUE ** 2
                par = np.conj(mx - my) * SPIN_VALUE ** 2
                if abs(anti) > 0:
                    mi.append(key[0]); mj.append(key[1]); mk.append(_lib.MOVE_PAIR_ANTI)
                    mc.append([anti.real, anti.imag, 0.0, 0.0])
                if abs(par) > 0:
                    mi.append(key[0]); mj.append(key[1]); mk.append(_lib.MOVE_PAIR_PAR)
                    mc.append([par.real, par.imag, 0.0, 0.0])
        diag_vals = list(zf.values()) + list(zz.values())
        if any(abs(np.imag(v)) > 0 for v in diag_vals):
            raise NotImplementedError("complex diagonal couplings are not lowered")
        is_real = all(abs(c[1]) == 0 and abs(c[2]) == 0 and abs(c[3]) == 0 for c in mc)
        return LoweredHamiltonian(
            ns=self.ns,
            move_i=np.asarray(mi, dtype=np.int32).reshape(-1),
            move_j=np.asarray(mj, dtype=np.int32).reshape(-1),
            move_kind=np.asarray(mk, dtype=np.int32).reshape(-1),
            move_coef=np.asarray(mc, dtype=np.float32).reshape(-1, 4),
            zf_site=np.asarray(list(zf.keys()), dtype=np.int32),
            zf_h=np.asarray([np.real(v) for v in zf.values()], dtype=np.float32),
            zz_i=np.asarray([k[0] for k in zz.keys()], dtype=np.int32),
            zz_j=np.asarray([k[1] for k in zz.keys()], dtype=np.int32),
            zz_J=np.asarray([np.real(v) for v in zz.values()], dtype=np.float32),
            is_real=is_real,
        )

    def neighbor_table(self, order=1):
        return get_neighbor_table(self.lattice, order=order)


class TransverseFieldIsing(SpinHamiltonian):
    def __init__(self, lattice, hilbert_space=None, j=1.0, hx=1.0, hz=1.0, operator_family="auto",
                 dtype=np.float64, backend="default", **kwargs):
        super().__init__(lattice, hilbert_space, dtype, backend, **kwargs)
        self._name = "Transverse Field Ising Model"
        ns = self.ns
        self._j, self._hx, self._hz = _coupling(j, ns), _coupling(hx, ns), _coupling(hz, ns)
        for i in range(ns):
            if _nz(self._hx, i):
                self.add("x", -self._hx[i], [i])
        for i in range(ns):
            if _nz(self._hz, i):
                self.add("z", -self._hz[i], [i])
        for i in range(ns):
            for nidx in range(lattice.get_nn_forward_num(i)):
                jn = lattice.get_nn_forward(i, num=nidx)
                if lattice.wrong_nei(jn):
                    continue
                phase = lattice.boundary_phase_from_winding(*lattice.bond_winding(i, jn))
                if not _nz(self._j, i):
                    continue
                self.add("z", -self._j[i] * phase, [i, int(jn)])


class XXZ(SpinHamiltonian):
    def __init__(self, lattice, hilbert_space=None, jxy=1.0, jz=1.0, delta=None, hx=0.0, hz=0.0,
                 operator_family="auto", dtype=np.float64, backend="default", **kwargs):
        super().__init__(lattice, hilbert_space, dtype, backend, **kwargs)
        self._name = "XXZ"
        ns = self.ns
        self._jxy = _coupling(jxy, ns)
        self._jz = _coupling(jz, ns)
        if delta is not None:
            self._jz = self._jxy * _coupling(delta, ns)
        self._hx, self._hz = _coupling(hx, ns), _coupling(hz, ns)
        if self._hx is not None:
            for i in range(ns):
                if not np.isclose(self._hx[i], 0.0):
                    self.add("x", -self._hx[i], [i])
        if self._hz is not None:
            for i in range(ns):
                if not np.isclose(self._hz[i], 0.0):
                    self.add("z", -self._hz[i], [i])
        for i in range(ns):
            for nidx in range(lattice.get_nn_forward_num(i)):
                jn = lattice.get_nn_forward(i, num=nidx)
                if lattice.wrong_nei(jn):
                    continue
                phase = lattice.boundary_phase_from_winding(*lattice.bond_winding(i, jn))
                if self._jxy is not None:
                    cxy = self._jxy[i] * phase
                    if not np.isclose(cxy, 0.0):
                        self.add("x", -cxy, [i, int(jn)])
                        self.add("y", -cxy, [i, int(jn)])
                if self._jz is not None:
                    cz = self._jz[i] * phase
                    if not np.isclose(cz, 0.0):
                        self.add("z", -cz, [i, int(jn)])


class J1J2Model(SpinHamiltonian):
    def __init__(self, lattice, J1=1.0, J2=0.0, *, hilbert_space=None, hx=None, hy=None, hz=None,
                 impurities=None, operator_family="auto", dtype=np.float64, backend="default",
                 use_forward=True, **kwargs):
        super().__init__(lattice, hilbert_space, dtype, backend, **kwargs)
        if impurities:
            raise NotImplementedError("classical impurities are outside the RBM-VMC path")
        self._name = "J1-J2"
        ns = self.ns
        self._j1, self._j2 = _coupling(J1, ns), _coupling(J2, ns)
        self._hx, self._hy, self._hz = _coupling(hx, ns), _coupling(hy, ns), _coupling(hz, ns)
        for i in range(ns):
            if _nz(self._hx, i):
                self.add("x", -self._hx[i], [i])
            if _nz(self._hy, i):
                self.add("y", -self._hy[i], [i])
            if _nz(self._hz, i):
                self.add("z", -self._hz[i], [i])

        def exch(mult, i, j):
            if np.isclose(mult, 0.0):
                return
            self.add("x", mult, [i, j])
            self.add("y", mult, [i, j])
            self.add("z", mult, [i, j])

        for i in range(ns):
            for nidx in range(lattice.get_nn_forward_num(i)):
                j = lattice.get_nn_forward(i, num=nidx)
                if lattice.wrong_nei(j) or int(j) == i:
                    continue
                phase = lattice.boundary_phase_from_winding(*lattice.bond_winding(i, j))
                exch(-phase * self._j1[i], i, int(j))
        if hasattr(lattice, "get_nnn_forward_num"):
            for i in range(ns):
                for nidx in range(lattice.get_nnn_forward_num(i)):
                    j = lattice.get_nnn_forward(i, num=nidx)
                    if lattice.wrong_nei(j) or int(j) == i:
                        continue
                    phase = lattice.boundary_phase_from_winding(*lattice.bond_winding(i, j))
                    exch(-phase * self._j2[i], i, int(j))


class SpinOperator(SpinHamiltonian):
    """A spin-1/2 operator on a lattice as an ordered term list, evaluated by the same lowering and
    ratio kernel as the models (observables of ``NQS.compute_observable`` / ``NQS.measure``).

    Terms use the reference's operator conventions (X flips with 0.5**k, Y flips with prod(i 0.5 sigma)
    on the state before the flip, Z keeps the state with prod(0.5 sigma);
    ``QES/Algebra/Operator/impl/jax/operators_spin.py:131-143,220-248,353-370``); z terms act on one or
    two sites, x / y terms flip one or two sites.  The constructors below build the common ones."""

    def __init__(self, lattice, terms=(), name="O", **kwargs):
        super().__init__(lattice, **kwargs)
        self.name = name
        for op, mult, sites in terms:
            self.add(op, mult, sites)

    @classmethod
    def sigma(cls, lattice, op, site, mult=1.0):
        """S^op on one site (op in x, y, z)."""
        return cls(lattice, [(op, mult, (site,))], name=f"S{op}_{site}")

    @classmethod
    def magnetization(cls, lattice, op="z"):
        """(1 / N) sum_i S^op_i."""
        return cls(lattice, [(op, 1.0 / lattice.ns, (i,)) for i in range(lattice.ns)], name=f"M{op}")

    @classmethod
    def correlation(cls, lattice, i, j, op="z"):
        """S^op_i S^op_j (i != j)."""
        if i == j:
            raise ValueError("correlation needs two distinct sites")
        return cls(lattice, [(op, 1.0, (i, j))], name=f"S{op}{op}_{i}_{j}")

    @classmethod
    def exchange(cls, lattice, i, j):
        """S_i . S_j = SxSx + SySy + SzSz on two distinct sites."""
        if i == j:
            raise ValueError("exchange needs two distinct sites")
        return cls(lattice, [("x", 1.0, (i, j)), ("y", 1.0, (i, j)), ("z", 1.0, (i, j))], name=f"SS_{i}_{j}")
