"""GPU Lanczos ground energy and matrix-free H x against the oracle's sparse S^z-basis H."""

import ctypes as C

import numpy as np
import pytest
import torch

from oracle import lattice as olat, hamiltonian as oH, ed as oed
import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib

pytestmark = pytest.mark.gpu


def _models():
    return [
        ("tfim_chain12", qb.TransverseFieldIsing(qb.SquareLattice(1, 12, 1, bc="pbc"), j=1.0, hx=0.7, hz=0.0),
         oH.tfim_terms(olat.SquareLattice(1, 12, 1, "pbc"), 1.0, 0.7, 0.0)),
        ("tfim_4x4_hz", qb.TransverseFieldIsing(qb.SquareLattice(2, 4, 4, bc="pbc"), j=1.0, hx=3.04, hz=0.2),
         oH.tfim_terms(olat.SquareLattice(2, 4, 4, "pbc"), 1.0, 3.04, 0.2)),
        ("xxz_4x4", qb.XXZ(qb.SquareLattice(2, 4, 4, bc="pbc"), jxy=-1.0, jz=-1.0),
         oH.xxz_terms(olat.SquareLattice(2, 4, 4, "pbc"), -1.0, -1.0)),
        ("j1j2_4x4", qb.J1J2Model(qb.SquareLattice(2, 4, 4, bc="pbc"), J1=-1.0, J2=-0.5),
         oH.j1j2_terms(olat.SquareLattice(2, 4, 4, "pbc"), -1.0, -0.5)),
    ]


def _bitrev(idx, ns):
    out = np.zeros_like(idx)
    for i in range(ns):
        out |= ((idx >> (ns - 1 - i)) & 1) << i
    return out


@pytest.mark.parametrize("k", range(4))
def test_ed_matvec_matches_oracle_matrix(k):
    name, model, terms = _models()[k]
    ns = model.ns
    H, basis = oH.sparse_hamiltonian(terms, ns, n_up=None)
    rng = np.random.default_rng(k)
    x_or = rng.normal(size=1 << ns)
    y_or = (H @ x_or).real
    perm = _bitrev(basis, ns)             # oracle row r (site i = bit ns-1-i) -> library index (site i = bit i)
    x = np.empty_like(x_or)
    x[perm] = x_or
    dh = dv.DeviceHamiltonian(model.lower())
    xd = torch.as_tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    _lib.call("qes_ed_matvec", ns, C.byref(dh.struct), _lib.ptr(xd), _lib.ptr(yd), _lib.stream_ptr())
    y = yd.cpu().numpy()[perm]
    assert np.max(np.abs(y - y_or)) <= 1e-5 * np.max(np.abs(y_or)), name   # float32 coefficients


@pytest.mark.parametrize("k", range(4))
def test_ed_lanczos_ground_energy_matches_oracle(k):
    name, model, terms = _models()[k]
    e_ref = oed.ground_energy(terms, model.ns, n_up=None)
    e = model.diagonalize(method="lanczos")[0]
    assert abs(e - e_ref) <= 1e-6 * abs(e_ref), (name, e, e_ref)


def test_ed_rejects_large_or_bad_input():
    model = qb.TransverseFieldIsing(qb.SquareLattice(1, 40, 1, bc="pbc"), j=1.0, hx=1.0, hz=0.0)
    with pytest.raises(_lib.QESError):
        model.diagonalize()


# ------------------------------------------------------------------------- S^z sectors and spin-flip parity
@pytest.mark.gpu
def test_sector_lanczos_matches_oracle_and_full_basis():
    """S^z-sector Lanczos (colex-ranked basis) against the oracle's sector ED, and the spin-flip
    parities against the sector: min over parities = the sector's ground energy."""
    L, OL = qb.SquareLattice(2, 4, 4), olat.SquareLattice(2, 4, 4)
    model = qb.J1J2Model(L, J1=-1.0, J2=-0.5)
    terms = oH.j1j2_terms(OL, -1.0, -0.5)
    e8 = float(model.diagonalize(n_up=8)[0])
    assert e8 == pytest.approx(oed.ground_energy(terms, 16, n_up=8), rel=1e-6)
    e7 = float(model.diagonalize(n_up=7)[0])
    assert e7 == pytest.approx(oed.ground_energy(terms, 16, n_up=7), rel=1e-6)
    ep = float(model.diagonalize(n_up=8, spin_flip=+1)[0])
    em = float(model.diagonalize(n_up=8, spin_flip=-1)[0])
    assert min(ep, em) == pytest.approx(e8, rel=1e-8) and max(ep, em) >= e8 - 1e-9
    full = float(model.diagonalize()[0])
    assert min(e8, e7) == pytest.approx(full, rel=1e-8) or full < min(e8, e7)


@pytest.mark.gpu
def test_sector_lanczos_xxz_chain_all_sectors():
    L, OL = qb.SquareLattice(1, 12), olat.SquareLattice(1, 12)
    model = qb.XXZ(L, jxy=-1.0, jz=-0.6, hz=0.3)
    terms = oH.xxz_terms(OL, -1.0, -0.6, hz=0.3)
    es = [float(model.diagonalize(n_up=u)[0]) for u in range(13)]
    # the lowered couplings are float32 (0.6 / 4 is not exact): 1e-6 relative
    for u in (0, 3, 6, 11):
        assert es[u] == pytest.approx(oed.ground_energy(terms, 12, n_up=u), rel=1e-6, abs=1e-10)
    assert min(es) == pytest.approx(float(model.diagonalize()[0]), rel=1e-8)
    with pytest.raises(_lib.QESError):
        model.diagonalize(n_up=6, spin_flip=1)             # a z field breaks the spin-flip parity
    tfim = qb.TransverseFieldIsing(L, j=1.0, hx=0.5, hz=0.0)
    with pytest.raises(_lib.QESError):
        tfim.diagonalize(n_up=6)                           # single flips do not conserve S^z


# ------------------------------------------------------------------------- translation sectors
def _j1j2(lx, ly, j2):
    dim = 2 if ly > 1 else 1
    return (qb.J1J2Model(qb.SquareLattice(dim, lx, ly), J1=-1.0, J2=-j2),
            oH.j1j2_terms(olat.SquareLattice(dim, lx, ly), -1.0, -j2))


@pytest.mark.parametrize("lx,ly,j2,sectors", [
    (10, 1, 0.0, [(0, 0, 0), (0, 5, 0), (1, 0, 0), (1, 5, 0), (-1, 0, 0), (-1, 5, 0)]),
    (12, 1, 0.3, [(0, 0, 0), (1, 6, 0), (-1, 6, 0)]),
    (4, 4, 0.5, [(0, 0, 0), (0, 2, 2), (1, 0, 0), (1, 2, 0), (1, 0, 2), (1, 2, 2), (-1, 0, 0), (-1, 2, 2)]),
    (4, 2, 0.5, [(1, 0, 1), (-1, 2, 0)]),
    (3, 3, 0.0, [(0, 0, 0)]),
])
def test_symm_lanczos_matches_projector_oracle(lx, ly, j2, sectors):
    """Translation (+ spin-flip) reduced Lanczos against the oracle's H + lam (1 - P) in the full
    S^z sector (no representatives, no orbit norms), and the sector dimension against trace P."""
    model, terms = _j1j2(lx, ly, j2)
    ns = lx * ly
    n_up = ns // 2
    for parity, nx, ny in sectors:
        kx, ky = int(nx != 0), int(ny != 0)
        e = float(model.diagonalize(n_up=n_up, spin_flip=parity, momentum=(nx, ny))[0])
        e_ref = oed.symmetric_ground_energy(terms, lx, ly, n_up, parity, kx, ky)
        assert e == pytest.approx(e_ref, rel=1e-9, abs=1e-9), (parity, nx, ny, e, e_ref)
        assert model.sector_dim == oed.symmetric_sector_dim(lx, ly, n_up, parity, kx, ky)


def test_symm_lanczos_ground_sector_and_xxz_field():
    """The 4x4 J1-J2 ground state sits at k = 0 with even flip parity: that sector's energy equals
    the S^z sector's; an XXZ chain in a uniform field (no parity) against the oracle."""
    model, _ = _j1j2(4, 4, 0.5)
    e_sz = float(model.diagonalize(n_up=8)[0])
    e_k0 = float(model.diagonalize(n_up=8, spin_flip=1, momentum=(0, 0))[0])
    assert e_k0 == pytest.approx(e_sz, rel=1e-10)
    assert model.sector_dim == 441
    L, OL = qb.SquareLattice(1, 12), olat.SquareLattice(1, 12)
    xxz = qb.XXZ(L, jxy=-1.0, jz=-0.6, hz=0.3)
    terms = oH.xxz_terms(OL, -1.0, -0.6, hz=0.3)
    for n_up, n in ((5, 0), (6, 6), (4, 6)):
        e = float(xxz.diagonalize(n_up=n_up, momentum=n)[0])
        e_ref = oed.symmetric_ground_energy(terms, 12, 1, n_up, 0, int(n != 0), 0)
        assert e == pytest.approx(e_ref, rel=1e-6, abs=1e-8)      # float32 couplings (0.6 / 4)


def test_symm_lanczos_rejects():
    L = qb.SquareLattice(1, 12)
    with pytest.raises(_lib.QESError):                                    # single flips
        qb.TransverseFieldIsing(L, j=1.0, hx=0.5, hz=0.0).diagonalize(n_up=6, momentum=0)
    j1 = np.ones(12)
    j1[3] = 0.7
    with pytest.raises(_lib.QESError):                                    # not translation invariant
        qb.J1J2Model(L, J1=-j1, J2=0.0).diagonalize(n_up=6, momentum=0)
    with pytest.raises(_lib.QESError):                                    # a field breaks the flip parity
        qb.XXZ(L, jxy=-1.0, jz=-1.0, hz=0.3).diagonalize(n_up=6, spin_flip=1, momentum=0)
    with pytest.raises(NotImplementedError):                              # complex characters
        qb.J1J2Model(L, J1=-1.0, J2=0.0).diagonalize(n_up=6, momentum=3)
    with pytest.raises(ValueError):                                       # open boundaries
        qb.J1J2Model(qb.SquareLattice(1, 12, bc="obc"), J1=-1.0, J2=0.0).diagonalize(n_up=6, momentum=0)
    with pytest.raises(ValueError):                                       # empty sector
        qb.J1J2Model(qb.SquareLattice(1, 4), J1=-1.0, J2=0.0).diagonalize(n_up=2, spin_flip=-1, momentum=0)


def test_symm_dim_6x6_matches_burnside():
    """Device enumeration of the 6x6 S^z = 0 sectors (4.5e9 / 9.1e9 ranks) against the oracle's
    fixed-point count."""
    for parity, kx, ky in ((1, 0, 0), (-1, 1, 1), (0, 1, 0)):
        nb = C.c_size_t(0)
        _lib.call("qes_ed_symm_workspace_bytes", 6, 6, 18, parity, kx, ky, C.c_uint64(0), C.byref(nb))
        ws = torch.empty((int(nb.value),), dtype=torch.uint8, device="cuda")
        dim = C.c_uint64(0)
        _lib.call("qes_ed_symm_dim", 6, 6, 18, parity, kx, ky, C.byref(dim), _lib.ptr(ws), int(ws.numel()),
                  _lib.stream_ptr())
        assert dim.value == oed.symmetric_sector_dim_burnside(6, 6, 18, parity, kx, ky)
