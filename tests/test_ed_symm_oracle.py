"""The oracle's momentum / spin-flip sector ED against its plain S^z-sector ED (CPU only)."""

import numpy as np
import pytest

from oracle import lattice as olat, hamiltonian as oH, ed as oed


@pytest.mark.parametrize("L,k_gs", [(8, 0), (10, 1)])
def test_symmetric_oracle_ground_sector(L, k_gs):
    """Heisenberg chain: the ground state has momentum 0 for even N/2 and pi for odd N/2, flip
    parity (-1)^(N/2); the sector energy equals the S^z sector's, the other sectors lie above."""
    terms = oH.xxz_terms(olat.SquareLattice(1, L), -1.0, -1.0)
    n_up = L // 2
    e_sz = oed.ground_energy(terms, L, n_up=n_up)
    p_gs = 1 if n_up % 2 == 0 else -1
    e = {(p, k): oed.symmetric_ground_energy(terms, L, 1, n_up, p, k, 0) for p in (1, -1) for k in (0, 1)}
    assert e[(p_gs, k_gs)] == pytest.approx(e_sz, rel=1e-10)
    assert min(e.values()) == pytest.approx(e_sz, rel=1e-10)
    e0 = {k: oed.symmetric_ground_energy(terms, L, 1, n_up, 0, k, 0) for k in (0, 1)}
    assert e0[k_gs] == pytest.approx(e_sz, rel=1e-10)


def test_symmetric_oracle_dims_add_up():
    """With both flip parities the dimensions add up to the parity-free sector's."""
    for lx, ly in ((8, 1), (4, 2)):
        n_up = lx * ly // 2
        for kx in (0, 1):
            for ky in ((0, 1) if ly % 2 == 0 else (0,)):
                d0 = oed.symmetric_sector_dim(lx, ly, n_up, 0, kx, ky)
                dp = oed.symmetric_sector_dim(lx, ly, n_up, 1, kx, ky)
                dm = oed.symmetric_sector_dim(lx, ly, n_up, -1, kx, ky)
                assert d0 == dp + dm
    assert oed.symmetric_sector_dim(4, 4, 8, 1, 0, 0) == 441


def test_burnside_dims_match_enumeration():
    for lx, ly, n_up in ((8, 1, 4), (10, 1, 5), (10, 1, 3), (4, 2, 4), (4, 4, 8), (4, 4, 6), (3, 3, 4)):
        for parity in ((0, 1, -1) if 2 * n_up == lx * ly else (0,)):
            for kx in ((0, 1) if lx % 2 == 0 else (0,)):
                for ky in ((0, 1) if ly % 2 == 0 else (0,)):
                    assert oed.symmetric_sector_dim_burnside(lx, ly, n_up, parity, kx, ky) == \
                        oed.symmetric_sector_dim(lx, ly, n_up, parity, kx, ky), (lx, ly, n_up, parity, kx, ky)
    # the 6x6 J1-J2 workload's ground-state sector (k = 0, even flip, S^z = 0)
    assert oed.symmetric_sector_dim_burnside(6, 6, 18, 1, 0, 0) == 126056625


def test_ed_6x6_fixture_consistent():
    """The committed 6x6 J1-J2 energies: sector dimensions match the fixed-point count, and the
    recorded ground energy is the lowest J2 = 0.5 sector."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "ed_j1j2_6x6.json")) as f:
        fx = json.load(f)
    for r in fx["sectors"]:
        kx, ky = (int(m != 0) for m in r["momentum"])
        assert r["sector_dim"] == oed.symmetric_sector_dim_burnside(6, 6, r["n_up"], r["spin_flip"], kx, ky)
    e05 = [r["e0"] for r in fx["sectors"] if r["j2"] == 0.5]
    assert len(e05) >= 3 and fx["e0_j2_0.5"] == min(e05) == e05[0]
