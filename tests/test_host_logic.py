"""Host-side logic of the package against the oracle, and the C-ABI library exports (no GPU)."""

import ctypes
import os
import re

import numpy as np
import pytest
import torch

from oracle import lattice as olat, hamiltonian as oH
import pyqusolver_b200 as qb
from pyqusolver_b200 import _lib, device as dv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _models():
    out = []
    l1 = qb.SquareLattice(1, 8, bc="pbc")
    o1 = olat.SquareLattice(1, 8, bc="pbc")
    out.append(("tfim1d", qb.TransverseFieldIsing(l1, j=1.0, hx=0.7, hz=0.3), oH.tfim_terms(o1, 1.0, 0.7, 0.3), 8))
    l2 = qb.SquareLattice(2, 4, 4, bc="pbc")
    o2 = olat.SquareLattice(2, 4, 4, bc="pbc")
    out.append(("xxz2d", qb.XXZ(l2, jxy=-1.0, jz=-0.7, hx=0.2), oH.xxz_terms(o2, -1.0, -0.7, hx=0.2), 16))
    out.append(("j1j2", qb.J1J2Model(l2, J1=-1.0, J2=-0.5, hy=0.3, hz=0.1),
                oH.j1j2_terms(o2, -1.0, -0.5, hy=0.3, hz=0.1), 16))
    l3 = qb.SquareLattice(1, 6, bc="obc")
    o3 = olat.SquareLattice(1, 6, bc="obc")
    out.append(("tfim_obc", qb.TransverseFieldIsing(l3, j=[1.0, 0.5, 0.0, 2.0, 1.0, 1.0], hx=1.0, hz=0.0),
                oH.tfim_terms(o3, [1.0, 0.5, 0.0, 2.0, 1.0, 1.0], 1.0, 0.0), 6))
    return out


@pytest.mark.parametrize("name,model,terms,ns", _models(), ids=[m[0] for m in _models()])
def test_term_lists_and_raw_slots_bit_exact(name, model, terms, ns):
    pkg = [(t.op, t.sites, complex(t.mult)) for t in model.terms]
    ora = [(t.op, tuple(t.sites), complex(t.mult)) for t in terms]
    assert pkg == ora
    rng = np.random.default_rng(0)
    for _ in range(5):
        s = np.where(rng.random(ns) < 0.5, 0.5, -0.5)
        st_p, co_p = model.connected(s)
        st_o, co_o = oH.connected_raw(terms, s)
        assert np.array_equal(st_p, st_o)
        assert np.array_equal(co_p, co_o)


def _lowered_merged(low, s):
    """Evaluate the lowered move table on one state: {sigma' tuple: conj(coefficient)} plus diagonal."""
    sig = np.where(np.asarray(s) > 0, 1, -1)
    out = {}
    diag = float(np.sum(low.zf_h * sig[low.zf_site])) + float(np.sum(low.zz_J * sig[low.zz_i] * sig[low.zz_j]))
    out[tuple(sig.tolist())] = diag
    for k in range(low.n_moves):
        i, j, kind = int(low.move_i[k]), int(low.move_j[k]), int(low.move_kind[k])
        c = low.move_coef[k]
        if kind == _lib.MOVE_FLIP1:
            coef = complex(c[0], c[1]) + sig[i] * complex(c[2], c[3])
            new = sig.copy()
            new[i] = -new[i]
        else:
            if (kind == _lib.MOVE_PAIR_ANTI) != (sig[i] != sig[j]):
                continue
            coef = complex(c[0], c[1])
            new = sig.copy()
            new[i] = -new[i]
            new[j] = -new[j]
        key = tuple(new.tolist())
        out[key] = out.get(key, 0) + coef
    return {k: v for k, v in out.items() if abs(v) > 1e-7}


@pytest.mark.parametrize("name,model,terms,ns", _models(), ids=[m[0] for m in _models()])
def test_lowered_moves_match_merged_connected_set(name, model, terms, ns):
    low = model.lower()
    rng = np.random.default_rng(1)
    for _ in range(8):
        s = np.where(rng.random(ns) < 0.5, 0.5, -0.5)
        ref = oH.connected_merged(terms, s)
        ref = {k: np.conj(v) for k, v in ref.items() if abs(v) > 1e-7}   # E_loc uses conj(<s'|H|s>)
        got = _lowered_merged(low, s)
        assert set(ref) == set(got)
        for k in ref:
            assert got[k] == pytest.approx(ref[k], abs=1e-6)


def test_isotropic_models_have_no_parallel_pair_moves():
    l2 = qb.SquareLattice(2, 6, 6, bc="pbc")
    low = qb.J1J2Model(l2, J1=-1.0, J2=-0.5).lower()
    assert set(low.move_kind.tolist()) == {_lib.MOVE_PAIR_ANTI}
    assert low.n_moves == 72 + 72
    low = qb.XXZ(qb.SquareLattice(2, 10, 10), jxy=-1.0, jz=-1.0).lower()
    assert low.n_moves == 200 and low.zz_i.size == 200


def test_neighbor_tables_match_oracle():
    for dim, lx, ly, bc in [(1, 7, 1, "pbc"), (2, 4, 4, "pbc"), (2, 6, 6, "pbc"), (2, 3, 5, "obc")]:
        a = qb.get_neighbor_table(qb.SquareLattice(dim, lx, ly, bc=bc))
        b = olat.neighbor_table(olat.SquareLattice(dim, lx, ly, bc=bc))
        assert np.array_equal(a, b)
    a = qb.get_neighbor_table(qb.SquareLattice(2, 5, 5), order=2)
    b = olat.neighbor_table(olat.SquareLattice(2, 5, 5), order=2)
    assert np.array_equal(a, b)


def test_pack_unpack_round_trip_cpu():
    rng = np.random.default_rng(5)
    for ns in (1, 16, 31, 32, 33, 100, 400):
        s = np.where(rng.random((7, ns)) < 0.5, 0.5, -0.5).astype(np.float32)
        w = dv.pack_states(s, device="cpu")
        assert w.shape == (7, (ns + 31) // 32)
        back = dv.unpack_states(w, ns).numpy()
        assert np.array_equal(back, s)


def test_hilbert_integer_convention():
    h = qb.HilbertSpace(ns=4)
    st = h.int_to_state(0b0010)
    assert st.tolist() == [-0.5, -0.5, 0.5, -0.5]
    assert h.state_to_int(st) == 2


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "qes_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qes_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert _header_symbols() == sorted(_lib.SIGNATURES)


def test_library_loads_and_exports_every_header_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in _header_symbols():
        assert hasattr(lib, name), name
    # host-only calls need no GPU
    lib.qes_version.restype = ctypes.c_int
    assert lib.qes_version() >= 100
    nb = ctypes.c_size_t(0)
    _lib.load()
    assert _lib.call("qes_sr_workspace_bytes", 1, 100, 200, 16384, ctypes.byref(nb)) == 0 and nb.value > 0
    assert _lib.call("qes_local_energy_workspace_bytes", 1, 100, 200, 16384, 200, ctypes.byref(nb)) == 0


def test_library_rejects_bad_arguments_without_gpu():
    _lib.load()
    with pytest.raises(_lib.QESError) as e:
        _lib.call("qes_init_chains", 1, 99, 0, 0, 4, 10, None, None)
    assert e.value.code == _lib.QES_ERR_ARG
    with pytest.raises(_lib.QESError):
        _lib.call("qes_rbm_forward", 7, 4, 4, 1, None, None, None, None, None, None, None, None)
    with pytest.raises(_lib.QESError) as e:
        _lib.call("qes_sampler_set_capped", 3)
    assert e.value.code == _lib.QES_ERR_ARG


def test_torch_ops_are_registered():
    import torch
    import pyqusolver_b200.ops  # noqa: F401  (registration only; no GPU call)
    for name in ("rbm_forward", "log_derivatives", "logpsi_vjp", "sr_matvec", "sr_solve_cg", "loss_stats"):
        assert hasattr(torch.ops.qes_b200, name)


def test_checkpoint_manager_roundtrip(tmp_path):
    from pyqusolver_b200.checkpoint import NQSCheckpointManager
    from pyqusolver_b200.rbm import rbm_leaves
    mgr = NQSCheckpointManager(tmp_path, max_to_keep=2)
    rng = np.random.default_rng(0)
    params = {"visible_bias": rng.normal(size=4) + 1j,
              "VisibleToHidden": {"kernel": rng.normal(size=(4, 8)) - 2j, "bias": rng.normal(size=8) + 0j}}
    for step in (1, 2, 3):
        mgr.save(step, params, {"energy": complex(-1.5, 0.0), "lr": 0.01})
    assert mgr.list_checkpoints() == [2, 3]                 # max_to_keep prunes the oldest
    assert mgr.latest_step == 3
    assert not (tmp_path / "metadata_1.json").exists() and not (tmp_path / "checkpoint_1.json").exists()
    tree = mgr.load()
    assert sorted(tree) == ["VisibleToHidden/bias", "VisibleToHidden/kernel", "visible_bias"]
    a, b, W = rbm_leaves(tree)
    assert np.array_equal(a, params["visible_bias"]) and np.array_equal(W, params["VisibleToHidden"]["kernel"])
    assert np.array_equal(b, params["VisibleToHidden"]["bias"])
    meta = mgr.load_metadata(3)
    assert meta["step"] == 3 and meta["lr"] == 0.01
    assert meta["energy"] == {"__complex__": True, "real": -1.5, "imag": 0.0}
    # a custom file name keeps its metadata beside it
    p = mgr.save("x", params, {"lr": 0.5}, filename="custom.h5")
    assert p.name == "custom.npz" and (tmp_path / "custom.json").exists()
    assert mgr.load_metadata(filename="custom.h5")["lr"] == 0.5
    assert sorted(mgr.load(filename="custom.h5")) == sorted(tree)


def test_checkpoint_reads_files_in_the_reference_layout(tmp_path):
    """Files as the reference's HDF5-less path writes them (QES/NQS/src/nqs_checkpoint_manager.py:
    np.savez of the "/"-flattened tree, metadata_<step>.json with the complex encoding of
    _make_json_serializable), read back by this package's manager and RBM tree reader."""
    import json
    from pyqusolver_b200.checkpoint import NQSCheckpointManager
    from pyqusolver_b200.rbm import rbm_leaves
    rng = np.random.default_rng(3)
    a = rng.normal(size=6) + 1j * rng.normal(size=6)
    W = rng.normal(size=(6, 12)) + 1j * rng.normal(size=(6, 12))
    b = rng.normal(size=12) + 1j * rng.normal(size=12)
    np.savez(tmp_path / "checkpoint_7.npz", **{"visible_bias": a, "VisibleToHidden/kernel": W,
                                               "VisibleToHidden/bias": b})
    (tmp_path / "metadata_7.json").write_text(json.dumps(
        {"step": 7, "E": {"__complex__": True, "real": -3.25, "imag": 0.5}}, indent=2))
    mgr = NQSCheckpointManager(tmp_path)
    assert mgr.list_checkpoints() == [7] and mgr.latest_step == 7
    ga, gb, gW = rbm_leaves(mgr.load(7))
    assert np.array_equal(ga, a) and np.array_equal(gb, b) and np.array_equal(gW, W)
    assert mgr.load_metadata(7)["E"]["real"] == -3.25
    # the names of the older flat layout are read as well
    ga, gb, gW = rbm_leaves({"params": {"visible_bias": a, "hidden_bias": b, "W": W}})
    assert np.array_equal(gW, W) and np.array_equal(gb, b)


def test_tdvp_initial_guess_selection():
    """TDVP._solve_handle_x0 mirrors QES/NQS/src/tdvp.py:1346-1380: a fixed sr_lin_x0, or the previous
    solution divided by rhs_prefactor when use_old_result is set; None (zero start) when the shape
    does not match."""
    import torch
    from pyqusolver_b200.tdvp import TDVP
    td = TDVP(rhs_prefactor=-2.0)
    assert td._solve_handle_x0(5, False) is None
    td._solution = torch.arange(5, dtype=torch.float64)
    assert td._solve_handle_x0(5, False) is None
    x0 = td._solve_handle_x0(5, True)
    assert torch.allclose(x0, torch.arange(5, dtype=torch.float64) / -2.0)
    assert td._solve_handle_x0(6, True) is None
    td2 = TDVP(rhs_prefactor=-1.0, sr_lin_x0=torch.ones(4, dtype=torch.float64))
    assert torch.equal(td2._solve_handle_x0(4, False), torch.ones(4, dtype=torch.float64))
    assert td2._solve_handle_x0(3, False) is None


def test_oracle_pcg_matches_scipy_cg_with_jacobi_preconditioner():
    """The oracle's preconditioned CG (z = M r, stopping rule on ||r||) reproduces SciPy's cg(M=...)
    iterate for iterate on a weighted SR system."""
    import numpy as np
    import scipy.sparse.linalg as sla
    from oracle import sr as osr
    rng = np.random.default_rng(3)
    O = rng.normal(size=(300, 40)) + 1j * rng.normal(size=(300, 40))
    O[:, :5] *= 10.0                                       # badly scaled columns: Jacobi matters
    e = rng.normal(size=300) + 1j * rng.normal(size=300)
    w = rng.random(300) + 0.5
    ec, Oc, w_, _, _ = osr.prepare(e, O, w)
    A = osr.s_matrix(Oc, w_) + 1e-3 * np.eye(40)
    F = osr.force(Oc, ec, w_)
    minv = osr.jacobi_minv(Oc, w_, 1e-3)
    x, it, res, conv = osr.cg(lambda v: A @ v, F, rtol=1e-10, maxiter=500, minv=minv)
    count = [0]
    xs, info = sla.cg(A, F, rtol=1e-10, atol=0.0, maxiter=500, M=sla.LinearOperator(A.shape, matvec=lambda r: minv * r,
                                                                                     dtype=A.dtype),
                      callback=lambda xk: count.__setitem__(0, count[0] + 1))
    assert conv and info == 0
    assert it == count[0]
    assert np.allclose(x, xs, rtol=1e-9, atol=1e-12 * np.abs(xs).max())
    _, it_plain, _, _ = osr.cg(lambda v: A @ v, F, rtol=1e-10, maxiter=500)
    assert it < it_plain


def test_oracle_minres_matches_scipy_minres():
    """The oracle's MINRES restatement follows SciPy's minres iterates on a Hermitian positive-definite
    SR system (same solution; its residual recurrence equals the true residual norm)."""
    import numpy as np
    import scipy.sparse.linalg as sla
    from oracle import sr as osr
    rng = np.random.default_rng(4)
    O = rng.normal(size=(200, 30)) + 1j * rng.normal(size=(200, 30))
    e = rng.normal(size=200) + 1j * rng.normal(size=200)
    ec, Oc, w_, _, _ = osr.prepare(e, O, None)
    A = osr.s_matrix(Oc, w_) + 1e-2 * np.eye(30)
    F = osr.force(Oc, ec, w_)
    x, it, phibar, conv, acond = osr.minres(lambda v: A @ v, F, rtol=1e-10, maxiter=300)
    assert conv
    assert abs(phibar - np.linalg.norm(A @ x - F)) <= 1e-6 * np.linalg.norm(F)
    xs, info = sla.minres(A, F, rtol=1e-12, maxiter=300)
    assert np.allclose(x, xs, rtol=1e-7, atol=1e-9 * np.abs(xs).max())
    ev = np.linalg.eigvalsh(A)
    assert 0.1 * ev[-1] / ev[0] <= acond <= 10 * ev[-1] / ev[0]


def test_oracle_fast_log_psi_matches_numpy_path():
    """oracle.fast (the CPU baseline's multi-core log cosh sum) gives the NumPy oracle's log psi."""
    import numpy as np
    import pytest
    from oracle import fast, rbm
    for cplx in (True, False):
        p = rbm.random_params(30, 60, complex_=cplx, scale=0.8, seed=2)
        sig = np.where(np.random.default_rng(1).random((5000, 30)) < 0.5, 1.0, -1.0)
        ref = rbm.log_psi(p, sig)
        if not fast.enable():
            pytest.skip("numba not available")
        try:
            got = rbm.log_psi(p, sig)
        finally:
            fast.disable()
        assert np.allclose(got, ref, rtol=0, atol=1e-11)
