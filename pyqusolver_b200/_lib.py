"""ctypes binding of libqes_b200.so (the C ABI declared in include/qes_b200.h).

Loading never falls back to anything: if the library is missing the import of
the compute path raises, and every call that returns a nonzero status raises
``QESError`` with the library's message.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqes_b200.so")

QES_OK = 0
QES_ERR_ARG = 1
QES_ERR_CUDA = 2
QES_ERR_WORKSPACE = 3
QES_ERR_NOT_CONVERGED = 4
QES_ERR_TIMEOUT = 5
QES_ERR_SIZE = 6

DTYPE_F32 = 0
DTYPE_C64 = 1

INIT_RND, INIT_RND_FIXED, INIT_UP, INIT_DOWN = 0, 1, 2, 3
RULE_LOCAL, RULE_EXCHANGE = 0, 1
MOVE_FLIP1, MOVE_PAIR_ANTI, MOVE_PAIR_PAR = 0, 1, 2

_vp = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_u64 = C.c_uint64
_sz = C.c_size_t


class QESError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"qes status {code}: {msg}")
        self.code = code


class SamplerConfig(C.Structure):
    _fields_ = [
        ("rule", C.c_int), ("ns", C.c_int), ("nh", C.c_int), ("n_chains", C.c_int),
        ("chain_offset", _i64), ("num_samples", C.c_int), ("therm_steps_total", _i64),
        ("sweep_steps", C.c_int), ("recompute_every", C.c_int), ("mu", C.c_float), ("beta", C.c_float),
        ("seed", _u64), ("deg", C.c_int),
    ]


class BatchInstance(C.Structure):
    """``qes_batch_instance``: one problem of a batch (offsets in elements / words)."""
    _fields_ = [
        ("ns", _i32), ("nh", _i32), ("n_moves", _i32), ("n_zz", _i32), ("n_zfield", _i32),
        ("n_chains", _i32), ("num_samples", _i32), ("sweep_steps", _i32),
        ("therm_steps_total", _i64), ("seed", _u64),
        ("param_off", _i64), ("chain_off", _i64), ("chain_word_off", _i64), ("sample_off", _i64),
        ("sample_word_off", _i64), ("tanh_off", _i64), ("flip_off", _i64), ("move_table_off", _i64),
        ("move_off", _i64), ("zz_off", _i64), ("zf_off", _i64), ("eloc_part_off", _i64), ("sr_part_off", _i64),
    ]


class Hamiltonian(C.Structure):
    _fields_ = [
        ("n_moves", C.c_int), ("move_i", _vp), ("move_j", _vp), ("move_kind", _vp), ("move_coef", _vp),
        ("n_zfield", C.c_int), ("zf_site", _vp), ("zf_h", _vp),
        ("n_zz", C.c_int), ("zz_i", _vp), ("zz_j", _vp), ("zz_J", _vp),
    ]


class SROptions(C.Structure):
    _fields_ = [
        ("shift", C.c_double), ("rtol", C.c_double), ("atol", C.c_double), ("maxiter", C.c_int),
        ("check_every", C.c_int), ("rhs_prefactor", C.c_double), ("precond", C.c_int),
        ("skip_true_residual", C.c_int),
    ]


PRECOND_NONE, PRECOND_JACOBI = 0, 1


class SRResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("converged", C.c_int), ("residual", C.c_double), ("rhs_norm", C.c_double),
        ("e_mean_re", C.c_double), ("e_mean_im", C.c_double), ("true_residual", C.c_double),
        ("acond", C.c_double),
    ]


# name -> argtypes ; every symbol declared in include/qes_b200.h
SIGNATURES = {
    "qes_last_error": [],
    "qes_version": [],
    "qes_launch_count": [C.c_int],
    "qes_init_chains": [C.c_int, C.c_int, _u64, _i64, C.c_int, C.c_int, _vp, _vp],
    "qes_rbm_move_tables": [C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_int, _vp, _vp, _vp, C.c_int, _vp, _vp, _vp, _vp],
    "qes_rbm_forward": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_sampler_run": [C.c_int, C.POINTER(SamplerConfig), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int,
                        _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_local_energy_workspace_bytes": [C.c_int, C.c_int, C.c_int, _i64, C.c_int, C.POINTER(_sz)],
    "qes_local_energy": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, C.POINTER(Hamiltonian), _vp, _vp, _vp, _vp,
                         _sz, _vp, _vp],
    "qes_local_energy_noalloc": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, C.POINTER(Hamiltonian), _vp, _vp, _vp,
                                 _vp, _vp],
    "qes_sampler_run_betas": [C.c_int, C.POINTER(SamplerConfig), _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                              C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_set_pdl": [C.c_int],
    "qes_set_cg_device_loop": [C.c_int],
    "qes_sampler_set_capped": [C.c_int],
    "qes_sampler_set_wide": [C.c_int],
    "qes_sampler_tanh_cache": [C.c_int, _i64, _vp, _vp, _vp],
    "qes_pt_swap": [C.c_int, C.c_int, C.c_int, _vp, _vp, C.c_float, _u64, _i64, _vp, _vp],
    "qes_pt_collect": [C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_float, _vp, _vp, _vp, _vp, _vp],
    "qes_loss_stats_workspace_bytes": [_i64, C.POINTER(_sz)],
    "qes_loss_stats": [_i64, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_loss_rhat_workspace_bytes": [_i64, C.c_int, C.POINTER(_sz)],
    "qes_loss_rhat": [_i64, C.c_int, _vp, _vp, _vp, _sz, _vp],
    "qes_rbm_log_derivatives": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _i64, _vp],
    "qes_sr_workspace_bytes": [C.c_int, C.c_int, C.c_int, _i64, C.POINTER(_sz)],
    "qes_set_sr_impl": [C.c_int],
    "qes_sr_uses_tensor_cores": [C.c_int, C.c_int, C.c_int, _i64, C.POINTER(C.c_int)],
    "qes_sr_tc_plan": [C.c_int, C.c_int, C.c_int, _i64, _vp, C.c_int],
    "qes_sr_set_tiling": [C.c_int, C.c_int, C.c_int],
    "qes_sr_set_ohu_pairs": [C.c_int],
    "qes_sr_set_fused_sv": [C.c_int],
    "qes_sr_set_ov_split": [C.c_int],
    "qes_sr_set_ovz": [C.c_int],
    "qes_set_cg_graphs": [C.c_int],
    "qes_set_cg_fused": [C.c_int],
    "qes_set_cg_single_reduction": [C.c_int],
    "qes_set_reduce_bulk": [C.c_int],
    "qes_set_cg_xrp": [C.c_int],
    "qes_set_cg_fused_pdl": [C.c_int],
    "qes_sr_set_prefetch": [C.c_int],
    "qes_sr_set_barrier_test": [C.c_uint, C.c_uint],
    "qes_rbm_forward_tc_workspace_bytes": [C.c_int, C.c_int, C.c_int, _i64, C.POINTER(_sz)],
    "qes_rbm_forward_tc": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_set_l2_persist": [C.c_int],
    "qes_profile_enable": [C.c_int],
    "qes_profile_read": [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_int],
    "qes_sr_force": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_sr_matvec": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, C.c_double, _vp, _vp, _vp, _sz, _vp],
    "qes_sr_solve_cg": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, C.POINTER(SROptions), _vp,
                        C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_sr_solve_cg_x0": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, C.POINTER(SROptions), _vp, _vp,
                           C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_sr_force_weighted": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_sr_matvec_weighted": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, C.c_double, _vp, _vp, _vp, _sz,
                               _vp],
    "qes_sr_solve_cg_weighted": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, C.POINTER(SROptions), _vp,
                                 _vp, C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_sr_solve_minres_weighted": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, C.POINTER(SROptions), _vp,
                                     _vp, C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_sr_dense_workspace_bytes": [C.c_int, C.c_int, C.c_int, _i64, C.c_int, C.POINTER(_sz)],
    "qes_sr_gram": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_sr_solve_dense": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, C.POINTER(SROptions), _vp,
                           C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_sr_minsr_workspace_bytes": [C.c_int, C.c_int, C.c_int, _i64, C.POINTER(_sz)],
    "qes_sr_solve_minsr": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, C.POINTER(SROptions), _vp,
                           C.POINTER(SRResult), _vp, _sz, _vp],
    "qes_rbm_logpsi_vjp": [C.c_int, C.c_int, C.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _sz, _vp],
    "qes_param_update": [C.c_int, _i64, C.c_double, _vp, _vp, _vp, _vp],
    "qes_swap_region": [_i64, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_ed_workspace_bytes": [C.c_int, C.POINTER(_sz)],
    "qes_ed_sector_dim": [C.c_int, C.c_int, C.c_int, C.POINTER(_u64)],
    "qes_ed_sector_workspace_bytes": [C.c_int, C.c_int, C.c_int, C.POINTER(_sz)],
    "qes_ed_lanczos_sector": [C.c_int, C.c_int, C.c_int, C.POINTER(Hamiltonian), C.c_int, C.c_double, _u64,
                              C.POINTER(C.c_double), C.POINTER(C.c_int), _vp, _sz, _vp],
    "qes_ed_symm_workspace_bytes": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _u64, C.POINTER(_sz)],
    "qes_ed_symm_dim": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_u64), _vp, _sz, _vp],
    "qes_ed_lanczos_symm": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(Hamiltonian), C.c_int,
                            C.c_double, _u64, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(_u64), _vp, _sz,
                            _vp],
    "qes_ed_matvec": [C.c_int, C.POINTER(Hamiltonian), _vp, _vp, _vp],
    "qes_ed_lanczos": [C.c_int, C.POINTER(Hamiltonian), C.c_int, C.c_double, _u64, C.POINTER(C.c_double),
                       C.POINTER(C.c_int), _vp, _sz, _vp],
    "qes_batch_move_tables": [C.c_int, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                              _vp],
    "qes_batch_sampler_run": [C.c_int, C.c_int, _vp, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_float,
                              C.c_float, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_batch_rbm_forward": [C.c_int, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_batch_local_energy": [C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "qes_batch_loss_stats": [C.c_int, _vp, _vp, _vp, _vp],
    "qes_batch_sr_workspace_bytes": [C.c_int, C.c_int, _i64, _i64, _i64, C.POINTER(_sz)],
    "qes_batch_sr_solve_cg": [C.c_int, C.c_int, _vp, C.c_int, _vp, C.c_int, _vp, _i64, _i64, _i64, _vp, _vp, _vp,
                              C.POINTER(SROptions), _vp, _vp, _vp, _sz, _vp],
}

_LIB = None


def load(path: str = LIB_PATH):
    """Load the library once; raises OSError when it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with `python -m pyqusolver_b200.build`")
    lib = C.CDLL(path)
    for name, argt in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argt
        fn.restype = {"qes_last_error": C.c_char_p, "qes_launch_count": C.c_longlong}.get(name, C.c_int)
    _LIB = lib
    return lib


def check(code: int):
    if code != QES_OK:
        msg = _LIB.qes_last_error().decode() if _LIB is not None else "?"
        raise QESError(code, msg)
    return code


def call(name, *args, allow=()):
    rc = getattr(load(), name)(*args)
    if rc != QES_OK and rc not in allow:
        check(rc)
    return rc


SR_IMPL_AUTO, SR_IMPL_CUDA_CORES, SR_IMPL_TENSOR_CORES, SR_IMPL_FP64 = 0, 1, 2, 3


_SR_IMPL = [0]


def set_sr_impl(impl: int):
    """0 = tensor cores where the shapes allow (mixed form), 1 = CUDA cores only (plain FP32 form), 2 = tensor
    cores required, 3 = CUDA cores with float64 contractions (the float64 reference form).  Also selects the
    forward (theta) path used by the training step (tensor cores only in forms 0 and 2)."""
    call("qes_set_sr_impl", int(impl))
    _SR_IMPL[0] = int(impl)


def sr_impl() -> int:
    return _SR_IMPL[0]


TC_PLAN_FIELDS = ("uses", "big", "KC", "n_chunks", "nsplit", "n_tiles", "Kd", "NB", "Np", "MT", "NC", "NR", "nnc",
                  "SPC", "ov_stages", "cl", "sv", "sv_grid", "ovz")


def sr_tc_plan(dtype_code: int, ns: int, nh: int, n_samples: int) -> dict:
    buf = (C.c_int32 * len(TC_PLAN_FIELDS))()
    call("qes_sr_tc_plan", int(dtype_code), int(ns), int(nh), int(n_samples), C.cast(buf, C.c_void_p),
         len(TC_PLAN_FIELDS))
    return {k: int(buf[i]) for i, k in enumerate(TC_PLAN_FIELDS)}


def sr_uses_tensor_cores(dtype_code: int, ns: int, nh: int, n_samples: int) -> bool:
    u = C.c_int(0)
    call("qes_sr_uses_tensor_cores", int(dtype_code), int(ns), int(nh), int(n_samples), C.byref(u))
    return bool(u.value)


PROFILE_CLASSES = ("ov", "ohu", "reduce", "gram", "cholesky", "sv")


def profile_enable(on: bool):
    call("qes_profile_enable", 1 if on else 0)


def profile_read(reset=True):
    n = len(PROFILE_CLASSES)
    ms = (C.c_double * n)()
    cnt = (C.c_longlong * n)()
    call("qes_profile_read", 1 if reset else 0, ms, cnt, n)
    return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(PROFILE_CLASSES)}


def launch_count(reset=False) -> int:
    return int(load().qes_launch_count(1 if reset else 0))


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else _vp(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return _vp(s.cuda_stream)
