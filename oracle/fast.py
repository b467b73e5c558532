"""Multi-core kernels for the oracle's dominant loop, used by the timed CPU baseline.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  ``enable()`` makes
``oracle.rbm.log_psi`` sum the log cosh of theta with a Numba ``prange`` loop over
the rows instead of NumPy's single-threaded element-wise ufuncs (theta itself is
a BLAS matrix product, already multi-threaded).  Same formula as
``oracle.rbm.log_cosh`` (log cosh z = z_s + log(1 + e^{-2 z_s}) - log 2 with
z_s = sign(Re z) z); the results agree with the NumPy path to float64 rounding
(``tests/test_host_logic.py``).  Profiling the 10x10 Heisenberg step of the NumPy
oracle put 70% of it in that element-wise log cosh (the local energy re-evaluates
every connected state in full, as the reference's estimator does).

Without Numba ``enable()`` returns False and the NumPy path stays in place.
"""

from __future__ import annotations

import numpy as np

try:
    import numba
    _HAVE_NUMBA = True
except Exception:                                       # pragma: no cover - numba absent
    numba = None
    _HAVE_NUMBA = False

_LOG2 = float(np.log(2.0))
_kernels = {}


def _build():
    if _kernels:
        return _kernels

    @numba.njit(parallel=True, cache=False)
    def rowsum_logcosh_c(th):
        out = np.empty(th.shape[0], dtype=np.complex128)
        for r in numba.prange(th.shape[0]):
            acc = 0.0 + 0.0j
            for m in range(th.shape[1]):
                z = th[r, m]
                if z.real < 0.0:
                    z = -z
                acc += z + np.log(1.0 + np.exp(-2.0 * z)) - _LOG2
            out[r] = acc
        return out

    @numba.njit(parallel=True, cache=False)
    def rowsum_logcosh_r(th):
        out = np.empty(th.shape[0], dtype=np.float64)
        for r in numba.prange(th.shape[0]):
            acc = 0.0
            for m in range(th.shape[1]):
                z = abs(th[r, m])
                acc += z + np.log1p(np.exp(-2.0 * z)) - _LOG2
            out[r] = acc
        return out

    _kernels["c"] = rowsum_logcosh_c
    _kernels["r"] = rowsum_logcosh_r
    return _kernels


def rowsum_log_cosh(th):
    """sum_m log cosh th[r, m] for every row r (float64 / complex128, 2-D)."""
    k = _build()
    th = np.ascontiguousarray(th)
    if np.iscomplexobj(th):
        return k["c"](th.astype(np.complex128, copy=False))
    return k["r"](th.astype(np.float64, copy=False))


def enable() -> bool:
    """Route oracle.rbm.log_psi's log-cosh sum through the parallel kernel; compiles it once
    (the caller times after this returns)."""
    if not _HAVE_NUMBA:
        return False
    from . import rbm
    rowsum_log_cosh(np.zeros((2, 2), dtype=np.complex128))
    rowsum_log_cosh(np.zeros((2, 2), dtype=np.float64))
    rbm._ROWSUM_LOGCOSH = rowsum_log_cosh
    return True


def disable():
    from . import rbm
    rbm._ROWSUM_LOGCOSH = None


def threads() -> int:
    """Threads the parallel kernel runs on (Numba's pool), or 1 without Numba."""
    return int(numba.get_num_threads()) if _HAVE_NUMBA else 1
