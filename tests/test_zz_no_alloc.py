"""The allocation-free local energy (qes_local_energy_noalloc) through the C ABI.

Callers that cannot allocate device memory -- a host that hands the library a
fixed device budget, a loop that cannot pay for cudaMalloc's implicit
synchronisation, a foreign-language binding without a device allocator --
use this entry point: its scratch is a static array inside the library.  The
test compares it with the workspace entry point on two calls in a row (the
second on different samples and parameters, so stale contents of the shared
array would show), within the local-energy tolerance of the parity tests.
This file is collected last so that a failure here stops a -x run only after
every other test has run; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest
import torch

import pyqusolver_b200 as qb
from pyqusolver_b200 import _lib, device as dv
from pyqusolver_b200.rbm import RBM

pytestmark = pytest.mark.gpu

RTOL = 1e-5


def _problem(seed, n_samples):
    L = qb.SquareLattice(2, 6, 6)
    model = qb.J1J2Model(L, J1=-1.0, J2=-0.5)
    net = RBM((L.ns,), alpha=4, dtype="complex64", seed=seed, init_scale=0.05)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, L.ns, net.nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    bits = dv.init_chains(_lib.INIT_RND_FIXED, n_samples, L.ns, seed=seed, n_up=L.ns // 2)
    _, tn, _ = dv.rbm_forward(net.flat, L.ns, net.nh, bits, tanh=True, logpsi=False)
    return net, h, tables, bits, tn


def _noalloc(net, h, tables, bits, tn):
    out = torch.empty((bits.shape[0],), dtype=torch.complex64, device=bits.device)
    Ct, St, A = tables
    _lib.call("qes_local_energy_noalloc", dv.dtype_code(net.flat), net.ns, net.nh, int(bits.shape[0]),
              _lib.ptr(bits), _lib.ptr(tn), C.byref(h.struct), _lib.ptr(Ct), _lib.ptr(St), _lib.ptr(A),
              _lib.ptr(out), _lib.stream_ptr())
    return out


def test_noalloc_local_energy_matches_workspace_entry_point_twice():
    for seed, n in ((11, 3000), (12, 777)):
        net, h, tables, bits, tn = _problem(seed, n)
        ref = dv.local_energy(net.flat, net.ns, net.nh, bits, tn, h, tables).cpu().numpy()
        got = _noalloc(net, h, tables, bits, tn).cpu().numpy()
        err = np.max(np.abs(got - ref)) / max(1.0, np.max(np.abs(ref)))
        assert err <= RTOL, err


def test_noalloc_local_energy_rejects_oversized_requests():
    net, h, tables, bits, tn = _problem(13, 64)
    # ceil(144/32) = 5 move blocks * n * 8 bytes > 8 MiB for n = 2**18
    n_big = 1 << 18
    with pytest.raises(_lib.QESError) as e:
        _lib.call("qes_local_energy_noalloc", dv.dtype_code(net.flat), net.ns, net.nh, n_big, _lib.ptr(bits),
                  _lib.ptr(tn), C.byref(h.struct), None, None, None, None, _lib.stream_ptr())
    assert e.value.code == _lib.QES_ERR_SIZE
