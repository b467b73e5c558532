"""SR solver paths through the C ABI: bounded-wait time-outs of the fused CG kernel.

A time-out is made on purpose with the library's barrier test hook (one arrival
that never comes and a short poll limit); every wait stays bounded, the kernel
records the time-out in a status word and the solve returns QES_ERR_TIMEOUT.
"""

import numpy as np
import pytest
import torch

import pyqusolver_b200 as qb
from pyqusolver_b200 import device as dv, _lib
from pyqusolver_b200.rbm import RBM

pytestmark = pytest.mark.gpu


def _small_problem(cplx, n=700, ns=9, nh=18, seed=6):
    model = qb.XXZ(qb.SquareLattice(2, 3, 3), jxy=-1.0, jz=-1.0, hx=0.4)
    net = RBM((ns,), n_hidden=nh, dtype="complex64" if cplx else "float32", seed=seed, init_scale=0.2)
    rng = np.random.default_rng(seed)
    st = np.where(rng.random((n, ns)) < 0.5, 0.5, -0.5)
    bits = dv.pack_states(st)
    _, tn, _ = dv.rbm_forward(net.flat, ns, nh, bits, tanh=True, logpsi=False)
    h = dv.DeviceHamiltonian(model.lower())
    tables = dv.move_tables(net.flat, ns, nh, h.move_i, h.move_j, h.move_kind, move_major=False)
    eloc = dv.local_energy(net.flat, ns, nh, bits, tn, h, tables)
    return net, bits, tn, eloc


@pytest.mark.parametrize("device_loop", [0, 1])
@pytest.mark.parametrize("impl", [0, 1])
def test_fused_cg_barrier_timeout_is_reported_and_solver_recovers(impl, device_loop):
    net, bits, tn, eloc = _small_problem(cplx=True)
    _lib.set_sr_impl(impl)
    _lib.call("qes_set_cg_fused", 2)
    _lib.call("qes_set_cg_device_loop", device_loop)
    ref, info_ref = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10,
                                   maxiter=2000, check_every=4)
    try:
        _lib.call("qes_sr_set_barrier_test", 1, 1000)
        with pytest.raises(_lib.QESError) as ei:
            dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000,
                           check_every=4)
        assert ei.value.code == _lib.QES_ERR_TIMEOUT
    finally:
        _lib.call("qes_sr_set_barrier_test", 0, 0)
    try:
        x, info = dv.sr_solve_cg(net.flat, net.ns, net.nh, bits, tn, eloc, shift=1e-2, rtol=1e-10, maxiter=2000,
                                 check_every=4)
        assert info["converged"] and info["iterations"] == info_ref["iterations"]
        assert torch.equal(x, ref)
    finally:
        _lib.call("qes_set_cg_fused", 1)
        _lib.call("qes_set_cg_device_loop", 1)
        _lib.set_sr_impl(0)
