"""Minimal ``HilbertSpace`` for spin-1/2 lattices (the fields the NQS path reads).

State convention (``QES/Algebra/Hilbert/hilbert_base.py:206-225``, pinned by
``Python/tests/nqs/test_nqs_model_state_convention.py:42-55``): vectors hold
+-0.5 (``spin_pm``); integers are binary with site i at bit ns-1-i and
bit 1 <-> +0.5.
"""

from __future__ import annotations

import numpy as np


class HilbertSpace:
    def __init__(self, lattice=None, ns=None, is_manybody=True, local_space="spin-1/2", **_):
        if lattice is None and ns is None:
            raise ValueError("HilbertSpace needs a lattice or ns")
        self.lattice = lattice
        self.ns = int(ns) if ns is not None else int(lattice.ns)
        if local_space not in ("spin-1/2", "spin_half", "spin-1/2 "):
            raise ValueError("only spin-1/2 local spaces are supported on this path")
        self.local_space = "spin-1/2"

    @property
    def Ns(self):
        return self.ns

    @property
    def state_convention(self):
        return {
            "local_space_type": "spin-1/2",
            "integer_representation": "binary_01",
            "vector_representation": "spin_pm",
            "representation": "spin_pm",
            "spin": True,
            "integer_mode_repr": 1.0,
            "vector_mode_repr": 0.5,
            "mode_repr": 0.5,
        }

    # conversions between +-0.5 vectors and big-endian integers
    def int_to_state(self, n):
        n = np.asarray(n, dtype=np.int64)
        shifts = np.arange(self.ns - 1, -1, -1, dtype=np.int64)
        bits = (n[..., None] >> shifts) & 1
        return np.where(bits == 1, 0.5, -0.5).astype(np.float32)

    def state_to_int(self, states):
        s = np.asarray(states) > 0
        weights = (1 << np.arange(self.ns - 1, -1, -1, dtype=np.int64))
        return (s.astype(np.int64) * weights).sum(axis=-1)
