"""Philox4x32-10 counter-based RNG and the proposal-stream mapping (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Philox4x32-10 is the published algorithm of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of two
32x32->64 multiplies with a Weyl-sequence key schedule.  The reference sampler
draws from JAX's threefry keys (``QES/Solver/MonteCarlo/vmc.py:1023-1026``),
which cannot be reproduced without JAX; the build replaces it with Philox
streams addressed by (chain, step), so the GPU sampler and this oracle draw
identical numbers and their chains can be compared step by step.

Stream layout (shared with ``pyqusolver_b200/csrc/philox.cuh``):

* proposals: counter = (chain, step_lo, step_hi, 0), key = (seed_lo, seed_hi)
  r0 -> site i = (r0 * N) >> 32, r1 -> neighbour slot k = (r1 * deg) >> 32,
  r2 -> u = ((r2 >> 9) + 0.5) * 2**-23 in (0, 1), exact in float32.
* initial states: counter = (chain, word, 0, 1) for RND bits; Fisher-Yates for
  RND_FIXED uses counter = (chain, pos, 0, 2), j = (r0 * (pos + 1)) >> 32.
"""

from __future__ import annotations

import numpy as np

PHILOX_M0 = np.uint64(0xD2511F53)
PHILOX_M1 = np.uint64(0xCD9E8D57)
PHILOX_W0 = np.uint32(0x9E3779B9)
PHILOX_W1 = np.uint32(0xBB67AE85)
_MASK32 = np.uint64(0xFFFFFFFF)

STREAM_PROPOSAL = 0
STREAM_INIT_RND = 1
STREAM_INIT_FIXED = 2
STREAM_PT_PHASE = 4
STREAM_PT_SWAP = 5


def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Vectorised Philox4x32-10.  All inputs broadcast; returns four uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint64) & _MASK32
    c1 = np.asarray(c1, dtype=np.uint64) & _MASK32
    c2 = np.asarray(c2, dtype=np.uint64) & _MASK32
    c3 = np.asarray(c3, dtype=np.uint64) & _MASK32
    k0 = np.asarray(k0, dtype=np.uint64) & _MASK32
    k1 = np.asarray(k1, dtype=np.uint64) & _MASK32
    c0, c1, c2, c3, k0, k1 = np.broadcast_arrays(c0, c1, c2, c3, k0, k1)
    c0, c1, c2, c3 = c0.copy(), c1.copy(), c2.copy(), c3.copy()
    k0, k1 = k0.copy(), k1.copy()
    for rnd in range(10):
        if rnd > 0:
            k0 = (k0 + np.uint64(PHILOX_W0)) & _MASK32
            k1 = (k1 + np.uint64(PHILOX_W1)) & _MASK32
        p0 = PHILOX_M0 * c0
        p1 = PHILOX_M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0), lo1, (hi0 ^ c3 ^ k1), lo0
    return (c0.astype(np.uint32), c1.astype(np.uint32),
            c2.astype(np.uint32), c3.astype(np.uint32))


def seed_key(seed: int):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return seed & 0xFFFFFFFF, seed >> 32


def bounded(r, n):
    """Multiply-shift map of a uint32 to [0, n)."""
    return ((np.asarray(r, dtype=np.uint64) * np.uint64(n)) >> np.uint64(32)).astype(np.int64)


def uniform_open(r):
    """(0,1) uniform, exactly representable in float32: ((r >> 9) + 0.5) * 2^-23."""
    k = (np.asarray(r, dtype=np.uint64) >> np.uint64(9)).astype(np.float64)
    return (k + 0.5) * 2.0 ** -23


def proposal_draws(seed, chains, step):
    """The four words that drive proposal number ``step`` of each chain in ``chains``."""
    k0, k1 = seed_key(seed)
    step = np.asarray(step, dtype=np.uint64)
    lo = step & _MASK32
    hi = step >> np.uint64(32)
    return philox4x32_10(np.asarray(chains, dtype=np.uint64), lo, hi, STREAM_PROPOSAL, k0, k1)
