"""RBM log-amplitude, theta cache, fast ratios and log-derivatives (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference RBM (``general_python.ml.net_impl.networks.net_rbm``) is in the
empty submodule.  What the reference pins, and what this restatement keeps:

* parameters W (N, M), visible bias a (N,), hidden bias b (M,): P = N*M + N + M
  (``QES/NQS/src/network/presets.py:117-137``);
* inputs mapped to +-1 before the network (``in_activation``;
  ``Python/tests/nqs/test_network_representation_consistency.py:121-156``);
* ``log_psi_delta`` equals the direct difference and the updated theta cache
  equals a fresh cache of the proposed state
  (``Python/tests/nqs/test_rbm_fast_update.py:47-147``);
* per-sample flat gradients O_k = d log psi / d p_k, holomorphic for complex
  parameters (``QES/NQS/src/nqs_kernels.py:212-259``).

Unpinned choices (named, shared with the CUDA path): flat order [a, b, W]
with W row-major (site-major); log cosh without the log 2 constant, evaluated
on the branch s*z + log1p(exp(-2 s z)) - log 2 with s = sign(Re z).  Ratios,
E_loc and O do not depend on either choice.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

LOG2 = np.log(2.0)


@dataclass
class RBMParams:
    a: np.ndarray   # (N,)
    b: np.ndarray   # (M,)
    W: np.ndarray   # (N, M)

    @property
    def n_visible(self):
        return self.a.shape[0]

    @property
    def n_hidden(self):
        return self.b.shape[0]

    @property
    def is_complex(self):
        return np.iscomplexobj(self.W)

    def flat(self):
        return np.concatenate([self.a.ravel(), self.b.ravel(), self.W.ravel()])

    @staticmethod
    def from_flat(p, n, m):
        p = np.asarray(p)
        return RBMParams(p[:n].copy(), p[n:n + m].copy(), p[n + m:].reshape(n, m).copy())


def random_params(n, m, *, complex_=False, scale=0.01, seed=0):
    rng = np.random.default_rng(seed)

    def draw(*shape):
        x = rng.normal(0.0, scale, size=shape)
        if complex_:
            x = x + 1j * rng.normal(0.0, scale, size=shape)
        return x

    return RBMParams(draw(n), draw(m), draw(n, m))


def to_sigma(states):
    """+-0.5 (or any signed) vectors -> +-1 float64."""
    return np.where(np.asarray(states) > 0, 1.0, -1.0)


def log_cosh(z):
    z = np.asarray(z)
    s = np.where(np.real(z) < 0, -1.0, 1.0)
    zs = z * s
    return zs + np.log1p(np.exp(-2.0 * zs)) - LOG2


def theta(p: RBMParams, sigma):
    return np.asarray(sigma, dtype=np.float64) @ p.W + p.b


# set by oracle.fast.enable() (the timed CPU baseline): a multi-core row sum of log cosh, same formula,
# for the large row blocks of the local energy (thread start-up outweighs it on a few chains' rows)
_ROWSUM_LOGCOSH = None


def log_psi(p: RBMParams, sigma):
    sigma = np.asarray(sigma, dtype=np.float64)
    th = theta(p, sigma)
    if _ROWSUM_LOGCOSH is not None and th.ndim == 2 and th.shape[0] >= 4096:
        return sigma @ p.a + _ROWSUM_LOGCOSH(th)
    return sigma @ p.a + np.sum(log_cosh(th), axis=-1)


def log_psi_delta_flips(p: RBMParams, sigma, flips, cache=None):
    """Delta log psi for flipping the sites in ``flips`` (a list per sample); returns (delta, new_theta)."""
    sigma = np.atleast_2d(np.asarray(sigma, dtype=np.float64))
    th = theta(p, sigma) if cache is None else np.array(cache, copy=True)
    delta = np.zeros(sigma.shape[0], dtype=np.result_type(p.W, np.float64))
    new_th = th.copy()
    for r, fl in enumerate(flips):
        dv = 0.0
        t_new = th[r].copy()
        sg = sigma[r].copy()
        for i in fl:            # sequential: a site listed twice is flipped back
            dv = dv - 2.0 * sg[i] * p.a[i]
            t_new = t_new - 2.0 * sg[i] * p.W[i]
            sg[i] = -sg[i]
        delta[r] = dv + np.sum(log_cosh(t_new) - log_cosh(th[r]))
        new_th[r] = t_new
    return delta, new_th


def log_derivatives(p: RBMParams, sigma):
    """Flat O (Ns, P) in the order [a, b, W]: O_a = sigma, O_b = tanh(theta), O_W = sigma_i tanh(theta_m)."""
    sigma = np.atleast_2d(np.asarray(sigma, dtype=np.float64))
    t = np.tanh(theta(p, sigma))
    ns = sigma.shape[0]
    ow = (sigma[:, :, None] * t[:, None, :]).reshape(ns, -1)
    dt = np.result_type(p.W, np.float64)
    return np.concatenate([sigma.astype(dt), t.astype(dt), ow.astype(dt)], axis=1)
