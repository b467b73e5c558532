"""Exact ground-state energy (oracle side).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The reference diagonalises with ``model.diagonalize(method='lanczos')``
(``QES/Algebra/hamil.py:1809+`` -> ``QES/Algebra/Hamil/hamil_diag_engine.py:176-305``),
whose eigensolver is in the empty ``general_python`` submodule.  This
restatement builds the same sparse S^z-basis matrix from the oracle's term
list and calls SciPy's ARPACK Lanczos (``eigsh``, smallest algebraic).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as spla

from .hamiltonian import sparse_hamiltonian


def ground_energy(terms, ns, n_up=None, dense_below=64):
    H, _ = sparse_hamiltonian(terms, ns, n_up=n_up)
    if H.shape[0] <= dense_below:
        return float(np.min(np.linalg.eigvalsh(H.toarray())))
    Hr = H if np.abs(H.imag).max() > 0 else H.real
    vals = spla.eigsh(Hr, k=1, which="SA", tol=1e-12, return_eigenvectors=False)
    return float(np.real(vals[0]))
