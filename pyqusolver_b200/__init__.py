"""B200-native RBM variational Monte Carlo with QES's NQS / sampler / model API.

Public names follow QES (makskliczkowski/pyqusolver): ``NQS``, ``VMCSampler``,
``TDVP``, ``RBM``, ``TransverseFieldIsing``, ``XXZ``, ``J1J2Model``,
``SquareLattice``, ``HilbertSpace``.  The compute path is the C-ABI library
``libqes_b200.so`` (hand-written sm_100a kernels); importing the compute
modules does not fall back to anything when the library is missing -- the
first call raises.
"""

from .lattice import SquareLattice, get_neighbor_table
from .hilbert import HilbertSpace
from .hamiltonian import TransverseFieldIsing, XXZ, J1J2Model, SpinHamiltonian, SpinOperator

__all__ = [
    "SpinOperator",
    "SquareLattice", "get_neighbor_table", "HilbertSpace", "TransverseFieldIsing", "XXZ", "J1J2Model",
    "SpinHamiltonian", "RBM", "VMCSampler", "TDVP", "NQS", "NQSSingleStepResult", "NQSTrainStats", "NQSBatch",
]


def __getattr__(name):
    if name == "RBM":
        from .rbm import RBM
        return RBM
    if name == "VMCSampler":
        from .sampler import VMCSampler
        return VMCSampler
    if name == "TDVP":
        from .tdvp import TDVP
        return TDVP
    if name in ("NQS", "NQSSingleStepResult", "NQSTrainStats"):
        from . import nqs
        return getattr(nqs, name)
    if name == "ops":
        from . import ops
        return ops
    if name in ("NQSBatch", "NQSBatchStats"):
        from . import batch
        return getattr(batch, name)
    raise AttributeError(name)
