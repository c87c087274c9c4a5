"""feat3_b200 -- B200-native (sm_100a) geometric-multigrid Poisson path of FEAT3.

Operator layer: ``feat3_b200.lafem`` (SparseMatrixCSR/ELL, DenseVector, UnitFilter,
Transfer) over the C-ABI in ``include/feat3_b200.h``. Solver layer: ``feat3_b200.solver``
(multigrid hierarchy, PCG/Richardson, mixed precision, adjoint).
"""
from . import _lib  # noqa: F401

__all__ = ["lib", "version"]


def lib():
    """The loaded C-ABI library (built in-tree with nvcc if missing)."""
    return _lib.load()


def version():
    return _lib.load().fb_version().decode()
