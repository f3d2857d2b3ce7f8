"""B200-native twisted-mass Wilson operator and solvers (drop-in for the
reference library's e/o-preconditioned tm path).

The compute path is libtmsolve.so (nissa_b200/csrc, CUDA for sm_100a) behind
the C ABI of include/tmsolve.h; this package is its host-side mirror.
"""
from .tm import Lattice, TmError, PRECISION, STATUS  # noqa: F401
from . import workload  # noqa: F401

__all__ = ["Lattice", "TmError", "PRECISION", "STATUS", "workload"]
