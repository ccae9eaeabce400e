"""B200-native supernodal Cholesky factorization and triangular solve.

A drop-in for the numeric path of symPACK's ``symPACKMatrix2D`` (symbolic
factorize, distribute, factorize, solve, get solution): host C++ symbolic
analysis bit-exact with the reference, sm_100a kernels for the numeric work.
"""
from .solver import (DeviceTimeoutError, DistSparseMatrix, NotSPDError, RelaxationParameters, StateError, SymPACKError,
                     symPACKMatrix2D, symPACKOptions)
from . import generators

__all__ = ["DeviceTimeoutError", "DistSparseMatrix", "NotSPDError", "RelaxationParameters", "StateError", "SymPACKError",
           "symPACKMatrix2D", "symPACKOptions", "generators"]
