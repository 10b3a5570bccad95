"""B200 (sm_100a) solver for HPRMAT's dense complex R-matrix linear-solve path.

The CUDA library ``lib/libhprmat_b200.so`` (C ABI: ``include/hprmat_b200.h``) does the
work; this package is the host-side mirror of the reference interface.
"""
from .api import (Context, HprmatError, RMatrixSolver, SOLVER_B200, default_context, rmat_ini, rmatrix,
                  solve_rmatrix, wf_print)
from . import workloads

__all__ = ["Context", "HprmatError", "RMatrixSolver", "SOLVER_B200", "default_context", "rmat_ini", "rmatrix",
           "solve_rmatrix", "wf_print", "workloads"]
