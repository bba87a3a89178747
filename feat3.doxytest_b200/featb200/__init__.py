"""featb200: B200-native (sm_100a) geometric-multigrid Poisson solve path.

A drop-in for the reference's PCG + MultiGrid path (kernel/solver/pcg.hpp,
kernel/solver/multigrid.hpp) behind its LAFEM/Solver interfaces.  The compute runs in
libfeatb200.so (hand-written CUDA for sm_100a behind the C ABI in include/featb200.h); this package
is the host-side mirror of the reference's interface.
"""
from ._lib import FeatB200Error, exported_symbols, launch_count, lib  # noqa: F401
from .lafem import DenseVector, SparseMatrixCSR, Transfer, UnitFilter, arch  # noqa: F401
from .solver import (BatchPCG, MultiGrid, MultiGridAdaptCGC, MultiGridCycle, MultiGridHierarchy,  # noqa: F401
                     MultiRhsPCG, PCG, Status, build_hierarchy, build_pcg_multigrid, cycle_events,
                     new_coarse_inverse, new_jacobi_precond, new_multigrid, new_pcg, new_richardson, solve,
                     status_success, storage_plan)

__all__ = [n for n in dir() if not n.startswith("_")]
