"""cathode_b200 — B200-native implicit solve path of the microwave-cathode fluid code.

Layers:
  csrc/          CUDA kernels for sm_100a and the extern "C" ABI (libcathode_b200.so)
  capi.py        ctypes binding of that ABI (no CPU fallback)
  solvers.py     solver_SMG / solver_SOR mirrors of include/solverFuncs.hpp, Grid
  fluid.py       device field store and FluidModule kernels (fluidModule.hpp)
  workloads.py   seeded synthetic inputs in the reference's array shapes
  build.py       nvcc recipe (sm_100a)

The directory name is not a Python identifier; load it with
``__graft_entry__.load_package()`` (registered as ``cathode_b200``).
"""
from . import batch, capi, discharge, feed, fluid, learned, workloads  # noqa: F401
from .fluid import Fields  # noqa: F401
from .solvers import Grid, Microwave3, solver_SMG, solver_SOR  # noqa: F401

__all__ = ["batch", "capi", "discharge", "feed", "fluid", "learned", "workloads", "Fields", "Grid", "Microwave3", "solver_SMG", "solver_SOR"]
