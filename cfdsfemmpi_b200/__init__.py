"""B200-native (sm_100a) time-step library for the cfdsfemmpi stabilised
finite-element incompressible Navier-Stokes solver.

The CUDA library (libcfdgpu.so, C ABI in include/cfdgpu.h) holds the hot
path; this package is the host side: the reference's file formats (io), the
``StabFEM`` driver with the reference's method names (stabfem), synthetic case
generators (meshgen) and a VTU writer (vtu).
"""
from . import io, meshgen
from ._lib import Batch, CfdGpuError, Handle, load, pattern_build
from .stabfem import StabFEM, solver_options_from_petsc

__all__ = ["io", "meshgen", "Handle", "CfdGpuError", "load", "pattern_build", "StabFEM", "solver_options_from_petsc"]
