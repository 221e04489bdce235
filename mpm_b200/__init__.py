"""B200-native explicit MPM step (USF/USL) -- a drop-in for the MPMExplicit
hot path of geomechanics/mpm.

The arithmetic runs in libmpm_b200.so (hand-written CUDA for sm_100a) through
the C ABI of include/mpm_gpu.h; this package is the Python host side.
"""
from ._native import MPMError, lib  # noqa: F401
from .problems import Problem, build_solver  # noqa: F401
from .solver import Solver, material_stress_batch, pinned_empty  # noqa: F401

__all__ = ["Solver", "MPMError", "Problem", "build_solver", "material_stress_batch", "pinned_empty", "lib"]
