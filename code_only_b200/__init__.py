"""B200-native self-gravity FMG Poisson solver for block-structured AMR.

A drop-in for the reference's ``fmg_poisson`` (fmg.F90:63-74): the solve runs
as hand-written sm_100a kernels behind the C ABI of include/sfmg.h; this
package holds the CUDA sources (csrc/), the in-tree build, a ctypes binding
(abi.py), the Python mirror of the entry point (solver.py) and synthetic
workloads (workloads.py).
"""
from . import abi, workloads  # noqa: F401

__all__ = ["abi", "workloads"]
