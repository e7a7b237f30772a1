"""B200-native composite-geometry FFT / domain-decomposition Poisson solver (Focalors_Poisson's 2D path).

The compute path is libfpb200.so (hand-written sm_100a CUDA behind the C ABI of include/fp_capi.h);
this package only loads it, owns device memory through torch, and mirrors the reference's solver
interface for Python callers.
"""
from . import workloads  # noqa: F401

__all__ = ["workloads"]
