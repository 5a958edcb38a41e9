"""stkfmm_b200 -- B200-native (sm_100a) STKFMM kernel-evaluation path.

The compute lives in ``libstkfmm_b200.so`` (hand-written CUDA for sm_100a behind
the C ABI of include/stkfmm_b200.h).  This package is the thin host-side
mirror of the reference's Python binding (Python/PySTKFMM.py) plus torch
entry points for device-resident data.
"""
from ._lib import StkError, lib  # noqa: F401
from .stkfmm import (KERNEL, PAXIS, PPKERNEL, PRECISION, SUPPORTED_KERNELS, UKERNEL, Octree,  # noqa: F401
                     Stk3DFMM, StkWallFMM, device_count, evaluate_kernel, get_kernel_dimension, get_kernel_name, kernel_slot,
                     ukernel_dims)

__all__ = ["KERNEL", "PAXIS", "PPKERNEL", "PRECISION", "UKERNEL", "Stk3DFMM", "StkWallFMM", "Octree", "StkError",
           "evaluate_kernel", "get_kernel_dimension", "get_kernel_name", "kernel_slot", "ukernel_dims",
           "device_count", "lib", "SUPPORTED_KERNELS"]
