"""ctypes binding of libstkfmm_b200.so (the C ABI declared in include/stkfmm_b200.h).

The shared library is the product: it is loaded from the package directory,
built in-tree by ``stkfmm_b200/build.py`` if it is missing or stale.  There is
no CPU implementation behind these calls; without a CUDA device every compute
entry point returns STK_ERR_NO_DEVICE and the Python layer raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# STKFMM_B200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("STKFMM_B200_LIB") or os.path.join(HERE, "libstkfmm_b200.so")

c_int, c_uint, c_double, c_void_p, c_char_p, c_float, c_longlong = (
    ctypes.c_int, ctypes.c_uint, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_float,
    ctypes.c_longlong)
P_d = ctypes.POINTER(ctypes.c_double)
P_i = ctypes.POINTER(ctypes.c_int)
P_ll = ctypes.POINTER(ctypes.c_longlong)
P_f = ctypes.POINTER(ctypes.c_float)

# (name, restype, argtypes) for every exported entry point
SIGNATURES = [
    ("stk_status_string", c_char_p, [c_int]),
    ("stk_get_kernel_dimension", c_int, [c_uint, P_i]),
    ("stk_get_kernel_name", c_char_p, [c_uint]),
    ("stk_kernel_slot", c_int, [c_uint, c_int]),
    ("stk_ukernel_dims", c_int, [c_int, P_i, P_i]),
    ("stk_ukernel_aux_dim", c_int, [c_int]),
    ("stk_device_count", c_int, []),
    ("stk_measure_peaks", c_int, [P_d]),
    ("stk_evaluate_kernel", c_int, [c_uint, c_uint, c_int, P_d, P_d, c_int, P_d, P_d, c_int]),
    ("stk_evaluate_kernel_device", c_int, [c_uint, c_uint, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                           c_int, c_void_p]),
    ("stk_ukernel_direct_device", c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int,
                                          c_void_p]),
    ("stk_ukernel_direct_device_noalloc", c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                                  c_int, c_void_p]),
    ("stk_p2p_lists", c_int, [c_int, c_int, c_int, P_i, P_i, P_i, P_i, c_int, P_i, P_i, c_int, c_void_p, c_void_p,
                              c_int, c_void_p, c_void_p, c_double, c_void_p]),
    ("stk_p2p_lists_aux", c_int, [c_int, c_int, c_int, P_i, P_i, P_i, P_i, c_int, P_i, P_i, c_int, c_void_p,
                                  c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p]),
    ("stk_ukernel_direct_aux_device", c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                                              c_void_p, c_int, c_void_p]),
    ("stk_gemm_3xtf32", c_int, [c_int, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_int, c_int,
                                c_void_p]),
    ("stk_p2p_plan_create", c_void_p, [c_int, P_i, P_i, P_i, P_i, c_int, P_i, P_i, c_int, c_int, c_double, P_i]),
    ("stk_p2p_plan_execute", c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p]),
    ("stk_p2p_plan_pairs", c_longlong, [c_void_p]),
    ("stk_p2p_plan_destroy", None, [c_void_p]),
    ("Stk3DFMM_create", c_void_p, [c_int, c_int, c_int, c_uint]),
    ("Stk3DFMM_destroy", None, [c_void_p]),
    ("Stk3DFMM_set_points", c_int, [c_void_p, c_int, P_d, c_int, P_d, c_int, P_d]),
    ("Stk3DFMM_get_kernel_dimension", c_int, [c_uint, P_i]),
    ("Stk3DFMM_set_box", c_int, [c_void_p, P_d, c_double]),
    ("Stk3DFMM_setup_tree", c_int, [c_void_p, c_uint]),
    ("Stk3DFMM_clear_fmm", c_int, [c_void_p, c_uint]),
    ("Stk3DFMM_evaluate_fmm", c_int, [c_void_p, c_uint, c_int, P_d, c_int, P_d, c_int, P_d]),
    ("Stk3DFMM_show_active_kernels", c_int, [c_void_p]),
    ("Stk3DFMM_evaluate_kernel", c_int, [c_void_p, c_uint, c_int, c_uint, c_int, P_d, P_d, c_int, P_d, P_d]),
    ("Stk3DFMM_set_precision", c_int, [c_void_p, c_int]),
    ("Stk3DFMM_set_shard", c_int, [c_void_p, c_int, c_int]),
    ("Stk3DFMM_set_allreduce", c_int, [c_void_p, c_void_p, c_void_p]),
    ("stk_octree_far_owners", c_int, [c_void_p, c_int, P_i]),
    ("stk_kernel_scaling", c_int, [c_uint, c_double, P_d, P_d, P_d]),
    ("stk_surface", c_int, [c_int, P_d, c_double, c_int, P_d]),
    ("Stk3DFMM_set_far_field", c_int, [c_void_p, c_int]),
    ("stk_partition_lpt", c_int, [c_int, P_d, c_int, P_i]),
    ("Stk3DFMM_evaluate_near", c_int, [c_void_p, c_uint, c_int, P_d, c_int, P_d, c_int, P_d]),
    ("Stk3DFMM_evaluate_near_device", c_int, [c_void_p, c_uint, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("Stk3DFMM_evaluate_fmm_device", c_int, [c_void_p, c_uint, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("Stk3DFMM_last_kernel_ms", c_int, [c_void_p, c_uint, P_f]),
    ("Stk3DFMM_last_phase_ms", c_int, [c_void_p, c_uint, P_f]),
    ("Stk3DFMM_get_fmm_stats", c_int, [c_void_p, c_uint, P_ll]),
    ("Stk3DFMM_get_m2l_work", c_int, [c_void_p, c_uint, P_d]),
    ("Stk3DFMM_last_launch_count", c_int, [c_void_p, c_uint, P_i]),
    ("Stk3DFMM_get_tree_stats", c_int, [c_void_p, c_uint, P_ll]),
    ("Stk3DFMM_get_ulist", c_int, [c_void_p, c_uint, P_i] + [P_i] * 11),
    ("StkWallFMM_create", c_void_p, [c_int, c_int, c_int, c_uint]),
    ("StkWallFMM_destroy", None, [c_void_p]),
    ("StkWallFMM_set_points", c_int, [c_void_p, c_int, P_d, c_int, P_d, c_int, P_d]),
    ("StkWallFMM_get_kernel_dimension", c_int, [c_uint, P_i]),
    ("StkWallFMM_set_box", c_int, [c_void_p, P_d, c_double]),
    ("StkWallFMM_setup_tree", c_int, [c_void_p, c_uint]),
    ("StkWallFMM_clear_fmm", c_int, [c_void_p, c_uint]),
    ("StkWallFMM_evaluate_fmm", c_int, [c_void_p, c_uint, c_int, P_d, c_int, P_d, c_int, P_d]),
    ("StkWallFMM_show_active_kernels", c_int, [c_void_p]),
    ("StkWallFMM_set_precision", c_int, [c_void_p, c_int]),
    ("StkWallFMM_set_far_field", c_int, [c_void_p, c_int]),
    ("StkWallFMM_evaluate_fmm_device", c_int, [c_void_p, c_uint, c_void_p, c_void_p, c_void_p]),
    ("StkWallFMM_last_kernel_ms", c_int, [c_void_p, P_f]),
    ("StkWallFMM_last_launch_count", c_int, [c_void_p, c_uint, P_i]),
    ("stk_octree_build", c_void_p, [P_d, c_int, c_int, c_int, P_d, c_int, P_d, c_int, P_d, c_int]),
    ("stk_octree_free", None, [c_void_p]),
    ("stk_octree_sizes", c_int, [c_void_p, P_ll]),
    ("stk_octree_nodes", c_int, [c_void_p, P_i, P_i, P_i, P_i]),
    ("stk_octree_list", c_int, [c_void_p, c_int, P_i, P_i]),
    ("stk_octree_set", c_int, [c_void_p, c_int, P_i, P_i, P_i]),
    ("stk_ker_last_status", c_int, []),
]
KER_SHIMS = ["laplace_p", "laplace_pgrad", "laplace_dipolep", "laplace_dipolepgrad", "stokes_vel", "rpy_u",
             "rpy_ulapu", "stk_ulapu", "stokes_regvel", "stokes_pvel", "stokes_doublepvel", "laplace_pgradgrad",
             "laplace_dipolepgradgrad", "laplace_quadp", "laplace_quadpgradgrad", "stokes_pvelgrad",
             "stokes_doublepvelgrad", "stokes_pvellaplacian", "stokes_doublelaplacian", "stokes_traction",
             "stokes_doubletraction", "stokes_regftvel", "stokes_regftvelomega", "stokes_velomega"]
for _n in KER_SHIMS:
    SIGNATURES.append(("stk_ker_" + _n, None, [P_d, c_int, P_d, c_int, P_d, c_int, P_d, c_void_p]))

# the host-only tree library (no CUDA): the octree / list C ABI and the LPT split
OCTREE_LIB_PATH = os.path.join(HERE, "libstk_octree.so")
OCTREE_SIGNATURES = [
    ("stk_octree_build", c_void_p, [P_d, c_int, c_int, c_int, P_d, c_int, P_d, c_int, P_d, c_int]),
    ("stk_octree_free", None, [c_void_p]),
    ("stk_octree_sizes", c_int, [c_void_p, P_ll]),
    ("stk_octree_nodes", c_int, [c_void_p, P_i, P_i, P_i, P_i]),
    ("stk_octree_list", c_int, [c_void_p, c_int, P_i, P_i]),
    ("stk_octree_set", c_int, [c_void_p, c_int, P_i, P_i, P_i]),
    ("stk_partition_lpt", c_int, [c_int, P_d, c_int, P_i]),
    ("stk_octree_far_owners", c_int, [c_void_p, c_int, P_i]),
]

# the collective a sharded handle calls (Stk3DFMM_set_allreduce)
ALLREDUCE_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_longlong, c_void_p, c_void_p)

_lib = None
_octree_lib = None
_lock = threading.Lock()


def _stale() -> bool:
    if os.environ.get("STKFMM_B200_LIB"):
        return False  # an explicitly chosen build is used as is
    if not os.path.exists(LIB_PATH):
        return True
    import glob
    srcs = glob.glob(os.path.join(HERE, "csrc", "*")) + glob.glob(os.path.join(os.path.dirname(HERE), "include",
                                                                               "*.h"))
    return any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in srcs)


def lib():
    """Load (building first if needed) libstkfmm_b200.so and declare its signatures."""
    global _lib
    with _lock:
        if _lib is None:
            if _stale():
                from . import build as _build
                _build.build()
            L = ctypes.CDLL(LIB_PATH)
            for name, res, args in SIGNATURES:
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
    return _lib


def octree_lib():
    """Load (building first if needed) the host-only libstk_octree.so; it maps no CUDA library."""
    global _octree_lib
    with _lock:
        if _octree_lib is None:
            from . import build as _build
            _build.build_octree()
            L = ctypes.CDLL(OCTREE_LIB_PATH)
            for name, res, args in OCTREE_SIGNATURES:
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _octree_lib = L
    return _octree_lib


class StkError(RuntimeError):
    """A C-ABI call returned a non-zero status (the reference printed and exited instead)."""

    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = lib().stk_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})" if where else f"{msg} (status {status})")


def check(status: int, where: str = "") -> None:
    if status != 0:
        raise StkError(status, where)
