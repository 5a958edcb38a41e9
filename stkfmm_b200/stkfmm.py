"""Python interface mirroring the reference's ctypes binding (Python/PySTKFMM.py).

Same class, method and argument names as ``PySTKFMM.Stk3DFMM``
(Python/PySTKFMM.py:34-79): ``set_box``, ``get_kernel_dimension``,
``set_points``, ``setup_tree``, ``evaluate_fmm``, ``clear_fmm``,
``show_active_kernels``; arrays are C-contiguous float64 numpy arrays of shape
(n, 3) for coordinates and (n, kdim) for values, and ``evaluate_fmm`` /
``evaluate_kernel`` add into the target array as the reference does.  Where the
reference printed a message and called exit(1), these methods raise StkError.

Additions: ``evaluate_kernel`` (STKFMM::evaluateKernel, Lib/src/STKFMM.cpp:88-99),
``set_precision`` (FP64 / MIXED P2P arithmetic), ``evaluate_near`` (U-list part
only), ``tree_stats`` and ``ulist``.
"""
from __future__ import annotations

import ctypes
import enum

import numpy as np

from ._lib import P_d, P_f, P_i, P_ll, StkError, check, lib, octree_lib


class PAXIS(enum.IntEnum):
    """Lib/include/STKFMM/STKFMM_common.hpp:29-34"""
    NONE = 0
    PX = 1
    PXY = 2
    PXYZ = 3


class PPKERNEL(enum.IntEnum):
    """Lib/include/STKFMM/STKFMM_common.hpp:40-44"""
    SLS2T = 1
    DLS2T = 2
    L2T = 4


class KERNEL(enum.IntFlag):
    """Lib/include/STKFMM/STKFMM_common.hpp:46-62"""
    LapPGrad = 1
    LapPGradGrad = 2
    LapQPGradGrad = 4
    Stokes = 8
    RPY = 16
    StokesRegVel = 32
    StokesRegVelOmega = 64
    PVel = 128
    PVelGrad = 256
    PVelLaplacian = 512
    Traction = 1024


class PRECISION(enum.IntEnum):
    FP64 = 0
    MIXED = 1


class UKERNEL(enum.IntEnum):
    """Micro-kernels (one STKFMM uKerEval body each); see include/stkfmm_b200.h."""
    LAPLACE_P = 0
    LAPLACE_PGRAD = 1
    LAPLACE_DIPOLEP = 2
    LAPLACE_DIPOLEPGRAD = 3
    STOKES_VEL = 4
    RPY_U = 5
    RPY_ULAPU = 6
    STK_ULAPU = 7
    STOKES_REGVEL = 8
    STOKES_PVEL = 9
    STOKES_DOUBLEPVEL = 10
    LAPLACE_SLDL_PGRAD = 11
    STOKES_SLDL_PVEL = 12
    REGVEL_ADJ_SRC = 13  # adjoint of stokes_regvel: (dL/df, dL/deps, dL/dx) at the sources
    REGVEL_ADJ_TRG = 14  # adjoint of stokes_regvel: dL/dx at the targets
    LAPLACE_SLDL_P = 15  # laplace_p + laplace_dipolep at one point (fused S2M / S2L)
    LAPLACE_PGRADGRAD = 16
    LAPLACE_DIPOLEPGRADGRAD = 17
    LAPLACE_QUADP = 18
    LAPLACE_QUADPGRADGRAD = 19
    STOKES_PVELGRAD = 20
    STOKES_DOUBLEPVELGRAD = 21
    STOKES_PVELLAPLACIAN = 22
    STOKES_DOUBLELAPLACIAN = 23
    STOKES_TRACTION = 24
    STOKES_DOUBLETRACTION = 25
    STOKES_REGFTVEL = 26
    STOKES_REGFTVELOMEGA = 27
    STOKES_VELOMEGA = 28


SUPPORTED_KERNELS = (KERNEL.LapPGrad, KERNEL.LapPGradGrad, KERNEL.LapQPGradGrad, KERNEL.Stokes, KERNEL.RPY,
                     KERNEL.StokesRegVel, KERNEL.StokesRegVelOmega, KERNEL.PVel, KERNEL.PVelGrad,
                     KERNEL.PVelLaplacian, KERNEL.Traction)


def _arr(a, cols=None, name="array"):
    """Return a C-contiguous float64 array (a copy only if needed)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if cols is not None and a.size:
        a = a.reshape(-1, cols)
    return a


def _ptr(a):
    return a.ctypes.data_as(P_d) if a is not None and a.size else None


def get_kernel_dimension(kernel) -> np.ndarray:
    dims = np.zeros(3, dtype=np.int32)
    check(lib().stk_get_kernel_dimension(int(kernel), dims.ctypes.data_as(P_i)), "get_kernel_dimension")
    return dims


def get_kernel_name(kernel) -> str:
    n = lib().stk_get_kernel_name(int(kernel))
    if n is None:
        raise StkError(2, "get_kernel_name")
    return n.decode()


def kernel_slot(kernel, slot: int) -> int:
    return lib().stk_kernel_slot(int(kernel), int(slot))


def ukernel_dims(uk) -> tuple:
    s, t = ctypes.c_int(), ctypes.c_int()
    check(lib().stk_ukernel_dims(int(uk), ctypes.byref(s), ctypes.byref(t)), "ukernel_dims")
    return s.value, t.value


def device_count() -> int:
    return lib().stk_device_count()


def evaluate_kernel(kernel, p2p, src_coord, src_value, trg_coord, trg_value, precision=PRECISION.FP64):
    """trg_value += direct sum (STKFMM::evaluateKernel semantics), host arrays, accumulate in place."""
    sd, dd, td = get_kernel_dimension(kernel)
    # the sub-kernel must exist before the value layout can be checked (FMMData.cpp:261-273)
    uk = kernel_slot(kernel, {PPKERNEL.SLS2T: 0, PPKERNEL.DLS2T: 1, PPKERNEL.L2T: 6}[PPKERNEL(p2p)])
    if uk < 0:
        raise StkError(2, "evaluate_kernel")
    sdim = {PPKERNEL.SLS2T: sd, PPKERNEL.DLS2T: dd, PPKERNEL.L2T: ukernel_dims(uk)[0]}[PPKERNEL(p2p)]
    src = _arr(src_coord, 3)
    val = _arr(src_value, sdim)
    trg = _arr(trg_coord, 3)
    if not (isinstance(trg_value, np.ndarray) and trg_value.dtype == np.float64 and trg_value.flags.c_contiguous):
        raise TypeError("trg_value must be a C-contiguous float64 numpy array (accumulated in place)")
    if len(val) != len(src) or trg_value.size != len(trg) * td:
        raise StkError(4, "evaluate_kernel")
    check(lib().stk_evaluate_kernel(int(kernel), int(p2p), len(src), _ptr(src), _ptr(val), len(trg), _ptr(trg),
                                    _ptr(trg_value), int(precision)), "evaluate_kernel")
    return trg_value


class Stk3DFMM:
    """B200 counterpart of PySTKFMM.Stk3DFMM (Python/PySTKFMM.py:34-79)."""

    def __init__(self, mult_order, max_pts, pbc, kernels, precision=PRECISION.FP64, enable_ff=True):
        """enable_ff: the reference's enableFF (Lib/include/STKFMM/STKFMM.hpp:199-200); False
        stops a periodic sum at the images within two cells (no far-image operator)."""
        self.mult_order = int(mult_order)
        self.max_pts = int(max_pts)
        self.pbc = int(pbc)
        self.kernels = int(kernels)
        L = lib()
        self.fmm = L.Stk3DFMM_create(self.mult_order, self.max_pts, self.pbc, self.kernels)
        if not self.fmm:
            status = 6 if L.stk_device_count() <= 0 else 1
            raise StkError(status, "Stk3DFMM_create")
        self.set_precision(precision)
        self.set_far_field(enable_ff)
        self._n = (0, 0, 0)

    def set_far_field(self, enable):
        check(lib().Stk3DFMM_set_far_field(self.fmm, 1 if enable else 0), "set_far_field")
        self.enable_ff = bool(enable)

    def __del__(self):
        f = getattr(self, "fmm", None)
        if f:
            lib().Stk3DFMM_destroy(f)
            self.fmm = None

    def set_precision(self, precision):
        check(lib().Stk3DFMM_set_precision(self.fmm, int(precision)), "set_precision")
        self.precision = PRECISION(precision)

    def set_box(self, origin, length):
        origin = _arr(origin).reshape(3)
        check(lib().Stk3DFMM_set_box(self.fmm, origin.ctypes.data_as(P_d), float(length)), "set_box")

    def get_kernel_dimension(self, kernel):
        return get_kernel_dimension(kernel)

    def set_points(self, src_SL_coord, trg_coord, src_DL_coord):
        sl = _arr(src_SL_coord, 3)
        trg = _arr(trg_coord, 3)
        dl = _arr(src_DL_coord, 3) if src_DL_coord is not None else np.zeros((0, 3))
        check(lib().Stk3DFMM_set_points(self.fmm, len(sl), _ptr(sl), len(trg), _ptr(trg), len(dl), _ptr(dl)),
              "set_points")
        self._n = (len(sl), len(dl), len(trg))

    def setup_tree(self, kernel):
        check(lib().Stk3DFMM_setup_tree(self.fmm, int(kernel)), "setup_tree")

    def clear_fmm(self, kernel):
        check(lib().Stk3DFMM_clear_fmm(self.fmm, int(kernel)), "clear_fmm")

    def show_active_kernels(self):
        check(lib().Stk3DFMM_show_active_kernels(self.fmm), "show_active_kernels")

    def _eval(self, fn, name, kernel, src_SL_value, trg_value, src_DL_value):
        sd, dd, td = get_kernel_dimension(kernel)
        slv = _arr(src_SL_value, sd)
        dlv = _arr(src_DL_value, dd) if src_DL_value is not None else np.zeros((0, dd))
        if not (isinstance(trg_value, np.ndarray) and trg_value.dtype == np.float64 and trg_value.flags.c_contiguous):
            raise TypeError("trg_value must be a C-contiguous float64 numpy array (accumulated in place)")
        ntrg = trg_value.size // td if td else 0
        check(fn(self.fmm, int(kernel), len(slv), _ptr(slv), ntrg, _ptr(trg_value), len(dlv), _ptr(dlv)), name)
        return trg_value

    def evaluate_fmm(self, kernel, src_SL_value, trg_value, src_DL_value):
        return self._eval(lib().Stk3DFMM_evaluate_fmm, "evaluate_fmm", kernel, src_SL_value, trg_value, src_DL_value)

    def evaluate_near(self, kernel, src_SL_value, trg_value, src_DL_value):
        return self._eval(lib().Stk3DFMM_evaluate_near, "evaluate_near", kernel, src_SL_value, trg_value,
                          src_DL_value)

    def evaluate_near_device(self, kernel, d_sl, d_trg, d_dl=None, stream=None):
        """Device pointers (ints) in the caller's order; queued on `stream` (a cudaStream_t int or None)."""
        check(lib().Stk3DFMM_evaluate_near_device(self.fmm, int(kernel), d_sl, d_trg, d_dl, stream),
              "evaluate_near_device")

    def evaluate_fmm_device(self, kernel, d_sl, d_trg, d_dl=None, stream=None):
        """evaluate_fmm on device pointers (ints) in the caller's order, unit box only."""
        check(lib().Stk3DFMM_evaluate_fmm_device(self.fmm, int(kernel), d_sl, d_trg, d_dl, stream),
              "evaluate_fmm_device")

    def last_kernel_ms(self, kernel) -> float:
        ms = ctypes.c_float()
        check(lib().Stk3DFMM_last_kernel_ms(self.fmm, int(kernel), ctypes.byref(ms)), "last_kernel_ms")
        return ms.value

    def evaluate_kernel(self, kernel, nThreads, p2p, src_coord, src_value, trg_coord, trg_value):
        """STKFMM::evaluateKernel through the handle (uses the handle's precision)."""
        if not (int(kernel) & self.kernels):
            raise StkError(2, "evaluate_kernel")
        return evaluate_kernel(kernel, p2p, src_coord, src_value, trg_coord, trg_value, self.precision)

    PHASES = ("near", "s2m", "m2m", "m2l", "s2l", "l2l", "l2t", "m2t")

    def last_phase_ms(self, kernel) -> dict:
        """Device time (ms) per phase of the last evaluation (near-field-only calls: far phases 0)."""
        ms = np.zeros(8, dtype=np.float32)
        check(lib().Stk3DFMM_last_phase_ms(self.fmm, int(kernel), ms.ctypes.data_as(P_f)), "last_phase_ms")
        return dict(zip(self.PHASES, (float(v) for v in ms)))

    def set_shard(self, rank: int, nranks: int):
        """Evaluate only shard `rank` of `nranks` of the target-side work (sum over shards = full result)."""
        check(lib().Stk3DFMM_set_shard(self.fmm, int(rank), int(nranks)), "set_shard")

    def set_allreduce(self, fn):
        """The shard group's collective (Stk3DFMM_set_allreduce): fn(ptr, n, stream) sums the n
        float64 values at device address ptr over the ranks, ordered on the CUDA stream handle
        `stream`, and returns 0.  With it a sharded handle splits the far field's M2L / S2L as
        well.  None clears it."""
        from ._lib import ALLREDUCE_FN
        if fn is None:
            self._allreduce = None
            check(lib().Stk3DFMM_set_allreduce(self.fmm, None, None), "set_allreduce")
            return

        def _cb(ptr, n, stream, user):
            try:
                return int(fn(ptr, n, stream) or 0)
            except Exception:  # an exception cannot cross the C ABI: report a failed collective
                import traceback
                traceback.print_exc()
                return 1
        self._allreduce = ALLREDUCE_FN(_cb)  # kept alive as long as the handle
        check(lib().Stk3DFMM_set_allreduce(self.fmm, ctypes.cast(self._allreduce, ctypes.c_void_p), None),
              "set_allreduce")

    def last_launch_count(self, kernel) -> int:
        n = ctypes.c_int()
        check(lib().Stk3DFMM_last_launch_count(self.fmm, int(kernel), ctypes.byref(n)), "last_launch_count")
        return int(n.value)

    def fmm_stats(self, kernel) -> dict:
        """Pair counts of one evaluate_fmm (available after the first call)."""
        out = np.zeros(10, dtype=np.int64)
        check(lib().Stk3DFMM_get_fmm_stats(self.fmm, int(kernel), out.ctypes.data_as(P_ll)), "fmm_stats")
        keys = ["near_pairs_sl", "near_pairs_dl", "s2m_pairs", "s2l_pairs", "m2t_pairs", "l2t_pairs", "m2l_pairs",
                "surface_points", "m2l_rank",
                "launches"]
        return dict(zip(keys, (int(v) for v in out)))

    def m2l_work(self, kernel) -> dict:
        """Flops of one compressed M2L: algorithmic (true ranks, real pairs) and executed."""
        out = np.zeros(2)
        check(lib().Stk3DFMM_get_m2l_work(self.fmm, int(kernel), out.ctypes.data_as(P_d)), "m2l_work")
        return {"flops_algorithmic": float(out[0]), "flops_executed": float(out[1])}

    def tree_stats(self, kernel) -> dict:
        out = np.zeros(9, dtype=np.int64)
        check(lib().Stk3DFMM_get_tree_stats(self.fmm, int(kernel), out.ctypes.data_as(P_ll)), "tree_stats")
        keys = ["nodes", "leaves", "depth", "u_entries", "u_pairs_sl", "u_pairs_dl", "v_entries", "w_entries",
                "x_entries"]
        return dict(zip(keys, (int(v) for v in out)))

    def ulist(self, kernel) -> dict:
        """The U-list of the last setup_tree, in leaf-sorted indices (stk_p2p_lists layout)."""
        sizes = np.zeros(5, dtype=np.int32)
        L = lib()
        nulls = [None] * 11
        check(L.Stk3DFMM_get_ulist(self.fmm, int(kernel), sizes.ctypes.data_as(P_i), *nulls), "ulist")
        nn, ne, nsl, ndl, ntrg = (int(v) for v in sizes)
        arrs = dict(trg_begin=nn, trg_end=nn, list_off=nn + 1, list_ent=ne, sl_begin=nn, sl_end=nn, dl_begin=nn,
                    dl_end=nn, sl_perm=nsl, dl_perm=ndl, trg_perm=ntrg)
        out = {k: np.zeros(max(v, 1), dtype=np.int32) for k, v in arrs.items()}
        check(L.Stk3DFMM_get_ulist(self.fmm, int(kernel), sizes.ctypes.data_as(P_i),
                                   *[out[k].ctypes.data_as(P_i) for k in arrs]), "ulist")
        return {k: out[k][:v] for k, v in arrs.items()}


class StkWallFMM:
    """B200 counterpart of PySTKFMM.StkWallFMM (Python/PySTKFMM.py:82-127): Stokeslets
    (KERNEL.Stokes) or RPY spheres (KERNEL.RPY) above a no-slip wall at z = origin_z,
    points in [o, o+L)^2 x [o_z, o_z+L/2); pbc NONE, PX or PXY."""

    def __init__(self, mult_order, max_pts, pbc, kernels, precision=PRECISION.FP64, enable_ff=True):
        self.mult_order = int(mult_order)
        self.max_pts = int(max_pts)
        self.pbc = int(pbc)
        self.kernels = int(kernels)
        L = lib()
        self.fmm = L.StkWallFMM_create(self.mult_order, self.max_pts, self.pbc, self.kernels)
        if not self.fmm:
            status = 6 if L.stk_device_count() <= 0 else 1
            raise StkError(status, "StkWallFMM_create")
        self.set_precision(precision)
        self.set_far_field(enable_ff)

    def set_far_field(self, enable):
        check(lib().StkWallFMM_set_far_field(self.fmm, 1 if enable else 0), "set_far_field")
        self.enable_ff = bool(enable)

    def __del__(self):
        f = getattr(self, "fmm", None)
        if f:
            lib().StkWallFMM_destroy(f)
            self.fmm = None

    def set_precision(self, precision):
        check(lib().StkWallFMM_set_precision(self.fmm, int(precision)), "set_precision")
        self.precision = PRECISION(precision)

    def set_box(self, origin, length):
        origin = _arr(origin).reshape(3)
        check(lib().StkWallFMM_set_box(self.fmm, origin.ctypes.data_as(P_d), float(length)), "set_box")

    def get_kernel_dimension(self, kernel):
        return get_kernel_dimension(kernel)

    def set_points(self, src_SL_coord, trg_coord, src_DL_coord=None):
        sl = _arr(src_SL_coord, 3)
        trg = _arr(trg_coord, 3)
        dl = _arr(src_DL_coord, 3) if src_DL_coord is not None else np.zeros((0, 3))
        check(lib().StkWallFMM_set_points(self.fmm, len(sl), _ptr(sl), len(trg), _ptr(trg), len(dl), _ptr(dl)),
              "set_points")

    def setup_tree(self, kernel):
        check(lib().StkWallFMM_setup_tree(self.fmm, int(kernel)), "setup_tree")

    def clear_fmm(self, kernel):
        check(lib().StkWallFMM_clear_fmm(self.fmm, int(kernel)), "clear_fmm")

    def show_active_kernels(self):
        check(lib().StkWallFMM_show_active_kernels(self.fmm), "show_active_kernels")

    def evaluate_fmm(self, kernel, src_SL_value, trg_value, src_DL_value=None):
        sd, _, td = get_kernel_dimension(kernel)
        slv = _arr(src_SL_value, sd)
        if not (isinstance(trg_value, np.ndarray) and trg_value.dtype == np.float64 and trg_value.flags.c_contiguous):
            raise TypeError("trg_value must be a C-contiguous float64 numpy array (accumulated in place)")
        ntrg = trg_value.size // td if td else 0
        check(lib().StkWallFMM_evaluate_fmm(self.fmm, int(kernel), len(slv), _ptr(slv), ntrg, _ptr(trg_value), 0,
                                            None), "evaluate_fmm")
        return trg_value

    def evaluate_fmm_device(self, kernel, d_sl, d_trg, stream=None):
        """evaluate_fmm on device pointers (ints) in the caller's order, queued on `stream`."""
        check(lib().StkWallFMM_evaluate_fmm_device(self.fmm, int(kernel), d_sl, d_trg, stream),
              "evaluate_fmm_device")

    def last_kernel_ms(self) -> float:
        ms = ctypes.c_float()
        check(lib().StkWallFMM_last_kernel_ms(self.fmm, ctypes.byref(ms)), "last_kernel_ms")
        return ms.value

    def last_launch_count(self, kernel) -> int:
        c = ctypes.c_int()
        check(lib().StkWallFMM_last_launch_count(self.fmm, int(kernel), ctypes.byref(c)), "last_launch_count")
        return c.value


class Octree:
    """Host-only octree + KIFMM lists (no GPU needed); coordinates in [0,1)^3."""

    def __init__(self, tree_pts, max_pts, pbc=0, sl=None, dl=None, trg=None):
        L = octree_lib()
        tp = _arr(tree_pts, 3)
        sl = _arr(sl if sl is not None else np.zeros((0, 3)), 3)
        dl = _arr(dl if dl is not None else np.zeros((0, 3)), 3)
        trg = _arr(trg if trg is not None else np.zeros((0, 3)), 3)
        self.t = L.stk_octree_build(_ptr(tp), len(tp), int(max_pts), int(pbc), _ptr(sl), len(sl), _ptr(dl), len(dl),
                                    _ptr(trg), len(trg))
        if not self.t:
            raise StkError(7, "stk_octree_build")
        sizes = np.zeros(7, dtype=np.int64)
        check(L.stk_octree_sizes(self.t, sizes.ctypes.data_as(P_ll)))
        self.num_nodes, self.num_leaves, self.depth = int(sizes[0]), int(sizes[1]), int(sizes[2])
        self.list_sizes = dict(U=int(sizes[3]), V=int(sizes[4]), W=int(sizes[5]), X=int(sizes[6]))
        nn = self.num_nodes
        self.level = np.zeros(nn, np.int32)
        self.parent = np.zeros(nn, np.int32)
        self.first_child = np.zeros(nn, np.int32)
        self.ixyz = np.zeros((nn, 3), np.int32)
        check(L.stk_octree_nodes(self.t, self.level.ctypes.data_as(P_i), self.parent.ctypes.data_as(P_i),
                                 self.first_child.ctypes.data_as(P_i), self.ixyz.ctypes.data_as(P_i)))
        self.n = (len(sl), len(dl), len(trg))

    def __del__(self):
        t = getattr(self, "t", None)
        if t:
            octree_lib().stk_octree_free(t)
            self.t = None

    def list(self, which: str):
        w = "UVWX".index(which)
        off = np.zeros(self.num_nodes + 1, np.int32)
        ent = np.zeros(max(self.list_sizes[which], 1), np.int32)
        check(octree_lib().stk_octree_list(self.t, w, off.ctypes.data_as(P_i), ent.ctypes.data_as(P_i)))
        return off, ent[:self.list_sizes[which]]

    def far_owners(self, nranks: int):
        """Owner rank of each node's M2L / S2L in a far field split over nranks (stk_octree_far_owners)."""
        o = np.zeros(self.num_nodes, np.int32)
        check(octree_lib().stk_octree_far_owners(self.t, int(nranks), o.ctypes.data_as(P_i)))
        return o

    def point_set(self, k: int):
        n = self.n[k]
        perm = np.zeros(max(n, 1), np.int32)
        b = np.zeros(self.num_nodes, np.int32)
        e = np.zeros(self.num_nodes, np.int32)
        check(octree_lib().stk_octree_set(self.t, k, perm.ctypes.data_as(P_i), b.ctypes.data_as(P_i),
                                   e.ctypes.data_as(P_i)))
        return perm[:n], b, e


def device_view(ptr: int, n: int, dtype="float64"):
    """A torch CUDA tensor aliasing n values at device address ptr (no copy)."""
    import torch

    class _Arr:
        __cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str, "data": (int(ptr), False),
                                    "version": 2}
    return torch.as_tensor(_Arr(), device="cuda")


def torch_allreduce(group=None):
    """A collective for Stk3DFMM.set_allreduce over a torch.distributed process group
    (NCCL for one process per GPU): all_reduce (sum) of the library's device buffer on
    the library's stream."""
    import torch
    import torch.distributed as dist

    def fn(ptr, n, stream):
        t = device_view(ptr, n)
        with torch.cuda.stream(torch.cuda.ExternalStream(int(stream) if stream else 0)):
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return 0
    return fn
