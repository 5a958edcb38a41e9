"""CPU FP64 oracle -- TEST INFRASTRUCTURE ONLY.

ctypes access to ``oracle/liboracle.so`` (the C restatement in stk_oracle.c) and,
where it was built, ``oracle/_ref/libstk_ref.so`` (the reference's own
Test/SimpleKernel.cpp).  Only tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline legs import this module; the product package never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libstk_ref.so")

# micro-kernel ids (same numbering as include/stkfmm_b200.h, enum stk_ukernel)
UK_LAPLACE_P = 0
UK_LAPLACE_PGRAD = 1
UK_LAPLACE_DIPOLEP = 2
UK_LAPLACE_DIPOLEPGRAD = 3
UK_STOKES_VEL = 4
UK_RPY_U = 5
UK_RPY_ULAPU = 6
UK_STK_ULAPU = 7
UK_STOKES_REGVEL = 8
UK_STOKES_PVEL = 9
UK_STOKES_DOUBLEPVEL = 10
# 11 .. 15 are fused / adjoint device micro-kernels without an oracle body
UK_LAPLACE_PGRADGRAD = 16
UK_LAPLACE_DIPOLEPGRADGRAD = 17
UK_LAPLACE_QUADP = 18
UK_LAPLACE_QUADPGRADGRAD = 19
UK_STOKES_PVELGRAD, UK_STOKES_DOUBLEPVELGRAD, UK_STOKES_PVELLAPLACIAN, UK_STOKES_DOUBLELAPLACIAN, \
    UK_STOKES_TRACTION, UK_STOKES_DOUBLETRACTION, UK_STOKES_REGFTVEL, UK_STOKES_REGFTVELOMEGA, \
    UK_STOKES_VELOMEGA = range(20, 29)
UK_NAMES = ["laplace_p", "laplace_pgrad", "laplace_dipolep", "laplace_dipolepgrad", "stokes_vel",
            "rpy_u", "rpy_ulapu", "stk_ulapu", "stokes_regvel", "stokes_pvel", "stokes_doublepvel",
            None, None, None, None, None,
            "laplace_pgradgrad", "laplace_dipolepgradgrad", "laplace_quadp", "laplace_quadpgradgrad",
            "stokes_pvelgrad", "stokes_doublepvelgrad", "stokes_pvellaplacian", "stokes_doublelaplacian",
            "stokes_traction", "stokes_doubletraction", "stokes_regftvel", "stokes_regftvelomega",
            "stokes_velomega"]
UK_SDIM = [1, 1, 3, 3, 3, 4, 4, 3, 4, 4, 9, 0, 0, 0, 0, 0, 1, 3, 9, 9, 4, 9, 4, 9, 4, 9, 7, 7, 3]
UK_TDIM = [1, 4, 1, 4, 3, 3, 6, 6, 3, 4, 4, 0, 0, 0, 0, 0, 10, 10, 1, 10, 16, 16, 7, 7, 9, 9, 3, 6, 6]

# reference SimpleKernel selectors (oracle/ref_driver.cpp)
REF_STOKES_SL, REF_LAP_SL_PGRAD, REF_LAP_DL_PGRAD, REF_STOKES_SL_RPY, REF_STOKES_REG_SL_VEL, \
    REF_STOKES_SL_PVEL, REF_STOKES_DL_PVEL, REF_LAP_SL_PGRADGRAD, REF_LAP_DL_PGRADGRAD, \
    REF_LAP_QPGRADGRAD, REF_STOKES_SL_PVELGRAD, REF_STOKES_DL_PVELGRAD, REF_STOKES_SL_PVELLAP, \
    REF_STOKES_DL_PVELLAP, REF_STOKES_SL_TRACTION, REF_STOKES_DL_TRACTION, REF_STOKES_REG_SL_VELOMEGA = range(17)
REF_DIMS = {REF_STOKES_SL: (3, 6), REF_LAP_SL_PGRAD: (1, 4), REF_LAP_DL_PGRAD: (3, 4),
            REF_STOKES_SL_RPY: (4, 6), REF_STOKES_REG_SL_VEL: (4, 3), REF_STOKES_SL_PVEL: (4, 4),
            REF_STOKES_DL_PVEL: (9, 4), REF_LAP_SL_PGRADGRAD: (1, 10), REF_LAP_DL_PGRADGRAD: (3, 10),
            REF_LAP_QPGRADGRAD: (9, 10), REF_STOKES_SL_PVELGRAD: (4, 16), REF_STOKES_DL_PVELGRAD: (9, 16),
            REF_STOKES_SL_PVELLAP: (4, 7), REF_STOKES_DL_PVELLAP: (9, 7), REF_STOKES_SL_TRACTION: (4, 9),
            REF_STOKES_DL_TRACTION: (9, 9), REF_STOKES_REG_SL_VELOMEGA: (7, 6)}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


# Where this recipe looks for the reference source tree (STKFMM_REF_TREE overrides).
REF_TREE = os.environ.get("STKFMM_REF_TREE", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference tree is present)."""
    cmd = ["make", "-C", HERE]
    if os.path.isdir(REF_TREE):
        cmd.append("REF=" + REF_TREE)
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(HERE, "stk_oracle.c")):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_direct.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        _lib.oracle_lists.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _dp, _dp, _dp,
                                      _dp, ctypes.c_double, ctypes.c_int]
        _lib.oracle_surface.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int, _dp]
        _lib.oracle_uk_scale.restype = ctypes.c_double
        _lib.oracle_uk_pair.argtypes = [ctypes.c_int, _dp, _dp, _dp]
        _lib.oracle_regvel_adjoint.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, _dp, _dp,
                                               ctypes.c_int]
        _lib.oracle_ewald.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                      _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        _lib.oracle_ewald2d.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref_tree():
    """The reference source tree oracle/_ref was built from (recorded by
    oracle/Makefile), or None where it is absent."""
    path = os.path.join(HERE, "_ref", "ref_tree.txt")
    if not os.path.exists(path):
        return None
    tree = open(path).read().strip()
    return tree if os.path.isdir(tree) else None


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise FileNotFoundError("oracle/_ref/libstk_ref.so not built (needs the reference tree)")
        _ref = ctypes.CDLL(_REF)
        _ref.ref_simple_direct.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_int, _dp,
                                           _dp, ctypes.c_int, ctypes.c_int]
        _ref.ref_simple_lists.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, _ip, _ip, _ip, _ip, _dp, _dp,
                                          ctypes.c_int, _dp, _dp, ctypes.c_int, ctypes.c_int]
        _ref.ref_surface.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int, _dp]
        _ref.ref_ukernel_direct.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        _ref.ref_kernel_composition.argtypes = [ctypes.c_uint, _ip, _ip, ctypes.c_char_p, ctypes.c_int]
        _ref.ref_kernel_scaling.argtypes = [ctypes.c_uint, ctypes.c_double, _dp, _dp, _dp, _ip]
        _ref.ref_evaluate_kernel.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp,
                                             _dp]
        _ref.ref_periodize.argtypes = [ctypes.c_uint, ctypes.c_int, _dp, ctypes.c_int, _dp, _ip]
        _ref.ref_wall_direct.argtypes = [ctypes.c_uint, _dp, ctypes.c_double, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp,
                                         _dp]
        _ref.ref_stk3d_direct.argtypes = [ctypes.c_uint, _dp, ctypes.c_double, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                          _dp, _dp, ctypes.c_int, _dp, _dp]
    return _ref


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def uk_scale(uk: int) -> float:
    return lib().oracle_uk_scale(uk)


def direct(uk: int, src, sval, trg, out=None, nthreads: int = 0):
    """out += scale * sum_s K_uk(trg - src) sval   (FMMData::evaluateKernel semantics)."""
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), UK_SDIM[uk]) if len(src) else np.zeros((0, UK_SDIM[uk])))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), UK_TDIM[uk]))
    assert out.dtype == np.float64 and out.flags.c_contiguous
    rc = lib().oracle_direct(uk, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return out


def lists(uk: int, trg_begin, trg_end, list_off, list_src, list_shift, src_begin, src_end, src, sval, trg,
          out=None, period: float = 1.0, nthreads: int = 0):
    """out += sum over an explicit target-box / source-box list (see stk_oracle.c:oracle_lists)."""
    tb, ptb = _i(trg_begin)
    te, pte = _i(trg_end)
    lo, plo = _i(list_off)
    ls, pls = _i(list_src)
    if list_shift is None:
        psh = None
    else:
        lsh, psh = _i(list_shift)
    sb, psb = _i(src_begin)
    se, pse = _i(src_end)
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), UK_TDIM[uk]))
    rc = lib().oracle_lists(uk, len(tb), ptb, pte, plo, pls, psh, psb, pse, ps, pv, pt, out.ctypes.data_as(_dp),
                            period, nthreads)
    assert rc == 0
    return out


def surface(p: int, c, alpha: float, depth: int):
    n = 6 * (p - 1) ** 2 + 2
    c, pc = _d(np.asarray(c, dtype=np.float64).reshape(3))
    out = np.zeros((n, 3))
    rc = lib().oracle_surface(p, pc, alpha, depth, out.ctypes.data_as(_dp))
    assert rc == 0
    return out


def ref_surface(p: int, c, alpha: float, depth: int):
    """The reference's own stkfmm::surface (stkfmm_helpers.hpp:46-85), from oracle/_ref."""
    n = 6 * (p - 1) ** 2 + 2
    c, pc = _d(np.asarray(c, dtype=np.float64).reshape(3))
    out = np.zeros((n, 3))
    rc = ref().ref_surface(p, pc, alpha, depth, out.ctypes.data_as(_dp))
    assert rc == 0
    return out


def ref_ukernel_direct(uk: int, src, sval, trg, out=None):
    """The reference's own micro-kernel body for id `uk` (the uKerEval of the
    STKFMM struct, Lib/include/STKFMM/*Kernel.hpp, compiled in oracle/_ref) over
    all (target, source) pairs: out += scale * sum_s K(trg - src) sval."""
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), UK_SDIM[uk]))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), UK_TDIM[uk]))
    assert out.dtype == np.float64 and out.flags.c_contiguous
    rc = ref().ref_ukernel_direct(uk, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp))
    assert rc == 0, uk
    return out


def ref_kernel_composition(kernel: int):
    """(slots, dims, name) of the reference's composite for a top-level kernel, as
    its headers' BuildKernel calls record them: slots = micro-kernel ids of (S2T
    SL, S2T DL, S2M SL, S2M DL, M2M = M2L = L2L, M2T, L2T, S2L SL, S2L DL), -1
    for none; dims = (ker_dim[0], surf_dim or 0 where PVFMM's default applies,
    ker_dim[1])."""
    slots = np.zeros(9, dtype=np.int32)
    dims = np.zeros(3, dtype=np.int32)
    name = ctypes.create_string_buffer(64)
    rc = ref().ref_kernel_composition(kernel, slots.ctypes.data_as(_ip), dims.ctypes.data_as(_ip), name, 64)
    assert rc == 0, kernel
    return [int(x) for x in slots], [int(x) for x in dims], name.value.decode()


def ref_evaluate_kernel(kernel: int, p2p: int, src, sval, trg, tdim: int):
    """The reference's own FMMData::evaluateKernel (Lib/src/FMMData.cpp:252-283,
    compiled in oracle/_ref): (ntrg, tdim) += the sub-kernel p2p selects over all
    pairs (1 SLS2T, 2 DLS2T, 4 L2T); zeros where the kernel has no such sub-kernel."""
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), -1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    out = np.zeros((len(trg), tdim))
    rc = ref().ref_evaluate_kernel(kernel, p2p, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp))
    assert rc == 0, kernel
    return out


def ref_wall_direct(kernel: int, src, val, trg, origin=(0.0, 0.0, 0.0), box: float = 1.0):
    """The reference's own StkWallFMM (Lib/src/StkWallFMM.cpp), its FMMs replaced
    by exact direct sums: the wall image system as the reference composes it."""
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    val, pv = _d(np.asarray(val).reshape(len(src), -1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    o, po = _d(np.asarray(origin, dtype=np.float64).reshape(3))
    out = np.zeros((len(trg), 3 if kernel == 8 else 6))
    rc = ref().ref_wall_direct(kernel, po, box, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp))
    assert rc == 0, kernel
    return out


def ref_stk3d_direct(kernel: int, sl, slv, trg, tdim: int, dl=None, dlv=None, origin=(0.0, 0.0, 0.0),
                     box: float = 1.0):
    """The reference's own Stk3DFMM (Lib/src/Stk3DFMM.cpp: box scaling, scaleSrc /
    scaleTrg) in free space, its FMM replaced by the exact direct sum."""
    sl, psl = _d(np.asarray(sl).reshape(-1, 3))
    slv, pslv = _d(np.asarray(slv).reshape(len(sl), -1))
    ndl = 0 if dl is None else len(dl)
    dl, pdl = _d(np.zeros((1, 3)) if dl is None else np.asarray(dl).reshape(-1, 3))
    dlv, pdlv = _d(np.zeros((1, 1)) if dlv is None else np.asarray(dlv).reshape(ndl, -1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    o, po = _d(np.asarray(origin, dtype=np.float64).reshape(3))
    out = np.zeros((len(trg), tdim))
    rc = ref().ref_stk3d_direct(kernel, po, box, len(sl), psl, pslv, ndl, pdl, pdlv, len(trg), pt,
                                out.ctypes.data_as(_dp))
    assert rc == 0, kernel
    return out


def ref_periodize(kernel: int, p: int, equiv):
    """1 + what the reference's own FMMData::periodizeFMM (FMMData.cpp:203-247)
    adds to each target component, for a triply periodic FMM of order p whose
    root upward-equivalent density is `equiv` (stand-in FMM, unit box).  Needs
    $PVFMM_DIR/pdata/M2C_<kernel>_3D3D_p<p> to exist (its values are unused)."""
    equiv, pe = _d(np.asarray(equiv, dtype=np.float64).reshape(-1))
    trg = np.zeros(16)
    kdim = np.zeros(1, dtype=np.int32)
    rc = ref().ref_periodize(kernel, p, pe, len(equiv), trg.ctypes.data_as(_dp), kdim.ctypes.data_as(_ip))
    assert rc == 0, kernel
    return trg[:kdim[0]].copy()


def ref_kernel_scaling(kernel: int, sf: float):
    """(sl, dl, trg) factors the reference's own FMMData applies around the FMM
    for a box with scale factor sf (scaleSrc / scaleTrg, Lib/src/FMMData.cpp:285-470,
    compiled in oracle/_ref); dl is empty for kernels without a double layer."""
    sl, dl, trg = np.zeros(16), np.zeros(16), np.zeros(16)
    dims = np.zeros(3, dtype=np.int32)
    rc = ref().ref_kernel_scaling(kernel, sf, sl.ctypes.data_as(_dp), dl.ctypes.data_as(_dp), trg.ctypes.data_as(_dp),
                                  dims.ctypes.data_as(_ip))
    assert rc == 0, kernel
    return sl[:dims[0]].copy(), dl[:dims[1]].copy(), trg[:dims[2]].copy()


def regvel_adjoint(src, sval, trg, w, nthreads: int = 0):
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1, 4))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    w, pw = _d(np.asarray(w).reshape(-1, 3))
    gf = np.zeros((len(src), 3))
    gx = np.zeros((len(src), 3))
    rc = lib().oracle_regvel_adjoint(len(src), ps, pv, len(trg), pt, pw, gf.ctypes.data_as(_dp),
                                     gx.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return gf, gx


def ref_direct(which: int, src, sval, trg, out=None, nthreads: int = 0):
    """Run the reference's own SimpleKernel over all pairs (runSimpleKernel protocol)."""
    sd, td = REF_DIMS[which]
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1, sd))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    rc = ref().ref_simple_direct(which, len(src), ps, pv, sd, len(trg), pt, out.ctypes.data_as(_dp), td, nthreads)
    assert rc == 0
    return out


def ref_lists(which: int, trg_begin, trg_end, list_off, list_src, src_begin, src_end, src, sval, trg, out=None,
              nthreads: int = 0):
    sd, td = REF_DIMS[which]
    tb, ptb = _i(trg_begin)
    te, pte = _i(trg_end)
    lo, plo = _i(list_off)
    ls, pls = _i(list_src)
    sb, psb = _i(src_begin)
    se, pse = _i(src_end)
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    rc = ref().ref_simple_lists(which, len(tb), ptb, pte, plo, pls, psb, pse, ps, pv, sd, pt,
                                out.ctypes.data_as(_dp), td, nthreads)
    assert rc == 0
    return out


# The reference's micro-kernel bodies in a PVFMM-style SIMD pair loop
# (ref_simd.cpp, oracle/_ref/libstk_ref_simd_{avx512,avx2}.so): selector -> (micro-kernel id, sdim, tdim)
REF_SIMD = {0: (UK_LAPLACE_PGRAD, 1, 4), 1: (UK_LAPLACE_DIPOLEPGRAD, 3, 4), 2: (UK_RPY_ULAPU, 4, 6),
            3: (UK_STOKES_REGVEL, 4, 3), 4: (UK_STOKES_PVEL, 4, 4), 5: (UK_STOKES_DOUBLEPVEL, 9, 4)}
REF_SIMD_LAP_PGRAD, REF_SIMD_LAP_DIPOLEPGRAD = 0, 1
_ref_simd = None


def _cpu_has_avx512() -> bool:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return " avx512f " in line + " "
    except OSError:
        pass
    return False


def ref_simd_path():
    """The SIMD baseline library for this host's vector ISA (AVX-512 when the CPU has it)."""
    return os.path.join(HERE, "_ref", "libstk_ref_simd_%s.so" % ("avx512" if _cpu_has_avx512() else "avx2"))


def ref_simd_available() -> bool:
    return os.path.exists(ref_simd_path())


def ref_simd():
    global _ref_simd
    if _ref_simd is None:
        L = ctypes.CDLL(ref_simd_path())
        L.ref_simd_lists.argtypes = [ctypes.c_int, ctypes.c_int] + [_ip] * 7 + [_dp] * 3 + [ctypes.c_double, _dp,
                                                                                         ctypes.c_int]
        L.ref_simd_direct.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
        _ref_simd = L
    return _ref_simd


def ref_simd_lists(which: int, trg_begin, trg_end, list_off, list_src, list_shift, src_begin, src_end, src, sval,
                   trg, out=None, period: float = 1.0, nthreads: int = 0):
    """out += the reference micro-kernel `which` (REF_SIMD) over an explicit list, PVFMM's SIMD loop."""
    _, sd, td = REF_SIMD[which]
    tb, ptb = _i(trg_begin)
    te, pte = _i(trg_end)
    lo, plo = _i(list_off)
    ls, pls = _i(list_src)
    lsh, plsh = _i(list_shift) if list_shift is not None else (None, None)
    sb, psb = _i(src_begin)
    se, pse = _i(src_end)
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape[1] == td
    rc = ref_simd().ref_simd_lists(which, len(tb), ptb, pte, plo, pls, plsh, psb, pse, ps, pv, pt, period,
                                   out.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return out


def ref_simd_direct(which: int, src, sval, trg, out=None, nthreads: int = 0):
    """out += the reference micro-kernel `which` (REF_SIMD) over all sources, PVFMM's SIMD loop."""
    _, sd, td = REF_SIMD[which]
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(-1))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    rc = ref_simd().ref_simd_direct(which, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return out


def regvel_fd_local(idx, nb_off, nb, x, val, w, h=1e-6, nthreads=0):
    """Central differences (step h, FP64) of L = sum w.u for the regularized-Stokeslet sum over a
    fixed pair set with sources = targets: dL/dx_i (point moved as source and target) and dL/df_i
    for each checked point i = idx[c], over the pairs that involve it (its neighbour list
    nb[nb_off[c]:nb_off[c+1]], i included).  Returns (gx, gf), each (len(idx), 3)."""
    idx, pidx = _i(idx)
    nb_off, po = _i(nb_off)
    nb, pn = _i(nb)
    x, px = _d(np.asarray(x).reshape(-1, 3))
    val, pv = _d(np.asarray(val).reshape(-1, 4))
    w, pw = _d(np.asarray(w).reshape(-1, 3))
    gx = np.zeros((len(idx), 3))
    gf = np.zeros((len(idx), 3))
    L = lib()
    L.oracle_regvel_fd_local.argtypes = [ctypes.c_int, _ip, _ip, _ip, _dp, _dp, _dp, ctypes.c_double, _dp, _dp,
                                         ctypes.c_int]
    rc = L.oracle_regvel_fd_local(len(idx), pidx, po, pn, px, pv, pw, h, gx.ctypes.data_as(_dp),
                                  gf.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return gx, gf


EWALD_LAPLACE, EWALD_STOKES = 0, 1


def ewald(kind: int, src, sval, trg, xi: float = 7.0, nreal: int = 1, nwave: int = 14, out=None, nthreads: int = 0):
    """out += triply periodic (unit cell) sum by Ewald summation (see stk_oracle.c:oracle_ewald).

    kind EWALD_LAPLACE: charges (n, 1) -> potential + gradient (n, 4), zero-mean Green's function;
    kind EWALD_STOKES: forces (n, 3) -> velocity (n, 3); kind EWALD_PVEL: (f, trD) (n, 4) -> pressure and
    velocity of stokes_pvel (n, 4); kind EWALD_LAPLACE_HESS: charges -> potential, gradient and
    Hessian (n, 10).  Defaults (xi = 7, one real-space image
    shell, |m| <= 14) converge to ~1e-15 for points in [0, 1)^3.
    """
    sd, td = {EWALD_LAPLACE: (1, 4), EWALD_STOKES: (3, 3), 2: (4, 4), 3: (1, 10)}[kind]
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), sd))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    assert out.dtype == np.float64 and out.flags.c_contiguous
    rc = lib().oracle_ewald(kind, xi, nreal, nwave, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return out


EWALD_PVEL = 2
# Laplace charges -> potential, gradient and Hessian (xx xy xz yy yz zz), laplace_pgradgrad's layout
EWALD_LAPLACE_HESS = 3


def ewald_cells(kind: int, src, sval, trg, xi: float = 16.0, nwave: int = 28, out=None, nthreads: int = 0):
    """The triply periodic sums of ewald() (kinds EWALD_LAPLACE, EWALD_STOKES, EWALD_LAPLACE_HESS) for
    millions of sources: real space through a cell list (cutoff 5.3 / xi, below 1/3), wave space
    through structure factors over the sphere |m| <= nwave (stk_oracle.c:oracle_ewald_cells).  The
    defaults converge to ~1e-13 for points in [0, 1)^3."""
    sd, td = {EWALD_LAPLACE: (1, 4), EWALD_STOKES: (3, 3), 3: (1, 10)}[kind]
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), sd))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    L = lib()
    L.oracle_ewald_cells.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, _dp,
                                     ctypes.c_int, _dp, _dp, ctypes.c_int]
    rc = L.oracle_ewald_cells(kind, xi, nwave, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp), nthreads)
    assert rc == 0, rc
    return out


def ewald_stokes_laplacian_cells(src, f, trg, **kw):
    """ewald_stokes_laplacian through ewald_cells (for millions of sources)."""
    src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(f, dtype=np.float64).reshape(len(src), 3)
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    sym = [[4, 5, 6], [5, 7, 8], [6, 8, 9]]
    out = np.zeros((len(trg), 3))
    for j in range(3):
        h = ewald_cells(EWALD_LAPLACE_HESS, src, f[:, j:j + 1], trg, **kw)
        for i in range(3):
            out[:, i] -= h[:, sym[i][j]]
    out += f.sum(0)
    return out




def ewald_stokes_laplacian(src, f, trg):
    """Laplacian of the triply periodic Stokeslet velocity (the unit cell's
    Hasimoto sum of stokes_vel, 1/8pi (delta/r + r r^T/r^3), k = 0 mode dropped;
    M2L/Stokeslet/Stokes3D3D.cpp:19-68) at trg, away from the sources: the
    laplacian output of rpy_ulapu / stk_ulapu (RPYKernel.hpp:52-129) summed over
    all images.  In Fourier space -k^2 G(k) = -8 pi delta + 8 pi k k^T / k^2;
    the second part is -2 d_i d_j of the periodic 1/r, the first the periodic
    delta minus its mean, which off the sources leaves + delta_ij per unit volume.
    So lap u_i = -sum_j H_ij[f_j] + F_i, with H[q] the Hessian of the zero-mean
    periodic potential of charges q (ewald kind EWALD_LAPLACE_HESS) and F the
    net force."""
    src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(f, dtype=np.float64).reshape(len(src), 3)
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    # Hessian entries (xx xy xz yy yz zz) at columns 4..9 of the EWALD_LAPLACE_HESS output
    sym = [[4, 5, 6], [5, 7, 8], [6, 8, 9]]
    out = np.zeros((len(trg), 3))
    for j in range(3):
        h = ewald(EWALD_LAPLACE_HESS, src, f[:, j:j + 1], trg)
        for i in range(3):
            out[:, i] -= h[:, sym[i][j]]
    out += f.sum(0)
    return out


def pvel_pxyz_terms(src, sval, trg):
    """What the reference's triply periodic StokesPVel far field adds to the Ewald
    sum of (f, trD) sources, as (pressure, velocity) at trg (unit cell, points in
    [0, 1)^3):

    * pressure (x - 1/2) . F with F = sum f, a mean pressure gradient that balances
      a net force (M2L/StokesPVel/StokesPVel3D3D.cpp:203-206, in the M2C operator);
    * velocity (1/2) sum y trD, half the trD dipole moment: the M2C operator adds
      half of each root equivalent point's position wrapped into the cell
      (StokesPVel3D3D.cpp:211-218) and FMMData::periodizeFMM the unwrapped rest
      (Lib/src/FMMData.cpp:203-247); the root's equivalent density has the
      sources' trD dipole moment.

    The velocity term applies to PVel, PVelGrad and PVelLaplacian.  The pressure
    term is fitted through the local expansion like every M2C value, and with no
    velocity beside it it is not a Stokes flow, so an FMM reproduces it only
    approximately; it vanishes for force-free sources.
    """
    src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
    sval = np.asarray(sval, dtype=np.float64).reshape(len(src), 4)
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((len(trg), 4))
    out[:, 0] = (trg - 0.5) @ sval[:, :3].sum(0)
    out[:, 1:] = 0.5 * (src * sval[:, 3:4]).sum(0)
    return out


def laplace_pxyz_neutraliser(total_charge: float, trg):
    """Potential and gradient (n, 4) at trg of the reference's triply periodic
    Laplace neutraliser: each equivalent charge of the root is paired with an
    opposite one at the cell centre N = (1/2, 1/2, 1/2)
    (M2L/Laplace/Laplace3D3D.cpp:266-273), whose periodic sum is taken without
    the 5 x 5 x 5 block of images nearest to N (DIRECTLAYER = 2,
    M2L/SVD_pvfmm.hpp:34).  For a total charge Q it contributes
    -Q [G_ewald(x - N) - sum_{|s_i| <= 2} 1 / (4 pi |x - N - s|)]."""
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    cen = np.array([[0.5, 0.5, 0.5]])
    one = np.ones((1, 1))
    g = ewald(EWALD_LAPLACE, cen, one, trg)
    near = np.zeros((len(trg), 4))
    for a in range(-2, 3):
        for b in range(-2, 3):
            for c in range(-2, 3):
                direct(UK_LAPLACE_PGRAD, cen + np.array([a, b, c]), one, trg, out=near)
    return -total_charge * (g - near)


def ewald2d(kind: int, src, sval, trg, out=None, nthreads: int = 0):
    """out += doubly periodic (x, y; z free) sum per pair (see stk_oracle.c:oracle_ewald2d).

    kind EWALD_LAPLACE: (n, 1) -> (n, 4) potential + gradient; EWALD_STOKES: (n, 3) -> (n, 3);
    EWALD_PVEL: (f, trD) (n, 4) -> (pressure, velocity) (n, 4); EWALD_LAPLACE_HESS: (n, 1) -> (n, 10).
    """
    sd, td = {EWALD_LAPLACE: (1, 4), EWALD_STOKES: (3, 3), EWALD_PVEL: (4, 4), EWALD_LAPLACE_HESS: (1, 10)}[kind]
    src, ps = _d(np.asarray(src).reshape(-1, 3))
    sval, pv = _d(np.asarray(sval).reshape(len(src), sd))
    trg, pt = _d(np.asarray(trg).reshape(-1, 3))
    if out is None:
        out = np.zeros((len(trg), td))
    assert out.dtype == np.float64 and out.flags.c_contiguous
    rc = lib().oracle_ewald2d(kind, len(src), ps, pv, len(trg), pt, out.ctypes.data_as(_dp), nthreads)
    assert rc == 0
    return out



# ---------------------------------------------------------------------------
# No-slip wall image systems (StkWallFMM), restated over the oracle's sums.
# The wall is the plane z = z0; every source at height y3 = z - z0 > 0 has an
# image at z0 - y3.  The free-space sums are direct sums in physical units;
# pbc = 2 (PXY, unit period in x and y) uses the doubly periodic Ewald sums.
# ---------------------------------------------------------------------------
def _mirror(src, z0):
    img = np.array(src, dtype=np.float64, copy=True)
    img[:, 2] = 2.0 * z0 - img[:, 2]
    return img


def _ewald2d_dipole(src, d, trg):
    """Doubly periodic laplace_dipolepgrad sum: potential -d.grad G and gradient -d.grad grad G."""
    out = np.zeros((len(trg), 4))
    hidx = {(0, 0): 4, (0, 1): 5, (0, 2): 6, (1, 1): 7, (1, 2): 8, (2, 2): 9}
    for k in range(3):
        h = ewald2d(EWALD_LAPLACE_HESS, src, np.ascontiguousarray(d[:, k:k + 1]), trg)
        out[:, 0] -= h[:, 1 + k]
        for j in range(3):
            out[:, 1 + j] -= h[:, hidx[(min(j, k), max(j, k))]]
    return out


def wall_stokes(src, f, trg, z0: float = 0.0, pbc: int = 0):
    """Stokeslets above a no-slip wall: StkWallFMM::evalStokes (Lib/src/StkWallFMM.cpp:154-208).

    Stokes sum of (fx, fy, 0) at the sources and (-fx, -fy, 0) at the images;
    laplace_pgrad of charges -fz/2 (sources), +fz/2 (images) plus dipoles
    (-y3 fx, -y3 fy, y3 fz) at the images; laplace_pgradgrad of charges fz y3
    (sources), -fz y3 (images).  u_j = uS_j + uL2_{grad j} / 2 + x3 uL1D_{grad j},
    u_z -= uL1D_pot, with x3 the target's height above the wall.
    """
    src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
    f = np.asarray(f, dtype=np.float64).reshape(-1, 3)
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    n = len(src)
    img = _mirror(src, z0)
    s2 = np.concatenate([src, img])
    y3 = src[:, 2] - z0
    x3 = trg[:, 2] - z0
    v_stk = np.zeros((2 * n, 3))
    v_stk[:n, :2] = f[:, :2]
    v_stk[n:, :2] = -f[:, :2]
    v_l1 = np.concatenate([-0.5 * f[:, 2], 0.5 * f[:, 2]])[:, None]
    v_d = np.stack([-y3 * f[:, 0], -y3 * f[:, 1], y3 * f[:, 2]], 1)
    v_l2 = np.concatenate([f[:, 2] * y3, -f[:, 2] * y3])[:, None]
    if pbc == 0:
        u_s = direct(UK_STOKES_VEL, s2, v_stk, trg)
        u_l1d = direct(UK_LAPLACE_PGRAD, s2, v_l1, trg) + direct(UK_LAPLACE_DIPOLEPGRAD, img, v_d, trg)
        g_l2 = direct(UK_LAPLACE_PGRADGRAD, s2, v_l2, trg)[:, 1:4]
    elif pbc == 2:
        u_s = ewald2d(EWALD_STOKES, s2, v_stk, trg)
        u_l1d = ewald2d(EWALD_LAPLACE, s2, v_l1, trg) + _ewald2d_dipole(img, v_d, trg)
        g_l2 = ewald2d(EWALD_LAPLACE, s2, v_l2, trg)[:, 1:4]
    else:
        raise ValueError("pbc must be 0 or 2")
    u = u_s + 0.5 * g_l2 + x3[:, None] * u_l1d[:, 1:4]
    u[:, 2] -= u_l1d[:, 0]
    return u


def wall_rpy(src, fb, trg, z0: float = 0.0):
    """RPY spheres above a no-slip wall: StkWallFMM::evalRPY (Lib/src/StkWallFMM.cpp:210-292),
    free space.  fb rows (fx, fy, fz, b); output rows (u 3, lap u 3).

    rpy_ulapu of (fx, fy, 0, b) at the sources and (-fx, -fy, 0, b) at the images;
    SD: laplace_pgradgrad of charges -fz/2 (sources), +fz/2 (images) plus dipoles
    (-y3 fx, -y3 fy, y3 fz) at the images; SDZ: laplace_pgrad of charges y3 fz / 2,
    -y3 fz / 2 plus dipoles (0, 0, b^2 fz / 6) at sources and images; Q:
    laplace_quadpgradgrad of S = 2 b^2 / 6 (fz e_xx + fz e_yy + fx e_zx + fy e_zy)
    at the images.
    """
    src = np.asarray(src, dtype=np.float64).reshape(-1, 3)
    fb = np.asarray(fb, dtype=np.float64).reshape(-1, 4)
    trg = np.asarray(trg, dtype=np.float64).reshape(-1, 3)
    n = len(src)
    img = _mirror(src, z0)
    s2 = np.concatenate([src, img])
    y3 = src[:, 2] - z0
    x3 = trg[:, 2] - z0
    f1, f2, f3, b = fb[:, 0], fb[:, 1], fb[:, 2], fb[:, 3]
    v_rpy = np.zeros((2 * n, 4))
    v_rpy[:n, 0], v_rpy[:n, 1], v_rpy[:n, 3] = f1, f2, b
    v_rpy[n:, 0], v_rpy[n:, 1], v_rpy[n:, 3] = -f1, -f2, b
    v_ls = np.concatenate([-0.5 * f3, 0.5 * f3])[:, None]
    v_ld = np.stack([-y3 * f1, -y3 * f2, y3 * f3], 1)
    v_lsz = np.concatenate([0.5 * y3 * f3, -0.5 * y3 * f3])[:, None]
    v_ldz = np.zeros((2 * n, 3))
    v_ldz[:n, 2] = b * b * f3 / 6.0
    v_ldz[n:, 2] = b * b * f3 / 6.0
    q = np.zeros((n, 9))
    tb = 2.0 * b * b / 6.0
    q[:, 0], q[:, 4], q[:, 6], q[:, 7] = tb * f3, tb * f3, tb * f1, tb * f2
    u_rpy = direct(UK_RPY_ULAPU, s2, v_rpy, trg)
    sd = direct(UK_LAPLACE_PGRADGRAD, s2, v_ls, trg) + direct(UK_LAPLACE_DIPOLEPGRADGRAD, img, v_ld, trg)
    sdz = direct(UK_LAPLACE_PGRAD, s2, v_lsz, trg) + direct(UK_LAPLACE_DIPOLEPGRAD, s2, v_ldz, trg)
    qq = direct(UK_LAPLACE_QUADPGRADGRAD, img, q, trg)
    u = np.zeros((len(trg), 6))
    for j in range(3):
        u[:, j] = u_rpy[:, j] + sdz[:, 1 + j] + x3 * sd[:, 1 + j] + x3 * qq[:, 1 + j]
    u[:, 2] -= sd[:, 0] + qq[:, 0]
    for j, h in ((3, 6), (4, 8), (5, 9)):
        u[:, j] = u_rpy[:, j] + 2.0 * sd[:, h] + 2.0 * qq[:, h]
    return u
