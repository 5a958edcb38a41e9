"""The C ABI library on a machine without a GPU: it loads, exports every symbol
include/stkfmm_b200.h declares, describes the kernels as the reference does, and
refuses to compute without a device (there is no CPU path)."""
import ctypes
import os
import re

import numpy as np
import pytest

import stkfmm_b200 as S
from conftest import cuda_available
from stkfmm_b200._lib import LIB_PATH, P_i, SIGNATURES, lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "stkfmm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n.startswith(("stk_", "Stk3DFMM_"))))


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) >= 40
    so = ctypes.CDLL(LIB_PATH)
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing
    # every declared function has a Python signature, and vice versa
    bound = {n for n, _, _ in SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_kernel_descriptors_match_reference():
    # (kdimSL, kdimDL, kdimTrg) from getKernelDimension (Lib/src/STKFMM.cpp:33-40)
    expect = {1: (1, 3, 4), 8: (3, 6, 3), 16: (4, 7, 6), 32: (4, 7, 3), 128: (4, 9, 4), 256: (4, 9, 16),
              512: (4, 9, 7), 1024: (4, 9, 9), 2: (1, 3, 10), 4: (9, 12, 10), 64: (7, 10, 6)}
    for k, d in expect.items():
        assert tuple(S.get_kernel_dimension(k)) == d
    assert S.get_kernel_name(S.KERNEL.LapPGrad) == "laplace_PGrad"
    assert S.get_kernel_name(S.KERNEL.Stokes) == "stokes_vel"
    assert S.get_kernel_name(S.KERNEL.RPY) == "rpy_ulapu"
    assert S.get_kernel_name(S.KERNEL.StokesRegVel) == "stokes_regvel"
    assert S.get_kernel_name(S.KERNEL.PVel) == "stokes_PVel"
    with pytest.raises(S.StkError):
        S.get_kernel_dimension(3)
    # slot compositions (RPYKernel.hpp:137-154): s2t rpy_ulapu, s2m rpy_u, m2x stokes_vel, m2t/l2t stk_ulapu
    assert [S.kernel_slot(16, s) for s in range(9)] == [6, -1, 5, -1, 4, 7, 7, 5, -1]
    # LapPGrad (LaplaceLayerKernel.hpp:314-326)
    assert [S.kernel_slot(1, s) for s in range(9)] == [1, 3, 0, 2, 0, 1, 1, 0, 2]
    # StokesRegVel (StokesRegSingleLayerKernel.hpp:211-218)
    assert [S.kernel_slot(32, s) for s in range(9)] == [8, -1, 8, -1, 4, 4, 4, 8, -1]
    # LapPGradGrad (LaplaceLayerKernel.hpp:328-341), LapQPGradGrad (LaplaceLayerKernel.hpp:343-356)
    assert [S.kernel_slot(2, s) for s in range(9)] == [16, 17, 0, 2, 0, 16, 16, 0, 2]
    assert [S.kernel_slot(4, s) for s in range(9)] == [19, -1, 18, -1, 0, 16, 16, 18, -1]
    assert S.ukernel_dims(S.UKERNEL.STOKES_SLDL_PVEL) == (13, 4)
    assert S.ukernel_dims(S.UKERNEL.LAPLACE_QUADPGRADGRAD) == (9, 10)
    # PVelGrad / PVelLaplacian / Traction (StokesLayerKernel.hpp:52-94): stokes_PVel translations
    assert [S.kernel_slot(256, s) for s in range(9)] == [20, 21, 9, 10, 9, 20, 20, 9, 10]
    assert [S.kernel_slot(512, s) for s in range(9)] == [22, 23, 9, 10, 9, 22, 22, 9, 10]
    assert [S.kernel_slot(1024, s) for s in range(9)] == [24, 25, 9, 10, 9, 24, 24, 9, 10]
    assert S.ukernel_dims(S.UKERNEL.STOKES_DOUBLEPVELGRAD) == (9, 16)
    # StokesRegVelOmega (StokesRegSingleLayerKernel.hpp:220-232)
    assert [S.kernel_slot(64, s) for s in range(9)] == [27, -1, 26, -1, 4, 28, 28, 26, -1]


def test_status_strings():
    L = lib()
    for st in range(9):
        assert L.stk_status_string(st)
    assert L.stk_status_string(6).decode().startswith("no CUDA device")


@pytest.mark.skipif(cuda_available(), reason="checks the no-device behaviour")
def test_no_cpu_fallback():
    L = lib()
    assert L.stk_device_count() == 0
    src = np.random.default_rng(0).random((10, 3))
    out = np.zeros((10, 3))
    with pytest.raises(S.StkError) as e:
        S.evaluate_kernel(S.KERNEL.Stokes, S.PPKERNEL.SLS2T, src, src, src, out)
    assert e.value.status == 6
    assert np.all(out == 0)
    with pytest.raises(S.StkError):
        S.Stk3DFMM(8, 64, 0, S.KERNEL.Stokes)
    assert not L.Stk3DFMM_create(8, 64, 0, 8)
    with pytest.raises(S.StkError):
        S.StkWallFMM(8, 64, 0, S.KERNEL.Stokes)
    assert not L.StkWallFMM_create(8, 64, 0, 8)


def test_setters_reject_null_handles():
    """The handle setters refuse a null handle and invalid flags before any device work."""
    L = lib()
    invalid_arg = 1  # STK_ERR_INVALID_ARG
    for fn, arg in (("Stk3DFMM_set_far_field", 1), ("StkWallFMM_set_far_field", 0), ("Stk3DFMM_set_precision", 0),
                    ("StkWallFMM_set_precision", 0), ("Stk3DFMM_set_shard", 0)):
        args = (None, arg, 1) if fn == "Stk3DFMM_set_shard" else (None, arg)
        assert getattr(L, fn)(*args) == invalid_arg, fn


def test_wall_create_rejects_bad_arguments():
    """StkWallFMM_create refuses a triply periodic box, kernels without a wall
    image system and invalid orders before it needs a device."""
    L = lib()
    assert not L.StkWallFMM_create(8, 64, 3, 8)  # PXYZ
    assert not L.StkWallFMM_create(8, 64, 0, 1)  # LapPGrad only
    assert not L.StkWallFMM_create(1, 64, 0, 8)  # order below 2
    assert not L.StkWallFMM_create(8, 0, 0, 16)  # no points per leaf
    dims = np.zeros(3, dtype=np.int32)
    assert L.StkWallFMM_get_kernel_dimension(16, dims.ctypes.data_as(P_i)) == 0
    assert tuple(dims) == (4, 7, 6)


def test_header_is_plain_c(tmp_path):
    """A C99 caller of the reference's C ABI (STKFMM.h, Stk3DFMM-c.cpp:5-67)
    compiles against include/stkfmm_b200.h with -pedantic, links the library and
    runs the no-device path."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    src = tmp_path / "caller.c"
    src.write_text(
        '#include "stkfmm_b200.h"\n#include <stdio.h>\n'
        "int main(void) {\n"
        "    int dims[3];\n"
        "    int rc = Stk3DFMM_get_kernel_dimension(STK_PVel, dims);\n"
        "    StkWallFMM *w = StkWallFMM_create(8, 64, STK_PAXIS_PXYZ, STK_Stokes);\n"
        '    printf("%d %d %d %d %d\\n", rc, dims[0], dims[1], dims[2], w == NULL);\n'
        "    return 0;\n}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.dirname(HEADER),
                    str(src), "-L", libdir, "-lstkfmm_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out == ["0", "4", "9", "4", "1"]


def test_surface_helper_matches_oracle():
    """stk_surface (host only) gives the reference's KIFMM surface points in the
    reference's order (pinned against the reference's own stkfmm::surface in
    tests/test_oracle.py), and refuses invalid arguments."""
    from oracle import oracle as O
    from stkfmm_b200._lib import P_d
    L = lib()
    c = np.array([0.1, -0.3, 0.7])
    for p in (2, 6, 10, 16):
        for depth in (0, 2):
            for alpha in (1.05, 2.95):
                out = np.zeros((6 * (p - 1) ** 2 + 2, 3))
                assert L.stk_surface(p, c.ctypes.data_as(P_d), alpha, depth, out.ctypes.data_as(P_d)) == 0
                ref = O.ref_surface(p, c, alpha, depth) if O.ref_available() else O.surface(p, c, alpha, depth)
                assert np.abs(out - ref).max() <= 4 * np.finfo(float).eps * np.abs(ref).max()
    out = np.zeros((2, 3))
    assert L.stk_surface(1, c.ctypes.data_as(P_d), 1.0, 0, out.ctypes.data_as(P_d)) == 1
    assert L.stk_surface(2, None, 1.0, 0, out.ctypes.data_as(P_d)) == 1



def test_kernel_tables_match_reference_compositions():
    """The library's per-slot micro-kernels, names and dimensions against the
    reference's own compositions: the BuildKernel calls of its kernel headers
    (LaplaceLayerKernel.hpp, StokesLayerKernel.hpp, RPYKernel.hpp,
    StokesRegSingleLayerKernel.hpp) compiled in oracle/_ref, for every kernel of
    Lib/src/STKFMM.cpp:18-31.  surf_dim is compared where the headers set it."""
    from oracle import oracle as O
    if not O.ref_available():
        pytest.skip("oracle/_ref needs the reference tree")
    for k in (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024):
        slots, dims, name = O.ref_kernel_composition(k)
        assert [S.kernel_slot(k, s) for s in range(9)] == slots, k
        assert S.get_kernel_name(k) == name, k
        mine = tuple(S.get_kernel_dimension(k))
        assert (mine[0], mine[2]) == (dims[0], dims[2]), k
        if dims[1]:
            assert mine[1] == dims[1], k


def test_reference_python_binding_drives_this_library():
    """The reference's own ctypes binding (Python/PySTKFMM.py, unmodified) with its
    library load pointed at this library, as a maintainer would repoint it: every
    call it makes binds and runs.  It reports the reference's kernel dimensions,
    and without a device its calls on the null handle return without writing."""
    import importlib.util
    import sys
    import types
    from oracle import oracle as O
    tree = O.ref_tree()
    src = os.path.join(tree, "Python", "PySTKFMM.py") if tree else None
    if not src or not os.path.exists(src):
        pytest.skip("the reference tree is not present")
    real = ctypes.cdll.LoadLibrary
    saved = sys.modules.get("mpi4py")
    sys.modules["mpi4py"] = types.SimpleNamespace(MPI=types.SimpleNamespace())  # imported, unused by these classes
    ctypes.cdll.LoadLibrary = lambda name: real(LIB_PATH if name == "libSTKFMM_SHARED.so" else name)
    try:
        spec = importlib.util.spec_from_file_location("PySTKFMM_reference", src)
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
    finally:
        ctypes.cdll.LoadLibrary = real
        if saved is None:
            sys.modules.pop("mpi4py", None)
        else:
            sys.modules["mpi4py"] = saved
    assert m.lib._name == LIB_PATH
    f = m.Stk3DFMM(8, 64, m.PAXIS.NONE, m.KERNEL.Stokes | m.KERNEL.PVel)
    for k in m.KERNEL:
        assert tuple(f.get_kernel_dimension(k)) == tuple(S.get_kernel_dimension(int(k)))
    w = m.StkWallFMM(8, 64, m.PAXIS.PXY, m.KERNEL.Stokes)
    assert tuple(w.get_kernel_dimension(m.KERNEL.RPY)) == (4, 7, 6)
    if not cuda_available():
        assert f.fmm.value is None and w.fmm.value is None
        pts = np.random.default_rng(0).random((10, 3))
        out = np.zeros((10, 3))
        f.set_box(np.zeros(3), 1.0)
        f.set_points(pts, pts, np.zeros((0, 3)))
        f.setup_tree(m.KERNEL.Stokes)
        f.evaluate_fmm(m.KERNEL.Stokes, pts, out, np.zeros((0, 3)))
        f.clear_fmm(m.KERNEL.Stokes)
        w.set_points(pts, pts, np.zeros((0, 3)))
        assert np.all(out == 0)
    del f, w


def test_reference_c_header_links_this_library(tmp_path):
    """A C caller compiled against the reference's own C header
    (Lib/include/STKFMM/STKFMM.h, whose functions return void) links this library
    and runs unchanged: the names, argument lists and calling convention match.
    Without a device, create returns NULL and the calls on it return."""
    import shutil
    import subprocess
    from oracle import oracle as O
    tree = O.ref_tree()
    hdir = os.path.join(tree, "Lib", "include", "STKFMM") if tree else None
    cc = shutil.which("gcc") or shutil.which("cc")
    if not hdir or not os.path.exists(os.path.join(hdir, "STKFMM.h")) or not cc:
        pytest.skip("the reference tree or a C compiler is not present")
    src = tmp_path / "caller.c"
    src.write_text(
        '#include <stdio.h>\n#include "STKFMM.h"\n'
        "int main(void) {\n"
        "    double xyz[6] = {0.1, 0.2, 0.3, 0.4, 0.5, 0.6}, f[6] = {1, 0, 0, 0, 1, 0}, u[6] = {0};\n"
        "    double origin[3] = {0, 0, 0};\n"
        "    Stk3DFMM *fmm = Stk3DFMM_create(8, 64, 0, 8);\n"
        "    Stk3DFMM_set_box(fmm, origin, 1.0);\n"
        "    Stk3DFMM_set_points(fmm, 2, xyz, 2, xyz, 0, NULL);\n"
        "    Stk3DFMM_setup_tree(fmm, 8);\n"
        "    Stk3DFMM_evaluate_fmm(fmm, 8, 2, f, 2, u, 0, NULL);\n"
        "    Stk3DFMM_show_active_kernels(fmm);\n"
        "    Stk3DFMM_destroy(fmm);\n"
        "    StkWallFMM *w = StkWallFMM_create(8, 64, 2, 8);\n"
        "    StkWallFMM_set_box(w, origin, 1.0);\n"
        "    StkWallFMM_destroy(w);\n"
        '    printf("%d %d %g\\n", fmm == NULL, w == NULL, u[0]);\n'
        "    return 0;\n}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", hdir, str(src), "-L", libdir, "-lstkfmm_b200",
                    "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    if not cuda_available():
        assert out[-3:] == ["1", "1", "0"]


def _cxx():
    import shutil
    return shutil.which("g++") or shutil.which("c++")


def _build(cxx, args, tmp_path, name):
    import subprocess
    libdir = os.path.dirname(LIB_PATH)
    exe = tmp_path / name
    subprocess.run([cxx, "-std=c++14"] + args + ["-L", libdir, "-lstkfmm_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    return exe


def test_cpp_interface(tmp_path):
    """include/stkfmm_b200.hpp mirrors the reference's C++ API (STKFMM.hpp,
    STKFMM_common.hpp): enums, asInteger, getKernelDimension / getKernelName,
    Stk3DFMM / StkWallFMM with the reference's constructors; a global
    `using Stk3DFMM = stkfmm::Stk3DFMM;` (as Test/Test.hpp writes) compiles; errors
    throw stkfmm::Error with the C status (LapGrad, outside the reference's kernel
    map, is refused; no device gives STK_ERR_NO_DEVICE)."""
    import subprocess
    cxx = _cxx()
    if not cxx:
        pytest.skip("no C++ compiler")
    src = tmp_path / "cpp_caller.cpp"
    src.write_text(r'''
#include "STKFMM/STKFMM.hpp"
#include <cstdio>
using Stk3DFMM = stkfmm::Stk3DFMM;
using StkWallFMM = stkfmm::StkWallFMM;
int main() {
    using namespace stkfmm;
    for (unsigned k = 1; k <= 1024; k *= 2) {
        auto d = getKernelDimension(static_cast<KERNEL>(k));
        std::printf("%u %d %d %d %s\n", k, std::get<0>(d), std::get<1>(d), std::get<2>(d),
                    getKernelName(static_cast<KERNEL>(k)).c_str());
    }
    try { getKernelDimension(KERNEL::LapGrad); } catch (const Error &e) { std::printf("lapgrad %d\n", e.status()); }
    try {
        auto fmm = Stk3DFMM(8, 64, PAXIS::PXY, asInteger(KERNEL::Stokes), false);
        std::printf("device %d\n", fmm.getMultOrder());
    } catch (const Error &e) { std::printf("nodevice %d\n", e.status()); }
    return 0;
}
''')
    exe = _build(cxx, ["-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.dirname(HEADER), str(src)], tmp_path,
                 "cpp_caller")
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    for line in lines[:11]:
        k, a, b, c, name = line.split()
        assert (int(a), int(b), int(c)) == tuple(S.get_kernel_dimension(int(k))) and name == S.get_kernel_name(int(k))
    assert lines[11] == "lapgrad 2"
    if not cuda_available():
        assert lines[12] == "nodevice 6"


def test_reference_demo_builds_against_this_library(tmp_path):
    """The reference's own Demo/Demo.cpp, unmodified, compiles against
    include/STKFMM/STKFMM.hpp (this library's C++ interface) and links
    libstkfmm_b200.so; MPI_Init / MPI_Finalize come from a two-line stand-in, as
    this library needs no MPI.  Without a device it stops with the library's
    no-device error."""
    import subprocess
    from oracle import oracle as O
    tree = O.ref_tree()
    demo = os.path.join(tree, "Demo", "Demo.cpp") if tree else None
    cxx = _cxx()
    if not demo or not os.path.exists(demo) or not cxx:
        pytest.skip("the reference tree or a C++ compiler is not present")
    stub = tmp_path / "mpistub"
    stub.mkdir()
    (stub / "mpi.h").write_text("#pragma once\ninline int MPI_Init(int *, char ***) { return 0; }\n"
                                "inline int MPI_Finalize() { return 0; }\n")
    exe = _build(cxx, ["-fopenmp", "-I", os.path.dirname(HEADER), "-I", str(stub), demo], tmp_path, "demo")
    if not cuda_available():
        r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
        assert r.returncode != 0 and "no CUDA device" in r.stderr


def test_reference_test_driver_built_on_this_library(tmp_path):
    """oracle/_ref/stkfmm_test_driver is the reference's own test driver
    (Test/Test.cpp, main.cpp, SimpleKernel.cpp, Util/PointDistribution.cpp)
    compiled against this library's C++ interface and a single-rank MPI stand-in
    (oracle/Makefile, target ref-driver).  It parses the reference's options, and
    without a device stops at the first FMM with the library's no-device error."""
    import subprocess
    drv = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "stkfmm_test_driver")
    if not os.path.exists(drv):
        pytest.skip("oracle/_ref/stkfmm_test_driver is built only where the reference tree is present")
    h = subprocess.run([drv, "--help"], capture_output=True, text=True, timeout=60)  # exits 1, as the reference's does
    assert "--verify" in h.stdout and "--wall" in h.stdout
    if not cuda_available():
        # -T is the driver's mesh parameter, not a point count: keep it small
        r = subprocess.run([drv, "-S", "1", "-T", "20", "-K", "1", "-M", "8"], capture_output=True, text=True,
                           timeout=120, cwd=str(tmp_path))
        assert r.returncode != 0 and "no CUDA device" in r.stderr


def test_box_scaling_matches_reference_fmmdata():
    """The library's box scaling (stk_kernel_scaling: the factors its evaluation
    applies to single-layer, double-layer and target values) against the
    reference's own FMMData::scaleSrc / scaleTrg (Lib/src/FMMData.cpp:285-470),
    compiled in oracle/_ref and run around a stub FMM, for every kernel."""
    from oracle import oracle as O
    from stkfmm_b200._lib import P_d
    if not O.ref_available():
        pytest.skip("oracle/_ref needs the reference tree")
    L = lib()
    for k in (1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024):
        for sf in (0.5, 1.0 / 3.0):
            rsl, rdl, rtrg = O.ref_kernel_scaling(k, sf)
            sl, dl, trg = np.zeros(16), np.zeros(16), np.zeros(16)
            assert L.stk_kernel_scaling(k, sf, sl.ctypes.data_as(P_d), dl.ctypes.data_as(P_d),
                                        trg.ctypes.data_as(P_d)) == 0
            assert np.array_equal(sl[:len(rsl)], rsl), (k, sl, rsl)
            assert np.array_equal(dl[:len(rdl)], rdl), (k, dl, rdl)
            assert np.allclose(trg[:len(rtrg)], rtrg, rtol=1e-15, atol=0), (k, trg, rtrg)
