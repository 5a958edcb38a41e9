"""GPU parity: U-list P2P over the same lists as the oracle, and the Stk3DFMM handle.

FP64: 1e-12 relative L2 against the oracle on the very same lists (the
north-star bar for the plain path); mixed: 1e-6.
"""
import numpy as np
import pytest

from conftest import component_errors, rel_l2
from helpers import UK_FORWARD, UK_NAMES, UK_TDIM, clustered_points, uk_values
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-6}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def run_lists(torch, uk, prec, tb, te, off, ent, sb, se, src_sorted, val_sorted, trg_sorted, period=1.0):
    from stkfmm_b200 import lib
    from stkfmm_b200._lib import P_i
    L = lib()
    s, v, t = dev(torch, src_sorted), dev(torch, val_sorted), dev(torch, trg_sorted)
    o = torch.zeros((len(trg_sorted), UK_TDIM[uk]), dtype=torch.float64, device="cuda")
    arrs = [np.ascontiguousarray(x, dtype=np.int32) for x in (tb, te, off, ent, sb, se)]
    ptrs = [a.ctypes.data_as(P_i) for a in arrs]
    rc = L.stk_p2p_lists(uk, prec, len(tb), ptrs[0], ptrs[1], ptrs[2], ptrs[3], len(sb), ptrs[4], ptrs[5],
                         len(src_sorted), s.data_ptr(), v.data_ptr(), len(trg_sorted), t.data_ptr(), o.data_ptr(),
                         period, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return o.cpu().numpy()


def oracle_ulist(uk, tb, te, off, ent, sb, se, src_sorted, val_sorted, trg_sorted, period=1.0):
    if uk == 11:
        return (oracle_ulist(1, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, :1], trg_sorted, period)
                + oracle_ulist(3, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, 1:4], trg_sorted, period))
    if uk == 12:
        return (oracle_ulist(9, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, :4], trg_sorted, period)
                + oracle_ulist(10, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, 4:], trg_sorted, period))
    if uk == 15:
        return (oracle_ulist(0, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, :1], trg_sorted, period)
                + oracle_ulist(2, tb, te, off, ent, sb, se, src_sorted, val_sorted[:, 1:4], trg_sorted, period))
    return O.lists(uk, tb, te, off, ent >> 5, ent & 31, sb, se, src_sorted, val_sorted, trg_sorted, period=period)


def tree_case(seed, n, pbc, max_pts, dist="clustered", separate_trg=False):
    from stkfmm_b200 import Octree
    rng = np.random.default_rng(seed)
    pts = clustered_points(rng, n, nclusters=6, sigma=0.03) if dist == "clustered" else rng.random((n, 3))
    trg = rng.random((n // 2, 3)) if separate_trg else pts
    t = Octree(pts, max_pts, pbc, sl=pts, trg=trg)
    sperm, sb, se = t.point_set(0)
    tperm, tb, te = t.point_set(2)
    off, ent = t.list("U")
    return rng, pts[sperm], trg[tperm], (tb, te, off, ent, sb, se)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("uk", UK_FORWARD)
def test_ulist_all_ukernels(torch_cuda, uk, prec):
    rng, src, trg, L = tree_case(uk, 6000, 0, 64)
    val = uk_values(rng, uk, len(src))
    out = run_lists(torch_cuda, uk, prec, *L, src, val, trg)
    ref = oracle_ulist(uk, *L, src, val, trg)
    err = rel_l2(out, ref)
    assert err < TOL[prec], (UK_NAMES[uk], prec, err)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("uk", [11, 4, 1])
def test_ulist_repeatable(torch_cuda, uk, prec):
    """Every target is owned by one work item (no atomics): results are bitwise repeatable."""
    rng, src, trg, L = tree_case(uk, 6000, 0, 64)
    val = uk_values(rng, uk, len(src))
    ref = oracle_ulist(uk, *L, src, val, trg)
    first = run_lists(torch_cuda, uk, prec, *L, src, val, trg)
    errs = []
    for _ in range(12):
        out = run_lists(torch_cuda, uk, prec, *L, src, val, trg)
        bad = np.flatnonzero(np.any(out != first, axis=1))
        errs.append((len(bad), bad[:4].tolist(), rel_l2(out, ref)))
    assert rel_l2(first, ref) < TOL[prec], rel_l2(first, ref)
    assert all(d == 0 and e < TOL[prec] for d, _, e in errs), errs


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("pbc", [1, 2, 3])
def test_ulist_periodic(torch_cuda, pbc, prec):
    rng, src, trg, L = tree_case(40 + pbc, 5000, pbc, 48, dist="uniform")
    for uk in (4, 6, 9):
        val = uk_values(rng, uk, len(src))
        out = run_lists(torch_cuda, uk, prec, *L, src, val, trg)
        ref = oracle_ulist(uk, *L, src, val, trg)
        assert rel_l2(out, ref) < TOL[prec], (UK_NAMES[uk], pbc, prec)


@pytest.mark.parametrize("prec", [0, 1])
def test_ulist_separate_targets_and_uneven(torch_cuda, prec):
    """Targets distinct from sources; very uneven leaves (tight clusters, small max_pts)."""
    rng, src, trg, L = tree_case(77, 8000, 0, 20, separate_trg=True)
    val = uk_values(rng, 1, len(src))
    out = run_lists(torch_cuda, 1, prec, *L, src, val, trg)
    ref = oracle_ulist(1, *L, src, val, trg)
    assert rel_l2(out, ref) < TOL[prec]


def test_lists_reject_bad_indices(torch_cuda):
    """Out-of-range list / range indices are refused on the host before any launch."""
    from stkfmm_b200 import lib
    from stkfmm_b200._lib import P_i
    L = lib()
    x = torch_cuda.zeros((10, 3), dtype=torch_cuda.float64, device="cuda")
    o = torch_cuda.zeros((10, 4), dtype=torch_cuda.float64, device="cuda")
    good = dict(tb=[0], te=[10], off=[0, 1], ent=[(0 << 5) | 13], sb=[0], se=[10])
    bad_cases = [dict(good, ent=[(5 << 5) | 13]), dict(good, se=[11]), dict(good, te=[11]), dict(good, ent=[27]),
                 dict(good, off=[0, 2])]
    for case in bad_cases:
        arrs = [np.array(case[k], dtype=np.int32) for k in ("tb", "te", "off", "ent", "sb", "se")]
        if len(arrs[3]) < arrs[2][-1]:
            arrs[3] = np.concatenate([arrs[3], arrs[3]])
            arrs[3][-1] = (7 << 5) | 13
        p = [a.ctypes.data_as(P_i) for a in arrs]
        rc = L.stk_p2p_lists(1, 0, 1, p[0], p[1], p[2], p[3], 1, p[4], p[5], 10, x.data_ptr(), x.data_ptr(), 10,
                             x.data_ptr(), o.data_ptr(), 1.0, 0)
        assert rc != 0, case


# ---- the Stk3DFMM handle ------------------------------------------------------

def handle_case(kernel, n, pbc=0, max_pts=64, seed=0, origin=(0.0, 0.0, 0.0), box=1.0, same_dl=True):
    import stkfmm_b200 as S
    rng = np.random.default_rng(seed)
    # keep clear of the upper box face so (x * box + origin - origin) / box stays below 1
    pts = np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.04), 0.999) * box + np.array(origin)
    sd, dd, td = S.get_kernel_dimension(kernel)
    has_dl = S.kernel_slot(kernel, 1) >= 0
    dl = pts.copy() if same_dl else (clustered_points(rng, n // 2, nclusters=3) * box + np.array(origin))
    slv = uk_values(rng, S.kernel_slot(kernel, 0), n)
    if kernel == 16:
        # RPY radii of the RPY workload, b ~ U(1e-4, 5e-4): the far-field RPY form the
        # reference evaluates assumes radii well below the pair distances
        slv[:, 3] = rng.uniform(1e-4, 5e-4, n) * box
    dlv = rng.normal(size=(len(dl), dd)) if has_dl else None
    return pts, (dl if has_dl else None), slv, dlv, td


@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
@pytest.mark.parametrize("prec", [0, 1])
def test_handle_evaluate_near(torch_cuda, kernel, prec):
    """Stk3DFMM_evaluate_near against the oracle on the handle's own U-list (SL and DL)."""
    import stkfmm_b200 as S
    pts, dl, slv, dlv, td = handle_case(kernel, 5000, seed=kernel)
    fmm = S.Stk3DFMM(8, 64, 0, kernel, precision=prec)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, dl)
    fmm.setup_tree(kernel)
    out0 = np.random.default_rng(1).normal(size=(len(pts), td))
    out = out0.copy()
    fmm.evaluate_near(kernel, slv, out, dlv)
    u = fmm.ulist(kernel)
    lst = (u["trg_begin"], u["trg_end"], u["list_off"], u["list_ent"])
    sk = S.kernel_slot(kernel, 0)
    ref = np.zeros((len(pts), td))
    ref[u["trg_perm"]] = oracle_ulist(sk, *lst, u["sl_begin"], u["sl_end"], pts[u["sl_perm"]], slv[u["sl_perm"]],
                                      pts[u["trg_perm"]])
    if dl is not None:
        dk = S.kernel_slot(kernel, 1)
        ref[u["trg_perm"]] += oracle_ulist(dk, *lst, u["dl_begin"], u["dl_end"], dl[u["dl_perm"]],
                                           dlv[u["dl_perm"]], pts[u["trg_perm"]])
    assert rel_l2(out - out0, ref) < TOL[prec], component_errors(out - out0, ref)
    st = fmm.tree_stats(kernel)
    assert st["u_pairs_sl"] > 0 and st["u_entries"] == len(u["list_ent"])


@pytest.mark.parametrize("pbc", [0, 3])
@pytest.mark.parametrize("kernel", [1, 2, 128])
def test_handle_mixed_coincident_on_leaf_faces(torch_cuda, kernel, pbc):
    """The handle's mixed near field masks the coincidence only on tiles that can hold a
    source at a target's position (the target's own leaf, periodic images): targets that
    duplicate sources exactly, many of them on leaf faces and cell faces (coordinates on
    a 1/64 grid, 0 included), stay finite and within the mixed bar of the oracle."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(7)
    grid = rng.integers(0, 64, size=(1500, 3)) / 64.0     # on the faces of leaves down to level 6
    free = clustered_points(rng, 2500, nclusters=4, sigma=0.03)
    pts = np.concatenate([grid, free, grid[:300]])         # exact duplicates inside the source set too
    sd, dd, td = S.get_kernel_dimension(kernel)
    slv = uk_values(rng, S.kernel_slot(kernel, 0), len(pts))
    has_dl = S.kernel_slot(kernel, 1) >= 0
    dlv = rng.normal(size=(len(pts), dd)) if has_dl else None
    fmm = S.Stk3DFMM(8, 40, pbc, kernel, precision=1)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts if has_dl else None)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), td))
    fmm.evaluate_near(kernel, slv, out, dlv)
    assert np.all(np.isfinite(out))
    u = fmm.ulist(kernel)
    lst = (u["trg_begin"], u["trg_end"], u["list_off"], u["list_ent"])
    ref = np.zeros_like(out)
    ref[u["trg_perm"]] = oracle_ulist(S.kernel_slot(kernel, 0), *lst, u["sl_begin"], u["sl_end"], pts[u["sl_perm"]],
                                      slv[u["sl_perm"]], pts[u["trg_perm"]])
    if has_dl:
        ref[u["trg_perm"]] += oracle_ulist(S.kernel_slot(kernel, 1), *lst, u["dl_begin"], u["dl_end"],
                                           pts[u["dl_perm"]], dlv[u["dl_perm"]], pts[u["trg_perm"]])
    assert rel_l2(out, ref) < 1e-6, component_errors(out, ref)


@pytest.mark.parametrize("kernel", [1, 2, 128])
def test_handle_separate_dl_points(torch_cuda, kernel):
    """SL and DL at different points: separate (unfused) passes."""
    import stkfmm_b200 as S
    pts, dl, slv, dlv, td = handle_case(kernel, 4000, seed=3, same_dl=False)
    fmm = S.Stk3DFMM(8, 50, 0, kernel)
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, dl)
    fmm.setup_tree(kernel)
    out = np.zeros((len(pts), td))
    fmm.evaluate_near(kernel, slv, out, dlv)
    u = fmm.ulist(kernel)
    lst = (u["trg_begin"], u["trg_end"], u["list_off"], u["list_ent"])
    ref = np.zeros_like(out)
    ref[u["trg_perm"]] = oracle_ulist(S.kernel_slot(kernel, 0), *lst, u["sl_begin"], u["sl_end"], pts[u["sl_perm"]],
                                      slv[u["sl_perm"]], pts[u["trg_perm"]])
    ref[u["trg_perm"]] += oracle_ulist(S.kernel_slot(kernel, 1), *lst, u["dl_begin"], u["dl_end"],
                                       dl[u["dl_perm"]], dlv[u["dl_perm"]], pts[u["trg_perm"]])
    assert rel_l2(out, ref) < 1e-12


@pytest.mark.parametrize("kernel", [1, 2, 4, 16, 64, 128, 256, 1024])
def test_handle_box_scaling(torch_cuda, kernel):
    """A box (origin o, length L) gives sF^k times the unit-box result (scaleSrc / scaleTrg)."""
    import stkfmm_b200 as S
    o, Lb = np.array([1.0, -2.0, 3.0]), 4.0
    pts, dl, slv, dlv, td = handle_case(kernel, 3000, seed=5)
    unit = S.Stk3DFMM(8, 64, 0, kernel)
    unit.set_box(np.zeros(3), 1.0)
    unit.set_points(pts, pts, dl)
    unit.setup_tree(kernel)
    big = S.Stk3DFMM(8, 64, 0, kernel)
    big.set_box(o, Lb)
    P = pts * Lb + o
    D = dl * Lb + o if dl is not None else None
    big.set_points(P, P, D)
    big.setup_tree(kernel)
    sf = 1.0 / Lb
    # physical values that map onto the unit-box values after scaleSrc
    slv_big = slv.copy()
    if kernel in (16, 128, 256, 1024):
        slv_big[:, -1] /= sf
    if kernel == 64:  # torque and regularisation scale like a double layer
        slv_big[:, 3:] /= sf
    dlv_big = dlv / sf if dlv is not None else None
    a = np.zeros((len(pts), td))
    b = np.zeros((len(pts), td))
    unit.evaluate_near(kernel, slv, a, dlv)
    big.evaluate_near(kernel, slv_big, b, dlv_big)
    pows = {1: [1, 2, 2, 2], 2: [1, 2, 2, 2, 3, 3, 3, 3, 3, 3], 4: [3, 4, 4, 4, 5, 5, 5, 5, 5, 5],
            16: [1, 1, 1, 3, 3, 3], 128: [2, 1, 1, 1], 256: [2, 1, 1, 1, 3, 3, 3] + [2] * 9,
            1024: [2] * 9, 64: [1, 1, 1, 2, 2, 2]}[kernel]
    assert rel_l2(b, a * sf ** np.array(pows)) < 1e-12


def test_handle_errors(torch_cuda):
    import stkfmm_b200 as S
    fmm = S.Stk3DFMM(8, 64, 0, 1 | 8)
    with pytest.raises(S.StkError):
        fmm.setup_tree(1)  # points not set
    pts = np.random.default_rng(0).random((100, 3))
    fmm.set_box(np.zeros(3), 1.0)
    fmm.set_points(pts, pts, pts)
    with pytest.raises(S.StkError):
        fmm.setup_tree(16)  # kernel not activated
    fmm.setup_tree(8)
    with pytest.raises(S.StkError):
        fmm.evaluate_near(8, np.zeros((99, 3)), np.zeros((100, 3)), None)  # size mismatch
    with pytest.raises(S.StkError):
        fmm.set_points(pts + 2.0, pts, None)  # outside the free-space box
