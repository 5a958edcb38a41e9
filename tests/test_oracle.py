"""The CPU oracle pinned against the reference's own kernels (no GPU needed)."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import GOLDEN_MAP, load_golden, uk_values
from oracle import oracle as O


@pytest.mark.parametrize("name", sorted(GOLDEN_MAP))
def test_oracle_matches_golden(name):
    """The C restatement of each uKerEval reproduces the reference SimpleKernel fixtures."""
    g = load_golden(name)
    for uk, osl, vsl in GOLDEN_MAP[name]:
        for pre in ("", "fixed_"):
            out = O.direct(uk, g[pre + "src"], g[pre + "val"][:, vsl], g[pre + (
                "trg")])
            err = rel_l2(out, g[pre + "out"][:, osl])
            assert err < 1e-13, (name, O.UK_NAMES[uk], pre, err)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
@pytest.mark.parametrize("which,uk,osl", [
    (O.REF_STOKES_SL, O.UK_STOKES_VEL, slice(0, 3)),
    (O.REF_LAP_SL_PGRAD, O.UK_LAPLACE_PGRAD, slice(0, 4)),
    (O.REF_LAP_DL_PGRAD, O.UK_LAPLACE_DIPOLEPGRAD, slice(0, 4)),
    (O.REF_STOKES_SL_RPY, O.UK_RPY_ULAPU, slice(0, 6)),
    (O.REF_STOKES_REG_SL_VEL, O.UK_STOKES_REGVEL, slice(0, 3)),
    (O.REF_STOKES_SL_PVEL, O.UK_STOKES_PVEL, slice(0, 4)),
    (O.REF_STOKES_DL_PVEL, O.UK_STOKES_DOUBLEPVEL, slice(0, 4)),
    (O.REF_LAP_SL_PGRADGRAD, O.UK_LAPLACE_PGRADGRAD, slice(0, 10)),
    (O.REF_LAP_DL_PGRADGRAD, O.UK_LAPLACE_DIPOLEPGRADGRAD, slice(0, 10)),
    (O.REF_LAP_QPGRADGRAD, O.UK_LAPLACE_QUADPGRADGRAD, slice(0, 10)),
    (O.REF_STOKES_SL_PVELGRAD, O.UK_STOKES_PVELGRAD, slice(0, 16)),
    (O.REF_STOKES_DL_PVELGRAD, O.UK_STOKES_DOUBLEPVELGRAD, slice(0, 16)),
    (O.REF_STOKES_SL_PVELLAP, O.UK_STOKES_PVELLAPLACIAN, slice(0, 7)),
    (O.REF_STOKES_DL_PVELLAP, O.UK_STOKES_DOUBLELAPLACIAN, slice(0, 7)),
    (O.REF_STOKES_SL_TRACTION, O.UK_STOKES_TRACTION, slice(0, 9)),
    (O.REF_STOKES_DL_TRACTION, O.UK_STOKES_DOUBLETRACTION, slice(0, 9)),
    (O.REF_STOKES_REG_SL_VELOMEGA, O.UK_STOKES_REGFTVELOMEGA, slice(0, 6)),
])
def test_oracle_matches_live_reference(which, uk, osl, rng):
    """Fresh random inputs (clustered, with coincident points) through the compiled reference."""
    src = rng.random((400, 3)) * 0.1 + 0.45
    trg = np.concatenate([src[:100], rng.random((80, 3))])
    v = rng.uniform(-1, 1, size=(400, O.REF_DIMS[which][0]))
    if which in (O.REF_STOKES_SL_RPY, O.REF_STOKES_REG_SL_VEL):
        v[:, 3] = np.abs(v[:, 3]) * 1e-3
    if which == O.REF_STOKES_REG_SL_VELOMEGA:
        v[:, 6] = np.abs(v[:, 6]) * 1e-3
    ref = O.ref_direct(which, src, v, trg)[:, osl]
    out = O.direct(uk, src, v[:, :O.UK_SDIM[uk]], trg)
    assert rel_l2(out, ref) < 1e-13


def test_oracle_lists_equals_direct_on_full_list(rng):
    """A list covering every (target box, source box) pair equals the dense sum."""
    src = rng.random((300, 3))
    trg = rng.random((200, 3))
    v = rng.uniform(-1, 1, (300, 3))
    sb = np.array([0, 100, 250], np.int32)
    se = np.array([100, 250, 300], np.int32)
    tb = np.array([0, 77], np.int32)
    te = np.array([77, 200], np.int32)
    off = np.array([0, 3, 6], np.int32)
    ent = np.array([(s << 5) | 13 for _ in range(2) for s in range(3)], np.int32)
    out = O.lists(O.UK_STOKES_VEL, tb, te, off, ent >> 5, ent & 31, sb, se, src, v, trg)
    ref = O.direct(O.UK_STOKES_VEL, src, v, trg)
    assert rel_l2(out, ref) < 1e-14


def test_oracle_lists_on_tree_repeatable():
    """Tree lists include internal nodes whose (empty-list) target ranges overlap
    their leaves: the threaded oracle must give the same result every time, equal
    to a plain numpy sum over the leaves."""
    from helpers import clustered_points
    from stkfmm_b200 import Octree
    rng = np.random.default_rng(4)
    pts = clustered_points(rng, 3000, nclusters=4, sigma=0.05)
    t = Octree(pts, 24, 0, sl=pts, trg=pts)
    sp, sb, se = t.point_set(0)
    tp, tb, te = t.point_set(2)
    off, ent = t.list("U")
    src, trg = pts[sp], pts[tp]
    q = rng.uniform(-1, 1, (len(pts), 1))
    ref = np.zeros((len(pts), 4))
    for b in range(t.num_nodes):
        for e in ent[off[b]:off[b + 1]]:
            s = e >> 5
            ref[tb[b]:te[b]] += O.direct(O.UK_LAPLACE_PGRAD, src[sb[s]:se[s]], q[sb[s]:se[s]], trg[tb[b]:te[b]])
    for _ in range(8):
        out = O.lists(O.UK_LAPLACE_PGRAD, tb, te, off, ent >> 5, ent & 31, sb, se, src, q, trg, nthreads=8)
        assert rel_l2(out, ref) < 1e-14


def test_oracle_periodic_shift(rng):
    """Shift code s adds s*period to the source coordinate."""
    src = rng.random((50, 3))
    trg = rng.random((40, 3))
    v = rng.uniform(-1, 1, (50, 1))
    code = (1 + 1) + 3 * (0 + 1) + 9 * (-1 + 1)  # (sx, sy, sz) = (+1, 0, -1)
    out = O.lists(O.UK_LAPLACE_PGRAD, [0], [40], [0, 1], [0], [code], [0], [50], src, v, trg, period=2.0)
    ref = O.direct(O.UK_LAPLACE_PGRAD, src + np.array([2.0, 0.0, -2.0]), v, trg)
    assert rel_l2(out, ref) < 1e-14


def test_surface_points():
    """Cube surface: 6(p-1)^2+2 distinct points, all on the cube boundary, centred on c+alpha*r."""
    for p in (4, 6, 8, 10, 12):
        c = np.array([0.25, 0.5, 0.125])
        pts = O.surface(p, c, 2.95, 2)
        n = 6 * (p - 1) ** 2 + 2
        assert pts.shape == (n, 3)
        r = 0.5 * 0.5 ** 2
        u = (pts - c) / (2.95 * r) - 1.0  # back to [-1,1]^3
        assert np.allclose(np.abs(u).max(axis=1), 1.0)
        assert len(np.unique(np.round(u, 12), axis=0)) == n
        assert np.allclose(u.mean(axis=0), 0.0, atol=1e-14)


def test_regvel_adjoint_finite_difference(rng):
    """The hand-derived adjoint of the regularized Stokeslet sum against central differences."""
    ns, nt = 30, 25
    src = rng.random((ns, 3))
    trg = np.concatenate([src[:10], rng.random((nt - 10, 3))])
    sv = rng.uniform(-1, 1, (ns, 4))
    sv[:, 3] = np.abs(sv[:, 3]) * 0.05 + 0.01
    w = rng.normal(size=(nt, 3))
    gf, gx = O.regvel_adjoint(src, sv, trg, w)

    def loss(s, v):
        return float(np.sum(w * O.direct(O.UK_STOKES_REGVEL, s, v, trg)))

    h = 1e-6
    for i in (0, 3, 17):
        for k in range(3):
            vp, vm = sv.copy(), sv.copy()
            vp[i, k] += h
            vm[i, k] -= h
            fd = (loss(src, vp) - loss(src, vm)) / (2 * h)
            assert abs(fd - gf[i, k]) <= 1e-6 * max(1.0, abs(fd))
            sp, sm = src.copy(), src.copy()
            sp[i, k] += h
            sm[i, k] -= h
            # the target copies of points 0..9 stay fixed: this is the source-position gradient
            fd = (loss(sp, sv) - loss(sm, sv)) / (2 * h)
            assert abs(fd - gx[i, k]) <= 1e-5 * max(1.0, abs(fd))


# ---- triply periodic Ewald sums (the periodic FMM's oracle) ----------------------

@pytest.mark.parametrize("kind", [O.EWALD_LAPLACE, O.EWALD_STOKES])
def test_ewald_splitting_independent(kind):
    """The Ewald split (xi, image counts) must not change the periodic sum."""
    rng = np.random.default_rng(21 + kind)
    src = rng.random((200, 3))
    v = rng.normal(size=(200, 1 if kind == O.EWALD_LAPLACE else 3))
    v -= v.mean(0)
    trg = np.concatenate([rng.random((40, 3)), src[:10]])   # includes targets on source points
    a = O.ewald(kind, src, v, trg)
    b = O.ewald(kind, src, v, trg, xi=2.0, nreal=4, nwave=5)
    c = O.ewald(kind, src, v, trg, xi=4.0, nreal=2, nwave=9)
    assert np.abs(a - b).max() < 1e-13 * np.abs(a).max()
    assert np.abs(a - c).max() < 1e-13 * np.abs(a).max()
    # periodic in every axis
    d = O.ewald(kind, src, v, trg + np.array([1.0, -2.0, 3.0]))
    assert np.abs(a - d).max() < 1e-13 * np.abs(a).max()


def test_ewald_laplace_field_matches_image_sum():
    """For a cell whose charges have no net charge, dipole or quadrupole moment
    (alternating charges on the corners of small cubes) the field of the image
    lattice summed over growing cubes converges to the Ewald field."""
    import itertools
    rng = np.random.default_rng(5)
    c = rng.random((3, 3)) * 0.5 + 0.25
    sg = np.array(list(itertools.product([-1, 1], [-1, 1], [-1, 1])), dtype=np.float64)
    src = np.concatenate([ci + 0.04 * sg for ci in c])
    q = np.tile(sg.prod(1), 3)[:, None]
    trg = rng.random((5, 3))
    ew = O.ewald(O.EWALD_LAPLACE, src, q, trg)[:, 1:]
    errs = []
    for L in (2, 8):
        r = np.arange(-L, L + 1)
        shifts = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
        imgs = (src[None, :, :] + shifts[:, None, :]).reshape(-1, 3)
        direct = O.direct(O.UK_LAPLACE_PGRAD, imgs, np.tile(q, (len(shifts), 1)), trg)[:, 1:]
        errs.append(np.abs(direct - ew).max() / np.abs(ew).max())
    assert errs[1] < 1e-6 and errs[1] < errs[0] / 50, errs


def _zero_moment_cell(rng, ncube=3, h=0.04):
    """Charges / forces on the corners of small cubes with alternating signs:
    no net charge, dipole or quadrupole, so lattice sums converge fast."""
    import itertools
    c = rng.random((ncube, 3)) * 0.5 + 0.25
    sg = np.array(list(itertools.product([-1, 1], [-1, 1], [-1, 1])), dtype=np.float64)
    src = np.concatenate([ci + h * sg for ci in c])
    s = np.tile(sg.prod(1), ncube)[:, None]
    return src, s


@pytest.mark.parametrize("kind", [O.EWALD_LAPLACE, O.EWALD_STOKES, O.EWALD_LAPLACE_HESS])
def test_ewald_cells_matches_ewald(kind):
    """The cell-list Ewald sum (used for the 2M-point periodic fixture) against the
    image-sum form, targets on and off the sources, points outside [0, 1) too."""
    rng = np.random.default_rng(41 + kind)
    src = rng.random((300, 3))
    src[:20] += rng.integers(-2, 3, (20, 3))
    v = rng.normal(size=(300, 3 if kind == O.EWALD_STOKES else 1))
    v -= v.mean(0)
    trg = np.concatenate([rng.random((40, 3)), src[:10]])
    a = O.ewald(kind, src, v, trg, xi=7.0, nreal=2, nwave=20)
    b = O.ewald_cells(kind, src, v, trg)
    assert np.abs(a - b).max() < 3e-12 * np.abs(a).max()
    lap = O.ewald_stokes_laplacian_cells(src, rng.normal(size=(300, 3)), trg[:8])
    assert np.isfinite(lap).all()


def test_ewald_pvel_splitting_independent():
    rng = np.random.default_rng(31)
    src = rng.random((150, 3))
    v = rng.normal(size=(150, 4))
    v -= v.mean(0)
    trg = np.concatenate([rng.random((30, 3)), src[:5]])
    a = O.ewald(O.EWALD_PVEL, src, v, trg)
    b = O.ewald(O.EWALD_PVEL, src, v, trg, xi=2.0, nreal=4, nwave=5)
    assert np.abs(a - b).max() < 1e-13 * np.abs(a).max()


def test_ewald_pvel_pressure_matches_image_sum():
    rng = np.random.default_rng(32)
    src, s = _zero_moment_cell(rng)
    pv = np.concatenate([s * np.array([[0.3, -0.2, 0.5]]), 0.7 * s], axis=1)
    trg = rng.random((5, 3))
    ew = O.ewald(O.EWALD_PVEL, src, pv, trg)
    r = np.arange(-8, 9)
    sh = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    imgs = (src[None] + sh[:, None]).reshape(-1, 3)
    d = O.direct(O.UK_STOKES_PVEL, imgs, np.tile(pv, (len(sh), 1)), trg)
    assert np.abs(d[:, 0] - ew[:, 0]).max() < 1e-6 * np.abs(ew[:, 0]).max()
    assert np.abs(d[:, 1:] - ew[:, 1:]).max() < 1e-4 * np.abs(ew[:, 1:]).max()


@pytest.mark.parametrize("kind", [O.EWALD_LAPLACE, O.EWALD_STOKES, O.EWALD_PVEL])
def test_ewald2d_matches_image_sums(kind):
    """Doubly periodic sums against sums over growing squares of images (x, y)."""
    rng = np.random.default_rng(33 + kind)
    src, s = _zero_moment_cell(rng)
    val = {O.EWALD_LAPLACE: s, O.EWALD_STOKES: s * np.array([[0.3, -0.2, 0.5]]),
           O.EWALD_PVEL: np.concatenate([s * np.array([[0.3, -0.2, 0.5]]), 0.7 * s], axis=1)}[kind]
    uk = {O.EWALD_LAPLACE: O.UK_LAPLACE_PGRAD, O.EWALD_STOKES: O.UK_STOKES_VEL, O.EWALD_PVEL: O.UK_STOKES_PVEL}[kind]
    trg = rng.random((5, 3))
    ew = O.ewald2d(kind, src, val, trg)
    # periodic in x and y
    assert np.abs(O.ewald2d(kind, src, val, trg + np.array([2.0, -1.0, 0.0])) - ew).max() < 1e-13 * np.abs(ew).max()
    r = np.arange(-32, 33)
    sh = np.stack(np.meshgrid(r, r, [0], indexing="ij"), -1).reshape(-1, 3).astype(np.float64)
    imgs = (src[None] + sh[:, None]).reshape(-1, 3)
    d = O.direct(uk, imgs, np.tile(val, (len(sh), 1)), trg)
    assert np.abs(d - ew).max() < 1e-6 * np.abs(ew).max()


@pytest.mark.parametrize("fn", ["ewald", "ewald2d"])
def test_ewald_laplace_hessian(fn):
    """Potential, gradient and Hessian of the periodic Laplace sums: the Hessian
    equals central differences of the gradient, its trace vanishes for neutral
    charges, and at a target on a source (self image removed) it is the limit of
    the full sum minus that source's own singular Hessian."""
    f = getattr(O, fn)
    rng = np.random.default_rng(34)
    src = rng.random((40, 3))
    q = rng.uniform(-1, 1, (40, 1))
    q -= q.mean()
    trg = rng.random((30, 3))
    H = f(O.EWALD_LAPLACE_HESS, src, q, trg)
    assert np.array_equal(H[:, :4], f(O.EWALD_LAPLACE, src, q, trg))
    h = 1e-5
    fd = np.zeros((len(trg), 3, 3))
    for a in range(3):
        e = np.zeros(3)
        e[a] = h
        fd[:, a] = (f(O.EWALD_LAPLACE, src, q, trg + e)[:, 1:4] - f(O.EWALD_LAPLACE, src, q, trg - e)[:, 1:4]) / (2 * h)
    hm = np.stack([fd[:, i, j] for i, j in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))], 1)
    scale = np.abs(hm).max()
    assert np.abs(H[:, 4:] - hm).max() < 1e-7 * scale
    assert np.abs(H[:, 4] + H[:, 7] + H[:, 9]).max() < 1e-12 * scale
    # self image: second-order convergence of the symmetric limit
    t0 = src[:5]
    H0 = f(O.EWALD_LAPLACE_HESS, src, q, t0)[:, 4:]
    errs = []
    for s in (1e-3, 5e-4):
        d = np.array([1.0, -0.7, 0.5]) * s
        avg = 0.5 * (f(O.EWALD_LAPLACE_HESS, src, q, t0 + d) + f(O.EWALD_LAPLACE_HESS, src, q, t0 - d))[:, 4:]
        sing = O.direct(O.UK_LAPLACE_PGRADGRAD, np.zeros((1, 3)), np.ones((1, 1)), d[None])[0, 4:]
        errs.append(np.abs(avg - q[:5] * sing[None] - H0).max() / np.abs(H0).max())
    assert errs[0] < 1e-3 and 3.0 < errs[0] / errs[1] < 5.0, errs


@pytest.mark.parametrize("kind", ["stokes", "stokes_pxy", "rpy"])
def test_wall_image_system_no_slip(kind):
    """The restated wall image systems (StkWallFMM.cpp:154-292) give zero velocity
    on the wall z = z0 (to rounding), free space and doubly periodic."""
    rng = np.random.default_rng(35)
    z0 = 0.25
    src = rng.random((60, 3))
    src[:, 2] = z0 + 0.05 + 0.4 * rng.random(60)
    f = rng.normal(size=(60, 3))
    bulk = rng.random((20, 3))
    bulk[:, 2] = z0 + 0.5 * bulk[:, 2]
    wall = rng.random((20, 3))
    wall[:, 2] = z0
    if kind == "rpy":
        fb = np.concatenate([f, rng.uniform(1e-3, 5e-3, (60, 1))], 1)
        uw, ub = O.wall_rpy(src, fb, wall, z0=z0)[:, :3], O.wall_rpy(src, fb, bulk, z0=z0)[:, :3]
    else:
        pbc = 2 if kind == "stokes_pxy" else 0
        uw, ub = O.wall_stokes(src, f, wall, z0=z0, pbc=pbc), O.wall_stokes(src, f, bulk, z0=z0, pbc=pbc)
    assert np.abs(uw).max() < 1e-13 * np.abs(ub).max()



def test_velomega_is_unregularized_force_torque(rng):
    """stokes_velomega (the M2T / L2T kernel of StokesRegVelOmega) equals
    stokes_regftvelomega with no torque and eps = 0 away from the sources."""
    src = rng.random((300, 3))
    trg = rng.random((200, 3)) + 2.0
    f = rng.normal(size=(300, 3))
    ft = np.concatenate([f, np.zeros((300, 4))], axis=1)
    a = O.direct(O.UK_STOKES_VELOMEGA, src, f, trg)
    b = O.direct(O.UK_STOKES_REGFTVELOMEGA, src, ft, trg)
    assert np.abs(a - b).max() < 1e-13 * np.abs(b).max()


@pytest.mark.parametrize("ukg,ukt,sd", [(20, 24, 4), (21, 25, 9)])
def test_traction_is_stress_of_pvelgrad(rng, ukg, ukt, sd):
    """stokes_traction = -p I + grad u + grad u^T of stokes_pvelgrad (SL), and the
    same for the double layer (up to the reference's truncated 2/3)."""
    src = rng.random((50, 3))
    trg = rng.random((40, 3)) + 1.5
    v = rng.normal(size=(50, sd))
    G = O.direct(ukg, src, v, trg)
    T = O.direct(ukt, src, v, trg)
    g = G[:, 7:16].reshape(-1, 3, 3)
    comb = -G[:, 0][:, None, None] * np.eye(3)[None] + g + g.transpose(0, 2, 1)
    assert np.abs(comb.reshape(-1, 9) - T).max() < 1e-13 * np.abs(T).max()


def _root_equivalent(uk, p, src, sval):
    """The root's upward-equivalent density of the unit cell as PVFMM forms it:
    check potentials on the radius-2.95 surface, a pseudo-inverse solve (cut
    sqrt(machine eps), M2L/SVD_pvfmm.hpp:599-604) for densities on the
    radius-1.05 surface (surface layout of stkfmm_helpers.hpp:46-85)."""
    sd, td = O.UK_SDIM[uk], O.UK_TDIM[uk]
    ue = O.surface(p, np.full(3, -0.025), 1.05, 0)
    uc = O.surface(p, np.full(3, -0.975), 2.95, 0)
    A = np.zeros((len(uc) * td, len(ue) * sd))
    for j in range(len(ue)):
        for c in range(sd):
            e = np.zeros((1, sd))
            e[0, c] = 1.0
            A[:, j * sd + c] = O.direct(uk, ue[j:j + 1], e, uc).reshape(-1)
    chk = O.direct(uk, src, sval, uc).reshape(-1)
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    keep = s > s[0] * np.sqrt(np.finfo(float).eps)
    return ue, ((Vt[keep].T / s[keep]) @ (U[:, keep].T @ chk)).reshape(len(ue), sd)


def _image_block(uk, src, sval, trg, layers):
    out = np.zeros((len(trg), O.UK_TDIM[uk]))
    r = range(-layers, layers + 1)
    for a in r:
        for b in r:
            for c in r:
                O.direct(uk, src + np.array([a, b, c]), sval, trg, out=out)
    return out


def test_pvel_pxyz_terms_pin_the_root_chain(rng):
    """oracle.pvel_pxyz_terms against the reference's own root-level arithmetic:
    the images outside the directly summed block come from the root's equivalent
    density through the Ewald sum, plus half its wrapped trD dipole (M2C,
    StokesPVel3D3D.cpp:211-218) and half the unwrapped rest (periodizeFMM,
    FMMData.cpp:203-247).  The velocity is then the sources' Ewald sum plus half
    their trD dipole moment, with no drift; without the two terms it is off by
    half the equivalent density's dipole (its fit misses the sources' dipole)."""
    src, trg = rng.random((300, 3)), rng.random((40, 3))
    val = rng.normal(size=(300, 4))
    val -= val.mean(0)
    ue, veq = _root_equivalent(O.UK_STOKES_PVEL, 8, src, val)
    ew = O.ewald(O.EWALD_PVEL, src, val, trg)
    chain = (_image_block(O.UK_STOKES_PVEL, src, val, trg, 1) + O.ewald(O.EWALD_PVEL, np.mod(ue, 1.0), veq, trg)
             - _image_block(O.UK_STOKES_PVEL, ue, veq, trg, 1))
    chain[:, 1:] += 0.5 * (np.mod(ue, 1.0) * veq[:, 3:4]).sum(0) + 0.5 * (np.floor(ue) * veq[:, 3:4]).sum(0)
    ref = ew + O.pvel_pxyz_terms(src, val, trg)
    vel = chain[:, 1:] - ref[:, 1:]
    assert np.abs(vel).max() < 1e-6 * np.abs(ref[:, 1:]).max()
    assert np.abs(0.5 * ((ue * veq[:, 3:4]).sum(0) - (src * val[:, 3:4]).sum(0))).max() > 1e-3


def test_laplace_pxyz_neutraliser_pins_the_root_chain(rng):
    """oracle.laplace_pxyz_neutraliser against the reference's root-level
    arithmetic for a charged cell: every equivalent charge is paired with an
    opposite one at the centre (Laplace3D3D.cpp:266-273).  The gradient then
    matches the Ewald sum plus the neutraliser exactly; the potential up to a
    constant (the drift of a triply periodic potential)."""
    src, trg = rng.random((300, 3)), rng.random((40, 3))
    q = rng.normal(size=(300, 1)) + 0.3
    ue, qeq = _root_equivalent(O.UK_LAPLACE_P, 10, src, q)
    cen = np.array([[0.5, 0.5, 0.5]])
    far_n = O.ewald(O.EWALD_LAPLACE, cen, np.ones((1, 1)), trg) - _image_block(O.UK_LAPLACE_PGRAD, cen, np.ones((1, 1)),
                                                                               trg, 2)
    chain = (_image_block(O.UK_LAPLACE_PGRAD, src, q, trg, 1) + O.ewald(O.EWALD_LAPLACE, np.mod(ue, 1.0), qeq, trg)
             - _image_block(O.UK_LAPLACE_PGRAD, ue, qeq, trg, 1) - qeq.sum() * far_n)
    ref = O.ewald(O.EWALD_LAPLACE, src, q, trg) + O.laplace_pxyz_neutraliser(q.sum(), trg)
    d = chain - ref
    assert np.abs(d[:, 1:]).max() < 1e-6 * np.abs(ref[:, 1:]).max()
    assert np.ptp(d[:, 0]) < 1e-6 * np.abs(ref[:, 0]).max()
    plain = chain - O.ewald(O.EWALD_LAPLACE, src, q, trg)
    assert np.abs(plain[:, 1:] - plain[:, 1:].mean(0)).max() > 1e-2 * np.abs(ref[:, 1:]).max()


def test_stokes_ewald_reference_three_forces(rng):
    """The reference generator's own check (M2L/Stokeslet/Stokes3D3D.cpp:183-242):
    three point forces in the unit cell (net force (0, 1, 0)), the near block
    summed directly plus the root's equivalent density through the far-image
    sum, against the Ewald sum (here at its sample point (1/2, 1/2, 1/2) and 20
    more).  Pins the oracle's Hasimoto sum, net force included, to the
    root-level arithmetic."""
    src = np.array([[0.1, 0.55, 0.2], [0.5, 0.1, 0.3], [0.8, 0.5, 0.7]])
    f = np.array([[1.0, 0.0, 0.0], [-1.0, 1.0, 1.0], [0.0, 0.0, -1.0]])
    trg = np.concatenate([[[0.5, 0.5, 0.5]], rng.random((20, 3))])
    ue, feq = _root_equivalent(O.UK_STOKES_VEL, 10, src, f)
    chain = (_image_block(O.UK_STOKES_VEL, src, f, trg, 1) + O.ewald(O.EWALD_STOKES, np.mod(ue, 1.0), feq, trg)
             - _image_block(O.UK_STOKES_VEL, ue, feq, trg, 1))
    ew = O.ewald(O.EWALD_STOKES, src, f, trg)
    assert np.abs(chain - ew).max() < 1e-6 * np.abs(ew).max()


@pytest.mark.parametrize("net_force", [True, False])
def test_ewald_stokes_laplacian_by_finite_differences(net_force):
    """oracle.ewald_stokes_laplacian (the periodic Laplacian term of rpy_ulapu /
    stk_ulapu, lap u = -sum_j H[f_j] + F) against central differences of the
    oracle's own periodic Stokeslet velocity (Richardson-extrapolated, targets at
    least 0.08 from every source image), with and without a net force."""
    rng = np.random.default_rng(2)
    src = rng.random((20, 3))
    f = rng.normal(size=(20, 3))
    if not net_force:
        f -= f.mean(0)
    trg = rng.random((200, 3))
    d = np.linalg.norm(((trg[:, None] - src[None]) + 0.5) % 1.0 - 0.5, axis=-1).min(1)
    trg = trg[d > 0.08][:30]

    def second_differences(h):
        u0 = O.ewald(O.EWALD_STOKES, src, f, trg)
        lap = np.zeros((len(trg), 3))
        for a in range(3):
            e = np.zeros(3)
            e[a] = h
            lap += O.ewald(O.EWALD_STOKES, src, f, trg + e) - 2 * u0 + O.ewald(O.EWALD_STOKES, src, f, trg - e)
        return lap / (h * h)

    fd = (4 * second_differences(1e-3) - second_differences(2e-3)) / 3
    an = O.ewald_stokes_laplacian(src, f, trg)
    assert np.abs(fd - an).max() < 2e-6 * np.abs(an).max()


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
def test_surface_matches_reference():
    """The oracle's surface generator against the reference's own stkfmm::surface
    (stkfmm_helpers.hpp:46-85, compiled from the reference tree): the same points in
    the same order, to an ulp or two (the C++ build may contract (u + 1) b + c into
    an FMA)."""
    for p in (2, 3, 6, 8, 10, 12, 16):
        for depth in (0, 1, 3):
            for alpha in (1.05, 2.95):
                c = np.array([0.1, -0.3, 0.7])
                ref = O.ref_surface(p, c, alpha, depth)
                assert np.abs(O.surface(p, c, alpha, depth) - ref).max() <= 4 * np.finfo(float).eps * np.abs(ref).max()


# Every micro-kernel body STKFMM defines itself (PVFMM's stokes_vel, id 4, is not
# in the reference tree; ids 11-15 are this project's fused and adjoint forms).
REF_UKERNELS = [0, 1, 2, 3, 5, 6, 7, 8, 9, 10] + list(range(16, 29))


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
@pytest.mark.parametrize("uk", REF_UKERNELS)
def test_oracle_matches_reference_ukernel(uk):
    """The oracle's restatement against the reference's own uKerEval body of the
    same micro-kernel (Lib/include/STKFMM/*Kernel.hpp, compiled in place through
    oracle/stub/pvfmm.hpp), sources and targets partly coincident."""
    rng = np.random.default_rng(100 + uk)
    src = rng.random((150, 3))
    trg = np.concatenate([src[:25], rng.random((75, 3))])
    v = uk_values(rng, uk, len(src))
    ref = O.ref_ukernel_direct(uk, src, v, trg)
    assert rel_l2(O.direct(uk, src, v, trg), ref) < 1e-14


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
def test_evaluate_kernel_selection_matches_reference(kernel):
    """The reference's own FMMData::evaluateKernel (its PPKERNEL -> sub-kernel
    choice, FMMData.cpp:261-268, run over 4000-target chunks) against the oracle
    micro-kernel that the library's slot table gives for SLS2T, DLS2T and L2T
    (the table stk_evaluate_kernel uses).  A missing sub-kernel leaves the
    reference's output untouched (it returns after a message)."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(kernel)
    src = rng.random((300, 3))
    trg = np.concatenate([src[:40], rng.random((4100, 3))])  # two 4000-target chunks
    tdim = S.get_kernel_dimension(kernel)[2]
    for p2p, slot in ((1, 0), (2, 1), (4, 6)):
        uk = S.kernel_slot(kernel, slot)
        if uk < 0:
            v = rng.uniform(-1, 1, (len(src), 3))
            assert not O.ref_evaluate_kernel(kernel, p2p, src, v, trg, tdim).any()
            continue
        v = uk_values(rng, uk, len(src))
        ref = O.ref_evaluate_kernel(kernel, p2p, src, v, trg, tdim)
        assert rel_l2(O.direct(uk, src, v, trg), ref) < 1e-14, (kernel, p2p, O.UK_NAMES[uk])


def _wall_points(rng, n, box=1.0, origin=(0.0, 0.0, 0.0)):
    from helpers import clustered_points
    p = np.minimum(clustered_points(rng, n, nclusters=5, sigma=0.05), 0.999)
    p[:, 2] = 0.01 + 0.48 * p[:, 2]
    return p * box + np.asarray(origin)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
@pytest.mark.parametrize("kernel", [8, 16])
@pytest.mark.parametrize("box", [1.0, 3.0])
def test_wall_image_systems_match_reference(kernel, box):
    """oracle.wall_stokes / wall_rpy (what the GPU wall tests compare with)
    against the reference's own StkWallFMM (Lib/src/StkWallFMM.cpp: images,
    sub-FMM values, evalStokes / evalRPY assembly, box scaling) run with exact
    direct sums in place of its FMMs."""
    rng = np.random.default_rng(kernel + int(box))
    origin = np.zeros(3) if box == 1.0 else np.array([-1.0, 2.0, 0.5])
    src = _wall_points(rng, 300, box, origin)
    trg = np.concatenate([src[:50], _wall_points(rng, 200, box, origin)])
    f = rng.normal(size=(len(src), 3))
    if kernel == 8:
        val, mine = f, O.wall_stokes(src, f, trg, z0=origin[2])
    else:
        val = np.concatenate([f, rng.uniform(1e-4, 5e-4, (len(src), 1)) * box], axis=1)
        mine = O.wall_rpy(src, val, trg, z0=origin[2])
    ref = O.ref_wall_direct(kernel, src, val, trg, origin=origin, box=box)
    assert rel_l2(mine, ref) < 1e-12


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
@pytest.mark.parametrize("kernel", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
def test_box_flow_matches_reference(kernel):
    """The reference's own Stk3DFMM in a box [o, o + L)^3 (scaling to the unit
    box, scaleSrc / scaleTrg; Stk3DFMM.cpp, FMMData.cpp) with its FMM replaced by
    the exact sum equals the oracle's single- plus double-layer sums in physical
    coordinates: the physical answer the GPU box-scaling tests compare with."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(200 + kernel)
    o, L = np.array([-1.0, 2.0, 0.5]), 3.0
    sl = rng.random((200, 3)) * L + o
    trg = np.concatenate([sl[:30], rng.random((150, 3)) * L + o])
    uk_sl, uk_dl = S.kernel_slot(kernel, 0), S.kernel_slot(kernel, 1)
    slv = uk_values(rng, uk_sl, len(sl))
    if uk_sl in (5, 6, 8):
        slv[:, 3] *= L  # radius / regularisation in physical units
    if uk_sl in (26, 27):
        slv[:, 6] *= L
    want = O.direct(uk_sl, sl, slv, trg)
    dl = dlv = None
    if uk_dl >= 0:
        dl, dlv = sl.copy(), uk_values(rng, uk_dl, len(sl))
        O.direct(uk_dl, dl, dlv, trg, out=want)
    got = O.ref_stk3d_direct(kernel, sl, slv, trg, S.get_kernel_dimension(kernel)[2], dl, dlv, origin=o, box=L)
    assert rel_l2(got, want) < 1e-12


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref needs the reference tree")
def test_net_flux_correction_matches_reference_periodize(tmp_path, monkeypatch):
    """The triply periodic net-flux correction this library adds after the FMM
    (pvel_net_flux_kernel: velocity += 1/2 sum_i floor(y_i) trD_i over the root's
    upward-equivalent points y_i) against the reference's own
    FMMData::periodizeFMM (FMMData.cpp:203-247) on the same root density: PVel,
    PVelGrad and PVelLaplacian get it on components 1..3, Traction does not."""
    import stkfmm_b200 as S
    p = 4
    n = 6 * (p - 1) ** 2 + 2
    size = 4 * n  # the reference reads (and checks the indices of) its M2C file first; values unused here
    pdata = tmp_path / "pdata"
    pdata.mkdir()
    ij = np.indices((size, size)).reshape(2, -1).T
    np.savetxt(pdata / ("M2C_stokes_PVel_3D3D_p%d" % p), np.c_[ij, np.zeros(len(ij))], fmt="%d %d %.1f")
    monkeypatch.setenv("PVFMM_DIR", str(tmp_path))
    rng = np.random.default_rng(9)
    equiv = rng.normal(size=(n, 4))
    ue = O.ref_surface(p, np.full(3, -0.025), 1.05, 0)
    corr = 0.5 * (np.floor(ue) * equiv[:, 3:4]).sum(0)
    assert np.abs(corr).max() > 0.1
    for k in (128, 256, 512, 1024):
        got = O.ref_periodize(k, p, equiv)
        want = np.ones(S.get_kernel_dimension(k)[2])
        if k != 1024:
            want[1:4] += corr
        assert np.allclose(got, want, rtol=0, atol=1e-14), (k, got, want)


def test_regvel_local_finite_differences_match_full_recomputation():
    """The oracle's neighbourhood-local central differences of L = sum w.u (the regularized
    Stokeslet U-list sum, sources = targets) equal differences of the whole loss recomputed
    over every U-list pair (the check bench.py runs at 1M points on a 4,096-point sample)."""
    import stkfmm_b200 as S
    rng = np.random.default_rng(31)
    n = 1500
    pts = rng.random((n, 3))
    fe = np.concatenate([rng.normal(size=(n, 3)), np.full((n, 1), 1e-3)], axis=1)
    w = rng.normal(size=(n, 3))
    t = S.Octree(pts, 40, 0, sl=pts, trg=pts)
    perm, beg, end = t.point_set(0)
    off, ent = t.list("U")
    leaf = t.first_child < 0
    tb, te = beg, np.where(leaf, end, beg)

    def loss(x, v):
        out = O.lists(O.UK_STOKES_REGVEL, tb, te, off, ent >> 5, ent & 31, beg, end, x[perm], v[perm], x[perm])
        return float((out * w[perm]).sum())

    leaf_of = np.empty(n, np.int64)
    for b in np.flatnonzero(leaf):
        leaf_of[perm[beg[b]:end[b]]] = b
    samp = rng.choice(n, 6, replace=False)
    nb_off, nb = [0], []
    for i in samp:
        b = leaf_of[i]
        lst = np.concatenate([perm[beg[sb]:end[sb]] for sb in (ent[off[b]:off[b + 1]] >> 5)])
        nb.append(lst)
        nb_off.append(nb_off[-1] + len(lst))
    h = 1e-6
    gx, gf = O.regvel_fd_local(samp, np.array(nb_off), np.concatenate(nb), pts, fe, w, h=h)
    for c, i in enumerate(samp):
        for k in range(3):
            xp, xm = pts.copy(), pts.copy()
            xp[i, k] += h
            xm[i, k] -= h
            full = (loss(xp, fe) - loss(xm, fe)) / (2 * h)
            assert abs(full - gx[c, k]) <= 1e-6 * max(abs(full), np.linalg.norm(gx[c])), (i, k, full, gx[c, k])
            fp, fm = fe.copy(), fe.copy()
            fp[i, k] += h
            fm[i, k] -= h
            full = (loss(pts, fp) - loss(pts, fm)) / (2 * h)
            assert abs(full - gf[c, k]) <= 1e-6 * max(abs(full), np.linalg.norm(gf[c])), (i, k, full, gf[c, k])
