"""Shared test helpers: golden-fixture map, seeded workloads, list utilities."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

# golden fixture -> [(micro-kernel id, output column slice, value column slice)]
# micro-kernel ids as in include/stkfmm_b200.h (enum stk_ukernel)
GOLDEN_MAP = {
    "StokesSL": [(4, slice(0, 3), slice(0, 3)), (7, slice(0, 6), slice(0, 3))],
    "LaplaceSLPGrad": [(1, slice(0, 4), slice(0, 1)), (0, slice(0, 1), slice(0, 1))],
    "LaplaceDLPGrad": [(3, slice(0, 4), slice(0, 3)), (2, slice(0, 1), slice(0, 3))],
    "StokesSLRPY": [(6, slice(0, 6), slice(0, 4)), (5, slice(0, 3), slice(0, 4))],
    "StokesRegSLVel": [(8, slice(0, 3), slice(0, 4))],
    "StokesSLPVel": [(9, slice(0, 4), slice(0, 4))],
    "StokesDLPVel": [(10, slice(0, 4), slice(0, 9))],
    "LaplaceSLPGradGrad": [(16, slice(0, 10), slice(0, 1))],
    "LaplaceDLPGradGrad": [(17, slice(0, 10), slice(0, 3))],
    "LaplaceQPGradGrad": [(19, slice(0, 10), slice(0, 9)), (18, slice(0, 1), slice(0, 9))],
    "StokesSLPVelGrad": [(20, slice(0, 16), slice(0, 4))],
    "StokesDLPVelGrad": [(21, slice(0, 16), slice(0, 9))],
    "StokesSLPVelLaplacian": [(22, slice(0, 7), slice(0, 4))],
    "StokesDLPVelLaplacian": [(23, slice(0, 7), slice(0, 9))],
    "StokesSLTraction": [(24, slice(0, 9), slice(0, 4))],
    "StokesDLTraction": [(25, slice(0, 9), slice(0, 9))],
    "StokesRegSLVelOmega": [(27, slice(0, 6), slice(0, 7)), (26, slice(0, 3), slice(0, 7))],
}
UK_SDIM = [1, 1, 3, 3, 3, 4, 4, 3, 4, 4, 9, 4, 13, 3, 4, 4, 1, 3, 9, 9, 4, 9, 4, 9, 4, 9, 7, 7, 3]
UK_TDIM = [1, 4, 1, 4, 3, 3, 6, 6, 3, 4, 4, 4, 4, 7, 3, 1, 10, 10, 1, 10, 16, 16, 7, 7, 9, 9, 3, 6, 6]
UK_NAMES = ["laplace_p", "laplace_pgrad", "laplace_dipolep", "laplace_dipolepgrad", "stokes_vel", "rpy_u",
            "rpy_ulapu", "stk_ulapu", "stokes_regvel", "stokes_pvel", "stokes_doublepvel", "laplace_sldl_pgrad",
            "stokes_sldl_pvel", "regvel_adjoint_src", "regvel_adjoint_trg", "laplace_sldl_p", "laplace_pgradgrad",
            "laplace_dipolepgradgrad", "laplace_quadp", "laplace_quadpgradgrad", "stokes_pvelgrad",
            "stokes_doublepvelgrad", "stokes_pvellaplacian", "stokes_doublelaplacian", "stokes_traction",
            "stokes_doubletraction", "stokes_regftvel", "stokes_regftvelomega", "stokes_velomega"]
# forward micro-kernels (the adjoint ones, 13 and 14, need per-target values)
UK_FORWARD = list(range(13)) + list(range(15, 29))


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, "golden_%s.npz" % name)))


def uk_values(rng, uk, n, eps=1e-2):
    """Seeded source values for micro-kernel uk (U(-1,1); radius/eps component |v|*eps)."""
    v = rng.uniform(-1.0, 1.0, size=(n, UK_SDIM[uk]))
    if uk in (5, 6, 8):
        v[:, 3] = np.abs(v[:, 3]) * eps
    if uk in (26, 27):
        v[:, 6] = np.abs(v[:, 6]) * eps
    return v


def clustered_points(rng, n, nclusters=8, sigma=0.02):
    """Gaussian clusters with centres in [0.1, 0.9]^3, clipped into [0,1)^3."""
    c = rng.uniform(0.1, 0.9, size=(nclusters, 3))
    idx = rng.integers(0, nclusters, size=n)
    p = c[idx] + rng.normal(0.0, sigma, size=(n, 3))
    return np.clip(p, 0.0, np.nextafter(1.0, 0.0))


def sldl_values(sl, dl):
    """Fused SL+DL value rows (the layout of the fused micro-kernels)."""
    return np.concatenate([sl, dl], axis=1)
