"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs the reference's FP64 test kernels (Test/SimpleKernel.cpp of STKFMM, compiled
from the read-only reference tree into oracle/_ref/libstk_ref.so by
oracle/Makefile) over all (target, source) pairs with the protocol of
runSimpleKernel (Test/Test.cpp:478-510), on seeded inputs shaped like the
reference test's (values U(-1,1) as Test/Test.cpp:318-319; the last component of
RPY / regularized-Stokes values |v|*eps as Test/Test.cpp:321-328).  Two point
layouts per kernel:

  random: 160 sources in [0,1)^3, 96 targets of which the first 48 coincide with
          sources (self-interaction mask / regularized self term);
  fixed:  the 4-point source layout of PointDistribution::fixedPoints
          (Test/Util/PointDistribution.cpp:15-48, box 1, shift 0) evaluated on a
          5x5x5 target grid.

Usage (needs the reference tree, so only in the build container):
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CASES = {
    "StokesSL": O.REF_STOKES_SL,
    "LaplaceSLPGrad": O.REF_LAP_SL_PGRAD,
    "LaplaceDLPGrad": O.REF_LAP_DL_PGRAD,
    "StokesSLRPY": O.REF_STOKES_SL_RPY,
    "StokesRegSLVel": O.REF_STOKES_REG_SL_VEL,
    "StokesSLPVel": O.REF_STOKES_SL_PVEL,
    "StokesDLPVel": O.REF_STOKES_DL_PVEL,
    "LaplaceSLPGradGrad": O.REF_LAP_SL_PGRADGRAD,
    "LaplaceDLPGradGrad": O.REF_LAP_DL_PGRADGRAD,
    "LaplaceQPGradGrad": O.REF_LAP_QPGRADGRAD,
    "StokesSLPVelGrad": O.REF_STOKES_SL_PVELGRAD,
    "StokesDLPVelGrad": O.REF_STOKES_DL_PVELGRAD,
    "StokesSLPVelLaplacian": O.REF_STOKES_SL_PVELLAP,
    "StokesDLPVelLaplacian": O.REF_STOKES_DL_PVELLAP,
    "StokesSLTraction": O.REF_STOKES_SL_TRACTION,
    "StokesDLTraction": O.REF_STOKES_DL_TRACTION,
    "StokesRegSLVelOmega": O.REF_STOKES_REG_SL_VELOMEGA,
}
EPS = 1e-2


def values(rng, which, n):
    sd = O.REF_DIMS[which][0]
    v = rng.uniform(-1.0, 1.0, size=(n, sd))
    if which in (O.REF_STOKES_SL_RPY, O.REF_STOKES_REG_SL_VEL, O.REF_STOKES_REG_SL_VELOMEGA):
        v[:, -1] = np.abs(v[:, -1]) * EPS
    return v


def main():
    O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libstk_ref.so missing: the reference tree is required")
    fixed_src = np.array([[0.1, 0.1, 0.1], [0.2, 0.2, 0.2], [0.3, 0.3, 0.3], [0.4, 0.4, 0.4]])
    g = (np.arange(5) + 0.5) / 5.0
    grid = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    for seed, (name, which) in enumerate(CASES.items()):
        rng = np.random.default_rng(1000 + seed)
        src = rng.random((160, 3))
        trg = np.concatenate([src[:48], rng.random((48, 3))])
        val = values(rng, which, len(src))
        out = O.ref_direct(which, src, val, trg)
        fval = values(rng, which, len(fixed_src))
        fout = O.ref_direct(which, fixed_src, fval, grid)
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % name), src=src, val=val, trg=trg, out=out,
                            fixed_src=fixed_src, fixed_val=fval, fixed_trg=grid, fixed_out=fout)
        print(name, out.shape, float(np.abs(out).max()))


if __name__ == "__main__":
    main()
