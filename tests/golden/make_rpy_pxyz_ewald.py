"""Generate tests/golden/rpy_pxyz_2m_ewald.npz: the triply periodic RPY velocity and its
Laplacian at a sample of the 2,097,152-point RPY workload, by Ewald summation.

Workload (the same numpy calls, in the same order, as the benchmark's RPY PXYZ workload):
default_rng(0); points ~ U[0,1)^3 (2,097,152 x 3); f ~ N(0,1)^3 minus its mean; b ~ U(1e-4, 5e-4).
Sample: default_rng(17).choice(n, 4096, replace=False).

Truth, with G the periodic Stokeslet (zero-mean force density, k = 0 mode dropped) and lap G its
Laplacian, both from the oracle's cell-list Ewald sums (oracle.ewald_cells, pinned against
oracle.ewald in tests/test_oracle.py):
    u     = G f + (1/6) lap G (b^2 f)     (RPY: u = (1 + b^2/6 lap) G f, summed over all images)
    lap u = lap G f
Relative accuracy of the truth ~1e-12 (Ewald splitting at xi = 16, real-space cutoff 5.3 / xi,
wave vectors |m| <= 28).

Usage (about 30-50 minutes on 8 host cores):
    python tests/golden/make_rpy_pxyz_ewald.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

N = 2097152
NSAMPLE = 4096
OUT = os.path.join(HERE, "rpy_pxyz_2m_ewald.npz")


def workload():
    rng = np.random.default_rng(0)
    pts = rng.random((N, 3))
    f = rng.normal(size=(N, 3))
    f -= f.mean(0)
    b = rng.uniform(1e-4, 5e-4, (N, 1))
    return pts, f, b


def sample():
    return np.sort(np.random.default_rng(17).choice(N, NSAMPLE, replace=False))


def main():
    O.build()
    pts, f, b = workload()
    idx = sample()
    trg = pts[idx]
    t0 = time.perf_counter()
    g = O.ewald_cells(O.EWALD_STOKES, pts, f, trg)
    print("stokes %.0f s" % (time.perf_counter() - t0), flush=True)
    lap_b2f = O.ewald_stokes_laplacian_cells(pts, b * b * f, trg)
    print("lap(b^2 f) %.0f s" % (time.perf_counter() - t0), flush=True)
    lap_f = O.ewald_stokes_laplacian_cells(pts, f, trg)
    print("lap(f) %.0f s" % (time.perf_counter() - t0), flush=True)
    truth = np.concatenate([g + lap_b2f / 6.0, lap_f], axis=1)
    np.savez_compressed(OUT, idx=idx.astype(np.int64), truth=truth, n=np.int64(N),
                        note=np.array("RPY PXYZ 2M workload, seed 0: (u, lap u) by Ewald summation"))
    print("wrote", OUT, truth.shape)


if __name__ == "__main__":
    main()
