/*
 * stk_oracle.c -- CPU FP64 oracle for the STKFMM direct kernel-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
 * compared against; it is never linked into, called by, or shipped with the
 * product library (stkfmm_b200/).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load it.
 *
 * What it restates (plain C, exact 1/sqrt, FP64):
 *   - every in-scope STKFMM micro-kernel ("uKerEval" body), one function each,
 *     with the reference's r^2 > 0 self-interaction mask;
 *   - the per-kernel scale factor that PVFMM's GenericKernel applies;
 *   - the dense direct sum of FMMData::evaluateKernel (Lib/src/FMMData.cpp:252-283);
 *   - a sum over an explicit target-box / source-box interaction list (the U/W/X
 *     list loops that PVFMM runs inside PtFMM_Evaluate), so the GPU list kernels
 *     can be checked on the very same lists;
 *   - the KIFMM cube-surface point generator (Lib/include/STKFMM/stkfmm_helpers.hpp:46-85);
 *   - the adjoint of the regularized Stokeslet sum (no reference counterpart;
 *     derived by hand from the forward formula and checked by finite differences).
 *
 * Parity pin: tests/golden/ holds outputs of the reference's own FP64 test
 * kernels (Test/SimpleKernel.cpp, compiled by oracle/Makefile into oracle/_ref/)
 * on seeded inputs; tests/test_oracle.py checks this file against them.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Micro-kernel ids.  Must match stkfmm_b200/csrc/stk_kernels.cuh and
 * include/stkfmm_b200.h (enum stk_ukernel). */
enum {
    UK_LAPLACE_P = 0,           /* q(1)      -> p(1)              LaplaceLayerKernel.hpp:41-65   */
    UK_LAPLACE_PGRAD = 1,       /* q(1)      -> p,grad p(4)       LaplaceLayerKernel.hpp:67-96   */
    UK_LAPLACE_DIPOLEP = 2,     /* d(3)      -> p(1)              LaplaceLayerKernel.hpp:98-113  */
    UK_LAPLACE_DIPOLEPGRAD = 3, /* d(3)      -> p,grad p(4)       LaplaceLayerKernel.hpp:115-136 */
    UK_STOKES_VEL = 4,          /* f(3)      -> u(3)              PVFMM stokes_vel (StokesLayerKernel.hpp:39-42) */
    UK_RPY_U = 5,               /* f,a(4)    -> u(3)              RPYKernel.hpp:17-45            */
    UK_RPY_ULAPU = 6,           /* f,a(4)    -> u,lap u(6)        RPYKernel.hpp:52-90            */
    UK_STK_ULAPU = 7,           /* f(3)      -> u,lap u(6)        RPYKernel.hpp:97-129           */
    UK_STOKES_REGVEL = 8,       /* f,eps(4)  -> u(3)              StokesRegSingleLayerKernel.hpp:17-41 */
    UK_STOKES_PVEL = 9,         /* f,trD(4)  -> p,u(4)            StokesSingleLayerKernel.hpp:27-47 */
    UK_STOKES_DOUBLEPVEL = 10,  /* D(9)      -> p,u(4)            StokesDoubleLayerKernel.hpp:25-57 */
    /* 11 .. 15: fused / adjoint device micro-kernels, no oracle body (tests compose them) */
    UK_LAPLACE_PGRADGRAD = 16,       /* q(1) -> p,grad,Hessian(10)  LaplaceLayerKernel.hpp:138-166 */
    UK_LAPLACE_DIPOLEPGRADGRAD = 17, /* d(3) -> (10)                LaplaceLayerKernel.hpp:168-200 */
    UK_LAPLACE_QUADP = 18,           /* S(9) -> p(1)                LaplaceLayerKernel.hpp:202-232 */
    UK_LAPLACE_QUADPGRADGRAD = 19,   /* S(9) -> (10)                LaplaceLayerKernel.hpp:234-301 */
    UK_STOKES_PVELGRAD = 20,         /* f,trD(4) -> (16)            StokesSingleLayerKernel.hpp:54-111 */
    UK_STOKES_DOUBLEPVELGRAD = 21,   /* D(9) -> (16)                StokesDoubleLayerKernel.hpp:64-143 */
    UK_STOKES_PVELLAPLACIAN = 22,    /* f,trD(4) -> (7)             StokesSingleLayerKernel.hpp:118-155 */
    UK_STOKES_DOUBLELAPLACIAN = 23,  /* D(9) -> (7)                 StokesDoubleLayerKernel.hpp:150-206 */
    UK_STOKES_TRACTION = 24,         /* f,trD(4) -> (9)             StokesSingleLayerKernel.hpp:162-199 */
    UK_STOKES_DOUBLETRACTION = 25,   /* D(9) -> (9)                 StokesDoubleLayerKernel.hpp:213-276 */
    UK_STOKES_REGFTVEL = 26,         /* f,t,eps(7) -> u(3)          StokesRegSingleLayerKernel.hpp:48-89 */
    UK_STOKES_REGFTVELOMEGA = 27,    /* f,t,eps(7) -> u,omega(6)    StokesRegSingleLayerKernel.hpp:96-151 */
    UK_STOKES_VELOMEGA = 28,         /* f(3) -> u,omega(6)          StokesRegSingleLayerKernel.hpp:158-203 */
    UK_COUNT = 29
};

static const int uk_sdim[UK_COUNT] = {1, 1, 3, 3, 3, 4, 4, 3, 4, 4, 9, 0, 0, 0, 0, 0, 1, 3, 9, 9,
                                      4, 9, 4, 9, 4, 9, 7, 7, 3};
static const int uk_tdim[UK_COUNT] = {1, 4, 1, 4, 3, 3, 6, 6, 3, 4, 4, 0, 0, 0, 0, 0, 10, 10, 1, 10,
                                      16, 16, 7, 7, 9, 9, 3, 6, 6};

static int uk_valid(int uk) { return uk >= 0 && uk < UK_COUNT && uk_sdim[uk] > 0; }

static const double PI_ = 3.14159265358979323846264338327950288;

int oracle_uk_dims(int uk, int *sdim, int *tdim) {
    if (!uk_valid(uk)) return 1;
    *sdim = uk_sdim[uk];
    *tdim = uk_tdim[uk];
    return 0;
}

/* ScaleFactor() of each micro-kernel: 1/(4 pi) for Laplace, 1/(8 pi) for the
 * Stokes family (e.g. LaplaceLayerKernel.hpp:44-46, RPYKernel.hpp:20-22). */
double oracle_uk_scale(int uk) {
    if (uk == UK_STOKES_TRACTION) return -3.0 / (4.0 * PI_);       /* StokesSingleLayerKernel.hpp:166-168 */
    if (uk == UK_STOKES_DOUBLETRACTION) return -3.0 / (8.0 * PI_); /* StokesDoubleLayerKernel.hpp:217-219 */
    if (uk >= UK_STOKES_PVELGRAD) return 1.0 / (8.0 * PI_);
    return (uk <= UK_LAPLACE_DIPOLEPGRAD || uk >= UK_LAPLACE_PGRADGRAD) ? 1.0 / (4.0 * PI_) : 1.0 / (8.0 * PI_);
}

/* Exact masked 1/sqrt: the reference's approx_rsqrt<digits>(r2, r2 > 0) returns
 * 0 where the mask is false and ~1/sqrt(r2) elsewhere. */
static inline double rsqrt_mask(double r2) { return r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0; }

/* One (target, source) pair, unscaled, accumulated into u.  r = x_trg - x_src. */
static void uk_pair(int uk, const double r[3], const double *f, double *u) {
    const double dx = r[0], dy = r[1], dz = r[2];
    switch (uk) {
    case UK_LAPLACE_P: { /* LaplaceLayerKernel.hpp:59-64 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        u[0] += f[0] * rinv;
    } break;
    case UK_LAPLACE_PGRAD: { /* LaplaceLayerKernel.hpp:85-95 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double sv = f[0] * rinv * rinv * rinv;
        u[0] += sv * r2;
        u[1] -= sv * dx;
        u[2] -= sv * dy;
        u[3] -= sv * dz;
    } break;
    case UK_LAPLACE_DIPOLEP: { /* LaplaceLayerKernel.hpp:105-112 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rdotn = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += rinv3 * rdotn;
    } break;
    case UK_LAPLACE_DIPOLEPGRAD: { /* LaplaceLayerKernel.hpp:122-135 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double rinv3 = rinv2 * rinv;
        double rinv5 = rinv3 * rinv2;
        double rdotn = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += rdotn * rinv3;
        u[1] += (f[0] * r2 - 3.0 * rdotn * dx) * rinv5;
        u[2] += (f[1] * r2 - 3.0 * rdotn * dy) * rinv5;
        u[3] += (f[2] * r2 - 3.0 * rdotn * dz) * rinv5;
    } break;
    case UK_STOKES_VEL: {
        /* Stokeslet u = f/r + r (f.r)/r^3 (times 1/8pi).  The body lives in PVFMM
         * (not vendored); restated from the Stokeslet formula and pinned by the
         * reference test kernel StokesSL (Test/SimpleKernel.cpp:986-1023, a = 0). */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += f[0] * rinv + dx * fdotr * rinv3;
        u[1] += f[1] * rinv + dy * fdotr * rinv3;
        u[2] += f[2] * rinv + dz * fdotr * rinv3;
    } break;
    case UK_RPY_U: { /* RPYKernel.hpp:24-44; note the truncated 1/3 constant */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        double fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        double three_fdotr_rinv5 = 3.0 * fdotr * rinv5;
        double a2_over_three = 0.3333333333333 * f[3] * f[3];
        u[0] += (r2 * f[0] + dx * fdotr) * rinv3 + a2_over_three * (f[0] * rinv3 - three_fdotr_rinv5 * dx);
        u[1] += (r2 * f[1] + dy * fdotr) * rinv3 + a2_over_three * (f[1] * rinv3 - three_fdotr_rinv5 * dy);
        u[2] += (r2 * f[2] + dz * fdotr) * rinv3 + a2_over_three * (f[2] * rinv3 - three_fdotr_rinv5 * dz);
    } break;
    case UK_RPY_ULAPU: { /* RPYKernel.hpp:59-89 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        double fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        double fdotr_rinv3 = fdotr * rinv3;
        double three_fdotr_rinv5 = 3.0 * fdotr * rinv5;
        double a2_over_three = 0.3333333333333 * f[3] * f[3];
        double cx = f[0] * rinv3 - three_fdotr_rinv5 * dx;
        double cy = f[1] * rinv3 - three_fdotr_rinv5 * dy;
        double cz = f[2] * rinv3 - three_fdotr_rinv5 * dz;
        u[0] += f[0] * rinv + dx * fdotr_rinv3 + a2_over_three * cx;
        u[1] += f[1] * rinv + dy * fdotr_rinv3 + a2_over_three * cy;
        u[2] += f[2] * rinv + dz * fdotr_rinv3 + a2_over_three * cz;
        u[3] += 2.0 * cx;
        u[4] += 2.0 * cy;
        u[5] += 2.0 * cz;
    } break;
    case UK_STK_ULAPU: { /* RPYKernel.hpp:104-128 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        double fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        double fdotr_rinv3 = fdotr * rinv3;
        double three_fdotr_rinv5 = 3.0 * fdotr * rinv5;
        u[0] += f[0] * rinv + dx * fdotr_rinv3;
        u[1] += f[1] * rinv + dy * fdotr_rinv3;
        u[2] += f[2] * rinv + dz * fdotr_rinv3;
        u[3] += 2.0 * (f[0] * rinv3 - three_fdotr_rinv5 * dx);
        u[4] += 2.0 * (f[1] * rinv3 - three_fdotr_rinv5 * dy);
        u[5] += 2.0 * (f[2] * rinv3 - three_fdotr_rinv5 * dz);
    } break;
    case UK_STOKES_REGVEL: { /* StokesRegSingleLayerKernel.hpp:24-40; the self term is kept */
        double reg = f[3];
        double r2 = dx * dx + dy * dy + dz * dz + reg * reg;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double r2reg2 = r2 + reg * reg;
        double cc = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += rinv3 * (r2reg2 * f[0] + dx * cc);
        u[1] += rinv3 * (r2reg2 * f[1] + dy * cc);
        u[2] += rinv3 * (r2reg2 * f[2] + dz * cc);
    } break;
    case UK_STOKES_PVEL: { /* StokesSingleLayerKernel.hpp:34-46 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double cc = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += 2.0 * cc * rinv3;
        cc -= f[3];
        u[1] += rinv3 * (r2 * f[0] + dx * cc);
        u[2] += rinv3 * (r2 * f[1] + dy * cc);
        u[3] += rinv3 * (r2 * f[2] + dz * cc);
    } break;
    case UK_STOKES_DOUBLEPVEL: { /* StokesDoubleLayerKernel.hpp:32-56; D row-major */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        double cc = f[0] * dx * dx + f[4] * dy * dy + f[8] * dz * dz;
        cc += (f[1] + f[3]) * dx * dy;
        cc += (f[2] + f[6]) * dx * dz;
        cc += (f[5] + f[7]) * dy * dz;
        cc *= -3.0 * rinv5;
        double trace = f[0] + f[4] + f[8];
        u[0] += 2.0 * (cc + r2 * rinv5 * trace);
        u[1] += dx * cc;
        u[2] += dy * cc;
        u[3] += dz * cc;
    } break;
    case UK_LAPLACE_PGRADGRAD: { /* LaplaceLayerKernel.hpp:145-165 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double sv = f[0] * rinv2 * rinv;
        u[0] += sv * r2;
        u[1] -= sv * dx;
        u[2] -= sv * dy;
        u[3] -= sv * dz;
        sv *= rinv2;
        u[4] += sv * (3.0 * dx * dx - r2);
        u[5] += sv * 3.0 * dx * dy;
        u[6] += sv * 3.0 * dx * dz;
        u[7] += sv * (3.0 * dy * dy - r2);
        u[8] += sv * 3.0 * dy * dz;
        u[9] += sv * (3.0 * dz * dz - r2);
    } break;
    case UK_LAPLACE_DIPOLEPGRADGRAD: { /* LaplaceLayerKernel.hpp:175-199 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double rinv3 = rinv2 * rinv;
        double rinv5 = rinv2 * rinv3;
        double rinv7 = rinv2 * rinv5;
        double rd = dx * f[0] + dy * f[1] + dz * f[2];
        double t3 = 3.0 * r2;
        u[0] += rd * rinv3;
        u[1] += (f[0] * r2 - rd * 3.0 * dx) * rinv5;
        u[2] += (f[1] * r2 - rd * 3.0 * dy) * rinv5;
        u[3] += (f[2] * r2 - rd * 3.0 * dz) * rinv5;
        u[4] += (15.0 * dx * dx * rd - r2 * (3.0 * rd + 6.0 * dx * f[0])) * rinv7;
        u[5] += (15.0 * dx * dy * rd - t3 * (dx * f[1] + dy * f[0])) * rinv7;
        u[6] += (15.0 * dx * dz * rd - t3 * (dx * f[2] + dz * f[0])) * rinv7;
        u[7] += (15.0 * dy * dy * rd - r2 * (3.0 * rd + 6.0 * dy * f[1])) * rinv7;
        u[8] += (15.0 * dy * dz * rd - t3 * (dy * f[2] + dz * f[1])) * rinv7;
        u[9] += (15.0 * dz * dz * rd - r2 * (3.0 * rd + 6.0 * dz * f[2])) * rinv7;
    } break;
    case UK_LAPLACE_QUADP: { /* LaplaceLayerKernel.hpp:209-231; S row-major */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv5 = rinv * rinv;
        rinv5 = rinv5 * rinv5 * rinv;
        double c = f[0] * dx * dx;
        c += (f[1] + f[3]) * dx * dy;
        c += (f[2] + f[6]) * dx * dz;
        c += f[4] * dy * dy;
        c += (f[5] + f[7]) * dy * dz;
        c += f[8] * dz * dz;
        c *= 3.0;
        u[0] += (c - r2 * (f[0] + f[4] + f[8])) * rinv5;
    } break;
    case UK_LAPLACE_QUADPGRADGRAD: { /* LaplaceLayerKernel.hpp:241-300 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double rinv3 = rinv2 * rinv;
        double rinv5 = rinv3 * rinv2;
        double rinv7 = rinv5 * rinv2;
        double rinv9 = rinv7 * rinv2;
        const double sxx = f[0], sxy = f[1], sxz = f[2], syx = f[3], syy = f[4], syz = f[5];
        const double szx = f[6], szy = f[7], szz = f[8];
        double rrQ = dx * dx * sxx + dx * dy * (sxy + syx) + dx * dz * (sxz + szx) + dy * dy * syy +
                     dy * dz * (syz + szy) + dz * dz * szz;
        double c3 = rrQ * 3.0, c5 = rrQ * 5.0;
        double tr = sxx + syy + szz;
        /* row (S r) and column (S^T r) products */
        double ax = dx * sxx + dy * sxy + dz * sxz, ay = dx * syx + dy * syy + dz * syz;
        double az = dx * szx + dy * szy + dz * szz;
        double bx = dx * sxx + dy * syx + dz * szx, by = dx * sxy + dy * syy + dz * szy;
        double bz = dx * sxz + dy * syz + dz * szz;
        u[0] += (c3 - r2 * tr) * rinv5;
        double px = dx * c5 - r2 * (ax + bx + dx * tr);
        double py = dy * c5 - r2 * (ay + by + dy * tr);
        double pz = dz * c5 - r2 * (az + bz + dz * tr);
        u[1] -= 3.0 * px * rinv7;
        u[2] -= 3.0 * py * rinv7;
        u[3] -= 3.0 * pz * rinv7;
        double r4 = r2 * r2;
        u[4] += rinv9 * (105.0 * dx * dx * rrQ - r2 * 15.0 * (rrQ + dx * 2.0 * (ax + bx) + dx * dx * tr) +
                         3.0 * r4 * (tr + 2.0 * sxx));
        u[5] += rinv9 * (105.0 * (dx * dy * rrQ) - r2 * 15.0 * ((dy * ax + dy * bx + dx * ay + dx * by) + dx * dy * tr) +
                         3.0 * r4 * (sxy + syx));
        u[6] += rinv9 * (105.0 * (dx * dz * rrQ) - r2 * 15.0 * ((dz * ax + dz * bx + dx * az + dx * bz) + dx * dz * tr) +
                         3.0 * r4 * (sxz + szx));
        u[7] += rinv9 * (105.0 * dy * dy * rrQ - r2 * 15.0 * (rrQ + dy * 2.0 * (ay + by) + dy * dy * tr) +
                         3.0 * r4 * (tr + 2.0 * syy));
        u[8] += rinv9 * (105.0 * (dy * dz * rrQ) - r2 * 15.0 * ((dy * az + dy * bz + dz * ay + dz * by) + dy * dz * tr) +
                         3.0 * r4 * (syz + szy));
        u[9] += rinv9 * (105.0 * dz * dz * rrQ - r2 * 15.0 * (rrQ + dz * 2.0 * (az + bz) + dz * dz * tr) +
                         3.0 * r4 * (tr + 2.0 * szz));
    } break;
    case UK_STOKES_PVELGRAD:        /* StokesSingleLayerKernel.hpp:61-110 */
    case UK_STOKES_PVELLAPLACIAN: { /* StokesSingleLayerKernel.hpp:125-154 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        const double fx = f[0], fy = f[1], fz = f[2], tr = f[3];
        double cc = fx * dx + fy * dy + fz * dz;
        u[0] += 2.0 * rinv3 * cc;
        cc -= tr;
        u[1] += rinv3 * (r2 * fx + cc * dx);
        u[2] += rinv3 * (r2 * fy + cc * dy);
        u[3] += rinv3 * (r2 * fz + cc * dz);
        cc += tr;
        u[4] += 2.0 * (r2 * fx - 3.0 * dx * cc) * rinv5;
        u[5] += 2.0 * (r2 * fy - 3.0 * dy * cc) * rinv5;
        u[6] += 2.0 * (r2 * fz - 3.0 * dz * cc) * rinv5;
        if (uk == UK_STOKES_PVELLAPLACIAN) break;
        double qxx = r2 - 3.0 * dx * dx, qxy = -3.0 * dx * dy, qxz = -3.0 * dx * dz;
        double qyy = r2 - 3.0 * dy * dy, qyz = -3.0 * dy * dz, qzz = r2 - 3.0 * dz * dz;
        cc -= tr;
        u[7] += qxx * cc * rinv5;
        u[8] += (qxy * cc + r2 * (dx * fy - dy * fx)) * rinv5;
        u[9] += (qxz * cc + r2 * (dx * fz - dz * fx)) * rinv5;
        u[10] += (qxy * cc + r2 * (dy * fx - dx * fy)) * rinv5;
        u[11] += qyy * cc * rinv5;
        u[12] += (qyz * cc + r2 * (dy * fz - dz * fy)) * rinv5;
        u[13] += (qxz * cc + r2 * (dz * fx - dx * fz)) * rinv5;
        u[14] += (qyz * cc + r2 * (dz * fy - dy * fz)) * rinv5;
        u[15] += qzz * cc * rinv5;
    } break;
    case UK_STOKES_TRACTION: { /* StokesSingleLayerKernel.hpp:169-198 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rinv5 = rinv3 * rinv * rinv;
        const double tr = f[3];
        double cc = (f[0] * dx + f[1] * dy + f[2] * dz - tr) * rinv5;
        double diag = tr * r2 * rinv5 * 0.3333333333333333333;
        const double d[3] = {dx, dy, dz};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) u[3 * i + j] += d[i] * d[j] * cc + (i == j ? diag : 0.0);
    } break;
    case UK_STOKES_DOUBLEPVELGRAD:    /* StokesDoubleLayerKernel.hpp:71-142 */
    case UK_STOKES_DOUBLELAPLACIAN: { /* StokesDoubleLayerKernel.hpp:157-205 */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double rinv3 = rinv * rinv2;
        double rinv5 = rinv3 * rinv2;
        double rinv7 = rinv5 * rinv2;
        const double sxx = f[0], sxy = f[1], sxz = f[2], syx = f[3], syy = f[4], syz = f[5];
        const double szx = f[6], szy = f[7], szz = f[8];
        double cc = sxx * dx * dx + syy * dy * dy + szz * dz * dz;
        cc += (sxy + syx) * dx * dy;
        cc += (sxz + szx) * dx * dz;
        cc += (syz + szy) * dy * dz;
        double ccn3 = -3.0 * cc, cc5 = 5.0 * cc;
        const double trace = sxx + syy + szz;
        double ax = dx * sxx + dy * sxy + dz * sxz, ay = dx * syx + dy * syy + dz * syz;
        double az = dx * szx + dy * szy + dz * szz;
        double bx = dx * sxx + dy * syx + dz * szx, by = dx * sxy + dy * syy + dz * szy;
        double bz = dx * sxz + dy * syz + dz * szz;
        u[0] += 2.0 * (ccn3 + r2 * trace) * rinv5;
        u[1] += rinv5 * dx * ccn3;
        u[2] += rinv5 * dy * ccn3;
        u[3] += rinv5 * dz * ccn3;
        rinv7 *= -3.0;
        u[4] -= 2.0 * rinv7 * (dx * cc5 - r2 * ((ax + bx) + dx * trace));
        u[5] -= 2.0 * rinv7 * (dy * cc5 - r2 * ((ay + by) + dy * trace));
        u[6] -= 2.0 * rinv7 * (dz * cc5 - r2 * ((az + bz) + dz * trace));
        if (uk == UK_STOKES_DOUBLELAPLACIAN) break;
        /* rinv7 keeps its factor -3 here, as in the reference */
        double ccn1 = -cc;
        double e0 = -2.0 * dx * sxx - dy * (sxy + syx) - dz * (sxz + szx);
        double e1 = -2.0 * dy * syy - dx * (sxy + syx) - dz * (syz + szy);
        double e2 = -2.0 * dz * szz - dx * (sxz + szx) - dy * (syz + szy);
        const double d[3] = {dx, dy, dz}, e[3] = {e0, e1, e2};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                u[7 + 3 * i + j] += (5.0 * ccn1 * d[i] * d[j] - r2 * d[i] * e[j] - (i == j ? r2 * ccn1 : 0.0)) * rinv7;
    } break;
    case UK_STOKES_REGFTVEL:        /* StokesRegSingleLayerKernel.hpp:55-88 */
    case UK_STOKES_REGFTVELOMEGA: { /* StokesRegSingleLayerKernel.hpp:103-150; unmasked rsqrt as there */
        const double fx = f[0], fy = f[1], fz = f[2], tx = f[3], ty = f[4], tz = f[5], eps = f[6];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r4 = r2 * r2;
        double eps2 = eps * eps, eps4 = eps2 * eps2;
        double rinv = 1.0 / sqrt(eps2 + r2);
        double sd = rinv * rinv * rinv;
        double rd = 0.5 * sd * rinv * rinv;
        double dd = 0.5 * rd * rinv * rinv;
        double rc = (2.0 * r2 + 5.0 * eps2) * rd;
        double D1 = (10.0 * eps4 - 7.0 * eps2 * r2 - 2.0 * r4) * dd;
        double D2 = (21.0 * eps2 + 6.0 * r2) * dd;
        double H2 = sd, H1 = (r2 + 2.0 * eps2) * H2;
        double fcx = fy * dz - fz * dy, fcy = fz * dx - fx * dz, fcz = fx * dy - fy * dx;
        double tcx = ty * dz - tz * dy, tcy = tz * dx - tx * dz, tcz = tx * dy - ty * dx;
        double fdr = fx * dx + fy * dy + fz * dz, tdr = tx * dx + ty * dy + tz * dz;
        u[0] += H1 * fx + H2 * fdr * dx + rc * tcx;
        u[1] += H1 * fy + H2 * fdr * dy + rc * tcy;
        u[2] += H1 * fz + H2 * fdr * dz + rc * tcz;
        if (uk == UK_STOKES_REGFTVEL) break;
        u[3] += D1 * tx + D2 * tdr * dx + rc * fcx;
        u[4] += D1 * ty + D2 * tdr * dy + rc * fcy;
        u[5] += D1 * tz + D2 * tdr * dz + rc * fcz;
    } break;
    case UK_STOKES_VELOMEGA: { /* StokesRegSingleLayerKernel.hpp:165-202 */
        const double fx = f[0], fy = f[1], fz = f[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv3 = rinv * rinv * rinv;
        double rc = 2.0 * r2 * (0.5 * rinv3 * rinv * rinv);
        double H2 = rinv3, H1 = r2 * H2;
        double fdr = fx * dx + fy * dy + fz * dz;
        u[0] += H1 * fx + H2 * fdr * dx;
        u[1] += H1 * fy + H2 * fdr * dy;
        u[2] += H1 * fz + H2 * fdr * dz;
        u[3] += rc * (fy * dz - fz * dy);
        u[4] += rc * (fz * dx - fx * dz);
        u[5] += rc * (fx * dy - fy * dx);
    } break;
    case UK_STOKES_DOUBLETRACTION: { /* StokesDoubleLayerKernel.hpp:220-275; 2/3 truncated as there */
        double r2 = dx * dx + dy * dy + dz * dz;
        double rinv = rsqrt_mask(r2);
        double rinv2 = rinv * rinv;
        double rinv3 = rinv * rinv2;
        double rinv5 = rinv3 * rinv2;
        double rinv7 = rinv5 * rinv2;
        const double sxx = f[0], sxy = f[1], sxz = f[2], syx = f[3], syy = f[4], syz = f[5];
        const double szx = f[6], szy = f[7], szz = f[8];
        double cc = sxx * dx * dx + syy * dy * dy + szz * dz * dz;
        cc += (sxy + syx) * dx * dy;
        cc += (sxz + szx) * dx * dz;
        cc += (syz + szy) * dy * dz;
        double ccn3 = -3.0 * cc;
        double trace = sxx + syy + szz;
        double e0 = -2.0 * dx * sxx - dy * (sxy + syx) - dz * (sxz + szx);
        double e1 = -2.0 * dy * syy - dx * (sxy + syx) - dz * (syz + szy);
        double e2 = -2.0 * dz * szz - dx * (sxz + szx) - dy * (syz + szy);
        double np = r2 * 0.66666666666666 * rinv7 * (ccn3 + r2 * trace);
        const double d[3] = {dx, dy, dz}, e[3] = {e0, e1, e2};
        double tv[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                tv[3 * i + j] = (-5.0 * cc * d[i] * d[j] - r2 * d[i] * e[j] + (i == j ? r2 * cc : 0.0)) * rinv7;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) u[3 * i + j] += (i == j ? np : 0.0) + tv[3 * i + j] + tv[3 * j + i];
    } break;
    default:
        break;
    }
}

/* Public single-pair entry (unscaled, accumulating), used by the tests. */
void oracle_uk_pair(int uk, const double *r, const double *f, double *u) { uk_pair(uk, r, f, u); }

static int clamp_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads < 1 || nthreads > omp_get_max_threads()) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    return nthreads;
}

/* Dense direct sum, trg_val += scale * sum_s K(x_t - x_s) f_s.
 * Follows FMMData::evaluateKernel (Lib/src/FMMData.cpp:252-283): raw (unscaled)
 * coordinates, accumulate into the caller's output, targets split across threads. */
int oracle_direct(int uk, int nsrc, const double *src_xyz, const double *src_val, int ntrg,
                  const double *trg_xyz, double *trg_val, int nthreads) {
    if (!uk_valid(uk) || nsrc < 0 || ntrg < 0) return 1;
    const int sd = uk_sdim[uk], td = uk_tdim[uk];
    const double sc = oracle_uk_scale(uk);
    nthreads = clamp_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
    for (int t = 0; t < ntrg; t++) {
        double acc[16] = {0};
        const double *xt = trg_xyz + 3 * (size_t)t;
        for (int s = 0; s < nsrc; s++) {
            const double *xs = src_xyz + 3 * (size_t)s;
            double r[3] = {xt[0] - xs[0], xt[1] - xs[1], xt[2] - xs[2]};
            uk_pair(uk, r, src_val + (size_t)sd * s, acc);
        }
        for (int k = 0; k < td; k++) trg_val[(size_t)td * t + k] += sc * acc[k];
    }
    return 0;
}

/* Sum over an explicit interaction list.
 *   target box b owns targets [trg_begin[b], trg_end[b]) of trg_xyz / trg_val;
 *   source box s owns sources [src_begin[s], src_end[s]) of src_xyz / src_val;
 *   target box b interacts with entries list_off[b] .. list_off[b+1]-1, each a
 *   source box list_src[e] seen through periodic image shift list_shift[e]
 *   (code = (sx+1) + 3(sy+1) + 9(sz+1), image coordinate x_s + (sx,sy,sz)*period).
 * This is the U-list S2T loop of PVFMM's PtFMM_Evaluate restated over the same
 * lists that the GPU kernels receive. */
int oracle_lists(int uk, int n_trg_box, const int *trg_begin, const int *trg_end, const int *list_off,
                 const int *list_src, const int *list_shift, const int *src_begin, const int *src_end,
                 const double *src_xyz, const double *src_val, const double *trg_xyz, double *trg_val,
                 double period, int nthreads) {
    if (!uk_valid(uk)) return 1;
    const int sd = uk_sdim[uk], td = uk_tdim[uk];
    const double sc = oracle_uk_scale(uk);
    nthreads = clamp_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int b = 0; b < n_trg_box; b++) {
        /* Boxes without list entries contribute nothing and are skipped: in a
         * tree, internal nodes (empty lists) overlap their leaves' target
         * ranges, and touching their targets here would race with the thread
         * that owns the leaf.  Boxes with entries must be disjoint. */
        if (list_off[b] == list_off[b + 1]) continue;
        for (int t = trg_begin[b]; t < trg_end[b]; t++) {
            double acc[16] = {0};
            const double *xt = trg_xyz + 3 * (size_t)t;
            for (int e = list_off[b]; e < list_off[b + 1]; e++) {
                const int sb = list_src[e];
                const int code = list_shift ? list_shift[e] : 13;
                const double sh[3] = {(code % 3 - 1) * period, ((code / 3) % 3 - 1) * period,
                                      (code / 9 - 1) * period};
                for (int s = src_begin[sb]; s < src_end[sb]; s++) {
                    const double *xs = src_xyz + 3 * (size_t)s;
                    double r[3] = {xt[0] - (xs[0] + sh[0]), xt[1] - (xs[1] + sh[1]), xt[2] - (xs[2] + sh[2])};
                    uk_pair(uk, r, src_val + (size_t)sd * s, acc);
                }
            }
            for (int k = 0; k < td; k++) trg_val[(size_t)td * t + k] += sc * acc[k];
        }
    }
    return 0;
}

/* KIFMM cube surface: n = 6(p-1)^2+2 points on the surface of the cube
 * [-1,1]^3, mapped to (u+1)*alpha*r + c with r = 0.5*0.5^depth.
 * Restates stkfmm::surface (Lib/include/STKFMM/stkfmm_helpers.hpp:46-85). */
int oracle_surface(int p, const double *c, double alpha, int depth, double *coord) {
    if (p < 2) return 1;
    const int n = 6 * (p - 1) * (p - 1) + 2;
    int cnt = 0;
    coord[0] = coord[1] = coord[2] = -1.0;
    cnt = 1;
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            coord[3 * cnt + 0] = -1.0;
            coord[3 * cnt + 1] = (2.0 * (i + 1) - p + 1) / (p - 1);
            coord[3 * cnt + 2] = (2.0 * j - p + 1) / (p - 1);
        }
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            coord[3 * cnt + 0] = (2.0 * i - p + 1) / (p - 1);
            coord[3 * cnt + 1] = -1.0;
            coord[3 * cnt + 2] = (2.0 * (j + 1) - p + 1) / (p - 1);
        }
    for (int i = 0; i < p - 1; i++)
        for (int j = 0; j < p - 1; j++, cnt++) {
            coord[3 * cnt + 0] = (2.0 * (i + 1) - p + 1) / (p - 1);
            coord[3 * cnt + 1] = (2.0 * j - p + 1) / (p - 1);
            coord[3 * cnt + 2] = -1.0;
        }
    /* second half is the point reflection of the first half */
    for (int i = 0; i < (n / 2) * 3; i++) coord[3 * cnt + i] = -coord[i];
    const double r = 0.5 * pow(0.5, depth);
    const double b = alpha * r;
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) coord[3 * i + k] = (coord[3 * i + k] + 1.0) * b + c[k];
    return 0;
}

/* Adjoint of the regularized-Stokeslet direct sum (no reference counterpart).
 * Forward: u_t = 1/(8 pi) sum_s G_eps_s(x_t - x_s) f_s with
 *   G_eps(r) = ((|r|^2 + 2 eps^2) I + r r^T) / (|r|^2 + eps^2)^{3/2}.
 * For loss L = sum_t w_t . u_t:
 *   dL/df_s = 1/(8 pi) sum_t G_eps_s(x_t - x_s) w_t            (G symmetric, even)
 *   dL/dx_s = -1/(8 pi) sum_t grad_r [w_t . G_eps_s(r) f_s] at r = x_t - x_s
 *   grad_r [w.G.f] = (2 r (w.f) + w (f.r) + f (w.r)) / R^3
 *                    - 3 r ((|r|^2 + 2 eps^2)(w.f) + (w.r)(f.r)) / R^5,  R^2 = |r|^2 + eps^2.
 * src_val holds (f, eps) per source; grads are accumulated. */
int oracle_regvel_adjoint(int nsrc, const double *src_xyz, const double *src_val, int ntrg,
                          const double *trg_xyz, const double *trg_w, double *grad_f, double *grad_x,
                          int nthreads) {
    const double sc = 1.0 / (8.0 * PI_);
    nthreads = clamp_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
    for (int s = 0; s < nsrc; s++) {
        const double *xs = src_xyz + 3 * (size_t)s;
        const double *f = src_val + 4 * (size_t)s;
        const double eps2 = f[3] * f[3];
        double gf[3] = {0, 0, 0}, gx[3] = {0, 0, 0};
        for (int t = 0; t < ntrg; t++) {
            const double *xt = trg_xyz + 3 * (size_t)t;
            const double *w = trg_w + 3 * (size_t)t;
            const double r[3] = {xt[0] - xs[0], xt[1] - xs[1], xt[2] - xs[2]};
            const double rr = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
            const double R2 = rr + eps2;
            if (!(R2 > 0.0)) continue;
            const double Rinv = 1.0 / sqrt(R2);
            const double Rinv3 = Rinv * Rinv * Rinv;
            const double Rinv5 = Rinv3 * Rinv * Rinv;
            const double wr = w[0] * r[0] + w[1] * r[1] + w[2] * r[2];
            const double fr = f[0] * r[0] + f[1] * r[1] + f[2] * r[2];
            const double wf = w[0] * f[0] + w[1] * f[1] + w[2] * f[2];
            const double a = rr + 2.0 * eps2;
            for (int k = 0; k < 3; k++) {
                gf[k] += Rinv3 * (a * w[k] + r[k] * wr);
                double g = (2.0 * r[k] * wf + w[k] * fr + f[k] * wr) * Rinv3 -
                           3.0 * r[k] * (a * wf + wr * fr) * Rinv5;
                gx[k] -= g;
            }
        }
        for (int k = 0; k < 3; k++) {
            grad_f[3 * (size_t)s + k] += sc * gf[k];
            grad_x[3 * (size_t)s + k] += sc * gx[k];
        }
    }
    return 0;
}

/* Central finite differences (step h) of L = sum_t w_t . u_t, u the regularized-
 * Stokeslet sum (uk_pair's stokes_regvel, scale 1/8 pi) over a fixed set of
 * (target, source) pairs with sources = targets = the points x, with respect to
 * the position x_i (moved as a source and as a target) and the force f_i of each
 * checked point i.  The pairs that involve point i are given per checked point
 * as its neighbour list nb[nb_off[c] .. nb_off[c+1]) (i included: the pair
 * (i, i) has r = 0 whatever x_i is): those are the only terms of L that x_i or
 * f_i enter, so each difference is taken over them alone, in FP64.  Writes
 * gx[3c + k] = dL/dx_{i,k} and gf[3c + k] = dL/df_{i,k}.
 * val holds (f, eps) per point.  No reference counterpart (test infrastructure). */
static double regvel_local_loss(int i, const double *xi, const double *fi, int nn, const int *nb, const double *x,
                                const double *val, const double *w) {
    double acc = 0.0;
    for (int q = 0; q < nn; q++) {
        const int j = nb[q];
        if (j == i) { /* self pair: r = 0, G_eps(0) f_i = 2 f_i / eps */
            double r0[3] = {0.0, 0.0, 0.0}, u[3] = {0, 0, 0}, fe[4] = {fi[0], fi[1], fi[2], val[4 * (size_t)i + 3]};
            uk_pair(UK_STOKES_REGVEL, r0, fe, u);
            acc += w[3 * (size_t)i] * u[0] + w[3 * (size_t)i + 1] * u[1] + w[3 * (size_t)i + 2] * u[2];
            continue;
        }
        const double *xj = x + 3 * (size_t)j;
        /* i as a source seen at target j */
        double r1[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
        double u1[3] = {0, 0, 0}, fe[4] = {fi[0], fi[1], fi[2], val[4 * (size_t)i + 3]};
        uk_pair(UK_STOKES_REGVEL, r1, fe, u1);
        acc += w[3 * (size_t)j] * u1[0] + w[3 * (size_t)j + 1] * u1[1] + w[3 * (size_t)j + 2] * u1[2];
        /* j as a source seen at target i */
        double r2[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
        double u2[3] = {0, 0, 0};
        uk_pair(UK_STOKES_REGVEL, r2, val + 4 * (size_t)j, u2);
        acc += w[3 * (size_t)i] * u2[0] + w[3 * (size_t)i + 1] * u2[1] + w[3 * (size_t)i + 2] * u2[2];
    }
    return acc / (8.0 * PI_);
}

int oracle_regvel_fd_local(int ncheck, const int *idx, const int *nb_off, const int *nb, const double *x,
                           const double *val, const double *w, double h, double *gx, double *gf, int nthreads) {
    nthreads = clamp_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int c = 0; c < ncheck; c++) {
        const int i = idx[c];
        const int nn = nb_off[c + 1] - nb_off[c];
        const int *lst = nb + nb_off[c];
        for (int k = 0; k < 3; k++) {
            double xp[3] = {x[3 * (size_t)i], x[3 * (size_t)i + 1], x[3 * (size_t)i + 2]};
            double xm[3] = {xp[0], xp[1], xp[2]};
            xp[k] += h;
            xm[k] -= h;
            const double *fi = val + 4 * (size_t)i;
            gx[3 * (size_t)c + k] = (regvel_local_loss(i, xp, fi, nn, lst, x, val, w) -
                                     regvel_local_loss(i, xm, fi, nn, lst, x, val, w)) / (2.0 * h);
            const double *x0 = x + 3 * (size_t)i;
            double fp[3] = {fi[0], fi[1], fi[2]}, fm[3] = {fi[0], fi[1], fi[2]};
            fp[k] += h;
            fm[k] -= h;
            gf[3 * (size_t)c + k] = (regvel_local_loss(i, x0, fp, nn, lst, x, val, w) -
                                     regvel_local_loss(i, x0, fm, nn, lst, x, val, w)) / (2.0 * h);
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------
 * Triply periodic sums (unit cell) by Ewald summation.
 *
 * Restates the periodic Green's functions of the reference's M2C generator:
 *   Laplace   M2L/Laplace/Laplace3D3D.cpp:14-84  (freal, frealp, gKernelEwald:
 *             real terms erfc(xi r)/r, wave terms 4 pi cos(k.r) exp(-k^2/4xi^2)/k^2,
 *             self term -2 xi/sqrt(pi), constant -pi/xi^2; all / 4 pi), i.e. the
 *             zero-mean periodic Green's function;
 *   Stokeslet M2L/Stokeslet/Stokes3D3D.cpp:19-68 (AEW, BEW, GkernelEwald: real
 *             tensor A(xi, r), wave tensor B(xi, k) cos(k.r), self -4 xi/sqrt(pi) I,
 *             k = 0 dropped; all / 8 pi).
 * kind 0: q (1 value)  -> potential and gradient (4 outputs);
 * kind 1: f (3 values) -> velocity (3 outputs);
 * kind 2: (f, trD) (4 values) -> stokes_pvel's pressure and velocity (4 outputs):
 *         p = -grad(psi).f / 4 pi, u = G f / 8 pi + grad(psi) trD / 8 pi, with psi the
 *         Laplace sum above and G the Stokeslet sum;
 * kind 3: q (1 value)  -> potential, gradient and Hessian (xx xy xz yy yz zz; 10 outputs)
 *         of the Laplace sum (laplace_pgradgrad's layout).  Real-space Hessian
 *         f'' r r^T / r^2 + f'/r (I - r r^T / r^2) of f = erfc(xi r)/r; a target on a
 *         source gets the Hessian at 0 of the smooth remainder -erf(xi r)/r,
 *         4 xi^3 / (3 sqrt(pi)) I; wave terms -w k k^T cos(k.r).
 * Real-space images |s_i| <= nreal around the minimum-image displacement, wave
 * vectors k = 2 pi m with 0 < max|m_i| <= nwave (structure factors per k).  A
 * target on a source point gets that source's periodic images but not the source
 * itself (the self term).  out is accumulated.
 * ------------------------------------------------------------------------ */
int oracle_ewald(int kind, double xi, int nreal, int nwave, int nsrc, const double *src, const double *val,
                 int ntrg, const double *trg, double *out, int nthreads) {
    if (kind < 0 || kind > 3 || nsrc < 0 || ntrg < 0 || nreal < 0 || nwave < 0 || !(xi > 0)) return 1;
    const int hess = kind == 3;
    if (hess) kind = 0;
    const int sd = kind == 0 ? 1 : kind == 1 ? 3 : 4, td = hess ? 10 : kind == 1 ? 3 : 4;
    /* structure-factor columns: the values, plus f.k for kind 2 */
    const int ns = kind == 2 ? 5 : sd;
    const double sqpi = sqrt(PI_), xi2 = xi * xi;
    const double eps = 1e-13;
    nthreads = clamp_threads(nthreads);
    /* wave vectors and structure factors S_c = sum v cos(k.x), S_s = sum v sin(k.x) */
    const int nm = 2 * nwave + 1, nk = nm * nm * nm;
    double *Sc = (double *)calloc((size_t)nk * ns, sizeof(double));
    double *Ss = (double *)calloc((size_t)nk * ns, sizeof(double));
    if (!Sc || !Ss) {
        free(Sc);
        free(Ss);
        return 2;
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int ik = 0; ik < nk; ik++) {
        const int mx = ik % nm - nwave, my = (ik / nm) % nm - nwave, mz = ik / (nm * nm) - nwave;
        if (mx == 0 && my == 0 && mz == 0) continue;
        const double k[3] = {2 * PI_ * mx, 2 * PI_ * my, 2 * PI_ * mz};
        double c[5] = {0, 0, 0, 0, 0}, sn[5] = {0, 0, 0, 0, 0};
        for (int j = 0; j < nsrc; j++) {
            const double ph = k[0] * src[3 * (size_t)j] + k[1] * src[3 * (size_t)j + 1] + k[2] * src[3 * (size_t)j + 2];
            const double cp = cos(ph), sp = sin(ph);
            const double *v = val + (size_t)sd * j;
            for (int a = 0; a < sd; a++) {
                c[a] += v[a] * cp;
                sn[a] += v[a] * sp;
            }
            if (kind == 2) {
                const double fk = v[0] * k[0] + v[1] * k[1] + v[2] * k[2];
                c[4] += fk * cp;
                sn[4] += fk * sp;
            }
        }
        for (int a = 0; a < ns; a++) {
            Sc[(size_t)ns * ik + a] = c[a];
            Ss[(size_t)ns * ik + a] = sn[a];
        }
    }
    double qsum = 0;
    if (kind == 0)
        for (int j = 0; j < nsrc; j++) qsum += val[j];
#pragma omp parallel for schedule(dynamic, 8) num_threads(nthreads)
    for (int t = 0; t < ntrg; t++) {
        const double *x = trg + 3 * (size_t)t;
        double acc[4] = {0, 0, 0, 0}, H[6] = {0, 0, 0, 0, 0, 0};
        /* real space */
        for (int j = 0; j < nsrc; j++) {
            double d0[3];
            for (int a = 0; a < 3; a++) {
                d0[a] = x[a] - src[3 * (size_t)j + a];
                d0[a] -= floor(d0[a] + 0.5);
            }
            const double *v = val + (size_t)sd * j;
            for (int i = -nreal; i <= nreal; i++)
                for (int jj = -nreal; jj <= nreal; jj++)
                    for (int kk = -nreal; kk <= nreal; kk++) {
                        const double r[3] = {d0[0] + i, d0[1] + jj, d0[2] + kk};
                        const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                        if (rr < eps) {
                            /* the source itself: its self term instead (no gradient) */
                            if (kind == 0) {
                                acc[0] += -2 * xi / sqpi * v[0];
                                if (hess) {
                                    const double h0 = 4 * xi * xi2 / (3 * sqpi) * v[0];
                                    H[0] += h0;
                                    H[3] += h0;
                                    H[5] += h0;
                                }
                            } else if (kind == 1)
                                for (int a = 0; a < 3; a++) acc[a] += -4 * xi / sqpi * v[a];
                            else
                                for (int a = 0; a < 3; a++) acc[1 + a] += -4 * xi / sqpi * v[a];
                            continue;
                        }
                        if (xi * rr > 7.0) continue; /* erfc(7) ~ 4e-23 */
                        const double ex = exp(-xi2 * rr * rr), ec = erfc(xi * rr);
                        const double fp = -(2. * ex * xi) / (sqpi * rr) - ec / (rr * rr);
                        if (kind == 0) {
                            acc[0] += v[0] * ec / rr;
                            for (int a = 0; a < 3; a++) acc[1 + a] += v[0] * fp / rr * r[a];
                            if (hess) {
                                const double fpp = 2 * xi / sqpi * ex * (2 * xi2 + 2 / (rr * rr)) + 2 * ec / (rr * rr * rr);
                                const double hs = v[0] * (fpp - fp / rr) / (rr * rr), hd = v[0] * fp / rr;
                                int q = 0;
                                for (int a = 0; a < 3; a++)
                                    for (int b = a; b < 3; b++) H[q++] += hs * r[a] * r[b] + (a == b ? hd : 0.0);
                            }
                        } else {
                            const double c1 = 2 * (xi * ex / (sqpi * rr * rr) + ec / (2 * rr * rr * rr));
                            const double c2 = 4 * xi / sqpi * ex;
                            const double rf = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
                            if (kind == 1) {
                                for (int a = 0; a < 3; a++) acc[a] += c1 * (rr * rr * v[a] + r[a] * rf) - c2 * v[a];
                            } else {
                                /* accumulated in units of 1 / 4 pi; the velocity rows halve at the end */
                                acc[0] -= fp / rr * rf;
                                for (int a = 0; a < 3; a++)
                                    acc[1 + a] += c1 * (rr * rr * v[a] + r[a] * rf) - c2 * v[a] + fp / rr * r[a] * v[3];
                            }
                        }
                    }
        }
        /* wave space */
        for (int ik = 0; ik < nk; ik++) {
            const int mx = ik % nm - nwave, my = (ik / nm) % nm - nwave, mz = ik / (nm * nm) - nwave;
            if (mx == 0 && my == 0 && mz == 0) continue;
            const double k[3] = {2 * PI_ * mx, 2 * PI_ * my, 2 * PI_ * mz};
            const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            const double ph = k[0] * x[0] + k[1] * x[1] + k[2] * x[2];
            const double cp = cos(ph), sp = sin(ph);
            const double g = exp(-k2 / (4 * xi2));
            if (kind == 0) {
                const double w = 4 * PI_ * g / k2;
                /* sum_j q cos(k.(x - x_j)) and sum_j q sin(k.(x - x_j)) */
                const double C = cp * Sc[ik] + sp * Ss[ik];
                const double Sn = sp * Sc[ik] - cp * Ss[ik];
                acc[0] += w * C;
                for (int a = 0; a < 3; a++) acc[1 + a] -= w * k[a] * Sn;
                if (hess) {
                    int q = 0;
                    for (int a = 0; a < 3; a++)
                        for (int b = a; b < 3; b++) H[q++] -= w * k[a] * k[b] * C;
                }
            } else {
                const double w = 8 * PI_ * (1 + k2 / (4 * xi2)) * g / (k2 * k2);
                const int o = kind == 1 ? 0 : 1;
                double C[3];
                for (int a = 0; a < 3; a++) C[a] = cp * Sc[(size_t)ns * ik + a] + sp * Ss[(size_t)ns * ik + a];
                const double kC = k[0] * C[0] + k[1] * C[1] + k[2] * C[2];
                for (int a = 0; a < 3; a++) acc[o + a] += w * (k2 * C[a] - k[a] * kC);
                if (kind == 2) {
                    const double wl = 4 * PI_ * g / k2;
                    /* sum_j (f_j.k) sin(k.(x - x_j)) and sum_j trD_j sin(k.(x - x_j)) */
                    const double Sfk = sp * Sc[(size_t)ns * ik + 4] - cp * Ss[(size_t)ns * ik + 4];
                    const double St = sp * Sc[(size_t)ns * ik + 3] - cp * Ss[(size_t)ns * ik + 3];
                    acc[0] += wl * Sfk;
                    for (int a = 0; a < 3; a++) acc[1 + a] -= wl * k[a] * St;
                }
            }
        }
        if (kind == 0) {
            acc[0] -= PI_ / xi2 * qsum;
            for (int a = 0; a < 4; a++) out[(size_t)td * t + a] += acc[a] / (4 * PI_);
            if (hess)
                for (int a = 0; a < 6; a++) out[(size_t)td * t + 4 + a] += H[a] / (4 * PI_);
        } else if (kind == 1) {
            for (int a = 0; a < 3; a++) out[(size_t)td * t + a] += acc[a] / (8 * PI_);
        } else {
            out[(size_t)td * t] += acc[0] / (4 * PI_);
            for (int a = 0; a < 3; a++) out[(size_t)td * t + 1 + a] += acc[1 + a] / (8 * PI_);
        }
    }
    free(Sc);
    free(Ss);
    return 0;
}

/* The sums of oracle_ewald kinds 0 / 3 (Laplace) and 1 (Stokes) for many
 * sources, same conventions and formulas, arranged for millions of sources:
 *   real space: pairs closer than rc = 5.3 / xi (erfc(5.3) < 1e-13), found with a
 *     cell list of the unit cell (cells of side >= rc, the 27 around the
 *     target's cell, periodic wrap, minimum image), so rc must stay below 1/3;
 *   wave space: k = 2 pi m with |m| <= nwave (a sphere), half of it (the terms
 *     are even in k: each counted twice), structure factors summed source by
 *     source with per-axis phase recurrences (e^{i 2 pi m x} from m = 1).
 * Test infrastructure: pinned against oracle_ewald in tests/test_oracle.py. */
typedef struct {
    int mx, my, mz;
} KVec;

int oracle_ewald_cells(int kind, double xi, int nwave, int nsrc, const double *src, const double *val, int ntrg,
                       const double *trg, double *out, int nthreads) {
    if (!(kind == 0 || kind == 1 || kind == 3) || nsrc < 0 || ntrg < 0 || nwave < 1 || !(xi > 0)) return 1;
    const double rc = 5.3 / xi;
    int nc = (int)floor(1.0 / rc);
    if (nc < 3) return 3; /* rc >= 1/3: use oracle_ewald */
    const int hess = kind == 3;
    const int lap = kind != 1;
    const int sd = lap ? 1 : 3, td = hess ? 10 : lap ? 4 : 3;
    const double sqpi = sqrt(PI_), xi2 = xi * xi;
    nthreads = clamp_threads(nthreads);
    /* ---- wave vectors: half of the sphere |m| <= nwave ---- */
    const int M = nwave;
    int nk = 0;
    KVec *kv = (KVec *)malloc(sizeof(KVec) * (size_t)(2 * M + 1) * (2 * M + 1) * (2 * M + 1));
    if (!kv) return 2;
    for (int mx = 0; mx <= M; mx++)
        for (int my = -M; my <= M; my++)
            for (int mz = -M; mz <= M; mz++) {
                if (mx * mx + my * my + mz * mz > M * M) continue;
                if (mx == 0 && (my < 0 || (my == 0 && mz <= 0))) continue; /* the other half and k = 0 */
                kv[nk].mx = mx;
                kv[nk].my = my;
                kv[nk].mz = mz;
                nk++;
            }
    /* ---- structure factors S(k) = sum_j v_j e^{-i k.x_j}: per-thread partial sums ---- */
    double *S = (double *)calloc((size_t)nthreads * nk * sd * 2, sizeof(double));
    if (!S) {
        free(kv);
        return 2;
    }
#pragma omp parallel num_threads(nthreads)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double *Sp = S + (size_t)tid * nk * sd * 2;
        double *E = (double *)malloc(sizeof(double) * 3 * (2 * M + 1) * 2);
#pragma omp for schedule(static)
        for (int j = 0; j < nsrc; j++) {
            /* E[a][m + M] = e^{-i 2 pi m x_a}, m = -M .. M */
            for (int a = 0; a < 3; a++) {
                const double ph = 2 * PI_ * src[3 * (size_t)j + a];
                const double c1 = cos(ph), s1 = -sin(ph);
                double *e = E + (size_t)a * (2 * M + 1) * 2;
                e[2 * M] = 1.0;
                e[2 * M + 1] = 0.0;
                double c = 1.0, sn = 0.0;
                for (int m = 1; m <= M; m++) {
                    const double cn = c * c1 - sn * s1, snn = c * s1 + sn * c1;
                    c = cn;
                    sn = snn;
                    e[2 * (M + m)] = c;
                    e[2 * (M + m) + 1] = sn;
                    e[2 * (M - m)] = c;
                    e[2 * (M - m) + 1] = -sn;
                }
            }
            const double *v = val + (size_t)sd * j;
            const double *ex = E, *ey = E + (size_t)(2 * M + 1) * 2, *ez = E + (size_t)2 * (2 * M + 1) * 2;
            for (int q = 0; q < nk; q++) {
                const double *a = ex + 2 * (kv[q].mx + M), *b = ey + 2 * (kv[q].my + M), *cc = ez + 2 * (kv[q].mz + M);
                const double abr = a[0] * b[0] - a[1] * b[1], abi = a[0] * b[1] + a[1] * b[0];
                const double pr = abr * cc[0] - abi * cc[1], pi = abr * cc[1] + abi * cc[0];
                double *o = Sp + (size_t)q * sd * 2;
                for (int t = 0; t < sd; t++) {
                    o[2 * t] += v[t] * pr;
                    o[2 * t + 1] += v[t] * pi;
                }
            }
        }
        free(E);
    }
    for (int th = 1; th < nthreads; th++)
        for (size_t i = 0; i < (size_t)nk * sd * 2; i++) S[i] += S[(size_t)th * nk * sd * 2 + i];
    double qsum = 0;
    if (lap)
        for (int j = 0; j < nsrc; j++) qsum += val[j];
    /* ---- cell list of the sources ---- */
    const double h = 1.0 / nc;
    const int ncell = nc * nc * nc;
    int *cstart = (int *)calloc((size_t)ncell + 1, sizeof(int)), *order = (int *)malloc(sizeof(int) * (size_t)(nsrc > 0 ? nsrc : 1));
    int *cof = (int *)malloc(sizeof(int) * (size_t)(nsrc > 0 ? nsrc : 1));
    if (!cstart || !order || !cof) {
        free(kv);
        free(S);
        free(cstart);
        free(order);
        free(cof);
        return 2;
    }
    for (int j = 0; j < nsrc; j++) {
        int ci[3];
        for (int a = 0; a < 3; a++) {
            double x = src[3 * (size_t)j + a];
            x -= floor(x);
            ci[a] = (int)(x / h);
            if (ci[a] >= nc) ci[a] = nc - 1;
        }
        cof[j] = ci[0] + nc * (ci[1] + nc * ci[2]);
        cstart[cof[j] + 1]++;
    }
    for (int c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
    {
        int *fill = (int *)malloc(sizeof(int) * (size_t)ncell);
        for (int c = 0; c < ncell; c++) fill[c] = cstart[c];
        for (int j = 0; j < nsrc; j++) order[fill[cof[j]]++] = j;
        free(fill);
    }
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int t = 0; t < ntrg; t++) {
        const double *x = trg + 3 * (size_t)t;
        double acc[4] = {0, 0, 0, 0}, H[6] = {0, 0, 0, 0, 0, 0};
        int ci[3];
        for (int a = 0; a < 3; a++) {
            double xx = x[a] - floor(x[a]);
            ci[a] = (int)(xx / h);
            if (ci[a] >= nc) ci[a] = nc - 1;
        }
        /* real space over the 27 cells around the target's */
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int cx = (ci[0] + dx + nc) % nc, cy = (ci[1] + dy + nc) % nc, cz = (ci[2] + dz + nc) % nc;
                    const int c = cx + nc * (cy + nc * cz);
                    for (int e = cstart[c]; e < cstart[c + 1]; e++) {
                        const int j = order[e];
                        double r[3];
                        for (int a = 0; a < 3; a++) {
                            r[a] = x[a] - src[3 * (size_t)j + a];
                            r[a] -= floor(r[a] + 0.5);
                        }
                        const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                        const double *v = val + (size_t)sd * j;
                        if (rr < 1e-13) {
                            if (lap) {
                                acc[0] += -2 * xi / sqpi * v[0];
                                if (hess) {
                                    const double h0 = 4 * xi * xi2 / (3 * sqpi) * v[0];
                                    H[0] += h0;
                                    H[3] += h0;
                                    H[5] += h0;
                                }
                            } else
                                for (int a = 0; a < 3; a++) acc[a] += -4 * xi / sqpi * v[a];
                            continue;
                        }
                        if (rr > rc) continue;
                        const double ex = exp(-xi2 * rr * rr), ec = erfc(xi * rr);
                        const double fp = -(2. * ex * xi) / (sqpi * rr) - ec / (rr * rr);
                        if (lap) {
                            acc[0] += v[0] * ec / rr;
                            for (int a = 0; a < 3; a++) acc[1 + a] += v[0] * fp / rr * r[a];
                            if (hess) {
                                const double fpp = 2 * xi / sqpi * ex * (2 * xi2 + 2 / (rr * rr)) + 2 * ec / (rr * rr * rr);
                                const double hs = v[0] * (fpp - fp / rr) / (rr * rr), hd = v[0] * fp / rr;
                                int q = 0;
                                for (int a = 0; a < 3; a++)
                                    for (int b = a; b < 3; b++) H[q++] += hs * r[a] * r[b] + (a == b ? hd : 0.0);
                            }
                        } else {
                            const double c1 = 2 * (xi * ex / (sqpi * rr * rr) + ec / (2 * rr * rr * rr));
                            const double c2 = 4 * xi / sqpi * ex;
                            const double rf = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
                            for (int a = 0; a < 3; a++) acc[a] += c1 * (rr * rr * v[a] + r[a] * rf) - c2 * v[a];
                        }
                    }
                }
        /* wave space: the half sphere, each term twice */
        double ph[3][2];
        for (int a = 0; a < 3; a++) {
            ph[a][0] = cos(2 * PI_ * x[a]);
            ph[a][1] = sin(2 * PI_ * x[a]);
        }
        for (int q = 0; q < nk; q++) {
            const double k[3] = {2 * PI_ * kv[q].mx, 2 * PI_ * kv[q].my, 2 * PI_ * kv[q].mz};
            const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            const double pk = k[0] * x[0] + k[1] * x[1] + k[2] * x[2];
            const double cp = cos(pk), sp = sin(pk);
            const double g = exp(-k2 / (4 * xi2));
            const double *Sq = S + (size_t)q * sd * 2;
            /* S stores sum v e^{-i k.x_j} = Sc - i Ss with oracle_ewald's Sc, Ss */
            if (lap) {
                const double Sc = Sq[0], Ss = -Sq[1];
                const double w = 2 * 4 * PI_ * g / k2;
                const double C = cp * Sc + sp * Ss, Sn = sp * Sc - cp * Ss;
                acc[0] += w * C;
                for (int a = 0; a < 3; a++) acc[1 + a] -= w * k[a] * Sn;
                if (hess) {
                    int qq = 0;
                    for (int a = 0; a < 3; a++)
                        for (int b = a; b < 3; b++) H[qq++] -= w * k[a] * k[b] * C;
                }
            } else {
                const double w = 2 * 8 * PI_ * (1 + k2 / (4 * xi2)) * g / (k2 * k2);
                double C[3];
                for (int a = 0; a < 3; a++) C[a] = cp * Sq[2 * a] - sp * Sq[2 * a + 1];
                const double kC = k[0] * C[0] + k[1] * C[1] + k[2] * C[2];
                for (int a = 0; a < 3; a++) acc[a] += w * (k2 * C[a] - k[a] * kC);
            }
        }
        (void)ph;
        if (lap) {
            acc[0] -= PI_ / xi2 * qsum;
            for (int a = 0; a < 4; a++) out[(size_t)td * t + a] += acc[a] / (4 * PI_);
            if (hess)
                for (int a = 0; a < 6; a++) out[(size_t)td * t + 4 + a] += H[a] / (4 * PI_);
        } else {
            for (int a = 0; a < 3; a++) out[(size_t)td * t + a] += acc[a] / (8 * PI_);
        }
    }
    free(kv);
    free(S);
    free(cstart);
    free(order);
    free(cof);
    return 0;
}

/* ------------------------------------------------------------------------
 * Doubly periodic sums (period 1 in x and y, z free), per pair, restating the
 * reference's generator: Laplace potential M2L/Laplace/Laplace2D3D.cpp:12-83,
 * Laplace gradient M2L/StokesPVel/StokesPVel2D3D.cpp:167-240, Stokeslet
 * M2L/Stokeslet/Stokes2D3D.cpp:19-168 (xi = 2; 11 x 11 real images and wave
 * vectors, as there).  Values without the 1/(4 pi) or 1/(8 pi) factors.
 * ------------------------------------------------------------------------ */
static const double XI2D = 2.0;
static const int NR2D = 5, NW2D = 5;

/* Potential, gradient and (hess != NULL) Hessian xx xy xz yy yz zz.  The Hessian
 * terms: real space as in oracle_ewald (kind 3); wave terms of
 * pi cos(k.r) g(z) / k with g = e+ + e-, g' = k (e+ - e-) (the two Gaussian
 * terms of the reference's gradient cancel), g'' = k^2 g - 4 xi k / sqrt(pi)
 * exp(-k^2/4xi^2 - xi^2 z^2); the k = 0 term's d2/dz2 = -4 sqrt(pi) xi exp(-xi^2 z^2). */
static void ewald2_laplace_h(const double r0[3], double *pot, double grad[3], double *hess) {
    const double xi = XI2D, z = r0[2], sp = sqrt(PI_);
    double p = 0.0, g[3] = {0, 0, 0}, H[6] = {0, 0, 0, 0, 0, 0};
    for (int a = -NR2D; a <= NR2D; a++)
        for (int b = -NR2D; b <= NR2D; b++) {
            const double r[3] = {r0[0] + a, r0[1] + b, z};
            const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (rr < 1e-13) {
                p += -2 * xi / sp;
                const double h0 = 4 * xi * xi * xi / (3 * sp);
                H[0] += h0;
                H[3] += h0;
                H[5] += h0;
                continue;
            }
            p += erfc(xi * rr) / rr;
            const double fp = -(2. * exp(-rr * rr * xi * xi) * xi) / (sp * rr) - erfc(rr * xi) / (rr * rr);
            for (int k = 0; k < 3; k++) g[k] += fp / rr * r[k];
            if (hess) {
                const double fpp = 2 * xi / sp * exp(-rr * rr * xi * xi) * (2 * xi * xi + 2 / (rr * rr)) +
                                   2 * erfc(xi * rr) / (rr * rr * rr);
                const double hs = (fpp - fp / rr) / (rr * rr), hd = fp / rr;
                int q = 0;
                for (int i = 0; i < 3; i++)
                    for (int j = i; j < 3; j++) H[q++] += hs * r[i] * r[j] + (i == j ? hd : 0.0);
            }
        }
    for (int a = -NW2D; a <= NW2D; a++)
        for (int b = -NW2D; b <= NW2D; b++) {
            if (a == 0 && b == 0) continue;
            const double kx = 2 * PI_ * a, ky = 2 * PI_ * b, k = sqrt(kx * kx + ky * ky);
            const double ph = kx * r0[0] + ky * r0[1];
            const double ep = exp(k * z) * erfc(xi * z + k / (2 * xi));
            const double em = exp(-k * z) * erfc(-xi * z + k / (2 * xi));
            const double gz = k * ep - k * em +
                              (2 * xi / sp) * (exp(-pow(-xi * z + k / (2 * xi), 2) - k * z) -
                                               exp(-pow(xi * z + k / (2 * xi), 2) + k * z));
            p += PI_ * cos(ph) * (ep + em) / k;
            g[0] += -PI_ * sin(ph) * (ep + em) / k * kx;
            g[1] += -PI_ * sin(ph) * (ep + em) / k * ky;
            g[2] += PI_ * cos(ph) * gz / k;
            if (hess) {
                const double gg = ep + em, c = cos(ph), s = sin(ph);
                const double gzz = k * k * gg - 4 * xi * k / sp * exp(-k * k / (4 * xi * xi) - xi * xi * z * z);
                H[0] -= PI_ * c * gg / k * kx * kx;
                H[1] -= PI_ * c * gg / k * kx * ky;
                H[2] -= PI_ * s * gz / k * kx;
                H[3] -= PI_ * c * gg / k * ky * ky;
                H[4] -= PI_ * s * gz / k * ky;
                H[5] += PI_ * c * gzz / k;
            }
        }
    p -= 2 * sp * (exp(-xi * xi * z * z) / xi + sp * z * erf(xi * z));
    g[2] += -2 * PI_ * erf(xi * z);
    H[5] -= 4 * sp * xi * exp(-xi * xi * z * z);
    *pot = p;
    for (int k = 0; k < 3; k++) grad[k] = g[k];
    if (hess)
        for (int k = 0; k < 6; k++) hess[k] = H[k];
}

static void ewald2_laplace(const double r0[3], double *pot, double grad[3]) { ewald2_laplace_h(r0, pot, grad, NULL); }

static void ewald2_stokes(const double r0[3], double G[3][3]) {
    const double xi = XI2D, xi2 = xi * xi, z = r0[2], sp = sqrt(PI_);
    double A[3][3] = {{0}};
    for (int a = -NR2D; a <= NR2D; a++)
        for (int b = -NR2D; b <= NR2D; b++) {
            const double r[3] = {r0[0] + a, r0[1] + b, z};
            const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
            if (rr < 1e-13) {
                for (int i = 0; i < 3; i++) A[i][i] += -4 * xi / sp;
                continue;
            }
            const double e2 = exp(-xi2 * rr * rr);
            const double s1 = 2 * (xi * e2 / (sp * rr * rr) + erfc(xi * rr) / (2 * rr * rr * rr));
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    A[i][j] += s1 * ((i == j) * rr * rr + r[i] * r[j]) - (i == j) * 4 * xi / sp * e2;
        }
    for (int a = -NW2D; a <= NW2D; a++)
        for (int b = -NW2D; b <= NW2D; b++) {
            if (a == 0 && b == 0) continue;
            const double kk[2] = {2 * PI_ * a, 2 * PI_ * b};
            const double k = sqrt(kk[0] * kk[0] + kk[1] * kk[1]);
            const double lam = exp(-k * k / (4 * xi2) - xi2 * z * z);
            const double thp = exp(k * z) * erfc(k / (2 * xi) + xi * z);
            const double thm = exp(-k * z) * erfc(k / (2 * xi) - xi * z);
            const double J00 = sp * lam * xi;
            const double J10 = PI_ * (thp + thm) / (4 * k);
            const double J20 = sp * lam / (4 * k * k * xi) +
                               PI_ * ((thp + thm) / (8 * k * k * k) + (thm - thp) * z / (8 * k * k) -
                                      (thp + thm) / (16 * k * xi2));
            const double J12 = PI_ * (-thp - thm) * k / 4 + sp * lam * xi;
            const double J22 = PI_ * ((thp + thm) * k / (16 * xi2) + (thp + thm) / (8 * k) + (thp - thm) * z / 8) -
                               sp * lam / (4 * xi);
            const double K11 = PI_ * (thm - thp) / 4;
            const double K12 = PI_ * ((thp - thm) / (16 * xi2) + (thm + thp) * z / (8 * k));
            const double ph = kk[0] * r0[0] + kk[1] * r0[1], c = cos(ph), s = sin(ph);
            const double fI = 2 * (J00 / (4 * xi2) + J10);
            const double fR = -2 * (J10 / (4 * xi2) + J20), fZ = -2 * (J12 / (4 * xi2) + J22);
            const double fM = -2 * (K11 / (4 * xi2) + K12);
            for (int i = 0; i < 2; i++)
                for (int j = 0; j < 2; j++) A[i][j] += 4 * c * ((i == j) * fI + fR * kk[i] * kk[j]);
            A[2][2] += 4 * c * (fI + fZ);
            for (int i = 0; i < 2; i++) {
                A[i][2] -= 4 * s * fM * kk[i];
                A[2][i] -= 4 * s * fM * kk[i];
            }
        }
    const double k0 = -4 * (PI_ * z * erf(z * xi) + sp / (2 * xi) * exp(-z * z * xi2));
    A[0][0] += k0;
    A[1][1] += k0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) G[i][j] = A[i][j];
}

/* out += doubly periodic sum, per pair (O(ntrg nsrc)).
 * kind 0: q (1) -> potential, gradient (4); kind 1: f (3) -> velocity (3);
 * kind 2: (f, trD) (4) -> (pressure, velocity) (4) of stokes_pvel;
 * kind 3: q (1) -> potential, gradient, Hessian (10). */
int oracle_ewald2d(int kind, int nsrc, const double *src, const double *val, int ntrg, const double *trg,
                   double *out, int nthreads) {
    if (kind < 0 || kind > 3 || nsrc < 0 || ntrg < 0) return 1;
    const int sd = kind == 0 || kind == 3 ? 1 : kind == 1 ? 3 : 4, td = kind == 3 ? 10 : kind == 1 ? 3 : 4;
    nthreads = clamp_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
    for (int t = 0; t < ntrg; t++) {
        double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int j = 0; j < nsrc; j++) {
            double r[3];
            for (int k = 0; k < 3; k++) r[k] = trg[3 * (size_t)t + k] - src[3 * (size_t)j + k];
            r[0] -= floor(r[0] + 0.5);
            r[1] -= floor(r[1] + 0.5);
            const double *v = val + (size_t)sd * j;
            if (kind == 3) {
                double pot, g[3], h[6];
                ewald2_laplace_h(r, &pot, g, h);
                acc[0] += v[0] * pot / (4 * PI_);
                for (int k = 0; k < 3; k++) acc[1 + k] += v[0] * g[k] / (4 * PI_);
                for (int k = 0; k < 6; k++) acc[4 + k] += v[0] * h[k] / (4 * PI_);
            }
            if (kind == 0 || kind == 2) {
                double pot, g[3];
                ewald2_laplace(r, &pot, g);
                if (kind == 0) {
                    acc[0] += v[0] * pot / (4 * PI_);
                    for (int k = 0; k < 3; k++) acc[1 + k] += v[0] * g[k] / (4 * PI_);
                } else {
                    /* p = -grad(psi) . f / 4pi, u += grad(psi) trD / 8pi */
                    acc[0] -= (g[0] * v[0] + g[1] * v[1] + g[2] * v[2]) / (4 * PI_);
                    for (int k = 0; k < 3; k++) acc[1 + k] += g[k] * v[3] / (8 * PI_);
                }
            }
            if (kind == 1 || kind == 2) {
                double G[3][3];
                ewald2_stokes(r, G);
                const int o = kind == 1 ? 0 : 1;
                for (int a = 0; a < 3; a++)
                    acc[o + a] += (G[a][0] * v[0] + G[a][1] * v[1] + G[a][2] * v[2]) / (8 * PI_);
            }
        }
        for (int k = 0; k < td; k++) out[(size_t)td * t + k] += acc[k];
    }
    return 0;
}
