// stk_ukernels.cuh -- STKFMM pair micro-kernels as sm_100a device functions.
//
// Each struct restates one STKFMM "uKerEval" body: the contribution of one
// source to one target, r = x_trg - x_src, unscaled, accumulated.  The bodies are
// written once for a value type V and instantiated twice:
//   V = double : the plain FP64 path (one source, one target);
//   V = F2     : the mixed path, Blackwell packed FP32 (fma.rn.f32x2 & co.),
//                two sources against one target per instruction.
// The algebra is regrouped to use fewer operations than the reference's
// expressions (e.g. u = rinv (f + r (f.r)/r^2) for the Stokeslet); both
// precision paths share it, and the FP64 path still matches the reference
// bodies to ~1e-15 (checked by the parity tests against the oracle, which
// keeps the reference's own operation order).
//
// Source values are "staged" once per source before the pair loop
// (Uk<ID>::stage): derived per-source quantities (2q, symmetric parts of the
// double-layer tensor, a^2/3, eps^2 ...) are computed there, not per pair.
// Target components may carry a constant factor applied after the sum
// (Uk<ID>::comp_scale), e.g. the pressure's factor 2.
//
// Reference bodies:
//   laplace_p            Lib/include/STKFMM/LaplaceLayerKernel.hpp:41-65
//   laplace_pgrad        Lib/include/STKFMM/LaplaceLayerKernel.hpp:67-96
//   laplace_dipolep      Lib/include/STKFMM/LaplaceLayerKernel.hpp:98-113
//   laplace_dipolepgrad  Lib/include/STKFMM/LaplaceLayerKernel.hpp:115-136
//   stokes_vel           PVFMM (not vendored); Stokeslet pinned by Test/SimpleKernel.cpp:986-1023
//   rpy_u                Lib/include/STKFMM/RPYKernel.hpp:17-45
//   rpy_ulapu            Lib/include/STKFMM/RPYKernel.hpp:52-90
//   stk_ulapu            Lib/include/STKFMM/RPYKernel.hpp:97-129
//   stokes_regvel        Lib/include/STKFMM/StokesRegSingleLayerKernel.hpp:17-41
//   stokes_pvel          Lib/include/STKFMM/StokesSingleLayerKernel.hpp:27-47
//   stokes_doublepvel    Lib/include/STKFMM/StokesDoubleLayerKernel.hpp:25-57
//   laplace_pgradgrad    Lib/include/STKFMM/LaplaceLayerKernel.hpp:138-166
//   laplace_dipolepgradgrad Lib/include/STKFMM/LaplaceLayerKernel.hpp:168-200
//   laplace_quadp        Lib/include/STKFMM/LaplaceLayerKernel.hpp:202-232
//   laplace_quadpgradgrad Lib/include/STKFMM/LaplaceLayerKernel.hpp:234-301
//   stokes_pvelgrad      Lib/include/STKFMM/StokesSingleLayerKernel.hpp:54-111
//   stokes_pvellaplacian Lib/include/STKFMM/StokesSingleLayerKernel.hpp:118-155
//   stokes_traction      Lib/include/STKFMM/StokesSingleLayerKernel.hpp:162-199
//   stokes_doublepvelgrad Lib/include/STKFMM/StokesDoubleLayerKernel.hpp:64-143
//   stokes_doublelaplacian Lib/include/STKFMM/StokesDoubleLayerKernel.hpp:150-206
//   stokes_doubletraction Lib/include/STKFMM/StokesDoubleLayerKernel.hpp:213-276
//   stokes_regftvel      Lib/include/STKFMM/StokesRegSingleLayerKernel.hpp:48-89
//   stokes_regftvelomega Lib/include/STKFMM/StokesRegSingleLayerKernel.hpp:96-151
//   stokes_velomega      Lib/include/STKFMM/StokesRegSingleLayerKernel.hpp:158-203
// Two fused variants (no single reference function) evaluate a single-layer
// and a double-layer source at the same point in one pass:
//   laplace_pgrad + laplace_dipolepgrad, stokes_pvel + stokes_doublepvel.
#pragma once
#include <cuda_runtime.h>

namespace stk {

// ---------------------------------------------------------------------------
// packed FP32 pair (two sources in one register pair).  MASK: whether rsq()
// zeroes coincident pairs; the list kernel evaluates tiles that cannot hold a
// source at a target's position with the unmasked type (F2U), which saves two
// compare-and-select steps per packed rsqrt.
// ---------------------------------------------------------------------------
template <bool MASK> struct F2T {
    float2 v;
};
using F2 = F2T<true>;
using F2U = F2T<false>;
__device__ __forceinline__ F2 splat(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ F2 mk(float a, float b) { return {make_float2(a, b)}; }
template <bool M> __device__ __forceinline__ F2T<M> operator+(F2T<M> a, F2T<M> b) { return {__fadd2_rn(a.v, b.v)}; }
template <bool M> __device__ __forceinline__ F2T<M> operator*(F2T<M> a, F2T<M> b) { return {__fmul2_rn(a.v, b.v)}; }
// a - b as one exactly rounded fma(b, -1, a)
template <bool M> __device__ __forceinline__ F2T<M> operator-(F2T<M> a, F2T<M> b) {
    return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)};
}
template <bool M> __device__ __forceinline__ F2T<M> fmav(F2T<M> a, F2T<M> b, F2T<M> c) {
    return {__ffma2_rn(a.v, b.v, c.v)};
}
__device__ __forceinline__ double fmav(double a, double b, double c) { return fma(a, b, c); }

template <class V> __device__ __forceinline__ V cst(double c);
template <> __device__ __forceinline__ double cst<double>(double c) { return c; }
template <> __device__ __forceinline__ F2 cst<F2>(double c) { return splat((float)c); }
template <> __device__ __forceinline__ F2U cst<F2U>(double c) { return {make_float2((float)c, (float)c)}; }

// masked reciprocal square root: 0 where r2 == 0 (the reference's
// approx_rsqrt<digits>(r2, r2 > 0))
#ifndef STK_RSQ64_NEWTON
// refinement of the hardware approximation: -1 = one third-order step (below),
// n > 0 = n Newton-Raphson steps, 0 = CUDA's rsqrt
#define STK_RSQ64_NEWTON -1
#endif
#if STK_RSQ64_NEWTON < 0
// Hardware approximation (MUFU, rsqrt.approx.ftz.f64; relative error ~1e-6 as
// measured here) refined by one step of the third-order Householder iteration
// for 1/sqrt: with e = 1 - r2 y^2, 1/sqrt(r2) = y (1 - e)^(-1/2) and
// (1 - e)^(-1/2) = 1 + e/2 + 3 e^2/8 + O(e^3), so y <- y + y e (1/2 + 3e/8)
// leaves ~(5/16) e^3 ~ 1e-19 before rounding (5 FP64 operations, against 8 for
// two Newton steps).  r2 below the smallest normal double counts as coincident
// (|r| < 1.5e-154).
__device__ __forceinline__ double rsq(double r2) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r2));
    const double e = fma(-(r2 * y), y, 1.0);
    const double t = e * fma(e, 0.375, 0.5);
    y = fma(y, t, y);
    // r2 >= smallest normal double, read off the high word (an integer compare
    // instead of an FP64 one; r2 is a sum of squares, so never negative)
    return __double2hiint(r2) >= 0x00100000 ? y : 0.0;
}
#elif STK_RSQ64_NEWTON
// Hardware approximation refined by Newton-Raphson steps y <- y + y e / 2 with
// e = 1 - r2 y^2 (quadratic convergence; e from one rounded product and one fma).
__device__ __forceinline__ double rsq(double r2) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r2));
#pragma unroll
    for (int it = 0; it < STK_RSQ64_NEWTON; it++) {
        const double e = fma(-(r2 * y), y, 1.0);
        y = fma(0.5 * y, e, y);
    }
    return r2 >= 2.2250738585072014e-308 ? y : 0.0;
}
#else
__device__ __forceinline__ double rsq(double r2) { return r2 > 0.0 ? rsqrt(r2) : 0.0; }
#endif

// Mixed path: hardware approximate rsqrt (MUFU, one per lane half) plus one
// Newton-Raphson step y <- y (3 - r2 y^2) / 2 in packed FP32.  Masked (F2):
// pairs closer than the smallest normal FP32 r^2 (|r| < 1.1e-19) count as
// coincident.  Unmasked (F2U): only for pairs known to be apart.
template <bool M> __device__ __forceinline__ F2T<M> rsq(F2T<M> r2) {
    float y0, y1;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(r2.v.x));
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y1) : "f"(r2.v.y));
    F2T<M> y{make_float2(y0, y1)};
    const F2T<M> h = r2 * F2T<M>{make_float2(-0.5f, -0.5f)};
    const F2T<M> t = fmav(h, y * y, F2T<M>{make_float2(1.5f, 1.5f)});
    y = y * t;
    if constexpr (M) {
        y.v.x = r2.v.x >= 1.17549435e-38f ? y.v.x : 0.0f;
        y.v.y = r2.v.y >= 1.17549435e-38f ? y.v.y : 0.0f;
    }
    return y;
}

template <class V> __device__ __forceinline__ V norm2(V dx, V dy, V dz) { return fmav(dx, dx, fmav(dy, dy, dz * dz)); }

// micro-kernel ids, identical to enum stk_ukernel in include/stkfmm_b200.h
enum UkId : int {
    UK_LAPLACE_P = 0,
    UK_LAPLACE_PGRAD = 1,
    UK_LAPLACE_DIPOLEP = 2,
    UK_LAPLACE_DIPOLEPGRAD = 3,
    UK_STOKES_VEL = 4,
    UK_RPY_U = 5,
    UK_RPY_ULAPU = 6,
    UK_STK_ULAPU = 7,
    UK_STOKES_REGVEL = 8,
    UK_STOKES_PVEL = 9,
    UK_STOKES_DOUBLEPVEL = 10,
    UK_LAPLACE_SLDL_PGRAD = 11,  // values (q, d0, d1, d2)
    UK_STOKES_SLDL_PVEL = 12,    // values (f0, f1, f2, trD, D00 .. D22)
    UK_REGVEL_ADJ_SRC = 13,      // adjoint of stokes_regvel, source side (see below)
    UK_REGVEL_ADJ_TRG = 14,      // adjoint of stokes_regvel, target positions
    UK_LAPLACE_SLDL_P = 15,      // values (q, d0, d1, d2): laplace_p + laplace_dipolep (S2M / S2L)
    UK_LAPLACE_PGRADGRAD = 16,
    UK_LAPLACE_DIPOLEPGRADGRAD = 17,
    UK_LAPLACE_QUADP = 18,
    UK_LAPLACE_QUADPGRADGRAD = 19,
    UK_STOKES_PVELGRAD = 20,
    UK_STOKES_DOUBLEPVELGRAD = 21,
    UK_STOKES_PVELLAPLACIAN = 22,
    UK_STOKES_DOUBLELAPLACIAN = 23,
    UK_STOKES_TRACTION = 24,
    UK_STOKES_DOUBLETRACTION = 25,
    UK_STOKES_REGFTVEL = 26,       // values (f, t, eps) -> u
    UK_STOKES_REGFTVELOMEGA = 27,  // values (f, t, eps) -> (u, omega)
    UK_STOKES_VELOMEGA = 28,       // values f -> (u, omega)
    UK_COUNT = 29
};

constexpr double kInv4Pi = 0.079577471545947667884441881686257181;  // 1/(4 pi)
constexpr double kInv8Pi = 0.039788735772973833942220940843128591;  // 1/(8 pi)
constexpr double kTracSL = -0.23873241463784300365332564505877155;  // -3/(4 pi), stokes_traction
constexpr double kTracDL = -0.11936620731892150182666282252938578;  // -3/(8 pi), stokes_doubletraction
// the reference's truncated 2/3 of stokes_doubletraction (StokesDoubleLayerKernel.hpp:234)
constexpr double kTwoThirdsTrunc = 0.66666666666666;
// the reference's truncated 1/3 of rpy_u / rpy_ulapu (RPYKernel.hpp:30,66)
constexpr double kRpyThird = 0.3333333333333;

template <int ID> struct Uk;

// laplace_p: u0 += q / r
template <> struct Uk<UK_LAPLACE_P> {
    static constexpr int SDIM = 1, TDIM = 1, NV = 1;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { v[0] = f[0]; }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        u[0] = fmav(v[0], rinv, u[0]);
    }
};

// laplace_pgrad: p = q/r, grad p = -q r / r^3.  staged (q, -q)
template <> struct Uk<UK_LAPLACE_PGRAD> {
    static constexpr int SDIM = 1, TDIM = 4, NV = 2;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = -f[0];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        u[0] = fmav(v[0], rinv, u[0]);
        V w = (v[1] * (rinv * rinv)) * rinv;
        u[1] = fmav(w, dx, u[1]);
        u[2] = fmav(w, dy, u[2]);
        u[3] = fmav(w, dz, u[3]);
    }
};

// laplace_dipolep: p = (d.r) / r^3
template <> struct Uk<UK_LAPLACE_DIPOLEP> {
    static constexpr int SDIM = 3, TDIM = 1, NV = 3;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rdn = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        u[0] = fmav(rdn, (rinv * rinv) * rinv, u[0]);
    }
};

// laplace_dipolepgrad: p = (d.r)/r^3, grad p = (d - 3 (d.r) r / r^2) / r^3
template <> struct Uk<UK_LAPLACE_DIPOLEPGRAD> {
    static constexpr int SDIM = 3, TDIM = 4, NV = 3;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rdn = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        u[0] = fmav(rdn, rinv3, u[0]);
        V nA = (rdn * rinv2) * cst<V>(-3.0);
        u[1] = fmav(fmav(nA, dx, v[0]), rinv3, u[1]);
        u[2] = fmav(fmav(nA, dy, v[1]), rinv3, u[2]);
        u[3] = fmav(fmav(nA, dz, v[2]), rinv3, u[3]);
    }
};

// stokes_vel (Stokeslet): u = (f + r (f.r)/r^2) / r
template <> struct Uk<UK_STOKES_VEL> {
    static constexpr int SDIM = 3, TDIM = 3, NV = 3;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V c = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * (rinv * rinv);
        u[0] = fmav(fmav(c, dx, v[0]), rinv, u[0]);
        u[1] = fmav(fmav(c, dy, v[1]), rinv, u[1]);
        u[2] = fmav(fmav(c, dz, v[2]), rinv, u[2]);
    }
};

// rpy_u: u = f (1/r + a^2/3 / r^3) + r (f.r)/r^2 (1/r - a^2 / r^3).
// staged (f, a^2/3, -a^2) with the reference's truncated 1/3
template <> struct Uk<UK_RPY_U> {
    static constexpr int SDIM = 4, TDIM = 3, NV = 5;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = kRpyThird * f[3] * f[3];
        v[4] = -3.0 * v[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * rinv2;
        V P = fmav(v[3], rinv3, rinv);
        V Q = c * fmav(v[4], rinv3, rinv);
        u[0] = fmav(Q, dx, fmav(v[0], P, u[0]));
        u[1] = fmav(Q, dy, fmav(v[1], P, u[1]));
        u[2] = fmav(Q, dz, fmav(v[2], P, u[2]));
    }
};

// rpy_ulapu: C = (f - 3 r (f.r)/r^2) / r^3, u = (f + r (f.r)/r^2)/r + a^2/3 C,
// lap u = 2 C (the factor 2 applied after the sum).  staged (f, a^2/3)
template <> struct Uk<UK_RPY_ULAPU> {
    static constexpr int SDIM = 4, TDIM = 6, NV = 4;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int k) { return k >= 3 ? 2.0 : 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = kRpyThird * f[3] * f[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * rinv2;
        V nc3 = c * cst<V>(-3.0);
        V Cx = fmav(nc3, dx, v[0]) * rinv3;
        V Cy = fmav(nc3, dy, v[1]) * rinv3;
        V Cz = fmav(nc3, dz, v[2]) * rinv3;
        u[0] = fmav(v[3], Cx, fmav(fmav(c, dx, v[0]), rinv, u[0]));
        u[1] = fmav(v[3], Cy, fmav(fmav(c, dy, v[1]), rinv, u[1]));
        u[2] = fmav(v[3], Cz, fmav(fmav(c, dz, v[2]), rinv, u[2]));
        u[3] = u[3] + Cx;
        u[4] = u[4] + Cy;
        u[5] = u[5] + Cz;
    }
};

// stk_ulapu: u = (f + r (f.r)/r^2)/r, lap u = 2 (f - 3 r (f.r)/r^2)/r^3
template <> struct Uk<UK_STK_ULAPU> {
    static constexpr int SDIM = 3, TDIM = 6, NV = 3;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int k) { return k >= 3 ? 2.0 : 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * rinv2;
        V nc3 = c * cst<V>(-3.0);
        u[0] = fmav(fmav(c, dx, v[0]), rinv, u[0]);
        u[1] = fmav(fmav(c, dy, v[1]), rinv, u[1]);
        u[2] = fmav(fmav(c, dz, v[2]), rinv, u[2]);
        u[3] = fmav(fmav(nc3, dx, v[0]), rinv3, u[3]);
        u[4] = fmav(fmav(nc3, dy, v[1]), rinv3, u[4]);
        u[5] = fmav(fmav(nc3, dz, v[2]), rinv3, u[5]);
    }
};

// stokes_regvel: R^2 = r^2 + eps^2, u = ((R^2 + eps^2) f + r (f.r)) / R^3; the
// self term is kept (mask on R^2).  staged (f, eps^2)
template <> struct Uk<UK_STOKES_REGVEL> {
    static constexpr int SDIM = 4, TDIM = 3, NV = 4;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = f[3] * f[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V R2 = fmav(dx, dx, fmav(dy, dy, fmav(dz, dz, v[3])));
        V rinv = rsq(R2);
        V rinv3 = (rinv * rinv) * rinv;
        V al = (R2 + v[3]) * rinv3;
        V be = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * rinv3;
        u[0] = fmav(be, dx, fmav(al, v[0], u[0]));
        u[1] = fmav(be, dy, fmav(al, v[1], u[1]));
        u[2] = fmav(be, dz, fmav(al, v[2], u[2]));
    }
};

// stokes_pvel: p = 2 (f.r)/r^3 (factor 2 after the sum),
// u = f / r + r ((f.r) - trD) / r^3.  values (f, trD)
template <> struct Uk<UK_STOKES_PVEL> {
    static constexpr int SDIM = 4, TDIM = 4, NV = 4;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int k) { return k == 0 ? 2.0 : 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = f[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv3 = (rinv * rinv) * rinv;
        V fdr = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        u[0] = fmav(fdr, rinv3, u[0]);
        V c = (fdr - v[3]) * rinv3;
        u[1] = fmav(c, dx, fmav(v[0], rinv, u[1]));
        u[2] = fmav(c, dy, fmav(v[1], rinv, u[2]));
        u[3] = fmav(c, dz, fmav(v[2], rinv, u[3]));
    }
};

// stokes_doublepvel: m = r^T D r / r^2, p = 2 (tr D - 3 m) / r^3 (factor 2
// after the sum), u = -3 m r / r^3.  staged symmetric parts
// (D00, D11, D22, D01+D10, D02+D20, D12+D21, tr D)
template <> struct Uk<UK_STOKES_DOUBLEPVEL> {
    static constexpr int SDIM = 9, TDIM = 4, NV = 7;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int k) { return k == 0 ? 2.0 : 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[4];
        v[2] = f[8];
        v[3] = f[1] + f[3];
        v[4] = f[2] + f[6];
        v[5] = f[5] + f[7];
        v[6] = f[0] + f[4] + f[8];
    }
    template <class V> static __device__ __forceinline__ V rdr(V dx, V dy, V dz, const V *s) {
        V a = fmav(s[4], dz, fmav(s[3], dy, s[0] * dx));
        V b = fmav(s[5], dz, s[1] * dy);
        return fmav(dx, a, fmav(dy, b, dz * (s[2] * dz)));
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V nm3 = (rdr(dx, dy, dz, v) * rinv2) * cst<V>(-3.0);
        u[0] = fmav(v[6] + nm3, rinv3, u[0]);
        V w = nm3 * rinv3;
        u[1] = fmav(w, dx, u[1]);
        u[2] = fmav(w, dy, u[2]);
        u[3] = fmav(w, dz, u[3]);
    }
};

// laplace_pgrad + laplace_dipolepgrad at one point, values (q, d):
// w = q + (d.r)/r^2, p = w / r, grad p = (d - r (q + 3 (d.r)/r^2)) / r^3.
// staged (q, 2q, d)
template <> struct Uk<UK_LAPLACE_SLDL_PGRAD> {
    static constexpr int SDIM = 4, TDIM = 4, NV = 5;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = 2.0 * f[0];
        v[2] = f[1];
        v[3] = f[2];
        v[4] = f[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rdn = fmav(v[2], dx, fmav(v[3], dy, v[4] * dz));
        V w = fmav(rdn, rinv2, v[0]);
        u[0] = fmav(w, rinv, u[0]);
        V nA = fmav(w, cst<V>(-3.0), v[1]);  // -(q + 3 (d.r)/r^2)
        V rinv3 = rinv2 * rinv;
        u[1] = fmav(fmav(nA, dx, v[2]), rinv3, u[1]);
        u[2] = fmav(fmav(nA, dy, v[3]), rinv3, u[2]);
        u[3] = fmav(fmav(nA, dz, v[4]), rinv3, u[3]);
    }
};

// stokes_pvel + stokes_doublepvel at one point, values (f, trD, D):
// m = r^T D r / r^2, p = 2 ((f.r) + tr D - 3 m) / r^3,
// u = f / r + r ((f.r) - trD - 3 m) / r^3.  staged (f, trD, D symmetric parts, tr D)
template <> struct Uk<UK_STOKES_SLDL_PVEL> {
    static constexpr int SDIM = 13, TDIM = 4, NV = 11;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int k) { return k == 0 ? 2.0 : 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = f[3];
        Uk<UK_STOKES_DOUBLEPVEL>::stage(f + 4, v + 4);
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V fdr = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        V nm3 = (Uk<UK_STOKES_DOUBLEPVEL>::rdr(dx, dy, dz, v + 4) * rinv2) * cst<V>(-3.0);
        V fm = fdr + nm3;
        u[0] = fmav(fm + v[10], rinv3, u[0]);
        V c = (fm - v[3]) * rinv3;
        u[1] = fmav(c, dx, fmav(v[0], rinv, u[1]));
        u[2] = fmav(c, dy, fmav(v[1], rinv, u[2]));
        u[3] = fmav(c, dz, fmav(v[2], rinv, u[3]));
    }
};

// ---------------------------------------------------------------------------
// Adjoint of the regularized Stokeslet sum (no reference counterpart).
// Forward: u_t = 1/(8 pi) sum_s G_{eps_s}(x_t - x_s) f_s with
//   G_eps(r) = ((|r|^2 + 2 eps^2) I + r r^T) / R^3,  R^2 = |r|^2 + eps^2.
// For a loss L = sum_t w_t . u_t, with F(r) = w . G_eps(r) f (F is even in r):
//   dL/df_s   = 1/(8 pi) sum_t G_{eps_s}(x_t - x_s) w_t
//   dL/deps_s = 1/(8 pi) sum_t eps_s (4 (w.f) - 3 m) / R^3,  m = ((|r|^2+2eps^2)(w.f) + (w.r)(f.r)) / R^2
//   dL/dx_s   = 1/(8 pi) sum_t grad F (x_s - x_t)
//   dL/dx_t   = 1/(8 pi) sum_s grad F (x_t - x_s)
//   grad F(d) = (d (2 (w.f) - 3 m) + w (f.d) + f (w.d)) / R^3.
// Both gradient sums are P2P sums over the displacement d = (output point) -
// (input point), so they run on the list kernel with per-output-point values:
// ---------------------------------------------------------------------------

// Source side: output points are the forward sources with per-point values
// (f, eps) (TV = 4, staged as f, eps^2, eps); input points are the forward
// targets with values w.  Outputs (dL/df 3, dL/deps 1, dL/dx_s 3).
template <> struct Uk<UK_REGVEL_ADJ_SRC> {
    static constexpr int SDIM = 3, TDIM = 7, NV = 3, TV = 4, NTV = 5;
    static constexpr double SCALE = kInv8Pi;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
    }
    static __device__ void stage_aux(const double *a, double *t) {
        t[0] = a[0];
        t[1] = a[1];
        t[2] = a[2];
        t[3] = a[3] * a[3];
        t[4] = a[3];
    }
    template <class V>
    static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *w, const V *t) {
        V R2 = fmav(dx, dx, fmav(dy, dy, fmav(dz, dz, t[3])));
        V Rinv = rsq(R2);
        V Rinv2 = Rinv * Rinv;
        V Rinv3 = Rinv2 * Rinv;
        V a = R2 + t[3];  // |d|^2 + 2 eps^2
        V wd = fmav(w[0], dx, fmav(w[1], dy, w[2] * dz));
        V fd = fmav(t[0], dx, fmav(t[1], dy, t[2] * dz));
        V wf = fmav(w[0], t[0], fmav(w[1], t[1], w[2] * t[2]));
        V al = a * Rinv3, be = wd * Rinv3;
        u[0] = fmav(be, dx, fmav(al, w[0], u[0]));
        u[1] = fmav(be, dy, fmav(al, w[1], u[1]));
        u[2] = fmav(be, dz, fmav(al, w[2], u[2]));
        V m = fmav(a, wf, wd * fd) * Rinv2;
        u[3] = fmav(fmav(wf, cst<V>(4.0), m * cst<V>(-3.0)), t[4] * Rinv3, u[3]);
        V c = fmav(m, cst<V>(-3.0), wf + wf);
        u[4] = fmav(fmav(c, dx, fmav(fd, w[0], wd * t[0])), Rinv3, u[4]);
        u[5] = fmav(fmav(c, dy, fmav(fd, w[1], wd * t[1])), Rinv3, u[5]);
        u[6] = fmav(fmav(c, dz, fmav(fd, w[2], wd * t[2])), Rinv3, u[6]);
    }
};

// Target positions: output points are the forward targets with per-point
// values w (TV = 3); input points are the forward sources with values (f, eps)
// (staged f, eps^2).  Output dL/dx_t (3).
template <> struct Uk<UK_REGVEL_ADJ_TRG> {
    static constexpr int SDIM = 4, TDIM = 3, NV = 4, TV = 3, NTV = 3;
    static constexpr double SCALE = kInv8Pi;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = f[3] * f[3];
    }
    static __device__ void stage_aux(const double *a, double *t) {
        t[0] = a[0];
        t[1] = a[1];
        t[2] = a[2];
    }
    template <class V>
    static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *f, const V *w) {
        V R2 = fmav(dx, dx, fmav(dy, dy, fmav(dz, dz, f[3])));
        V Rinv = rsq(R2);
        V Rinv2 = Rinv * Rinv;
        V Rinv3 = Rinv2 * Rinv;
        V a = R2 + f[3];
        V wd = fmav(w[0], dx, fmav(w[1], dy, w[2] * dz));
        V fd = fmav(f[0], dx, fmav(f[1], dy, f[2] * dz));
        V wf = fmav(w[0], f[0], fmav(w[1], f[1], w[2] * f[2]));
        V m = fmav(a, wf, wd * fd) * Rinv2;
        V c = fmav(m, cst<V>(-3.0), wf + wf);
        u[0] = fmav(fmav(c, dx, fmav(fd, w[0], wd * f[0])), Rinv3, u[0]);
        u[1] = fmav(fmav(c, dy, fmav(fd, w[1], wd * f[1])), Rinv3, u[1]);
        u[2] = fmav(fmav(c, dz, fmav(fd, w[2], wd * f[2])), Rinv3, u[2]);
    }
};

// laplace_p + laplace_dipolep at one point (the check potentials of S2M / S2L when
// SL and DL sit at the same points): p = (q + (d.r) / r^2) / r.  staged (q, d)
template <> struct Uk<UK_LAPLACE_SLDL_P> {
    static constexpr int SDIM = 4, TDIM = 1, NV = 4;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = f[1];
        v[2] = f[2];
        v[3] = f[3];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rdn = fmav(v[1], dx, fmav(v[2], dy, v[3] * dz));
        u[0] = fmav(fmav(rdn, rinv * rinv, v[0]), rinv, u[0]);
    }
};

// Second derivatives: outputs (p, grad p, H_xx, H_xy, H_xz, H_yy, H_yz, H_zz).

// laplace_pgradgrad: p = q/r, grad p = -q r / r^3,
// H = q (3 r r^T - r^2 I) / r^5 = 3 q r r^T / r^5 + (grad p / r) I.  staged (q, -q, 3q)
template <> struct Uk<UK_LAPLACE_PGRADGRAD> {
    static constexpr int SDIM = 1, TDIM = 10, NV = 3;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = f[0];
        v[1] = -f[0];
        v[2] = 3.0 * f[0];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        u[0] = fmav(v[0], rinv, u[0]);
        V w = v[1] * rinv3;  // -q / r^3
        u[1] = fmav(w, dx, u[1]);
        u[2] = fmav(w, dy, u[2]);
        u[3] = fmav(w, dz, u[3]);
        V s3 = (v[2] * rinv3) * rinv2;  // 3 q / r^5
        V sx = s3 * dx, sy = s3 * dy;
        u[4] = fmav(sx, dx, u[4] + w);
        u[5] = fmav(sx, dy, u[5]);
        u[6] = fmav(sx, dz, u[6]);
        u[7] = fmav(sy, dy, u[7] + w);
        u[8] = fmav(sy, dz, u[8]);
        u[9] = fmav(s3 * dz, dz, u[9] + w);
    }
};

// laplace_dipolepgradgrad, A = (d.r)/r^2:
//   p = (d.r)/r^3, grad p = (d - 3 A r) / r^3,
//   H_kl = (15 A r_k r_l - 3 (r_k d_l + r_l d_k)) / r^5 - 3 A d_kl / r^3
//        = (r_k h_l + r_l h_k) / r^5 - 3 A d_kl / r^3  with h = 7.5 A r - 3 d.   staged (d, -3d)
template <> struct Uk<UK_LAPLACE_DIPOLEPGRADGRAD> {
    static constexpr int SDIM = 3, TDIM = 10, NV = 6;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        for (int k = 0; k < 3; k++) {
            v[k] = f[k];
            v[3 + k] = -3.0 * f[k];
        }
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V rdn = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        V A = rdn * rinv2;
        u[0] = fmav(rdn, rinv3, u[0]);
        V nA = A * cst<V>(-3.0);
        u[1] = fmav(fmav(nA, dx, v[0]), rinv3, u[1]);
        u[2] = fmav(fmav(nA, dy, v[1]), rinv3, u[2]);
        u[3] = fmav(fmav(nA, dz, v[2]), rinv3, u[3]);
        V c = rinv3 * rinv2;
        V a75 = A * cst<V>(7.5);
        V hx = fmav(a75, dx, v[3]) * c, hy = fmav(a75, dy, v[4]) * c, hz = fmav(a75, dz, v[5]) * c;
        V dg = nA * rinv3;
        u[4] = fmav(dx + dx, hx, u[4] + dg);
        u[5] = fmav(dx, hy, fmav(dy, hx, u[5]));
        u[6] = fmav(dx, hz, fmav(dz, hx, u[6]));
        u[7] = fmav(dy + dy, hy, u[7] + dg);
        u[8] = fmav(dy, hz, fmav(dz, hy, u[8]));
        u[9] = fmav(dz + dz, hz, u[9] + dg);
    }
};

// laplace_quadp: p = (3 r^T S r - r^2 tr S) / r^5 (only the symmetric part of S
// enters).  staged symmetric parts (3 S00, 3 S11, 3 S22, 3 (S01+S10), 3 (S02+S20),
// 3 (S12+S21), -tr S)
template <> struct Uk<UK_LAPLACE_QUADP> {
    static constexpr int SDIM = 9, TDIM = 1, NV = 7;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = 3.0 * f[0];
        v[1] = 3.0 * f[4];
        v[2] = 3.0 * f[8];
        v[3] = 3.0 * (f[1] + f[3]);
        v[4] = 3.0 * (f[2] + f[6]);
        v[5] = 3.0 * (f[5] + f[7]);
        v[6] = -(f[0] + f[4] + f[8]);
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rr3 = Uk<UK_STOKES_DOUBLEPVEL>::rdr(dx, dy, dz, v);  // 3 r^T S r
        u[0] = fmav(fmav(rr3, rinv2, v[6]), rinv2 * rinv, u[0]);
    }
};

// laplace_quadpgradgrad, with P the symmetric part of S, g = P r, m = r^T P r / r^2,
// t = tr S and gamma = 3 t - 15 m (p = S_ij d_i d_j (1/r) and its derivatives):
//   p = (3 m - t) / r^3,  grad p = (gamma r + 6 g) / r^5,
//   H_kl = (r_k h_l + r_l h_k + gamma d_kl + 6 P_kl) / r^5,
//   h = ((52.5 m - 7.5 t) r - 30 g) / r^2.
// staged (6 P00, 6 P11, 6 P22, 6 P01, 6 P02, 6 P12, 3 t, -t)
template <> struct Uk<UK_LAPLACE_QUADPGRADGRAD> {
    static constexpr int SDIM = 9, TDIM = 10, NV = 8;
    static constexpr double SCALE = kInv4Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        v[0] = 6.0 * f[0];
        v[1] = 6.0 * f[4];
        v[2] = 6.0 * f[8];
        v[3] = 3.0 * (f[1] + f[3]);
        v[4] = 3.0 * (f[2] + f[6]);
        v[5] = 3.0 * (f[5] + f[7]);
        const double t = f[0] + f[4] + f[8];
        v[6] = 3.0 * t;
        v[7] = -t;
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c = rinv3 * rinv2;
        // g6 = 6 P r
        V gx = fmav(v[0], dx, fmav(v[3], dy, v[4] * dz));
        V gy = fmav(v[3], dx, fmav(v[1], dy, v[5] * dz));
        V gz = fmav(v[4], dx, fmav(v[5], dy, v[2] * dz));
        V m15 = (fmav(gx, dx, fmav(gy, dy, gz * dz)) * rinv2) * cst<V>(2.5);  // 15 m
        u[0] = fmav(fmav(m15, cst<V>(0.2), v[7]), rinv3, u[0]);
        V gam = v[6] - m15;
        u[1] = fmav(fmav(gam, dx, gx), c, u[1]);
        u[2] = fmav(fmav(gam, dy, gy), c, u[2]);
        u[3] = fmav(fmav(gam, dz, gz), c, u[3]);
        V ah = fmav(m15, cst<V>(3.5), v[6] * cst<V>(-2.5));  // 52.5 m - 7.5 t
        V cr = c * rinv2;
        V hx = fmav(ah, dx, gx * cst<V>(-5.0)) * cr;
        V hy = fmav(ah, dy, gy * cst<V>(-5.0)) * cr;
        V hz = fmav(ah, dz, gz * cst<V>(-5.0)) * cr;
        u[4] = fmav(dx + dx, hx, fmav(gam + v[0], c, u[4]));
        u[5] = fmav(dx, hy, fmav(dy, hx, fmav(v[3], c, u[5])));
        u[6] = fmav(dx, hz, fmav(dz, hx, fmav(v[4], c, u[6])));
        u[7] = fmav(dy + dy, hy, fmav(gam + v[1], c, u[7]));
        u[8] = fmav(dy, hz, fmav(dz, hy, fmav(v[5], c, u[8])));
        u[9] = fmav(dz + dz, hz, fmav(gam + v[2], c, u[9]));
    }
};

// ---------------------------------------------------------------------------
// Stokes pressure / velocity derivatives.  Outputs of the PVelGrad kernels:
// (p, u 3, grad p 3, grad u 9 with u[7 + 3i + j] = d u_i / d x_j); PVelLaplacian:
// (p, u 3, lap u 3); Traction: the 3x3 stress-like tensor, row-major.
// ---------------------------------------------------------------------------

// Single layer, values (f, trD), cc = f.r, c1 = cc - trD:
//   p = 2 cc / r^3, u = f / r + c1 r / r^3, grad p = lap u = 2 f / r^3 - 6 cc r / r^5,
//   d u_i / d x_j = c1 (d_ij r^2 - 3 r_i r_j) / r^5 + (r_i f_j - r_j f_i) / r^3.
// staged (f, trD, 2 f)
struct StokesSLGrad {
    static __device__ void stage(const double *f, double *v) {
        for (int k = 0; k < 4; k++) v[k] = f[k];
        for (int k = 0; k < 3; k++) v[4 + k] = 2.0 * f[k];
    }
    // p, u and grad p (= lap u): outputs 0..6; returns c1
    template <class V, int N>
    static __device__ __forceinline__ V pvel_gradp(V (&u)[N], V dx, V dy, V dz, const V *v, V rinv, V rinv2,
                                                   V rinv3) {
        V cc = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz));
        u[0] = fmav(cc + cc, rinv3, u[0]);
        V c1 = cc - v[3];
        V a = c1 * rinv3;
        u[1] = fmav(a, dx, fmav(v[0], rinv, u[1]));
        u[2] = fmav(a, dy, fmav(v[1], rinv, u[2]));
        u[3] = fmav(a, dz, fmav(v[2], rinv, u[3]));
        V g = (cc * rinv2) * (rinv3 * cst<V>(-6.0));
        u[4] = fmav(g, dx, fmav(v[4], rinv3, u[4]));
        u[5] = fmav(g, dy, fmav(v[5], rinv3, u[5]));
        u[6] = fmav(g, dz, fmav(v[6], rinv3, u[6]));
        return c1;
    }
};

template <> struct Uk<UK_STOKES_PVELGRAD> {
    static constexpr int SDIM = 4, TDIM = 16, NV = 7;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesSLGrad::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c1 = StokesSLGrad::pvel_gradp(u, dx, dy, dz, v, rinv, rinv2, rinv3);
        V a = c1 * rinv3;                             // d_ij part
        V b = (c1 * rinv2) * (rinv3 * cst<V>(-3.0));  // r_i r_j part
        V bx = b * dx, by = b * dy, bz = b * dz;
        V wxy = (dx * v[1] - dy * v[0]) * rinv3;
        V wxz = (dx * v[2] - dz * v[0]) * rinv3;
        V wyz = (dy * v[2] - dz * v[1]) * rinv3;
        V sxy = bx * dy, sxz = bx * dz, syz = by * dz;
        u[7] = u[7] + fmav(bx, dx, a);
        u[8] = u[8] + (sxy + wxy);
        u[9] = u[9] + (sxz + wxz);
        u[10] = u[10] + (sxy - wxy);
        u[11] = u[11] + fmav(by, dy, a);
        u[12] = u[12] + (syz + wyz);
        u[13] = u[13] + (sxz - wxz);
        u[14] = u[14] + (syz - wyz);
        u[15] = u[15] + fmav(bz, dz, a);
    }
};

template <> struct Uk<UK_STOKES_PVELLAPLACIAN> {
    static constexpr int SDIM = 4, TDIM = 7, NV = 7;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesSLGrad::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        (void)StokesSLGrad::pvel_gradp(u, dx, dy, dz, v, rinv, rinv2, rinv3);
    }
};

// stokes_traction (scale -3/(4 pi)): T_ij = (f.r - trD) r_i r_j / r^5 + d_ij trD / (3 r^3).
// staged (f, trD, trD / 3)
template <> struct Uk<UK_STOKES_TRACTION> {
    static constexpr int SDIM = 4, TDIM = 9, NV = 5;
    static constexpr double SCALE = kTracSL;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        for (int k = 0; k < 4; k++) v[k] = f[k];
        v[4] = f[3] * (1.0 / 3.0);
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V c = (fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) - v[3]) * (rinv3 * rinv2);
        V dg = v[4] * rinv3;
        V cx = c * dx, cy = c * dy, cz = c * dz;
        u[0] = u[0] + fmav(cx, dx, dg);
        u[1] = fmav(cx, dy, u[1]);
        u[2] = fmav(cx, dz, u[2]);
        u[3] = fmav(cy, dx, u[3]);
        u[4] = u[4] + fmav(cy, dy, dg);
        u[5] = fmav(cy, dz, u[5]);
        u[6] = fmav(cz, dx, u[6]);
        u[7] = fmav(cz, dy, u[7]);
        u[8] = u[8] + fmav(cz, dz, dg);
    }
};

// Double layer, D row-major, g = (D + D^T) r, C = r^T D r = (r.g)/2, C2 = C / r^2:
//   p = (2 tr - 6 C2) / r^3, u = -3 C2 r / r^3, grad p = lap u = 6 ((5 C2 - tr) r - g) / r^5,
//   d u_i / d x_j = -3 (r_i e_j + C d_ij) / r^5 with e = g - 5 C2 r.
// staged (2 D00, 2 D11, 2 D22, D01 + D10, D02 + D20, D12 + D21, -tr, 2 tr)
struct StokesDLGrad {
    static __device__ void stage(const double *f, double *v) {
        v[0] = 2.0 * f[0];
        v[1] = 2.0 * f[4];
        v[2] = 2.0 * f[8];
        v[3] = f[1] + f[3];
        v[4] = f[2] + f[6];
        v[5] = f[5] + f[7];
        const double tr = f[0] + f[4] + f[8];
        v[6] = -tr;
        v[7] = 2.0 * tr;
    }
    template <class V>
    static __device__ __forceinline__ V gvec(V dx, V dy, V dz, const V *v, V &gx, V &gy, V &gz) {
        gx = fmav(v[0], dx, fmav(v[3], dy, v[4] * dz));
        gy = fmav(v[3], dx, fmav(v[1], dy, v[5] * dz));
        gz = fmav(v[4], dx, fmav(v[5], dy, v[2] * dz));
        return fmav(gx, dx, fmav(gy, dy, gz * dz)) * cst<V>(0.5);  // C
    }
    // p, u and grad p: outputs 0..6
    template <class V, int N>
    static __device__ __forceinline__ void pvel_gradp(V (&u)[N], V dx, V dy, V dz, const V *v, V rinv3, V rinv5,
                                                      V C2, V gx, V gy, V gz) {
        u[0] = fmav(fmav(C2, cst<V>(-6.0), v[7]), rinv3, u[0]);
        V a = (C2 * cst<V>(-3.0)) * rinv3;
        u[1] = fmav(a, dx, u[1]);
        u[2] = fmav(a, dy, u[2]);
        u[3] = fmav(a, dz, u[3]);
        V h = fmav(C2, cst<V>(5.0), v[6]);
        V e6 = rinv5 * cst<V>(6.0);
        u[4] = fmav(e6, h * dx - gx, u[4]);
        u[5] = fmav(e6, h * dy - gy, u[5]);
        u[6] = fmav(e6, h * dz - gz, u[6]);
    }
};

template <> struct Uk<UK_STOKES_DOUBLEPVELGRAD> {
    static constexpr int SDIM = 9, TDIM = 16, NV = 8;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesDLGrad::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V rinv5 = rinv3 * rinv2;
        V gx, gy, gz;
        V C = StokesDLGrad::gvec(dx, dy, dz, v, gx, gy, gz);
        V C2 = C * rinv2;
        StokesDLGrad::pvel_gradp(u, dx, dy, dz, v, rinv3, rinv5, C2, gx, gy, gz);
        V m = C2 * cst<V>(-5.0);
        V s3 = rinv5 * cst<V>(-3.0);
        V ex = fmav(m, dx, gx) * s3, ey = fmav(m, dy, gy) * s3, ez = fmav(m, dz, gz) * s3;
        V dg = C * s3;
        u[7] = u[7] + fmav(dx, ex, dg);
        u[8] = fmav(dx, ey, u[8]);
        u[9] = fmav(dx, ez, u[9]);
        u[10] = fmav(dy, ex, u[10]);
        u[11] = u[11] + fmav(dy, ey, dg);
        u[12] = fmav(dy, ez, u[12]);
        u[13] = fmav(dz, ex, u[13]);
        u[14] = fmav(dz, ey, u[14]);
        u[15] = u[15] + fmav(dz, ez, dg);
    }
};

template <> struct Uk<UK_STOKES_DOUBLELAPLACIAN> {
    static constexpr int SDIM = 9, TDIM = 7, NV = 8;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesDLGrad::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V gx, gy, gz;
        V C = StokesDLGrad::gvec(dx, dy, dz, v, gx, gy, gz);
        StokesDLGrad::pvel_gradp(u, dx, dy, dz, v, rinv3, rinv3 * rinv2, C * rinv2, gx, gy, gz);
    }
};

// stokes_doubletraction (scale -3/(8 pi)):
//   T_ij = np d_ij + (r_i e_j + r_j e_i + 2 C d_ij) / r^5,
//   np = k (tr - 3 C2) / r^3 with the reference's k = 0.66666666666666.
// staged (2 D00, 2 D11, 2 D22, D01 + D10, D02 + D20, D12 + D21, k tr)
template <> struct Uk<UK_STOKES_DOUBLETRACTION> {
    static constexpr int SDIM = 9, TDIM = 9, NV = 7;
    static constexpr double SCALE = kTracDL;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        double w[8];
        StokesDLGrad::stage(f, w);
        for (int k = 0; k < 6; k++) v[k] = w[k];
        v[6] = kTwoThirdsTrunc * (f[0] + f[4] + f[8]);
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv2 = rinv * rinv;
        V rinv3 = rinv2 * rinv;
        V rinv5 = rinv3 * rinv2;
        V gx, gy, gz;
        V C = StokesDLGrad::gvec(dx, dy, dz, v, gx, gy, gz);
        V C2 = C * rinv2;
        V np = fmav(C2, cst<V>(-3.0 * kTwoThirdsTrunc), v[6]) * rinv3;
        V m = C2 * cst<V>(-5.0);
        V ex = fmav(m, dx, gx) * rinv5, ey = fmav(m, dy, gy) * rinv5, ez = fmav(m, dz, gz) * rinv5;
        V dg = fmav(C + C, rinv5, np);
        V txy = fmav(dx, ey, dy * ex), txz = fmav(dx, ez, dz * ex), tyz = fmav(dy, ez, dz * ey);
        u[0] = u[0] + fmav(dx + dx, ex, dg);
        u[1] = u[1] + txy;
        u[2] = u[2] + txz;
        u[3] = u[3] + txy;
        u[4] = u[4] + fmav(dy + dy, ey, dg);
        u[5] = u[5] + tyz;
        u[6] = u[6] + txz;
        u[7] = u[7] + tyz;
        u[8] = u[8] + fmav(dz + dz, ez, dg);
    }
};

// ---------------------------------------------------------------------------
// Regularized force + torque (values f, t, eps; R^2 = r^2 + eps^2, self term kept):
//   u = ((r^2 + 2 eps^2) f + (f.r) r) / R^3 + (r^2 + 2.5 eps^2) (t x r) / R^5,
//   omega = D1 t + D2 (t.r) r + (r^2 + 2.5 eps^2) (f x r) / R^5,
//   D1 = (2.5 eps^4 - 1.75 eps^2 r^2 - 0.5 r^4) / R^7, D2 = (5.25 eps^2 + 1.5 r^2) / R^7.
// Evaluated with q = r / R, a = eps^2 / R^2, b = r^2 / R^2 (all at most 1), so that
// only 1/R, 1/R^2 and 1/R^3 appear: u = ((b + 2a) f + (f.q) q) / R + (b + 2.5a)(t x q) / R^2,
// omega = ((2.5a^2 - 1.75ab - 0.5b^2) t + (5.25a + 1.5b)(t.q) q) / R^3 + (b + 2.5a)(f x q) / R^2
// (the FP32 path would overflow 1/R^5, 1/R^7 for R below ~1e-8 at coincident points).
// staged (f, t, eps^2)
struct StokesRegFT {
    static __device__ void stage(const double *f, double *v) {
        for (int k = 0; k < 6; k++) v[k] = f[k];
        v[6] = f[6] * f[6];
    }
    // velocity (outputs 0..2); returns q, a, b, 1/R^2 and (b + 2.5a) / R^2
    template <class V, int N>
    static __device__ __forceinline__ void vel(V (&u)[N], V dx, V dy, V dz, const V *v, V &qx, V &qy, V &qz, V &a,
                                               V &b, V &rinv, V &rinv2, V &rc) {
        V r2 = norm2(dx, dy, dz);
        rinv = rsq(r2 + v[6]);
        rinv2 = rinv * rinv;
        a = v[6] * rinv2;
        b = r2 * rinv2;
        qx = dx * rinv;
        qy = dy * rinv;
        qz = dz * rinv;
        V h1 = fmav(a, cst<V>(2.0), b) * rinv;
        V h2 = fmav(v[0], qx, fmav(v[1], qy, v[2] * qz)) * rinv;
        rc = fmav(a, cst<V>(2.5), b) * rinv2;
        u[0] = fmav(rc, v[4] * qz - v[5] * qy, fmav(h2, qx, fmav(h1, v[0], u[0])));
        u[1] = fmav(rc, v[5] * qx - v[3] * qz, fmav(h2, qy, fmav(h1, v[1], u[1])));
        u[2] = fmav(rc, v[3] * qy - v[4] * qx, fmav(h2, qz, fmav(h1, v[2], u[2])));
    }
};

template <> struct Uk<UK_STOKES_REGFTVEL> {
    static constexpr int SDIM = 7, TDIM = 3, NV = 7;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesRegFT::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V qx, qy, qz, a, b, rinv, rinv2, rc;
        StokesRegFT::vel(u, dx, dy, dz, v, qx, qy, qz, a, b, rinv, rinv2, rc);
    }
};

template <> struct Uk<UK_STOKES_REGFTVELOMEGA> {
    static constexpr int SDIM = 7, TDIM = 6, NV = 7;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) { StokesRegFT::stage(f, v); }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V qx, qy, qz, a, b, rinv, rinv2, rc;
        StokesRegFT::vel(u, dx, dy, dz, v, qx, qy, qz, a, b, rinv, rinv2, rc);
        V rinv3 = rinv2 * rinv;
        V d1 = fmav(a, fmav(a, cst<V>(2.5), b * cst<V>(-1.75)), (b * b) * cst<V>(-0.5)) * rinv3;
        V td = fmav(v[3], qx, fmav(v[4], qy, v[5] * qz)) * (fmav(a, cst<V>(5.25), b * cst<V>(1.5)) * rinv3);
        u[3] = fmav(rc, v[1] * qz - v[2] * qy, fmav(td, qx, fmav(d1, v[3], u[3])));
        u[4] = fmav(rc, v[2] * qx - v[0] * qz, fmav(td, qy, fmav(d1, v[4], u[4])));
        u[5] = fmav(rc, v[0] * qy - v[1] * qx, fmav(td, qz, fmav(d1, v[5], u[5])));
    }
};

// stokes_velomega: u = f / r + (f.r) r / r^3, omega = (f x r) / r^3 (masked at r = 0)
template <> struct Uk<UK_STOKES_VELOMEGA> {
    static constexpr int SDIM = 3, TDIM = 6, NV = 3;
    static constexpr double SCALE = kInv8Pi;
    static constexpr int TV = 0;
    static __host__ __device__ constexpr double comp_scale(int) { return 1.0; }
    static __device__ void stage(const double *f, double *v) {
        for (int k = 0; k < 3; k++) v[k] = f[k];
    }
    template <class V> static __device__ __forceinline__ void eval(V (&u)[TDIM], V dx, V dy, V dz, const V *v) {
        V rinv = rsq(norm2(dx, dy, dz));
        V rinv3 = (rinv * rinv) * rinv;
        V h2 = fmav(v[0], dx, fmav(v[1], dy, v[2] * dz)) * rinv3;
        u[0] = fmav(h2, dx, fmav(v[0], rinv, u[0]));
        u[1] = fmav(h2, dy, fmav(v[1], rinv, u[1]));
        u[2] = fmav(h2, dz, fmav(v[2], rinv, u[2]));
        u[3] = fmav(rinv3, v[1] * dz - v[2] * dy, u[3]);
        u[4] = fmav(rinv3, v[2] * dx - v[0] * dz, u[4]);
        u[5] = fmav(rinv3, v[0] * dy - v[1] * dx, u[5]);
    }
};

// Host/device tables for launch-time checks.
__host__ __device__ constexpr int uk_sdim(int id) {
    return id == UK_LAPLACE_P ? 1 : id == UK_LAPLACE_PGRAD ? 1 : id == UK_LAPLACE_DIPOLEP ? 3
         : id == UK_LAPLACE_DIPOLEPGRAD ? 3 : id == UK_STOKES_VEL ? 3 : id == UK_RPY_U ? 4
         : id == UK_RPY_ULAPU ? 4 : id == UK_STK_ULAPU ? 3 : id == UK_STOKES_REGVEL ? 4
         : id == UK_STOKES_PVEL ? 4 : id == UK_STOKES_DOUBLEPVEL ? 9 : id == UK_LAPLACE_SLDL_PGRAD ? 4
         : id == UK_STOKES_SLDL_PVEL ? 13 : id == UK_REGVEL_ADJ_SRC ? 3 : id == UK_REGVEL_ADJ_TRG ? 4
         : id == UK_LAPLACE_SLDL_P ? 4 : id == UK_LAPLACE_PGRADGRAD ? 1 : id == UK_LAPLACE_DIPOLEPGRADGRAD ? 3
         : id == UK_LAPLACE_QUADP ? 9 : id == UK_LAPLACE_QUADPGRADGRAD ? 9 : id == UK_STOKES_PVELGRAD ? 4
         : id == UK_STOKES_DOUBLEPVELGRAD ? 9 : id == UK_STOKES_PVELLAPLACIAN ? 4 : id == UK_STOKES_DOUBLELAPLACIAN ? 9
         : id == UK_STOKES_TRACTION ? 4 : id == UK_STOKES_DOUBLETRACTION ? 9 : id == UK_STOKES_REGFTVEL ? 7
         : id == UK_STOKES_REGFTVELOMEGA ? 7 : id == UK_STOKES_VELOMEGA ? 3 : 0;
}
__host__ __device__ constexpr int uk_tdim(int id) {
    return id == UK_LAPLACE_P ? 1 : id == UK_LAPLACE_PGRAD ? 4 : id == UK_LAPLACE_DIPOLEP ? 1
         : id == UK_LAPLACE_DIPOLEPGRAD ? 4 : id == UK_STOKES_VEL ? 3 : id == UK_RPY_U ? 3
         : id == UK_RPY_ULAPU ? 6 : id == UK_STK_ULAPU ? 6 : id == UK_STOKES_REGVEL ? 3
         : id == UK_STOKES_PVEL ? 4 : id == UK_STOKES_DOUBLEPVEL ? 4 : id == UK_LAPLACE_SLDL_PGRAD ? 4
         : id == UK_STOKES_SLDL_PVEL ? 4 : id == UK_REGVEL_ADJ_SRC ? 7 : id == UK_REGVEL_ADJ_TRG ? 3
         : id == UK_LAPLACE_SLDL_P ? 1 : id == UK_LAPLACE_PGRADGRAD ? 10 : id == UK_LAPLACE_DIPOLEPGRADGRAD ? 10
         : id == UK_LAPLACE_QUADP ? 1 : id == UK_LAPLACE_QUADPGRADGRAD ? 10 : id == UK_STOKES_PVELGRAD ? 16
         : id == UK_STOKES_DOUBLEPVELGRAD ? 16 : id == UK_STOKES_PVELLAPLACIAN ? 7 : id == UK_STOKES_DOUBLELAPLACIAN ? 7
         : id == UK_STOKES_TRACTION ? 9 : id == UK_STOKES_DOUBLETRACTION ? 9 : id == UK_STOKES_REGFTVEL ? 3
         : id == UK_STOKES_REGFTVELOMEGA ? 6 : id == UK_STOKES_VELOMEGA ? 6 : 0;
}
// per-output-point (target-side) values a micro-kernel reads
__host__ __device__ constexpr int uk_tvdim(int id) {
    return id == UK_REGVEL_ADJ_SRC ? 4 : id == UK_REGVEL_ADJ_TRG ? 3 : 0;
}
__host__ __device__ constexpr double uk_scale(int id) {
    return id == UK_STOKES_TRACTION ? kTracSL
         : id == UK_STOKES_DOUBLETRACTION ? kTracDL
         : id >= UK_STOKES_PVELGRAD ? kInv8Pi
         : id <= UK_LAPLACE_DIPOLEPGRAD || id == UK_LAPLACE_SLDL_PGRAD || id >= UK_LAPLACE_SLDL_P ? kInv4Pi
                                                                                                : kInv8Pi;
}

}  // namespace stk
