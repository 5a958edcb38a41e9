// stk_ukernels.cuh -- STKFMM pair micro-kernels as sm_100a device functions.
//
// Each struct restates one STKFMM "uKerEval" body (one (target, source) pair,
// unscaled, accumulated) for a real type R (double for the FP64 path, float for
// the mixed path).  r = x_trg - x_src.  The self-interaction mask of the
// reference (approx_rsqrt<digits>(r2, r2 > 0)) becomes a select on r2 > 0.
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
// Two fused variants (no reference counterpart as one function) evaluate a
// single-layer and a double-layer source that sit at the same point in one pass,
// sharing r^2 and 1/r:  laplace_pgrad + laplace_dipolepgrad, and
// stokes_pvel + stokes_doublepvel.
#pragma once
#include <cuda_runtime.h>

namespace stk {

// ---- masked reciprocal square root -----------------------------------------
template <class R> struct RSqrt;

template <> struct RSqrt<double> {
    // FP64 path: CUDA's double-precision rsqrt, masked at r2 == 0.
    static __device__ __forceinline__ double eval(double r2) { return r2 > 0.0 ? rsqrt(r2) : 0.0; }
};

template <> struct RSqrt<float> {
    // Mixed path: hardware approximate rsqrt (MUFU) plus one Newton-Raphson step
    // y <- y (3 - r2 y^2) / 2, masked at r2 == 0 (select, so inf never leaks).
    static __device__ __forceinline__ float eval(float r2) {
        float y;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(r2));
        float h = r2 * y;
        y = y * fmaf(-0.5f * h, y, 1.5f);
        return r2 > 0.0f ? y : 0.0f;
    }
};

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
    UK_LAPLACE_SLDL_PGRAD = 11,  // fused laplace_pgrad (q) + laplace_dipolepgrad (d), values (q, d)
    UK_STOKES_SLDL_PVEL = 12,    // fused stokes_pvel (f, trD) + stokes_doublepvel (D), values (f, trD, D)
    UK_COUNT = 13
};

constexpr double kInv4Pi = 0.079577471545947667884441881686257181;  // 1/(4 pi)
constexpr double kInv8Pi = 0.039788735772973833942220940843128591;  // 1/(8 pi)

template <int ID> struct Uk;

template <> struct Uk<UK_LAPLACE_P> {
    static constexpr int SDIM = 1, TDIM = 1;
    static constexpr double SCALE = kInv4Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        u[0] += f[0] * rinv;
    }
};

template <> struct Uk<UK_LAPLACE_PGRAD> {
    static constexpr int SDIM = 1, TDIM = 4;
    static constexpr double SCALE = kInv4Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R sv = f[0] * rinv * rinv * rinv;
        u[0] += sv * r2;
        u[1] -= sv * dx;
        u[2] -= sv * dy;
        u[3] -= sv * dz;
    }
};

template <> struct Uk<UK_LAPLACE_DIPOLEP> {
    static constexpr int SDIM = 3, TDIM = 1;
    static constexpr double SCALE = kInv4Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R rdotn = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += rinv3 * rdotn;
    }
};

template <> struct Uk<UK_LAPLACE_DIPOLEPGRAD> {
    static constexpr int SDIM = 3, TDIM = 4;
    static constexpr double SCALE = kInv4Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv2 = rinv * rinv;
        R rinv3 = rinv2 * rinv;
        R rinv5 = rinv3 * rinv2;
        R rdotn = f[0] * dx + f[1] * dy + f[2] * dz;
        R three = R(3);
        u[0] += rdotn * rinv3;
        u[1] += (f[0] * r2 - three * rdotn * dx) * rinv5;
        u[2] += (f[1] * r2 - three * rdotn * dy) * rinv5;
        u[3] += (f[2] * r2 - three * rdotn * dz) * rinv5;
    }
};

template <> struct Uk<UK_STOKES_VEL> {
    static constexpr int SDIM = 3, TDIM = 3;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R fdotr_rinv3 = (f[0] * dx + f[1] * dy + f[2] * dz) * rinv3;
        u[0] += f[0] * rinv + dx * fdotr_rinv3;
        u[1] += f[1] * rinv + dy * fdotr_rinv3;
        u[2] += f[2] * rinv + dz * fdotr_rinv3;
    }
};

template <> struct Uk<UK_RPY_U> {
    static constexpr int SDIM = 4, TDIM = 3;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R rinv5 = rinv3 * rinv * rinv;
        R fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        R three_fdotr_rinv5 = R(3) * fdotr * rinv5;
        R a2_over_three = R(0.3333333333333) * f[3] * f[3];  // the reference's truncated 1/3
        u[0] += (r2 * f[0] + dx * fdotr) * rinv3 + a2_over_three * (f[0] * rinv3 - three_fdotr_rinv5 * dx);
        u[1] += (r2 * f[1] + dy * fdotr) * rinv3 + a2_over_three * (f[1] * rinv3 - three_fdotr_rinv5 * dy);
        u[2] += (r2 * f[2] + dz * fdotr) * rinv3 + a2_over_three * (f[2] * rinv3 - three_fdotr_rinv5 * dz);
    }
};

template <> struct Uk<UK_RPY_ULAPU> {
    static constexpr int SDIM = 4, TDIM = 6;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R rinv5 = rinv3 * rinv * rinv;
        R fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        R fdotr_rinv3 = fdotr * rinv3;
        R three_fdotr_rinv5 = R(3) * fdotr * rinv5;
        R a2_over_three = R(0.3333333333333) * f[3] * f[3];
        R cx = f[0] * rinv3 - three_fdotr_rinv5 * dx;
        R cy = f[1] * rinv3 - three_fdotr_rinv5 * dy;
        R cz = f[2] * rinv3 - three_fdotr_rinv5 * dz;
        u[0] += f[0] * rinv + dx * fdotr_rinv3 + a2_over_three * cx;
        u[1] += f[1] * rinv + dy * fdotr_rinv3 + a2_over_three * cy;
        u[2] += f[2] * rinv + dz * fdotr_rinv3 + a2_over_three * cz;
        u[3] += R(2) * cx;
        u[4] += R(2) * cy;
        u[5] += R(2) * cz;
    }
};

template <> struct Uk<UK_STK_ULAPU> {
    static constexpr int SDIM = 3, TDIM = 6;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R rinv5 = rinv3 * rinv * rinv;
        R fdotr = f[0] * dx + f[1] * dy + f[2] * dz;
        R fdotr_rinv3 = fdotr * rinv3;
        R three_fdotr_rinv5 = R(3) * fdotr * rinv5;
        u[0] += f[0] * rinv + dx * fdotr_rinv3;
        u[1] += f[1] * rinv + dy * fdotr_rinv3;
        u[2] += f[2] * rinv + dz * fdotr_rinv3;
        u[3] += R(2) * (f[0] * rinv3 - three_fdotr_rinv5 * dx);
        u[4] += R(2) * (f[1] * rinv3 - three_fdotr_rinv5 * dy);
        u[5] += R(2) * (f[2] * rinv3 - three_fdotr_rinv5 * dz);
    }
};

template <> struct Uk<UK_STOKES_REGVEL> {
    static constexpr int SDIM = 4, TDIM = 3;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R reg2 = f[3] * f[3];
        R r2 = dx * dx + dy * dy + dz * dz + reg2;  // self term kept (mask on r^2 + eps^2)
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R r2reg2 = r2 + reg2;
        R cc = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += rinv3 * (r2reg2 * f[0] + dx * cc);
        u[1] += rinv3 * (r2reg2 * f[1] + dy * cc);
        u[2] += rinv3 * (r2reg2 * f[2] + dz * cc);
    }
};

template <> struct Uk<UK_STOKES_PVEL> {
    static constexpr int SDIM = 4, TDIM = 4;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv3 = rinv * rinv * rinv;
        R cc = f[0] * dx + f[1] * dy + f[2] * dz;
        u[0] += R(2) * cc * rinv3;
        cc -= f[3];
        u[1] += rinv3 * (r2 * f[0] + dx * cc);
        u[2] += rinv3 * (r2 * f[1] + dy * cc);
        u[3] += rinv3 * (r2 * f[2] + dz * cc);
    }
};

template <> struct Uk<UK_STOKES_DOUBLEPVEL> {
    static constexpr int SDIM = 9, TDIM = 4;
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv2 = rinv * rinv;
        R rinv5 = rinv2 * rinv2 * rinv;
        R cc = f[0] * dx * dx + f[4] * dy * dy + f[8] * dz * dz;
        cc += (f[1] + f[3]) * dx * dy;
        cc += (f[2] + f[6]) * dx * dz;
        cc += (f[5] + f[7]) * dy * dz;
        cc *= R(-3) * rinv5;
        R trace = f[0] + f[4] + f[8];
        u[0] += R(2) * (cc + r2 * rinv5 * trace);
        u[1] += dx * cc;
        u[2] += dy * cc;
        u[3] += dz * cc;
    }
};

template <> struct Uk<UK_LAPLACE_SLDL_PGRAD> {
    static constexpr int SDIM = 4, TDIM = 4;  // values (q, dx, dy, dz)
    static constexpr double SCALE = kInv4Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv2 = rinv * rinv;
        R rinv3 = rinv2 * rinv;
        R rinv5 = rinv3 * rinv2;
        R rdotn = f[1] * dx + f[2] * dy + f[3] * dz;
        R qr3 = f[0] * rinv3;
        R c = R(3) * rdotn * rinv5 + qr3;  // single-layer gradient and dipole radial part together
        u[0] += qr3 * r2 + rdotn * rinv3;
        u[1] += f[1] * r2 * rinv5 - c * dx;
        u[2] += f[2] * r2 * rinv5 - c * dy;
        u[3] += f[3] * r2 * rinv5 - c * dz;
    }
};

template <> struct Uk<UK_STOKES_SLDL_PVEL> {
    static constexpr int SDIM = 13, TDIM = 4;  // values (fx, fy, fz, trD, D00..D22)
    static constexpr double SCALE = kInv8Pi;
    template <class R>
    static __device__ __forceinline__ void eval(R (&u)[TDIM], R dx, R dy, R dz, const R *f) {
        R r2 = dx * dx + dy * dy + dz * dz;
        R rinv = RSqrt<R>::eval(r2);
        R rinv2 = rinv * rinv;
        R rinv3 = rinv2 * rinv;
        R rinv5 = rinv3 * rinv2;
        const R *D = f + 4;
        R cc = f[0] * dx + f[1] * dy + f[2] * dz;
        R dd = D[0] * dx * dx + D[4] * dy * dy + D[8] * dz * dz;
        dd += (D[1] + D[3]) * dx * dy;
        dd += (D[2] + D[6]) * dx * dz;
        dd += (D[5] + D[7]) * dy * dz;
        dd *= R(-3) * rinv5;
        R trace = D[0] + D[4] + D[8];
        u[0] += R(2) * (cc * rinv3 + dd + r2 * rinv5 * trace);
        R c2 = (cc - f[3]) * rinv3 + dd;
        R r2rinv3 = r2 * rinv3;
        u[1] += r2rinv3 * f[0] + dx * c2;
        u[2] += r2rinv3 * f[1] + dy * c2;
        u[3] += r2rinv3 * f[2] + dz * c2;
    }
};

// Host/device table of dimensions, for launch-time checks.
__host__ __device__ constexpr int uk_sdim(int id) {
    return id == UK_LAPLACE_P ? 1 : id == UK_LAPLACE_PGRAD ? 1 : id == UK_LAPLACE_DIPOLEP ? 3
         : id == UK_LAPLACE_DIPOLEPGRAD ? 3 : id == UK_STOKES_VEL ? 3 : id == UK_RPY_U ? 4
         : id == UK_RPY_ULAPU ? 4 : id == UK_STK_ULAPU ? 3 : id == UK_STOKES_REGVEL ? 4
         : id == UK_STOKES_PVEL ? 4 : id == UK_STOKES_DOUBLEPVEL ? 9 : id == UK_LAPLACE_SLDL_PGRAD ? 4
         : id == UK_STOKES_SLDL_PVEL ? 13 : 0;
}
__host__ __device__ constexpr int uk_tdim(int id) {
    return id == UK_LAPLACE_P ? 1 : id == UK_LAPLACE_PGRAD ? 4 : id == UK_LAPLACE_DIPOLEP ? 1
         : id == UK_LAPLACE_DIPOLEPGRAD ? 4 : id == UK_STOKES_VEL ? 3 : id == UK_RPY_U ? 3
         : id == UK_RPY_ULAPU ? 6 : id == UK_STK_ULAPU ? 6 : id == UK_STOKES_REGVEL ? 3
         : id == UK_STOKES_PVEL ? 4 : id == UK_STOKES_DOUBLEPVEL ? 4 : id == UK_LAPLACE_SLDL_PGRAD ? 4
         : id == UK_STOKES_SLDL_PVEL ? 4 : 0;
}
__host__ __device__ constexpr double uk_scale(int id) {
    return id <= UK_LAPLACE_DIPOLEPGRAD || id == UK_LAPLACE_SLDL_PGRAD ? kInv4Pi : kInv8Pi;
}

}  // namespace stk
