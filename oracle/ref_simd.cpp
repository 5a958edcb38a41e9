// ref_simd.cpp -- TEST INFRASTRUCTURE ONLY (the timed CPU baseline of bench.py).
//
// The reference's production pair loop on the host CPU: STKFMM's own micro-kernel
// bodies (the uKerEval of each struct in Lib/include/STKFMM/*Kernel.hpp, compiled
// in place from the reference tree by oracle/Makefile, never copied here), run
// the way PVFMM's GenericKernel drives them: target points in the lanes of a
// SIMD vector, one source broadcast at a time, the body accumulating into
// per-lane sums, the kernel's ScaleFactor applied once per target.  Two things
// PVFMM and SCTL supply are stood in for here:
//   * the vector type: VecD, 8 doubles (AVX-512) or 4 (AVX2), on GCC vector
//     extensions, with the comparison giving a lane mask;
//   * sctl::approx_rsqrt<digits>(r2, mask): the hardware reciprocal square-root
//     estimate (rsqrt14 on AVX-512, the single-precision rsqrt on AVX2) refined
//     by Newton-Raphson steps y <- y (3 - r2 y^2) / 2 to full double precision
//     (2 steps from 14 bits, 3 from 12), zero where the mask fails -- the
//     published scheme SCTL's approx_rsqrt follows.
// The list loop is the U-list (S2T) pass over the same CSR target-box / source-box
// lists the GPU path evaluates, OpenMP over target boxes.
#include <cmath>
#include <cstring>
#include <immintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include <pvfmm.hpp>  // the stand-in of oracle/stub (GenericKernel, sctl::const_pi, ...)

#if defined(__AVX512F__)
constexpr int kW = 8;
#elif defined(__AVX2__)
constexpr int kW = 4;
#else
#error "ref_simd.cpp needs AVX2 or AVX-512"
#endif

typedef double vd __attribute__((vector_size(kW * 8)));
typedef long long vm __attribute__((vector_size(kW * 8)));

struct VecD {
    using ScalarType = double;
    vd v;
    VecD() : v(vd{} + 0.0) {}
    VecD(double x) : v(vd{} + x) {}
    explicit VecD(vd x) : v(x) {}
    static VecD Zero() { return VecD(0.0); }
    VecD &operator+=(const VecD &o) {
        v += o.v;
        return *this;
    }
    VecD &operator-=(const VecD &o) {
        v -= o.v;
        return *this;
    }
    VecD &operator*=(const VecD &o) {
        v *= o.v;
        return *this;
    }
};
struct MaskD {
    vm m;
};
inline VecD operator+(const VecD &a, const VecD &b) { return VecD(a.v + b.v); }
inline VecD operator-(const VecD &a, const VecD &b) { return VecD(a.v - b.v); }
inline VecD operator*(const VecD &a, const VecD &b) { return VecD(a.v * b.v); }
inline VecD operator/(const VecD &a, const VecD &b) { return VecD(a.v / b.v); }
inline VecD operator-(const VecD &a) { return VecD(-a.v); }
inline MaskD operator>(const VecD &a, const VecD &b) { return MaskD{a.v > b.v}; }

namespace sctl {
// reciprocal square root: hardware estimate + Newton-Raphson steps to double precision
inline vd rsqrt_estimate(vd r2) {
#if defined(__AVX512F__)
    return (vd)_mm512_rsqrt14_pd((__m512d)r2);
#else
    return (vd)_mm256_cvtps_pd(_mm_rsqrt_ps(_mm256_cvtpd_ps((__m256d)r2)));
#endif
}
template <int digits>
inline VecD approx_rsqrt(const VecD &r2, const MaskD &mask) {
    vd y = rsqrt_estimate(r2.v);
    const vd h = r2.v * 0.5;
#if defined(__AVX512F__)
    constexpr int steps = 2;  // 14 -> 28 -> 56 bits
#else
    constexpr int steps = 3;  // 12 -> 24 -> 48 -> 96 bits
#endif
    for (int s = 0; s < steps; s++) y = y * (1.5 - h * y * y);
    return VecD((vd)((vm)y & mask.m));
}
template <int digits>
inline VecD approx_rsqrt(const VecD &r2) {
    return approx_rsqrt<digits>(r2, MaskD{r2.v == r2.v});
}
}  // namespace sctl

#include "STKFMM/LaplaceLayerKernel.hpp"
#include "STKFMM/RPYKernel.hpp"
#include "STKFMM/StokesDoubleLayerKernel.hpp"
#include "STKFMM/StokesRegSingleLayerKernel.hpp"
#include "STKFMM/StokesSingleLayerKernel.hpp"

namespace {

constexpr double kFar = 1.0e10;  // coordinate of the padding target lanes (results discarded)

// One target box: its targets in blocks of kW lanes against every source of its
// list entries (sources broadcast), as GenericKernel::Eval runs a uKerEval body.
template <class Ker, int SD, int TD>
void eval_box(int t0, int t1, int e0, int e1, const int *list_src, const int *list_shift, const int *src_begin,
              const int *src_end, const double *src, const double *val, const double *trg, double period,
              double *out) {
    const double scale = Ker::template ScaleFactor<double>();
    for (int tb = t0; tb < t1; tb += kW) {
        const int nt = t1 - tb < kW ? t1 - tb : kW;
        VecD tx, ty, tz;
        for (int l = 0; l < kW; l++) {
            tx.v[l] = l < nt ? trg[3 * (size_t)(tb + l) + 0] : kFar;
            ty.v[l] = l < nt ? trg[3 * (size_t)(tb + l) + 1] : kFar;
            tz.v[l] = l < nt ? trg[3 * (size_t)(tb + l) + 2] : kFar;
        }
        VecD u[TD];
        for (int e = e0; e < e1; e++) {
            const int sb = list_src[e];
            const int code = list_shift ? list_shift[e] : 13;
            const double shx = (code % 3 - 1) * period, shy = ((code / 3) % 3 - 1) * period,
                         shz = (code / 9 - 1) * period;
            for (int j = src_begin[sb]; j < src_end[sb]; j++) {
                const VecD r[3] = {tx - VecD(src[3 * (size_t)j] + shx), ty - VecD(src[3 * (size_t)j + 1] + shy),
                                   tz - VecD(src[3 * (size_t)j + 2] + shz)};
                VecD f[SD];
                for (int q = 0; q < SD; q++) f[q] = VecD(val[(size_t)SD * j + q]);
                Ker::template uKerEval<VecD, 16>(u, r, f, nullptr);
            }
        }
        for (int l = 0; l < nt; l++)
            for (int k = 0; k < TD; k++) out[(size_t)TD * (tb + l) + k] += scale * u[k].v[l];
    }
}

typedef void (*box_fn)(int, int, int, int, const int *, const int *, const int *, const int *, const double *,
                       const double *, const double *, double, double *);

// Selector values (stable, used by oracle/oracle.py):
//   0 laplace_pgrad (1 -> 4)   1 laplace_dipolepgrad (3 -> 4)   2 rpy_ulapu (4 -> 6)
//   3 stokes_regvel (4 -> 3)   4 stokes_pvel (4 -> 4)            5 stokes_doublepvel (9 -> 4)
box_fn pick(int which, int &sd, int &td) {
    switch (which) {
    case 0: sd = 1, td = 4; return eval_box<pvfmm::laplace_pgrad, 1, 4>;
    case 1: sd = 3, td = 4; return eval_box<pvfmm::laplace_dipolepgrad, 3, 4>;
    case 2: sd = 4, td = 6; return eval_box<pvfmm::rpy_ulapu, 4, 6>;
    case 3: sd = 4, td = 3; return eval_box<pvfmm::stokes_regvel, 4, 3>;
    case 4: sd = 4, td = 4; return eval_box<pvfmm::stokes_pvel, 4, 4>;
    case 5: sd = 9, td = 4; return eval_box<pvfmm::stokes_doublepvel, 9, 4>;
    default: return nullptr;
    }
}

}  // namespace

extern "C" int ref_simd_width() { return kW; }

// out += the micro-kernel's S2T sum over an explicit list: target box b owns
// targets [trg_begin[b], trg_end[b]), its entries list_off[b] .. list_off[b+1]-1
// name source boxes list_src[e] (records [src_begin, src_end) of src / val) with
// periodic shift codes list_shift[e] (may be null: no shift).  The layout of
// oracle_lists in stk_oracle.c.
extern "C" int ref_simd_lists(int which, int n_trg_box, const int *trg_begin, const int *trg_end,
                              const int *list_off, const int *list_src, const int *list_shift, const int *src_begin,
                              const int *src_end, const double *src, const double *val, const double *trg,
                              double period, double *out, int nthreads) {
    int sd = 0, td = 0;
    box_fn f = pick(which, sd, td);
    if (!f) return 1;
#ifdef _OPENMP
    if (nthreads < 1 || nthreads > omp_get_max_threads()) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(nthreads)
#endif
    for (int b = 0; b < n_trg_box; b++)
        f(trg_begin[b], trg_end[b], list_off[b], list_off[b + 1], list_src, list_shift, src_begin, src_end, src, val,
          trg, period, out);
    return 0;
}

// out += the micro-kernel's direct sum over all sources (FMMData::evaluateKernel's
// loop, targets in chunks over OpenMP threads).
extern "C" int ref_simd_direct(int which, int nsrc, const double *src, const double *val, int ntrg,
                               const double *trg, double *out, int nthreads) {
    int sd = 0, td = 0;
    box_fn f = pick(which, sd, td);
    if (!f) return 1;
    const int one_src[1] = {0};
    const int sb[1] = {0}, se[1] = {nsrc};
    const int chunk = 64;
    const int nchunk = (ntrg + chunk - 1) / chunk;
#ifdef _OPENMP
    if (nthreads < 1 || nthreads > omp_get_max_threads()) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int c = 0; c < nchunk; c++) {
        const int t0 = c * chunk, t1 = t0 + chunk < ntrg ? t0 + chunk : ntrg;
        f(t0, t1, 0, 1, one_src, nullptr, sb, se, src, val, trg, 1.0, out);
    }
    return 0;
}
