// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own FP64 test kernels (Test/SimpleKernel.cpp of STKFMM,
// compiled from the reference tree by oracle/Makefile, never copied here) over
// all (target, source) pairs, the same protocol as runSimpleKernel in
// Test/Test.cpp:478-510: a zeroed 20-slot result per pair, added into the target.
// The shared library it builds (oracle/_ref/libstk_ref.so) generates the golden
// fixtures under tests/golden/ and is the "reference" CPU baseline of bench.py.
// It also exposes the reference's KIFMM surface generator (stkfmm::surface,
// Lib/include/STKFMM/stkfmm_helpers.hpp:46-85), compiled from the reference's
// header with oracle/stub/pvfmm.hpp standing in for PVFMM's umbrella header.
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "STKFMM/stkfmm_helpers.hpp"
#include "SimpleKernel.hpp"

typedef void (*kernel_func)(double *, double *, double *, double *);

// Selector values (stable, used by oracle/oracle.py):
//   0 StokesSL  1 LaplaceSLPGrad  2 LaplaceDLPGrad  3 StokesSLRPY
//   4 StokesRegSLVel  5 StokesSLPVel  6 StokesDLPVel  7 LaplaceSLPGradGrad
//   8 LaplaceDLPGradGrad  9 LaplaceQPGradGrad  10 StokesSLPVelGrad  11 StokesDLPVelGrad
//   12 StokesSLPVelLaplacian  13 StokesDLPVelLaplacian  14 StokesSLTraction  15 StokesDLTraction
//   16 StokesRegSLVelOmega
static kernel_func pick(int which) {
    switch (which) {
    case 0: return StokesSL;
    case 1: return LaplaceSLPGrad;
    case 2: return LaplaceDLPGrad;
    case 3: return StokesSLRPY;
    case 4: return StokesRegSLVel;
    case 5: return StokesSLPVel;
    case 6: return StokesDLPVel;
    case 7: return LaplaceSLPGradGrad;
    case 8: return LaplaceDLPGradGrad;
    case 9: return LaplaceQPGradGrad;
    case 10: return StokesSLPVelGrad;
    case 11: return StokesDLPVelGrad;
    case 12: return StokesSLPVelLaplacian;
    case 13: return StokesDLPVelLaplacian;
    case 14: return StokesSLTraction;
    case 15: return StokesDLTraction;
    case 16: return StokesRegSLVelOmega;
    default: return nullptr;
    }
}

extern "C" int ref_simple_direct(int which, int nsrc, const double *src, const double *val, int sdim, int ntrg,
                                 const double *trg, double *out, int tdim, int nthreads) {
    kernel_func k = pick(which);
    if (!k || tdim > 20 || sdim > 20) return 1;
#ifdef _OPENMP
    if (nthreads < 1 || nthreads > omp_get_max_threads()) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int i = 0; i < ntrg; i++) {
        double t[3] = {trg[3 * i], trg[3 * i + 1], trg[3 * i + 2]};
        for (int j = 0; j < nsrc; j++) {
            double result[20];
            std::memset(result, 0, sizeof(result));
            double s[3] = {src[3 * j], src[3 * j + 1], src[3 * j + 2]};
            double v[20];
            for (int q = 0; q < sdim; q++) v[q] = val[(size_t)sdim * j + q];
            k(s, t, v, result);
            for (int q = 0; q < tdim; q++) out[(size_t)tdim * i + q] += result[q];
        }
    }
    return 0;
}

// Same protocol over an explicit target-box / source-box list (the list layout
// of oracle_lists in stk_oracle.c), so the reference kernels can be timed on the
// same U-list work as the GPU path.
extern "C" int ref_simple_lists(int which, int n_trg_box, const int *trg_begin, const int *trg_end,
                                const int *list_off, const int *list_src, const int *src_begin,
                                const int *src_end, const double *src, const double *val, int sdim,
                                const double *trg, double *out, int tdim, int nthreads) {
    kernel_func k = pick(which);
    if (!k || tdim > 20 || sdim > 20) return 1;
#ifdef _OPENMP
    if (nthreads < 1 || nthreads > omp_get_max_threads()) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int b = 0; b < n_trg_box; b++) {
        for (int i = trg_begin[b]; i < trg_end[b]; i++) {
            double t[3] = {trg[3 * i], trg[3 * i + 1], trg[3 * i + 2]};
            for (int e = list_off[b]; e < list_off[b + 1]; e++) {
                const int sb = list_src[e];
                for (int j = src_begin[sb]; j < src_end[sb]; j++) {
                    double result[20];
                    std::memset(result, 0, sizeof(result));
                    double s[3] = {src[3 * j], src[3 * j + 1], src[3 * j + 2]};
                    double v[20];
                    for (int q = 0; q < sdim; q++) v[q] = val[(size_t)sdim * j + q];
                    k(s, t, v, result);
                    for (int q = 0; q < tdim; q++) out[(size_t)tdim * i + q] += result[q];
                }
            }
        }
    }
    return 0;
}

// out[3 n] = stkfmm::surface(p, c, alpha, depth), n = 6 (p - 1)^2 + 2.
extern "C" int ref_surface(int p, const double *c, double alpha, int depth, double *out) {
    if (p < 2 || !c || !out) return 1;
    double cc[3] = {c[0], c[1], c[2]};
    const std::vector<double> v = stkfmm::surface<double>(p, cc, alpha, depth);
    std::memcpy(out, v.data(), v.size() * sizeof(double));
    return 0;
}
