// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own FP64 test kernels (Test/SimpleKernel.cpp of STKFMM,
// compiled from the reference tree by oracle/Makefile, never copied here) over
// all (target, source) pairs, the same protocol as runSimpleKernel in
// Test/Test.cpp:478-510: a zeroed 20-slot result per pair, added into the target.
// The shared library it builds (oracle/_ref/libstk_ref.so) generates the golden
// fixtures under tests/golden/ and is the "reference" CPU baseline of bench.py.
// It also exposes, compiled from the reference's headers with
// oracle/stub/pvfmm.hpp standing in for PVFMM's umbrella header:
//   * the KIFMM surface generator (stkfmm::surface, stkfmm_helpers.hpp:46-85);
//   * every micro-kernel body STKFMM defines (the uKerEval of each struct in
//     Lib/include/STKFMM/*Kernel.hpp), run over all pairs by the stub's driver;
//   * the composition of each top-level kernel (which micro-kernel fills which
//     FMM slot, as BuildKernel records it in those headers);
//   * the reference's FMMData (Lib/src/FMMData.cpp, with STKFMM.cpp for its
//     kernel map) around a stub FMM, to read off its source and target scaling;
//   * the reference's Stk3DFMM and StkWallFMM (Stk3DFMM.cpp, StkWallFMM.cpp)
//     over the stand-in FMM in its direct-sum mode: their box scaling, image
//     systems and assembly run as the reference wrote them, exactly.
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "STKFMM/STKFMM.hpp"
#include "STKFMM/STKFMM_impl.hpp"
#include "STKFMM/LaplaceLayerKernel.hpp"
#include "STKFMM/RPYKernel.hpp"
#include "STKFMM/StokesLayerKernel.hpp"
#include "STKFMM/StokesRegSingleLayerKernel.hpp"
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

typedef pvfmm::Kernel<double>::Ker_t ker_t;

namespace pvfmm {
int stub_fmm_direct = 0;  // the stand-in FMM's mode (oracle/stub/pvfmm.hpp)
std::vector<double> stub_root_equiv;
}  // namespace pvfmm

// The reference's micro-kernels by this project's micro-kernel ids (the
// numbering of include/stkfmm_b200.h).  Id 4, PVFMM's stokes_vel, is the stub's
// (its body is not in the reference tree); 11-15 have no reference struct.
static ker_t ukernel_fn(int uk) {
    using namespace pvfmm;
    switch (uk) {
    case 0: return laplace_p::Eval<double>;
    case 1: return laplace_pgrad::Eval<double>;
    case 2: return laplace_dipolep::Eval<double>;
    case 3: return laplace_dipolepgrad::Eval<double>;
    case 4: return stokes_vel::Eval<double>;
    case 5: return rpy_u::Eval<double>;
    case 6: return rpy_ulapu::Eval<double>;
    case 7: return stk_ulapu::Eval<double>;
    case 8: return stokes_regvel::Eval<double>;
    case 9: return stokes_pvel::Eval<double>;
    case 10: return stokes_doublepvel::Eval<double>;
    case 16: return laplace_pgradgrad::Eval<double>;
    case 17: return laplace_dipolepgradgrad::Eval<double>;
    case 18: return laplace_quadp::Eval<double>;
    case 19: return laplace_quadpgradgrad::Eval<double>;
    case 20: return stokes_pvelgrad::Eval<double>;
    case 21: return stokes_doublepvelgrad::Eval<double>;
    case 22: return stokes_pvellaplacian::Eval<double>;
    case 23: return stokes_doublelaplacian::Eval<double>;
    case 24: return stokes_traction::Eval<double>;
    case 25: return stokes_doubletraction::Eval<double>;
    case 26: return stokes_regftvel::Eval<double>;
    case 27: return stokes_regftvelomega::Eval<double>;
    case 28: return stokes_velomega::Eval<double>;
    default: return nullptr;
    }
}

static int ukernel_id(ker_t fn) {
    if (!fn) return -1;
    for (int uk = 0; uk < 29; uk++)
        if (ukernel_fn(uk) == fn) return uk;
    return -9;  // a function this driver does not know
}

// out[ntrg * tdim] += the reference micro-kernel `uk` over all (target, source)
// pairs (ScaleFactor included).  PVFMM's stokes_vel (id 4) is refused.
extern "C" int ref_ukernel_direct(int uk, int nsrc, const double *src, const double *val, int ntrg,
                                  const double *trg, double *out) {
    ker_t fn = uk == 4 ? nullptr : ukernel_fn(uk);
    if (!fn || nsrc < 0 || ntrg < 0) return 1;
    fn(const_cast<double *>(src), nsrc, const_cast<double *>(val), 1, const_cast<double *>(trg), ntrg, out, nullptr);
    return 0;
}

// The reference's map from KERNEL to its composite (Lib/src/STKFMM.cpp:18-31).
static const pvfmm::Kernel<double> *composite(unsigned id) {
    using namespace pvfmm;
    switch (id) {
    case 1: return &LaplaceLayerKernel<double>::PGrad();
    case 2: return &LaplaceLayerKernel<double>::PGradGrad();
    case 4: return &LaplaceLayerKernel<double>::QPGradGrad();
    case 8: return &StokesLayerKernel<double>::Vel();
    case 16: return &RPYKernel<double>::ulapu();
    case 32: return &StokesRegKernel<double>::Vel();
    case 64: return &StokesRegKernel<double>::FTVelOmega();
    case 128: return &StokesLayerKernel<double>::PVel();
    case 256: return &StokesLayerKernel<double>::PVelGrad();
    case 512: return &StokesLayerKernel<double>::PVelLaplacian();
    case 1024: return &StokesLayerKernel<double>::Traction();
    default: return nullptr;
    }
}

// For top-level kernel `id`: slots[9] = micro-kernel ids of (S2T single layer,
// S2T double layer, S2M single, S2M double, M2M, M2T, L2T, S2L single, S2L
// double), -1 where the slot's kernel has no such function, -2 where M2L or
// L2L differ from M2M; dims[3] = (ker_dim[0], surf_dim as the headers set it,
// 0 if they leave PVFMM's default, ker_dim[1]); name = ker_name.
extern "C" int ref_kernel_composition(unsigned id, int *slots, int *dims, char *name, int namelen) {
    const pvfmm::Kernel<double> *k = composite(id);
    if (!k || !slots || !dims) return 1;
    auto self = [k](const pvfmm::Kernel<double> *sub) { return sub ? sub : k; };
    slots[0] = ukernel_id(self(k->k_s2t)->ker_poten);
    slots[1] = ukernel_id(self(k->k_s2t)->dbl_layer_poten);
    slots[2] = ukernel_id(self(k->k_s2m)->ker_poten);
    slots[3] = ukernel_id(self(k->k_s2m)->dbl_layer_poten);
    slots[4] = ukernel_id(self(k->k_m2m)->ker_poten);
    if (ukernel_id(self(k->k_m2l)->ker_poten) != slots[4] || ukernel_id(self(k->k_l2l)->ker_poten) != slots[4])
        slots[4] = -2;
    slots[5] = ukernel_id(self(k->k_m2t)->ker_poten);
    slots[6] = ukernel_id(self(k->k_l2t)->ker_poten);
    slots[7] = ukernel_id(self(k->k_s2l)->ker_poten);
    slots[8] = ukernel_id(self(k->k_s2l)->dbl_layer_poten);
    dims[0] = k->ker_dim[0];
    dims[1] = k->surf_dim;
    dims[2] = k->ker_dim[1];
    if (name && namelen > 0) {
        std::strncpy(name, k->ker_name ? k->ker_name : "", (size_t)namelen - 1);
        name[namelen - 1] = 0;
    }
    return 0;
}

// The factors the reference's FMMData applies around the FMM for a box with
// scale factor sf (FMMData::scaleSrc / scaleTrg, Lib/src/FMMData.cpp:285-470),
// seen through its public evaluateFMM on one point per set: the source values
// (ones) are scaled in place before the stub FMM, which sets every target value
// to 1, so the targets come back as the target factors.  Free space.
// sl[kdimSL], dl[kdimDL] (empty without a double layer), trg[kdimTrg];
// dims = (kdimSL, kdimDL or 0, kdimTrg).
extern "C" int ref_kernel_scaling(unsigned id, double sf, double *sl, double *dl, double *trg, int *dims) {
    using namespace stkfmm;
    if (!composite(id) || !sl || !dl || !trg || !dims) return 1;
    pvfmm::stub_fmm_direct = 0;
    impl::FMMData fmm(static_cast<KERNEL>(id), PAXIS::NONE, 6, 50, true);
    const std::vector<double> pt = {0.5, 0.5, 0.5}, none;
    const bool has_dl = fmm.hasDL();
    fmm.setupTree(pt, has_dl ? pt : none, pt);
    std::vector<double> slv(fmm.kdimSL, 1.0), dlv(has_dl ? fmm.kdimDL : 0, 1.0), tv(fmm.kdimTrg, 0.0);
    fmm.evaluateFMM(slv, dlv, tv, sf);
    std::copy(slv.begin(), slv.end(), sl);
    std::copy(dlv.begin(), dlv.end(), dl);
    std::copy(tv.begin(), tv.end(), trg);
    dims[0] = fmm.kdimSL;
    dims[1] = has_dl ? fmm.kdimDL : 0;
    dims[2] = fmm.kdimTrg;
    return 0;
}

// The reference's own direct sum (FMMData::evaluateKernel, Lib/src/FMMData.cpp:252-283):
// out[ntrg * kdimTrg] += the sub-kernel that p2p (PPKERNEL: 1 SLS2T, 2 DLS2T,
// 4 L2T) selects, over all pairs; out is untouched where the kernel has none.
extern "C" int ref_evaluate_kernel(unsigned id, unsigned p2p, int nsrc, const double *src, const double *val,
                                   int ntrg, const double *trg, double *out) {
    using namespace stkfmm;
    if (!composite(id) || nsrc < 0 || ntrg < 0) return 1;
    impl::FMMData fmm(static_cast<KERNEL>(id), PAXIS::NONE, 6, 50, true);
    fmm.evaluateKernel(1, static_cast<PPKERNEL>(p2p), nsrc, const_cast<double *>(src), const_cast<double *>(val),
                       ntrg, const_cast<double *>(trg), out);
    return 0;
}

// The reference's own StkWallFMM (Lib/src/StkWallFMM.cpp: mirror images, the
// sub-FMMs' source values and the assembly of evalStokes / evalRPY) over the
// stand-in FMM in direct mode: the wall's exact image system in free space.
// kernel 8 (Stokes, f -> u) or 16 (RPY, (f, b) -> (u, lap u)); out += result.
extern "C" int ref_wall_direct(unsigned kernel, const double *origin, double len, int nsrc, const double *src,
                               const double *val, int ntrg, const double *trg, double *out) {
    using namespace stkfmm;
    if ((kernel != 8 && kernel != 16) || nsrc < 1 || ntrg < 1) return 1;
    pvfmm::stub_fmm_direct = 1;
    {
        StkWallFMM wall(6, 50, PAXIS::NONE, kernel, true);
        double o[3] = {origin[0], origin[1], origin[2]};
        wall.setBox(o, len);
        wall.setPoints(nsrc, src, ntrg, trg);
        wall.setupTree(static_cast<KERNEL>(kernel));
        wall.evaluateFMM(static_cast<KERNEL>(kernel), nsrc, val, ntrg, out);
    }
    pvfmm::stub_fmm_direct = 0;
    return 0;
}

// The reference's own Stk3DFMM (Lib/src/Stk3DFMM.cpp, STKFMM.cpp: box scaling,
// wrapping, scaleSrc / scaleTrg) over the stand-in FMM in direct mode, free
// space: out += the kernel's single- and double-layer sums in the caller's box.
extern "C" int ref_stk3d_direct(unsigned kernel, const double *origin, double len, int nsl, const double *sl,
                                const double *slv, int ndl, const double *dl, const double *dlv, int ntrg,
                                const double *trg, double *out) {
    using namespace stkfmm;
    if (!composite(kernel) || nsl < 1 || ntrg < 1) return 1;
    pvfmm::stub_fmm_direct = 1;
    {
        Stk3DFMM fmm(6, 50, PAXIS::NONE, kernel, true);
        double o[3] = {origin[0], origin[1], origin[2]};
        fmm.setBox(o, len);
        fmm.setPoints(nsl, sl, ntrg, trg, ndl, ndl > 0 ? dl : nullptr);
        fmm.setupTree(static_cast<KERNEL>(kernel));
        fmm.evaluateFMM(static_cast<KERNEL>(kernel), nsl, slv, ntrg, out, ndl, ndl > 0 ? dlv : nullptr);
    }
    pvfmm::stub_fmm_direct = 0;
    return 0;
}

// The reference's own periodizeFMM (Lib/src/FMMData.cpp:203-247) for a triply
// periodic FMMData of order p: with the root's upward-equivalent density set to
// equiv[n * kdim] and every FMM value 1 (the stand-in in ones mode, unit box),
// trg[kdimTrg] returns 1 + the correction periodizeFMM adds.  The reference
// reads its M2C operator from $PVFMM_DIR/pdata (FMMData.cpp:13-56) even though
// the stand-in FMM does not use it: the caller provides that file.
extern "C" int ref_periodize(unsigned id, int p, const double *equiv, int nequiv, double *trg, int *kdim_trg) {
    using namespace stkfmm;
    if (!composite(id) || !equiv || !trg || !kdim_trg) return 1;
    pvfmm::stub_fmm_direct = 0;
    pvfmm::stub_root_equiv.assign(equiv, equiv + nequiv);
    {
        impl::FMMData fmm(static_cast<KERNEL>(id), PAXIS::PXYZ, p, 50, true);
        const std::vector<double> pt = {0.5, 0.5, 0.5}, none;
        const bool has_dl = fmm.hasDL();
        fmm.setupTree(pt, has_dl ? pt : none, pt);
        std::vector<double> slv(fmm.kdimSL, 0.0), dlv(has_dl ? fmm.kdimDL : 0, 0.0), tv(fmm.kdimTrg, 0.0);
        fmm.evaluateFMM(slv, dlv, tv, 1.0);
        std::copy(tv.begin(), tv.end(), trg);
        *kdim_trg = fmm.kdimTrg;
    }
    pvfmm::stub_root_equiv.clear();
    return 0;
}
