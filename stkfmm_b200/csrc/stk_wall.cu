// stk_wall.cu -- StkWallFMM: Stokeslets and RPY spheres above a no-slip wall.
//
// Mirrors the reference's StkWallFMM (Lib/src/StkWallFMM.cpp, Lib/include/STKFMM/
// STKFMM.hpp:219-262, C ABI Lib/src/Stk3DFMM-c.cpp:37-67).  The user's box
// [o, o+L)^2 x [o_z, o_z + L/2) is scaled to [0,1)^2 x [0,0.5) and shifted to
// z in [0.5, 1) (StkWallFMM.cpp:41-88); the wall is the plane z = 0.5 and every
// source has an image at 1 - z.  The wall velocity is a combination of several
// free-space (or PX / PXY) FMMs over the sources and their images
// (evalStokes, StkWallFMM.cpp:154-208; evalRPY, StkWallFMM.cpp:210-292):
//   Stokes: stokes_vel (sources + images), laplace_PGrad (charges + image
//           dipoles), laplace_PGradGrad (charges);
//   RPY:    rpy_ulapu (sources + images), laplace_PGradGrad (charges + image
//           dipoles), laplace_PGrad (charges + dipoles), laplace_QPGradGrad
//           (image quadrupoles, tree refined on sources and images).
// Each sub-FMM is a unit-box Stk3DFMM handle of this library, so its trees,
// operators and work lists stay resident.  The source values of the sub-FMMs
// are formed on the device (one staging kernel), the sub-FMMs run concurrently
// on their own handles' streams, and one assembly kernel on the wall's stream
// combines their outputs with the targets' heights.  The reference's box scaling (scaleSrc / scaleTrg applied
// by each sub-FMM with the wall's scale factor) is applied in the staging and
// assembly kernels: DL values and RPY radii times sF, sub-FMM outputs times
// sF^k (the kernel's trg_scale_pow).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/stkfmm_b200.h"
#include "stk_handle.hpp"
#include "stk_kernel_table.hpp"

using namespace stk;

namespace {

constexpr int kFamilies = 2;  // 0 Stokes, 1 RPY
constexpr int kSubs = 4;

// sub-FMM kernels per family, in the order of the reference's eval functions
const unsigned kSubKernel[kFamilies][kSubs] = {
    {STK_Stokes, STK_LapPGrad, STK_LapPGradGrad, 0},
    {STK_RPY, STK_LapPGradGrad, STK_LapPGrad, STK_LapQPGradGrad},
};

struct SubScale {
    double a[kSubs][10];  // sF^k per output component of each sub-FMM (scaleTrg)
};

#define WCUDA(call)                                 \
    do {                                            \
        if ((call) != cudaSuccess) {                \
            cudaGetLastError();                     \
            return STK_ERR_CUDA;                    \
        }                                           \
    } while (0)

inline int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 8)); }

// ---- Stokes: sub-FMM source values (StkWallFMM.cpp:161-196) ----
// f (n x 3) and the internal height z of each source; y3 = (z - 1/2) / sF is the
// physical height above the wall.
__global__ void wall_stage_stokes(int n, const double *__restrict__ f, const double *__restrict__ z, double sf,
                                  double *__restrict__ v_stk, double *__restrict__ v_l1, double *__restrict__ v_d,
                                  double *__restrict__ v_l2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double f0 = f[3 * (size_t)i], f1 = f[3 * (size_t)i + 1], f2 = f[3 * (size_t)i + 2];
        const double y3 = (z[i] - 0.5) / sf;
        const size_t o = 3 * (size_t)i, m = 3 * ((size_t)n + i);
        v_stk[o] = f0;
        v_stk[o + 1] = f1;
        v_stk[o + 2] = 0.0;
        v_stk[m] = -f0;
        v_stk[m + 1] = -f1;
        v_stk[m + 2] = 0.0;
        v_l1[i] = -0.5 * f2;
        v_l1[n + i] = 0.5 * f2;
        // image dipoles, DL values times sF (scaleSrc)
        v_d[o] = -y3 * f0 * sf;
        v_d[o + 1] = -y3 * f1 * sf;
        v_d[o + 2] = y3 * f2 * sf;
        v_l2[i] = f2 * y3;
        v_l2[n + i] = -f2 * y3;
    }
}

// u_j += uS_j + uL2_{grad j} / 2 + x3 uL1D_{grad j};  u_z -= uL1D_pot  (StkWallFMM.cpp:198-207)
__global__ void wall_assemble_stokes(int n, const double *__restrict__ z, double sf, SubScale w,
                                     const double *__restrict__ u_s, const double *__restrict__ u_l1d,
                                     const double *__restrict__ u_l2, double *__restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x3 = (z[i] - 0.5) / sf;
        const size_t t = (size_t)i;
        for (int j = 0; j < 3; j++)
            out[3 * t + j] += w.a[0][j] * u_s[3 * t + j] + 0.5 * w.a[2][j + 1] * u_l2[10 * t + j + 1] +
                              x3 * w.a[1][j + 1] * u_l1d[4 * t + j + 1];
        out[3 * t + 2] -= w.a[1][0] * u_l1d[4 * t];
    }
}

// ---- RPY: sub-FMM source values (StkWallFMM.cpp:220-275) ----
// fb rows (fx, fy, fz, b).
__global__ void wall_stage_rpy(int n, const double *__restrict__ fb, const double *__restrict__ z, double sf,
                               double *__restrict__ v_rpy, double *__restrict__ v_ls, double *__restrict__ v_ld,
                               double *__restrict__ v_lsz, double *__restrict__ v_ldz, double *__restrict__ v_q) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const size_t s = (size_t)i, m = (size_t)n + i;
        const double f1 = fb[4 * s], f2 = fb[4 * s + 1], f3 = fb[4 * s + 2], b = fb[4 * s + 3];
        const double y3 = (z[i] - 0.5) / sf;
        // rpy_ulapu: radii scale like a double layer (scaleSrc)
        v_rpy[4 * s] = f1;
        v_rpy[4 * s + 1] = f2;
        v_rpy[4 * s + 2] = 0.0;
        v_rpy[4 * s + 3] = b * sf;
        v_rpy[4 * m] = -f1;
        v_rpy[4 * m + 1] = -f2;
        v_rpy[4 * m + 2] = 0.0;
        v_rpy[4 * m + 3] = b * sf;
        // SD: laplace_PGradGrad charges and image dipoles
        v_ls[s] = -0.5 * f3;
        v_ls[m] = 0.5 * f3;
        v_ld[3 * s] = -y3 * f1 * sf;
        v_ld[3 * s + 1] = -y3 * f2 * sf;
        v_ld[3 * s + 2] = y3 * f3 * sf;
        // SDZ: laplace_PGrad charges and dipoles (0, 0, b^2 fz / 6) at sources and images
        v_lsz[s] = 0.5 * y3 * f3;
        v_lsz[m] = -0.5 * y3 * f3;
        const double dz = b * b * f3 * (1.0 / 6.0) * sf;
        v_ldz[3 * s] = 0.0;
        v_ldz[3 * s + 1] = 0.0;
        v_ldz[3 * s + 2] = dz;
        v_ldz[3 * m] = 0.0;
        v_ldz[3 * m + 1] = 0.0;
        v_ldz[3 * m + 2] = dz;
        // Q: image quadrupoles 2 b^2 / 6 (fz e_xx + fz e_yy + fx e_zx + fy e_zy), row-major
        const double tb = 2.0 * b * b * (1.0 / 6.0);
        double *q = v_q + 9 * s;
        q[0] = tb * f3;
        q[1] = 0.0;
        q[2] = 0.0;
        q[3] = 0.0;
        q[4] = tb * f3;
        q[5] = 0.0;
        q[6] = tb * f1;
        q[7] = tb * f2;
        q[8] = 0.0;
    }
}

// StkWallFMM.cpp:278-291: u = rpy + SDZ_grad + x3 (SD_grad + Q_grad), u_z -= SD_pot + Q_pot,
// lap u = rpy_lap + 2 (SD + Q)_{xz, yz, zz}
__global__ void wall_assemble_rpy(int n, const double *__restrict__ z, double sf, SubScale w,
                                  const double *__restrict__ u_rpy, const double *__restrict__ u_sd,
                                  const double *__restrict__ u_sdz, const double *__restrict__ u_q,
                                  double *__restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double x3 = (z[i] - 0.5) / sf;
        const size_t t = (size_t)i;
        const double *r = u_rpy + 6 * t, *sd = u_sd + 10 * t, *sdz = u_sdz + 4 * t, *q = u_q + 10 * t;
        double *o = out + 6 * t;
        for (int j = 0; j < 3; j++)
            o[j] += w.a[0][j] * r[j] + w.a[2][j + 1] * sdz[j + 1] +
                    x3 * (w.a[1][j + 1] * sd[j + 1] + w.a[3][j + 1] * q[j + 1]);
        o[2] -= w.a[1][0] * sd[0] + w.a[3][0] * q[0];
        const int h[3] = {6, 8, 9};
        for (int j = 0; j < 3; j++)
            o[3 + j] += w.a[0][3 + j] * r[3 + j] + 2.0 * (w.a[1][h[j]] * sd[h[j]] + w.a[3][h[j]] * q[h[j]]);
    }
}

}  // namespace

struct StkWallFMM {
    int mult_order = 10, max_pts = 2000, pbc = 0;
    unsigned kernel_comb = 0;
    double origin[3] = {0, 0, 0};
    double len = 1.0, sf = 1.0;
    int precision = STK_FP64;
    bool enable_ff = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timed = false;
    bool points_set = false;
    int nsl = 0, ntrg = 0;
    // internal coordinates (unit box, z in [0.5, 1)): sources, images, both, targets
    std::vector<double> src, img, src2, trg;
    Stk3DFMM *sub[kFamilies][kSubs] = {};
    bool ready[kFamilies] = {false, false};
    cudaEvent_t ev_staged = nullptr, ev_done[kSubs] = {};  // sub-FMMs run concurrently on their own streams
    DevBuf d_zsrc, d_ztrg, d_in, d_out, d_val[6], d_sub[kSubs];
    ~StkWallFMM() {
        for (auto &fam : sub)
            for (auto &h : fam)
                if (h) Stk3DFMM_destroy(h);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_staged) cudaEventDestroy(ev_staged);
        for (auto &e : ev_done)
            if (e) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

static int family_of(unsigned kernel) {
    return kernel == STK_Stokes ? 0 : kernel == STK_RPY ? 1 : -1;
}

extern "C" StkWallFMM *StkWallFMM_create(int mult_order, int max_pts, int pbc, unsigned kernelComb) {
    // the wall system is periodic in x, y at most (triply periodic is not a wall problem)
    if (mult_order < 2 || max_pts < 1 || pbc < 0 || pbc > 2) return nullptr;
    if (!(kernelComb & (STK_Stokes | STK_RPY))) return nullptr;
    if (stk_device_count() <= 0) return nullptr;
    auto *w = new StkWallFMM();
    w->mult_order = mult_order;
    w->max_pts = max_pts;
    w->pbc = pbc;
    w->kernel_comb = kernelComb;
    if (cudaGetDevice(&w->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&w->ev0) != cudaSuccess || cudaEventCreate(&w->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&w->ev_staged, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        delete w;
        return nullptr;
    }
    for (auto &e : w->ev_done)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            delete w;
            return nullptr;
        }
    double o[3] = {0, 0, 0};
    for (int f = 0; f < kFamilies; f++) {
        if (!(kernelComb & (f == 0 ? STK_Stokes : STK_RPY))) continue;
        for (int k = 0; k < kSubs && kSubKernel[f][k]; k++) {
            Stk3DFMM *h = Stk3DFMM_create(mult_order, max_pts, pbc, kSubKernel[f][k]);
            if (!h || Stk3DFMM_set_box(h, o, 1.0) != STK_OK) {
                if (h) Stk3DFMM_destroy(h);
                delete w;
                return nullptr;
            }
            w->sub[f][k] = h;
        }
    }
    return w;
}

extern "C" void StkWallFMM_destroy(StkWallFMM *fmm) {
    if (!fmm) return;
    cudaSetDevice(fmm->device);
    delete fmm;
}

extern "C" int StkWallFMM_set_box(StkWallFMM *fmm, double *origin, double len) {
    if (!fmm || !origin || !(len > 0)) return STK_ERR_INVALID_ARG;
    for (int k = 0; k < 3; k++) fmm->origin[k] = origin[k];
    fmm->len = len;
    fmm->sf = 1.0 / len;
    return STK_OK;
}

extern "C" int StkWallFMM_get_kernel_dimension(unsigned kernel, int *dims) {
    return stk_get_kernel_dimension(kernel, dims);
}

// scale to [0,1)^2 x [0,1/2), wrap the periodic axes, shift z by 1/2 (StkWallFMM.cpp:54-64)
static int wall_coord(const StkWallFMM *w, int n, const double *in, std::vector<double> &out) {
    out.resize(3 * (size_t)n);
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) {
            double x = (in[3 * (size_t)i + k] - w->origin[k]) * w->sf;
            const bool periodic = (w->pbc >= 1 && k == 0) || (w->pbc >= 2 && k == 1);
            if (periodic) {
                x -= std::floor(x);
                if (x >= 1.0) x = 0.0;
            }
            const double hi = k == 2 ? 0.5 : 1.0;
            if (!(x >= 0.0 && x < hi)) return STK_ERR_OUT_OF_BOX;
            out[3 * (size_t)i + k] = k == 2 ? x + 0.5 : x;
        }
        if (!(out[3 * (size_t)i + 2] < 1.0)) return STK_ERR_OUT_OF_BOX;
    }
    return STK_OK;
}

extern "C" int StkWallFMM_set_points(StkWallFMM *fmm, const int nSL, double *src_SL_coord, const int nTrg,
                                     double *trg_coord, const int nDL, double *src_DL_coord) {
    (void)nDL;  // the wall FMM has no double layer (StkWallFMM.cpp:41-88 ignores it)
    (void)src_DL_coord;
    if (!fmm || nSL < 0 || nTrg < 0) return STK_ERR_INVALID_ARG;
    if ((nSL > 0 && !src_SL_coord) || (nTrg > 0 && !trg_coord)) return STK_ERR_INVALID_ARG;
    fmm->points_set = false;
    fmm->ready[0] = fmm->ready[1] = false;
    int rc = wall_coord(fmm, nSL, src_SL_coord, fmm->src);
    if (!rc) rc = wall_coord(fmm, nTrg, trg_coord, fmm->trg);
    if (rc) return rc;
    fmm->nsl = nSL;
    fmm->ntrg = nTrg;
    fmm->img = fmm->src;
    for (int i = 0; i < nSL; i++) fmm->img[3 * (size_t)i + 2] = 1.0 - fmm->src[3 * (size_t)i + 2];
    fmm->src2 = fmm->src;
    fmm->src2.insert(fmm->src2.end(), fmm->img.begin(), fmm->img.end());
    fmm->points_set = true;
    return STK_OK;
}

// one sub-FMM: its SL / DL point sets and, for the quadrupole FMM, the tree points
static int setup_sub(Stk3DFMM *h, unsigned kernel, std::vector<double> &sl, std::vector<double> *dl,
                     std::vector<double> &trg, const std::vector<double> *tree_pts) {
    int rc = Stk3DFMM_set_points(h, (int)(sl.size() / 3), sl.data(), (int)(trg.size() / 3), trg.data(),
                                 dl ? (int)(dl->size() / 3) : 0, dl ? dl->data() : nullptr);
    if (rc) return rc;
    if (tree_pts)
        h->tree_pts = *tree_pts;
    else
        h->tree_pts.clear();
    return Stk3DFMM_setup_tree(h, kernel);
}

// The precision choice applies to the Stokes / RPY sub-FMM.  The Laplace
// sub-FMMs stay FP64: near a source the wall velocity is the difference of
// their terms (e.g. grad(fz y3 / r) / 2 and x3 grad(-fz / 2r), each ~10x the
// result for clustered sources), so FP32 pair errors there would be amplified
// about tenfold.
static void apply_precision(StkWallFMM *w) {
    for (auto &fam : w->sub)
        for (int k = 0; k < kSubs; k++)
            if (fam[k]) Stk3DFMM_set_precision(fam[k], k == 0 ? w->precision : STK_FP64);
}

extern "C" int StkWallFMM_setup_tree(StkWallFMM *fmm, unsigned kernel) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    const int f = family_of(kernel);
    if (f < 0) return STK_ERR_NOT_SUPPORTED;  // only Stokes and RPY have a wall image system
    if (!fmm->sub[f][0]) return STK_ERR_KERNEL;
    if (!fmm->points_set) return STK_ERR_STATE;
    cudaSetDevice(fmm->device);
    fmm->ready[f] = false;
    Stk3DFMM **h = fmm->sub[f];
    int rc;
    if (f == 0) {  // StkWallFMM.cpp:92-95
        rc = setup_sub(h[0], STK_Stokes, fmm->src2, nullptr, fmm->trg, nullptr);
        if (!rc) rc = setup_sub(h[1], STK_LapPGrad, fmm->src2, &fmm->img, fmm->trg, nullptr);
        if (!rc) rc = setup_sub(h[2], STK_LapPGradGrad, fmm->src2, nullptr, fmm->trg, nullptr);
    } else {  // StkWallFMM.cpp:96-101
        rc = setup_sub(h[0], STK_RPY, fmm->src2, nullptr, fmm->trg, nullptr);
        if (!rc) rc = setup_sub(h[1], STK_LapPGradGrad, fmm->src2, &fmm->img, fmm->trg, nullptr);
        if (!rc) rc = setup_sub(h[2], STK_LapPGrad, fmm->src2, &fmm->src2, fmm->trg, nullptr);
        if (!rc) rc = setup_sub(h[3], STK_LapQPGradGrad, fmm->img, nullptr, fmm->trg, &fmm->src2);
    }
    if (rc) return rc;
    apply_precision(fmm);
    // internal heights of sources and targets for the staging / assembly kernels
    std::vector<double> zs(fmm->nsl), zt(fmm->ntrg);
    for (int i = 0; i < fmm->nsl; i++) zs[i] = fmm->src[3 * (size_t)i + 2];
    for (int i = 0; i < fmm->ntrg; i++) zt[i] = fmm->trg[3 * (size_t)i + 2];
    rc = fmm->d_zsrc.upload(zs.data(), zs.size() * sizeof(double), fmm->stream);
    if (!rc) rc = fmm->d_ztrg.upload(zt.data(), zt.size() * sizeof(double), fmm->stream);
    if (!rc && cudaStreamSynchronize(fmm->stream) != cudaSuccess) rc = STK_ERR_CUDA;
    if (rc) return rc;
    fmm->ready[f] = true;
    return STK_OK;
}

extern "C" int StkWallFMM_clear_fmm(StkWallFMM *fmm, unsigned kernel) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    const int f = family_of(kernel);
    if (f < 0) return STK_ERR_NOT_SUPPORTED;
    return fmm->sub[f][0] ? STK_OK : STK_ERR_KERNEL;
}

extern "C" int StkWallFMM_show_active_kernels(StkWallFMM *fmm) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    if (fmm->sub[0][0]) printf("enable Stokes image kernel\n");
    if (fmm->sub[1][0]) printf("enable RPY image kernel\n");
    return STK_OK;
}

// The reference's enableFF (StkWallFMM.cpp:5-32 hands it to every sub-FMM).
extern "C" int StkWallFMM_set_far_field(StkWallFMM *fmm, int enable) {
    if (!fmm || (enable != 0 && enable != 1)) return STK_ERR_INVALID_ARG;
    for (auto &fam : fmm->sub)
        for (int k = 0; k < kSubs; k++)
            if (fam[k]) {
                const int rc = Stk3DFMM_set_far_field(fam[k], enable);
                if (rc) return rc;
            }
    if (fmm->enable_ff != (enable == 1)) fmm->ready[0] = fmm->ready[1] = false;  // takes effect at setup_tree
    fmm->enable_ff = enable == 1;
    return STK_OK;
}

extern "C" int StkWallFMM_set_precision(StkWallFMM *fmm, int precision) {
    if (!fmm || (precision != STK_FP64 && precision != STK_MIXED)) return STK_ERR_INVALID_ARG;
    fmm->precision = precision;
    apply_precision(fmm);
    return STK_OK;
}

// The sub-FMMs of one evaluation: each on its own handle's stream after the
// staging kernel (event on s), s waits for all of them before the assembly.
// Their near-field kernels fill the GPU; the smaller far-field kernels and
// GEMMs of one sub-FMM overlap with the others'.
static int run_subs(StkWallFMM *w, int f, const double *const *sv, const double *const *dv, double *const *u,
                    cudaStream_t s) {
    WCUDA(cudaEventRecord(w->ev_staged, s));
    int rc = STK_OK;
    int k = 0;
    for (; k < kSubs && w->sub[f][k]; k++) {
        Stk3DFMM *h = w->sub[f][k];
        WCUDA(cudaStreamWaitEvent(h->stream, w->ev_staged, 0));
        rc = Stk3DFMM_evaluate_fmm_device(h, kSubKernel[f][k], sv[k], u[k], dv[k], h->stream);
        WCUDA(cudaEventRecord(w->ev_done[k], h->stream));
        if (rc) break;
    }
    for (int j = 0; j < k && j < kSubs && w->sub[f][j]; j++) WCUDA(cudaStreamWaitEvent(s, w->ev_done[j], 0));
    return rc;
}

// The wall evaluation on device buffers: d_trg_value (caller's order, kdimTrg per
// target) += wall FMM of d_src_SL_value (caller's order, kdimSL per source).
static int wall_eval(StkWallFMM *w, int f, const double *d_sl, double *d_out, cudaStream_t s) {
    const int n = w->nsl, nt = w->ntrg;
    Stk3DFMM **h = w->sub[f];
    SubScale sc{};
    for (int k = 0; k < kSubs; k++) {
        if (!h[k]) continue;
        const KernelInfo *ki = find_kernel(kSubKernel[f][k]);
        for (int c = 0; c < ki->kdim_trg && c < 10; c++) sc.a[k][c] = std::pow(w->sf, ki->trg_scale_pow[c]);
    }
    // sub-FMM value buffers (2n points at most, 9 values for the quadrupoles)
    const size_t vb[6] = {f == 0 ? 6 * (size_t)n : 8 * (size_t)n, 2 * (size_t)n, 3 * (size_t)n, 2 * (size_t)n,
                          6 * (size_t)n, 9 * (size_t)n};
    for (int k = 0; k < 6; k++)
        if (int rc = w->d_val[k].reserve(sizeof(double) * std::max<size_t>(vb[k], 1))) return rc;
    const int tdim[kFamilies][kSubs] = {{3, 4, 10, 0}, {6, 10, 4, 10}};
    for (int k = 0; k < kSubs; k++) {
        if (!tdim[f][k]) continue;
        const size_t bytes = sizeof(double) * (size_t)std::max(nt, 1) * tdim[f][k];
        if (int rc = w->d_sub[k].reserve(bytes)) return rc;
        WCUDA(cudaMemsetAsync(w->d_sub[k].ptr, 0, bytes, s));
    }
    double *v[6];
    for (int k = 0; k < 6; k++) v[k] = (double *)w->d_val[k].ptr;
    double *u[kSubs];
    for (int k = 0; k < kSubs; k++) u[k] = (double *)w->d_sub[k].ptr;
    const double *zs = (const double *)w->d_zsrc.ptr, *zt = (const double *)w->d_ztrg.ptr;
    if (f == 0) {
        if (n > 0) {
            wall_stage_stokes<<<grid_for(n), 256, 0, s>>>(n, d_sl, zs, w->sf, v[0], v[1], v[2], v[3]);
            WCUDA(cudaGetLastError());
        }
        const double *sv[kSubs] = {v[0], v[1], v[3], nullptr}, *dv[kSubs] = {nullptr, v[2], nullptr, nullptr};
        if (int rc2 = run_subs(w, f, sv, dv, u, s)) return rc2;
        if (nt > 0) {
            wall_assemble_stokes<<<grid_for(nt), 256, 0, s>>>(nt, zt, w->sf, sc, u[0], u[1], u[2], d_out);
            WCUDA(cudaGetLastError());
        }
    } else {
        if (n > 0) {
            wall_stage_rpy<<<grid_for(n), 256, 0, s>>>(n, d_sl, zs, w->sf, v[0], v[1], v[2], v[3], v[4], v[5]);
            WCUDA(cudaGetLastError());
        }
        const double *sv[kSubs] = {v[0], v[1], v[3], v[5]}, *dv[kSubs] = {nullptr, v[2], v[4], nullptr};
        if (int rc2 = run_subs(w, f, sv, dv, u, s)) return rc2;
        if (nt > 0) {
            wall_assemble_rpy<<<grid_for(nt), 256, 0, s>>>(nt, zt, w->sf, sc, u[0], u[1], u[2], u[3], d_out);
            WCUDA(cudaGetLastError());
        }
    }
    return STK_OK;
}

extern "C" int StkWallFMM_evaluate_fmm_device(StkWallFMM *fmm, unsigned kernel, const double *d_src_SL_value,
                                              double *d_trg_value, void *stream) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    const int f = family_of(kernel);
    if (f < 0) return STK_ERR_NOT_SUPPORTED;
    if (!fmm->sub[f][0]) return STK_ERR_KERNEL;
    if (!fmm->ready[f]) return STK_ERR_STATE;
    if ((fmm->nsl > 0 && !d_src_SL_value) || (fmm->ntrg > 0 && !d_trg_value)) return STK_ERR_INVALID_ARG;
    cudaSetDevice(fmm->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : fmm->stream;
    WCUDA(cudaEventRecord(fmm->ev0, s));
    const int rc = wall_eval(fmm, f, d_src_SL_value, d_trg_value, s);
    if (rc) return rc;
    WCUDA(cudaEventRecord(fmm->ev1, s));
    fmm->timed = true;
    return STK_OK;
}

// StkWallFMM::evaluateFMM (StkWallFMM.cpp:107-136): trg_value += wall FMM(sources);
// Stokes: 3 values per source -> 3 per target; RPY: (f, b) -> (u, lap u).
extern "C" int StkWallFMM_evaluate_fmm(StkWallFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value,
                                       const int nTrg, double *trg_value, const int nDL, double *src_DL_value) {
    (void)nDL;
    (void)src_DL_value;
    if (!fmm) return STK_ERR_INVALID_ARG;
    const int f = family_of(kernel);
    if (f < 0) return STK_ERR_NOT_SUPPORTED;
    if (!fmm->sub[f][0]) return STK_ERR_KERNEL;
    if (!fmm->ready[f]) return STK_ERR_STATE;
    if (nSL != fmm->nsl || nTrg != fmm->ntrg) return STK_ERR_SIZE;
    if ((nSL > 0 && !src_SL_value) || (nTrg > 0 && !trg_value)) return STK_ERR_INVALID_ARG;
    cudaSetDevice(fmm->device);
    const size_t nin = (size_t)nSL * (f == 0 ? 3 : 4), nout = (size_t)nTrg * (f == 0 ? 3 : 6);
    cudaStream_t s = fmm->stream;
    int rc = fmm->d_in.upload(src_SL_value, nin * sizeof(double), s);
    if (!rc) rc = fmm->d_out.upload(trg_value, nout * sizeof(double), s);
    if (rc) return rc;
    rc = StkWallFMM_evaluate_fmm_device(fmm, kernel, (const double *)fmm->d_in.ptr, (double *)fmm->d_out.ptr, s);
    if (rc) return rc;
    if (nout) WCUDA(cudaMemcpyAsync(trg_value, fmm->d_out.ptr, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
    WCUDA(cudaStreamSynchronize(s));
    return STK_OK;
}

// this library's kernels launched by the last evaluation: the sub-FMMs' plus staging and assembly
extern "C" int StkWallFMM_last_launch_count(StkWallFMM *fmm, unsigned kernel, int *count) {
    if (!fmm || !count) return STK_ERR_INVALID_ARG;
    const int f = family_of(kernel);
    if (f < 0) return STK_ERR_NOT_SUPPORTED;
    if (!fmm->sub[f][0]) return STK_ERR_KERNEL;
    if (!fmm->ready[f]) return STK_ERR_STATE;
    int total = 2;
    for (int k = 0; k < kSubs; k++) {
        if (!fmm->sub[f][k]) continue;
        int c = 0;
        if (int rc = Stk3DFMM_last_launch_count(fmm->sub[f][k], kSubKernel[f][k], &c)) return rc;
        total += c;
    }
    *count = total;
    return STK_OK;
}

extern "C" int StkWallFMM_last_kernel_ms(StkWallFMM *fmm, float *ms) {
    if (!fmm || !ms) return STK_ERR_INVALID_ARG;
    if (!fmm->timed) return STK_ERR_STATE;
    if (cudaEventSynchronize(fmm->ev1) != cudaSuccess || cudaEventElapsedTime(ms, fmm->ev0, fmm->ev1) != cudaSuccess) {
        cudaGetLastError();
        return STK_ERR_CUDA;
    }
    return STK_OK;
}
