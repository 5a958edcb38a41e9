// stk_handle.cu -- the Stk3DFMM handle of the C ABI.
//
// Mirrors the reference's Stk3DFMM (Lib/src/Stk3DFMM.cpp) and FMMData
// (Lib/src/FMMData.cpp): box scaling and periodic wrap of the coordinates
// (STKFMM.cpp:113-150), one tree + operator set per activated kernel, value
// scaling before evaluation (scaleSrc, FMMData.cpp:285-317), target rescaling
// after (scaleTrg, FMMData.cpp:319-470) and accumulation into the caller's
// array (Stk3DFMM.cpp:104-108).  Trees, lists, sorted coordinates and work
// items stay resident on the device between evaluations (setupTree once,
// evaluate many times, as in Python/example.py:88-100).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/stkfmm_b200.h"
#include "stk_farfield.hpp"
#include "stk_handle.hpp"
#include "stk_kernel_table.hpp"
#include "stk_p2p.cuh"
#include "stk_tree.hpp"
#include "stk_work.hpp"

using namespace stk;

namespace stk {

static bool verbose() {
    static const bool v = [] {
        const char *e = getenv("STKFMM_VERBOSE");
        return !(e == nullptr || e[0] == '0');
    }();
    return v;
}

#define HCUDA(call)                                                                                        \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            if (verbose()) fprintf(stderr, "stkfmm_b200: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return STK_ERR_CUDA;                                                                           \
        }                                                                                                  \
    } while (0)

void DevBuf::release() {
    owner.reset();  // cudaFree when this was the last owner
    ptr = nullptr;
    bytes = 0;
}

int DevBuf::reserve(size_t n) {
    if (n == 0) n = 16;
    if (n <= bytes && !shared()) return STK_OK;
    release();
    void *p = nullptr;
    if (cudaMalloc(&p, n) != cudaSuccess) {
        cudaGetLastError();
        return STK_ERR_CUDA;
    }
    owner = std::shared_ptr<void>(p, [](void *q) { cudaFree(q); });
    ptr = p;
    bytes = n;
    return STK_OK;
}

int DevBuf::upload(const void *src, size_t n, cudaStream_t s) {
    int rc = reserve(n);
    if (rc) return rc;
    if (n == 0) return STK_OK;
    HCUDA(cudaMemcpyAsync(ptr, src, n, cudaMemcpyHostToDevice, s));
    return STK_OK;
}

KernelData::~KernelData() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : ph)
        if (e) cudaEventDestroy(e);
}

}  // namespace stk

Stk3DFMM::~Stk3DFMM() {
    pool.clear();
    if (stream) cudaStreamDestroy(stream);
    if (aux_stream) cudaStreamDestroy(aux_stream);
    if (ev_out) cudaEventDestroy(ev_out);
}

extern "C" Stk3DFMM *Stk3DFMM_create(int mult_order, int max_pts, int pbc, unsigned kernelComb) {
    if (mult_order < 2 || max_pts < 1 || pbc < 0 || pbc > 3 || kernelComb == 0) return nullptr;
    if (stk_device_count() <= 0) return nullptr;
    auto *f = new Stk3DFMM();
    f->mult_order = mult_order;
    f->max_pts = max_pts;
    f->pbc = pbc;
    f->kernel_comb = kernelComb;
    if (cudaGetDevice(&f->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaDeviceGetAttribute(&f->sms, cudaDevAttrMultiProcessorCount, f->device) != cudaSuccess) {
        cudaGetLastError();
        delete f;
        return nullptr;
    }
    for (int i = 0; i < kNumKernels; i++) {
        if (kernelComb & kKernels[i].id) {
            f->pool[kKernels[i].id] = std::unique_ptr<KernelData>(new KernelData());
            f->pool[kKernels[i].id]->info = &kKernels[i];
        }
    }
    if (f->pool.empty()) {
        delete f;
        return nullptr;
    }
    return f;
}

extern "C" void Stk3DFMM_destroy(Stk3DFMM *fmm) {
    if (!fmm) return;
    cudaSetDevice(fmm->device);
    delete fmm;
}

extern "C" int Stk3DFMM_set_box(Stk3DFMM *fmm, double *origin, double len) {
    if (!fmm || !origin || !(len > 0)) return STK_ERR_INVALID_ARG;
    for (int k = 0; k < 3; k++) fmm->origin[k] = origin[k];
    fmm->len = len;
    fmm->scale_factor = 1.0 / len;  // STKFMM::setBox, Lib/src/STKFMM.cpp:74-86
    return STK_OK;
}

extern "C" int Stk3DFMM_get_kernel_dimension(unsigned kernel, int *dims) {
    return stk_get_kernel_dimension(kernel, dims);
}

// scale to the unit box and wrap periodic axes (STKFMM::scaleCoord / wrapCoord)
static int set_coord(const Stk3DFMM *f, int n, const double *src, std::vector<double> &dst) {
    dst.resize(3 * (size_t)n);
    const double sf = f->scale_factor;
    for (int i = 0; i < n; i++) {
        for (int k = 0; k < 3; k++) {
            double x = (src[3 * (size_t)i + k] - f->origin[k]) * sf;
            const bool periodic = (f->pbc >= 1 && k == 0) || (f->pbc >= 2 && k == 1) || (f->pbc >= 3 && k == 2);
            if (periodic) x = x - std::floor(x);  // fracwrap, stkfmm_helpers.hpp:34
            if (periodic && x >= 1.0) x = 0.0;      // x just below 0 rounds up to 1
            if (!(x >= 0.0 && x < 1.0)) return STK_ERR_OUT_OF_BOX;
            dst[3 * (size_t)i + k] = x;
        }
    }
    return STK_OK;
}

extern "C" int Stk3DFMM_set_points(Stk3DFMM *fmm, const int nSL, double *src_SL_coord, const int nTrg,
                                   double *trg_coord, const int nDL, double *src_DL_coord) {
    if (!fmm || nSL < 0 || nTrg < 0 || nDL < 0) return STK_ERR_INVALID_ARG;
    if ((nSL > 0 && !src_SL_coord) || (nTrg > 0 && !trg_coord)) return STK_ERR_INVALID_ARG;
    if (!(fmm->len > 0)) return STK_ERR_STATE;
    // all trees are invalidated (Stk3DFMM.cpp:35-43)
    for (auto &kv : fmm->pool) kv.second->tree_ready = false;
    fmm->points_set = false;
    int rc = set_coord(fmm, nSL, src_SL_coord, fmm->sl);
    if (!rc) rc = set_coord(fmm, nTrg, trg_coord, fmm->trg);
    if (!rc) {
        if (nDL > 0 && src_DL_coord)
            rc = set_coord(fmm, nDL, src_DL_coord, fmm->dl);
        else
            fmm->dl.clear();
    }
    if (rc) return rc;
    fmm->nsl = nSL;
    fmm->ntrg = nTrg;
    fmm->ndl = (int)(fmm->dl.size() / 3);
    fmm->sl_dl_same = fmm->nsl == fmm->ndl && fmm->nsl > 0 &&
                      std::memcmp(fmm->sl.data(), fmm->dl.data(), sizeof(double) * 3 * fmm->nsl) == 0;
    fmm->points_set = true;
    if (verbose()) printf("points set\n");
    return STK_OK;
}

static KernelData *get_kd(Stk3DFMM *f, unsigned kernel) {
    auto it = f->pool.find(kernel);
    return it == f->pool.end() ? nullptr : it->second.get();
}

static bool has_dl(const KernelData *kd) { return kd->info->slot[SLOT_S2T_DL] >= 0; }

static int fused_uk(const KernelData *kd) {
    if (kd->info->id == STK_LapPGrad) return UK_LAPLACE_SLDL_PGRAD;
    if (kd->info->id == STK_PVel) return UK_STOKES_SLDL_PVEL;
    return -1;
}

extern "C" int Stk3DFMM_setup_tree(Stk3DFMM *fmm, unsigned kernel) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kernel_supported(kd->info)) return STK_ERR_NOT_SUPPORTED;
    if (!fmm->points_set) return STK_ERR_STATE;
    cudaSetDevice(fmm->device);
    kd->tree_ready = false;
    kd->far_ready = false;
    const bool dl = has_dl(kd) && fmm->ndl > 0;
    const int nsl = fmm->nsl, ndl = dl ? fmm->ndl : 0, ntrg = fmm->ntrg;
    // tree points: the largest of SL / DL / targets, ties to targets (FMMData.cpp:123-135)
    const std::vector<double> *pts = &fmm->trg;
    if (nsl > ndl && nsl > ntrg)
        pts = &fmm->sl;
    else if (ndl > nsl && ndl > ntrg)
        pts = &fmm->dl;
    if (!fmm->tree_pts.empty()) pts = &fmm->tree_pts;
    Octree &T = kd->tree;
    std::string err = T.build(pts->data(), (int)(pts->size() / 3), fmm->max_pts, kMaxDepth, fmm->pbc);
    if (err.empty()) err = T.assign(0, fmm->sl.data(), nsl);
    if (err.empty()) err = T.assign(1, dl ? fmm->dl.data() : nullptr, ndl);
    if (err.empty()) err = T.assign(2, fmm->trg.data(), ntrg);
    if (!err.empty()) {
        if (verbose()) fprintf(stderr, "stkfmm_b200: %s\n", err.c_str());
        return STK_ERR_OUT_OF_BOX;
    }
    T.build_lists();
    kd->fused = dl && fmm->sl_dl_same && fused_uk(kd) >= 0;

    // ---- device-resident tree data ----
    cudaStream_t s = fmm->stream;
    const int nn = T.num_nodes();
    std::vector<double> centre(3 * (size_t)nn);
    for (int i = 0; i < nn; i++) T.centre(i, &centre[3 * (size_t)i]);
    int rc = STK_OK;
    auto up = [&](DevBuf &b, const void *p, size_t n) {
        if (!rc) rc = b.upload(p, n, s);
    };
    up(kd->d_centre, centre.data(), centre.size() * sizeof(double));
    for (int k = 0; k < 3; k++) {
        const PointSet &ps = T.sets[k];
        up(kd->d_xyz[k], ps.xyz.data(), ps.xyz.size() * sizeof(double));
        up(kd->d_perm[k], ps.perm.data(), ps.perm.size() * sizeof(int));
        up(kd->d_beg[k], ps.node_begin.data(), ps.node_begin.size() * sizeof(int));
        up(kd->d_end[k], ps.node_end.data(), ps.node_end.size() * sizeof(int));
    }
    up(kd->d_uent, T.U.ent.data(), T.U.ent.size() * sizeof(int));
    // U-list work items: per source set (SL, DL) or fused
    const PointSet &tg = T.sets[2];
    kd->u_pairs[0] = kd->u_pairs[1] = 0;
    for (int k = 0; k < 2; k++) {
        kd->n_items[k] = 0;
        if (k == 1 && (!dl || kd->fused)) continue;
        const PointSet &sp = T.sets[k];
        std::vector<WorkItem> items;
        long long pairs = 0;
        build_list_items(nn, tg.node_begin.data(), tg.node_end.data(), T.U.off.data(), T.U.ent.data(),
                         sp.node_begin.data(), sp.node_end.data(), items, pairs, fmm->sms * 12, fmm->shard_rank,
                         fmm->shard_n);
        kd->u_pairs[k] = pairs;
        kd->n_items[k] = (int)items.size();
        up(kd->d_items[k], items.data(), items.size() * sizeof(WorkItem));
    }
    if (kd->fused) kd->u_pairs[1] = kd->u_pairs[0];
    if (!rc) rc = kd->d_counter.reserve(64);
    if (!rc && !kd->ev0) {
        if (cudaEventCreate(&kd->ev0) != cudaSuccess || cudaEventCreate(&kd->ev1) != cudaSuccess) rc = STK_ERR_CUDA;
        for (int i = 0; i < KernelData::kPhases && !rc; i++)
            if (cudaEventCreate(&kd->ph[i]) != cudaSuccess) rc = STK_ERR_CUDA;
    }
    if (!rc && cudaStreamSynchronize(s) != cudaSuccess) rc = STK_ERR_CUDA;
    if (rc) return rc;
    kd->tree_ready = true;
    if (verbose())
        printf("tree: %d nodes, %zu leaves, depth %d, U entries %zu, U pairs SL %lld DL %lld\n", nn, T.leaves.size(),
               T.depth(), T.U.size(), kd->u_pairs[0], kd->u_pairs[1]);
    return STK_OK;
}

extern "C" int Stk3DFMM_clear_fmm(Stk3DFMM *fmm, unsigned kernel) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    return get_kd(fmm, kernel) ? STK_OK : STK_ERR_KERNEL;
}

extern "C" int Stk3DFMM_show_active_kernels(Stk3DFMM *fmm) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    printf("active kernels: ");
    for (int i = 0; i < kNumKernels; i++)
        if (fmm->kernel_comb & kKernels[i].id) printf("\t%s", kKernels[i].name);
    printf("\n");
    return STK_OK;
}

extern "C" int Stk3DFMM_set_shard(Stk3DFMM *fmm, int rank, int nranks) {
    if (!fmm || nranks < 1 || rank < 0 || rank >= nranks) return STK_ERR_INVALID_ARG;
    if (fmm->shard_rank != rank || fmm->shard_n != nranks)
        for (auto &kv : fmm->pool) {
            kv.second->tree_ready = false;  // work lists are rebuilt by the next setup_tree
            kv.second->far_ready = false;
        }
    fmm->shard_rank = rank;
    fmm->shard_n = nranks;
    return STK_OK;
}

extern "C" int Stk3DFMM_set_allreduce(Stk3DFMM *fmm, stk_allreduce_fn fn, void *user) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    if (fmm->allreduce != fn)
        for (auto &kv : fmm->pool) {
            kv.second->tree_ready = false;  // the far-field split is rebuilt by the next setup_tree
            kv.second->far_ready = false;
        }
    fmm->allreduce = fn;
    fmm->allreduce_user = user;
    return STK_OK;
}

extern "C" int Stk3DFMM_set_far_field(Stk3DFMM *fmm, int enable) {
    if (!fmm || (enable != 0 && enable != 1)) return STK_ERR_INVALID_ARG;
    if (fmm->enable_ff != (enable == 1))
        for (auto &kv : fmm->pool) {
            kv.second->tree_ready = false;  // takes effect at the next setup_tree
            kv.second->far_ready = false;
        }
    fmm->enable_ff = enable == 1;
    return STK_OK;
}

extern "C" int Stk3DFMM_set_precision(Stk3DFMM *fmm, int precision) {
    if (!fmm || (precision != STK_FP64 && precision != STK_MIXED)) return STK_ERR_INVALID_ARG;
    fmm->precision = precision;
    return STK_OK;
}

// Near-field (and with far = true, the KIFMM far-field) evaluation on device
// buffers in the caller's order.  d_sl / d_dl hold values already scaled
// (scaleSrc); d_out_user receives trg += sF^k * result (scaleTrg) in the
// caller's order.
int stk::near_device(Stk3DFMM *f, KernelData *kd, const double *d_sl, const double *d_dl, double *d_out_user,
                     cudaStream_t s, bool far, const std::function<int()> &before_scatter) {
    const KernelInfo *ki = kd->info;
    Octree &T = kd->tree;
    const int nn = T.num_nodes();
    const int ntrg = f->ntrg;
    const int td = ki->kdim_trg;
    const bool dl = has_dl(kd) && T.sets[1].n > 0;
    int rc = kd->d_out_sorted.reserve(sizeof(double) * std::max(1, ntrg) * td);
    if (rc) return rc;
    double *out = (double *)kd->d_out_sorted.ptr;
    HCUDA(cudaMemsetAsync(out, 0, sizeof(double) * ntrg * td, s));
    HCUDA(cudaEventRecord(kd->ev0, s));
    int launches = 0;
    for (int k = 0; k < 2; k++) {
        if (k == 1 && (!dl || kd->fused)) continue;
        // the FMM's near field: U list plus the W / X interactions evaluated directly
        const ListPass *fp = far ? &kd->far->near[k] : nullptr;
        const int n_items = far ? fp->n_items : kd->n_items[k];
        if (n_items == 0) continue;
        const int uk = kd->fused ? fused_uk(kd) : ki->slot[k == 0 ? SLOT_S2T_SL : SLOT_S2T_DL];
        const int rs = uk_record_stride(uk);
        const PointSet &sp = T.sets[k];
        rc = kd->d_rec[k].reserve(sizeof(double) * std::max(1, sp.n) * rs);
        if (rc) return rc;
        double *rec = (double *)kd->d_rec[k].ptr;
        if (kd->fused)
            HCUDA(launch_pack_records(sp.n, (const int *)kd->d_perm[0].ptr, (const double *)kd->d_xyz[0].ptr, d_sl,
                                      ki->kdim_sl, d_dl, ki->kdim_dl, rs, rec, s));
        else
            HCUDA(launch_pack_records(sp.n, (const int *)kd->d_perm[k].ptr, (const double *)kd->d_xyz[k].ptr,
                                      k == 0 ? d_sl : d_dl, k == 0 ? ki->kdim_sl : ki->kdim_dl, nullptr, 0, rs, rec,
                                      s));
        ListP2PArgs a{};
        a.src_rec = rec;
        a.src_box_begin = (const int *)kd->d_beg[k].ptr;
        a.src_box_end = (const int *)kd->d_end[k].ptr;
        a.list_ent = far ? (const int *)fp->ent.ptr : (const int *)kd->d_uent.ptr;
        a.items = far ? (const WorkItem *)fp->items.ptr : (const WorkItem *)kd->d_items[k].ptr;
        a.n_items = n_items;
        a.counter = (unsigned int *)kd->d_counter.ptr;
        a.trg_xyz = (const double *)kd->d_xyz[2].ptr;
        a.trg_out = out;
        a.box_centre = (const double *)kd->d_centre.ptr;
        a.period = 1.0;
        a.atomic_out = 0;
        // one octree holds the sources and the targets: coincident points share a leaf
        a.coincident_own_box = 1;
        HCUDA(launch_list_p2p(uk, f->precision, a, f->sms, s));
        launches += 2;  // record packing + list kernel
    }
    HCUDA(cudaEventRecord(kd->ph[0], s));
    kd->last_far = far;
    if (far) {
        rc = farfield_evaluate(f, kd, d_sl, dl ? d_dl : nullptr, out, s);
        if (rc) return rc;
    }
    HCUDA(cudaEventRecord(kd->ev1, s));
    // caller order + scaleTrg factors
    double alpha[16];
    for (int c = 0; c < td; c++) alpha[c] = std::pow(f->scale_factor, ki->trg_scale_pow[c]);
    rc = kd->d_alpha.upload(alpha, sizeof(double) * td, s);
    if (rc) return rc;
    (void)nn;
    if (before_scatter && (rc = before_scatter())) return rc;
    HCUDA(launch_scatter_add(ntrg, td, (const int *)kd->d_perm[2].ptr, out, (const double *)kd->d_alpha.ptr,
                             d_out_user, s));
    kd->launches = launches + (ntrg > 0 ? 1 : 0) + (far ? kd->far->launches : 0);
    kd->timed = true;
    return STK_OK;
}

static int check_eval_args(Stk3DFMM *fmm, unsigned kernel, int nSL, const double *slv, int nTrg, double *trgv,
                           int nDL, const double *dlv, KernelData *&kd) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready) return STK_ERR_STATE;
    if (nSL != fmm->nsl || nTrg != fmm->ntrg) return STK_ERR_SIZE;
    const bool dl = has_dl(kd) && fmm->ndl > 0;
    if (dl && nDL != fmm->ndl) return STK_ERR_SIZE;
    if ((nSL > 0 && !slv) || (nTrg > 0 && !trgv) || (dl && nDL > 0 && !dlv)) return STK_ERR_INVALID_ARG;
    return STK_OK;
}

// v[i stride + offset] *= a for i < n
__global__ void scale_strided_kernel(double *__restrict__ v, long long n, int stride, int offset, double a) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i * stride + offset] *= a;
}

static cudaError_t scale_strided(double *v, long long n, int stride, int offset, double a, cudaStream_t s) {
    if (n <= 0 || a == 1.0) return cudaSuccess;
    const int grid = (int)std::min<long long>((n + 255) / 256, 148 * 16);
    scale_strided_kernel<<<grid, 256, 0, s>>>(v, n, stride, offset, a);
    return cudaGetLastError();
}

static int ensure_far(Stk3DFMM *fmm, KernelData *kd);

// Host-array evaluation (evaluate_near / evaluate_fmm): the caller's arrays are
// copied straight to the device (DMA when they are pinned), scaleSrc runs on
// the device, the caller's target array is accumulated on the device and copied
// back in place: trg_value += result.
static int eval_host(Stk3DFMM *fmm, unsigned kernel, const int nSL, const double *src_SL_value, const int nTrg,
                     double *trg_value, const int nDL, const double *src_DL_value, bool far) {
    KernelData *kd = nullptr;
    int rc = check_eval_args(fmm, kernel, nSL, src_SL_value, nTrg, trg_value, nDL, src_DL_value, kd);
    if (rc) return rc;
    cudaSetDevice(fmm->device);
    if (far && (rc = ensure_far(fmm, kd))) return rc;
    const KernelInfo *ki = kd->info;
    const bool dl = has_dl(kd) && fmm->ndl > 0;
    cudaStream_t s = fmm->stream;
    const size_t nsl_v = (size_t)nSL * ki->kdim_sl, ndl_v = dl ? (size_t)nDL * ki->kdim_dl : 0;
    const size_t ntrg_v = (size_t)nTrg * ki->kdim_trg;
    rc = kd->d_val[0].upload(src_SL_value, nsl_v * sizeof(double), s);
    if (!rc && dl) rc = kd->d_val[1].upload(src_DL_value, ndl_v * sizeof(double), s);
    if (!rc) rc = kd->d_out_user.reserve(std::max<size_t>(ntrg_v, 1) * sizeof(double));
    if (rc) return rc;
    if (!fmm->aux_stream && cudaStreamCreateWithFlags(&fmm->aux_stream, cudaStreamNonBlocking) != cudaSuccess)
        return STK_ERR_CUDA;
    if (!fmm->ev_out && cudaEventCreateWithFlags(&fmm->ev_out, cudaEventDisableTiming) != cudaSuccess)
        return STK_ERR_CUDA;
    // the caller's target values go up on the side stream while the kernels run
    auto upload_out = [&]() -> int {
        if (ntrg_v)
            HCUDA(cudaMemcpyAsync(kd->d_out_user.ptr, trg_value, ntrg_v * sizeof(double), cudaMemcpyHostToDevice,
                                  fmm->aux_stream));
        HCUDA(cudaEventRecord(fmm->ev_out, fmm->aux_stream));
        HCUDA(cudaStreamWaitEvent(s, fmm->ev_out, 0));
        return STK_OK;
    };
    // scaleSrc (FMMData.cpp:285-317): DL values and a scaling last SL component times sF
    const double sf = fmm->scale_factor;
    if (dl) HCUDA(scale_strided((double *)kd->d_val[1].ptr, (long long)ndl_v, 1, 0, sf, s));
    for (int c = ki->kdim_sl - ki->sl_last_scales; c < ki->kdim_sl; c++)
        HCUDA(scale_strided((double *)kd->d_val[0].ptr, nSL, ki->kdim_sl, c, sf, s));
    rc = near_device(fmm, kd, (const double *)kd->d_val[0].ptr, dl ? (const double *)kd->d_val[1].ptr : nullptr,
                     (double *)kd->d_out_user.ptr, s, far, upload_out);
    if (rc) return rc;
    if (ntrg_v) HCUDA(cudaMemcpyAsync(trg_value, kd->d_out_user.ptr, ntrg_v * sizeof(double), cudaMemcpyDeviceToHost, s));
    HCUDA(cudaStreamSynchronize(s));
    return far ? farfield_status(kd) : STK_OK;
}

extern "C" int Stk3DFMM_evaluate_near(Stk3DFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value,
                                      const int nTrg, double *trg_value, const int nDL, double *src_DL_value) {
    return eval_host(fmm, kernel, nSL, src_SL_value, nTrg, trg_value, nDL, src_DL_value, false);
}

extern "C" int Stk3DFMM_evaluate_near_device(Stk3DFMM *fmm, unsigned kernel, const double *d_src_SL_value,
                                             double *d_trg_value, const double *d_src_DL_value, void *stream) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready) return STK_ERR_STATE;
    // device values are used as given: the caller's box must be the unit box (scaleSrc is then the identity)
    if (fmm->scale_factor != 1.0) return STK_ERR_NOT_SUPPORTED;
    const bool dl = has_dl(kd) && fmm->ndl > 0;
    if ((fmm->nsl > 0 && !d_src_SL_value) || (dl && !d_src_DL_value) || (fmm->ntrg > 0 && !d_trg_value))
        return STK_ERR_INVALID_ARG;
    cudaSetDevice(fmm->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : fmm->stream;
    return near_device(fmm, kd, d_src_SL_value, dl ? d_src_DL_value : nullptr, d_trg_value, s, false);
}

extern "C" int Stk3DFMM_last_kernel_ms(Stk3DFMM *fmm, unsigned kernel, float *ms) {
    if (!fmm || !ms) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->timed) return STK_ERR_STATE;
    if (cudaEventSynchronize(kd->ev1) != cudaSuccess) return STK_ERR_CUDA;
    if (cudaEventElapsedTime(ms, kd->ev0, kd->ev1) != cudaSuccess) return STK_ERR_CUDA;
    return kd->last_far ? farfield_status(kd) : STK_OK;
}

extern "C" int Stk3DFMM_last_phase_ms(Stk3DFMM *fmm, unsigned kernel, float *ms) {
    if (!fmm || !ms) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->timed) return STK_ERR_STATE;
    if (cudaEventSynchronize(kd->ev1) != cudaSuccess) return STK_ERR_CUDA;
    const int np = kd->last_far ? KernelData::kPhases : 1;
    cudaEvent_t prev = kd->ev0;
    for (int i = 0; i < KernelData::kPhases; i++) {
        ms[i] = 0.0f;
        if (i >= np) continue;
        if (cudaEventElapsedTime(&ms[i], prev, kd->ph[i]) != cudaSuccess) return STK_ERR_CUDA;
        prev = kd->ph[i];
    }
    return STK_OK;
}

extern "C" int Stk3DFMM_last_launch_count(Stk3DFMM *fmm, unsigned kernel, int *count) {
    if (!fmm || !count) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->timed) return STK_ERR_STATE;
    *count = kd->launches;
    return STK_OK;
}

extern "C" int Stk3DFMM_get_tree_stats(Stk3DFMM *fmm, unsigned kernel, long long *out) {
    if (!fmm || !out) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready) return STK_ERR_STATE;
    const Octree &T = kd->tree;
    out[0] = T.num_nodes();
    out[1] = (long long)T.leaves.size();
    out[2] = T.depth();
    out[3] = (long long)T.U.size();
    out[4] = kd->u_pairs[0];
    out[5] = kd->u_pairs[1];
    out[6] = (long long)T.V.size();
    out[7] = (long long)T.W.size();
    out[8] = (long long)T.X.size();
    return STK_OK;
}

extern "C" int Stk3DFMM_get_m2l_work(Stk3DFMM *fmm, unsigned kernel, double *out) {
    if (!fmm || !out) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready || !kd->far_ready) return STK_ERR_STATE;
    out[0] = kd->far->m2l_flops_alg;
    out[1] = kd->far->m2l_flops;
    return STK_OK;
}

extern "C" int Stk3DFMM_get_fmm_stats(Stk3DFMM *fmm, unsigned kernel, long long *out) {
    if (!fmm || !out) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready || !kd->far_ready) return STK_ERR_STATE;
    const FarField &F = *kd->far;
    out[0] = F.near[0].pairs;
    out[1] = kd->fused ? F.near[0].pairs : F.near[1].pairs;
    out[2] = F.s2m[0].pairs + F.s2m[1].pairs;
    out[3] = F.s2l[0].pairs + F.s2l[1].pairs;
    out[4] = F.m2t.pairs;
    out[5] = F.l2t.pairs;
    out[6] = F.m2l_pairs;
    out[7] = F.n;
    out[8] = F.m2l_rank;
    out[9] = kd->launches;
    return STK_OK;
}

extern "C" int Stk3DFMM_get_ulist(Stk3DFMM *fmm, unsigned kernel, int *sizes, int *trg_begin, int *trg_end,
                                  int *list_off, int *list_ent, int *sl_begin, int *sl_end, int *dl_begin,
                                  int *dl_end, int *sl_perm, int *dl_perm, int *trg_perm) {
    if (!fmm || !sizes) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready) return STK_ERR_STATE;
    const Octree &T = kd->tree;
    const int nn = T.num_nodes();
    sizes[0] = nn;
    sizes[1] = (int)T.U.size();
    sizes[2] = T.sets[0].n;
    sizes[3] = T.sets[1].n;
    sizes[4] = T.sets[2].n;
    auto cp = [](int *dst, const std::vector<int> &v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int));
    };
    cp(trg_begin, T.sets[2].node_begin);
    cp(trg_end, T.sets[2].node_end);
    cp(list_off, T.U.off);
    cp(list_ent, T.U.ent);
    cp(sl_begin, T.sets[0].node_begin);
    cp(sl_end, T.sets[0].node_end);
    cp(dl_begin, T.sets[1].node_begin);
    cp(dl_end, T.sets[1].node_end);
    cp(sl_perm, T.sets[0].perm);
    cp(dl_perm, T.sets[1].perm);
    cp(trg_perm, T.sets[2].perm);
    return STK_OK;
}

// The KIFMM operators and per-tree far-field data are built at the first
// evaluation after setupTree (the reference builds them in setupTree,
// FMMData.cpp:107-167); evaluate_near never needs them.
static int ensure_far(Stk3DFMM *fmm, KernelData *kd) {
    if (kd->far_ready) return STK_OK;
    const int rc = farfield_setup(fmm, kd);
    if (rc) return rc;
    kd->far_ready = true;
    return STK_OK;
}

extern "C" int Stk3DFMM_evaluate_fmm(Stk3DFMM *fmm, unsigned kernel, const int nSL, double *src_SL_value,
                                     const int nTrg, double *trg_value, const int nDL, double *src_DL_value) {
    return eval_host(fmm, kernel, nSL, src_SL_value, nTrg, trg_value, nDL, src_DL_value, true);
}

extern "C" int Stk3DFMM_evaluate_fmm_device(Stk3DFMM *fmm, unsigned kernel, const double *d_src_SL_value,
                                            double *d_trg_value, const double *d_src_DL_value, void *stream) {
    if (!fmm) return STK_ERR_INVALID_ARG;
    KernelData *kd = get_kd(fmm, kernel);
    if (!kd) return STK_ERR_KERNEL;
    if (!kd->tree_ready) return STK_ERR_STATE;
    if (fmm->scale_factor != 1.0) return STK_ERR_NOT_SUPPORTED;
    const bool dl = has_dl(kd) && fmm->ndl > 0;
    if ((fmm->nsl > 0 && !d_src_SL_value) || (dl && !d_src_DL_value) || (fmm->ntrg > 0 && !d_trg_value))
        return STK_ERR_INVALID_ARG;
    cudaSetDevice(fmm->device);
    const int rc = ensure_far(fmm, kd);
    if (rc) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : fmm->stream;
    return near_device(fmm, kd, d_src_SL_value, dl ? d_src_DL_value : nullptr, d_trg_value, s, true);
}

extern "C" int Stk3DFMM_evaluate_kernel(Stk3DFMM *fmm, unsigned kernel, int nThreads, unsigned p2p, int nSrc,
                                        double *srcCoord, double *srcValue, int nTrg, double *trgCoord,
                                        double *trgValue) {
    (void)nThreads;  // the GPU path ignores the OpenMP thread count
    if (!fmm) return STK_ERR_INVALID_ARG;
    if (!get_kd(fmm, kernel)) return STK_ERR_KERNEL;  // STKFMM.cpp:91-95
    cudaSetDevice(fmm->device);
    return stk_evaluate_kernel(kernel, p2p, nSrc, srcCoord, srcValue, nTrg, trgCoord, trgValue, fmm->precision);
}
