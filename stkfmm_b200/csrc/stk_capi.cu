// stk_capi.cu -- C ABI of the B200 STKFMM kernel-evaluation path.
//
// See include/stkfmm_b200.h for the contract of each entry point and the
// reference interface it replaces.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/stkfmm_b200.h"
#include "stk_kernel_table.hpp"
#include "stk_p2p.cuh"
#include "stk_tree.hpp"
#include "stk_umma.cuh"
#include "stk_work.hpp"

using namespace stk;

// ---------------------------------------------------------------------------
// verbosity: the reference's STKFMM_VERBOSE switch (Lib/src/STKFMM.cpp:7-16)
// ---------------------------------------------------------------------------
static bool stk_verbose() {
    static const bool v = [] {
        const char *e = getenv("STKFMM_VERBOSE");
        return !(e == nullptr || e[0] == '0');
    }();
    return v;
}

extern "C" const char *stk_status_string(int status) {
    switch (status) {
    case STK_OK: return "ok";
    case STK_ERR_INVALID_ARG: return "invalid argument";
    case STK_ERR_KERNEL: return "kernel not activated or sub-kernel not available";
    case STK_ERR_STATE: return "call order: set_points/setup_tree missing";
    case STK_ERR_SIZE: return "point/value count mismatch";
    case STK_ERR_CUDA: return "CUDA runtime error";
    case STK_ERR_NO_DEVICE: return "no CUDA device (this library has no CPU path)";
    case STK_ERR_OUT_OF_BOX: return "point outside the FMM box";
    case STK_ERR_NOT_SUPPORTED: return "not supported by this library";
    default: return "unknown status";
    }
}

extern "C" int stk_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" int stk_get_kernel_dimension(unsigned kernel, int *dims) {
    const KernelInfo *k = find_kernel(kernel);
    if (!k) return STK_ERR_KERNEL;
    if (!dims) return STK_ERR_INVALID_ARG;
    dims[0] = k->kdim_sl;
    dims[1] = k->kdim_dl;
    dims[2] = k->kdim_trg;
    return STK_OK;
}

// The factors applied around the unit-box FMM for a box with scale factor sf,
// read from the same table fields the evaluation uses (scaleSrc / scaleTrg of
// Lib/src/FMMData.cpp:285-470): the trailing sl_last_scales single-layer
// components, every double-layer value, and each target component to the power
// trg_scale_pow.  Host only.
extern "C" int stk_kernel_scaling(unsigned kernel, double sf, double *sl, double *dl, double *trg) {
    const KernelInfo *k = find_kernel(kernel);
    if (!k) return STK_ERR_KERNEL;
    if (!sl || !dl || !trg) return STK_ERR_INVALID_ARG;
    for (int c = 0; c < k->kdim_sl; c++) sl[c] = c >= k->kdim_sl - k->sl_last_scales ? sf : 1.0;
    for (int c = 0; c < k->kdim_dl; c++) dl[c] = sf;
    for (int c = 0; c < k->kdim_trg; c++) trg[c] = std::pow(sf, k->trg_scale_pow[c]);
    return STK_OK;
}

extern "C" const char *stk_get_kernel_name(unsigned kernel) {
    const KernelInfo *k = find_kernel(kernel);
    return k ? k->name : nullptr;
}

extern "C" int stk_kernel_slot(unsigned kernel, int slot) {
    const KernelInfo *k = find_kernel(kernel);
    if (!k || slot < 0 || slot >= SLOT_COUNT) return -1;
    return k->slot[slot];
}

extern "C" int stk_ukernel_dims(int uk, int *sdim, int *tdim) {
    if (uk < 0 || uk >= UK_COUNT || !sdim || !tdim) return STK_ERR_INVALID_ARG;
    *sdim = uk_sdim_host(uk);
    *tdim = uk_tdim_host(uk);
    return STK_OK;
}

extern "C" int stk_ukernel_aux_dim(int uk) { return (uk < 0 || uk >= UK_COUNT) ? -1 : uk_tvdim_host(uk); }

#define STK_CUDA(call)                                                                                     \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) {                                                                           \
            if (stk_verbose()) fprintf(stderr, "stkfmm_b200: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return STK_ERR_CUDA;                                                                           \
        }                                                                                                  \
    } while (0)

// ---------------------------------------------------------------------------
// direct sum on device pointers
// ---------------------------------------------------------------------------
static int direct_device(int uk, int nsrc, const double *d_src, const double *d_val, int ntrg, const double *d_trg,
                         double *d_out, int prec, cudaStream_t stream, Workspace &ws,
                         const double *d_trg_aux = nullptr) {
    if (uk < 0 || uk >= UK_COUNT || nsrc < 0 || ntrg < 0) return STK_ERR_INVALID_ARG;
    if (prec != PREC_FP64 && prec != PREC_MIXED) return STK_ERR_INVALID_ARG;
    if (nsrc == 0 || ntrg == 0) return STK_OK;
    if (!d_src || !d_val || !d_trg || !d_out) return STK_ERR_INVALID_ARG;
    if ((uk_tvdim_host(uk) > 0) != (d_trg_aux != nullptr)) return STK_ERR_INVALID_ARG;
    int rc = ws.ensure_device();
    if (rc) return rc;
    if ((rc = ws.begin(stream))) return rc;
    const int sd = uk_sdim_host(uk);
    const int rs = uk_record_stride(uk);
    // source records
    double *rec = ws.buf<double>(Workspace::kRec, (size_t)nsrc * rs);
    if (!rec) return STK_ERR_CUDA;
    STK_CUDA(launch_pack_records(nsrc, nullptr, d_src, d_val, sd, nullptr, 0, rs, rec, stream));
    // work list: 64-target chunks x source chunks
    std::vector<WorkItem> items;
    std::vector<int> sbeg, send, ent;
    build_direct_items(ntrg, nsrc, ws.num_sms(), items, sbeg, send, ent);
    int *d_sbeg = ws.buf<int>(Workspace::kSrcBeg, sbeg.size());
    int *d_send = ws.buf<int>(Workspace::kSrcEnd, send.size());
    int *d_ent = ws.buf<int>(Workspace::kEnt, ent.size());
    WorkItem *d_items = ws.buf<WorkItem>(Workspace::kItems, items.size());
    if (!d_sbeg || !d_send || !d_ent || !d_items) return STK_ERR_CUDA;
    STK_CUDA(cudaMemcpyAsync(d_sbeg, sbeg.data(), sbeg.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    STK_CUDA(cudaMemcpyAsync(d_send, send.data(), send.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    STK_CUDA(cudaMemcpyAsync(d_ent, ent.data(), ent.size() * sizeof(int), cudaMemcpyHostToDevice, stream));
    STK_CUDA(cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, stream));
    ListP2PArgs a{};
    a.src_rec = rec;
    a.src_box_begin = d_sbeg;
    a.src_box_end = d_send;
    a.list_ent = d_ent;
    a.items = d_items;
    a.n_items = (int)items.size();
    a.counter = ws.counter();
    a.trg_xyz = d_trg;
    a.trg_out = d_out;
    a.box_centre = nullptr;  // per-item origin: the item's first target
    a.period = 1.0;
    a.atomic_out = sbeg.size() > 1 ? 1 : 0;
    a.trg_aux = d_trg_aux;
    STK_CUDA(launch_list_p2p(uk, prec, a, ws.num_sms(), stream));
    // the host vectors may die at return: copies from pageable memory have been
    // staged by the time cudaMemcpyAsync returns, so no host wait is needed
    if ((rc = ws.end(stream))) return rc;
    return STK_OK;
}

extern "C" int stk_ukernel_direct_device(int ukernel, int nsrc, const double *d_src_coord, const double *d_src_value,
                                         int ntrg, const double *d_trg_coord, double *d_trg_value, int precision,
                                         void *stream) {
    return direct_device(ukernel, nsrc, d_src_coord, d_src_value, ntrg, d_trg_coord, d_trg_value, precision,
                         (cudaStream_t)stream, Workspace::thread_local_ws());
}

extern "C" int stk_ukernel_direct_aux_device(int ukernel, int nsrc, const double *d_src_coord,
                                             const double *d_src_value, int ntrg, const double *d_trg_coord,
                                             const double *d_trg_aux, double *d_trg_value, int precision,
                                             void *stream) {
    return direct_device(ukernel, nsrc, d_src_coord, d_src_value, ntrg, d_trg_coord, d_trg_value, precision,
                         (cudaStream_t)stream, Workspace::thread_local_ws(), d_trg_aux);
}

static int pick_ppkernel(unsigned kernel, unsigned ppkernel, int &uk) {
    const KernelInfo *k = find_kernel(kernel);
    if (!k) return STK_ERR_KERNEL;
    int slot = -1;
    if (ppkernel == STK_SLS2T) slot = SLOT_S2T_SL;
    else if (ppkernel == STK_DLS2T) slot = SLOT_S2T_DL;
    else if (ppkernel == STK_L2T) slot = SLOT_L2T;
    else return STK_ERR_INVALID_ARG;
    if (!kernel_supported(k)) return STK_ERR_NOT_SUPPORTED;
    uk = k->slot[slot];
    return uk < 0 ? STK_ERR_KERNEL : STK_OK;
}

extern "C" int stk_evaluate_kernel_device(unsigned kernel, unsigned ppkernel, int nsrc, const double *d_src_coord,
                                          const double *d_src_value, int ntrg, const double *d_trg_coord,
                                          double *d_trg_value, int precision, void *stream) {
    int uk = -1;
    int rc = pick_ppkernel(kernel, ppkernel, uk);
    if (rc) return rc;
    return direct_device(uk, nsrc, d_src_coord, d_src_value, ntrg, d_trg_coord, d_trg_value, precision,
                         (cudaStream_t)stream, Workspace::thread_local_ws());
}

// Host-array direct sum for micro-kernel uk (accumulate).  Targets are sorted in
// Morton order before upload so that 64-target items are compact (tight local
// origins for the mixed path); results are scattered back to the caller's order.
static int direct_host(int uk, int nsrc, const double *src, const double *val, int ntrg, const double *trg,
                       double *out, int prec) {
    if (uk < 0 || uk >= UK_COUNT || nsrc < 0 || ntrg < 0 || uk_tvdim_host(uk) > 0) return STK_ERR_INVALID_ARG;
    if (prec != PREC_FP64 && prec != PREC_MIXED) return STK_ERR_INVALID_ARG;
    if (nsrc == 0 || ntrg == 0) return STK_OK;
    if (!src || !val || !trg || !out) return STK_ERR_INVALID_ARG;
    Workspace &ws = Workspace::thread_local_ws();
    int rc = ws.ensure_device();
    if (rc) return rc;
    cudaStream_t s = ws.stream();
    const int sd = uk_sdim_host(uk), td = uk_tdim_host(uk);
    std::vector<int> order;
    std::vector<double> trg_sorted;
    morton_order(trg, ntrg, order, trg_sorted);
    double *d_src = ws.buf<double>(Workspace::kHostSrc, (size_t)nsrc * 3);
    double *d_val = ws.buf<double>(Workspace::kHostVal, (size_t)nsrc * sd);
    double *d_trg = ws.buf<double>(Workspace::kHostTrg, (size_t)ntrg * 3);
    double *d_out = ws.buf<double>(Workspace::kHostOut, (size_t)ntrg * td);
    if (!d_src || !d_val || !d_trg || !d_out) return STK_ERR_CUDA;
    STK_CUDA(cudaMemcpyAsync(d_src, src, sizeof(double) * 3 * nsrc, cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemcpyAsync(d_val, val, sizeof(double) * sd * nsrc, cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemcpyAsync(d_trg, trg_sorted.data(), sizeof(double) * 3 * ntrg, cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * td * ntrg, s));
    rc = direct_device(uk, nsrc, d_src, d_val, ntrg, d_trg, d_out, prec, s, ws);
    if (rc) return rc;
    std::vector<double> res((size_t)ntrg * td);
    STK_CUDA(cudaMemcpyAsync(res.data(), d_out, sizeof(double) * td * ntrg, cudaMemcpyDeviceToHost, s));
    STK_CUDA(cudaStreamSynchronize(s));
    for (int i = 0; i < ntrg; i++)
        for (int k = 0; k < td; k++) out[(size_t)order[i] * td + k] += res[(size_t)i * td + k];
    return STK_OK;
}

extern "C" int stk_evaluate_kernel(unsigned kernel, unsigned ppkernel, int nsrc, const double *src_coord,
                                   const double *src_value, int ntrg, const double *trg_coord, double *trg_value,
                                   int precision) {
    int uk = -1;
    int rc = pick_ppkernel(kernel, ppkernel, uk);
    if (rc) return rc;
    return direct_host(uk, nsrc, src_coord, src_value, ntrg, trg_coord, trg_value, precision);
}

// ---------------------------------------------------------------------------
// list-level P2P
// ---------------------------------------------------------------------------
static int p2p_lists(int ukernel, int precision, int n_trg_box, const int *trg_begin, const int *trg_end,
                     const int *list_off, const int *list_ent, int n_src_box, const int *src_begin, const int *src_end,
                     int nsrc, const double *d_src_coord, const double *d_src_value, int ntrg,
                     const double *d_trg_coord, const double *d_trg_aux, double *d_trg_value, double period,
                     void *stream) {
    if (ukernel < 0 || ukernel >= UK_COUNT || n_trg_box < 0 || n_src_box < 0 || nsrc < 0 || ntrg < 0)
        return STK_ERR_INVALID_ARG;
    if (precision != PREC_FP64 && precision != PREC_MIXED) return STK_ERR_INVALID_ARG;
    if (n_trg_box == 0 || ntrg == 0) return STK_OK;
    if (!trg_begin || !trg_end || !list_off || (list_off[n_trg_box] > 0 && !list_ent)) return STK_ERR_INVALID_ARG;
    if (n_src_box > 0 && (!src_begin || !src_end)) return STK_ERR_INVALID_ARG;
    // validate every index before anything reaches the GPU
    if (list_off[0] != 0) return STK_ERR_INVALID_ARG;
    for (int b = 0; b < n_trg_box; b++) {
        if (trg_begin[b] < 0 || trg_end[b] < trg_begin[b] || trg_end[b] > ntrg) return STK_ERR_INVALID_ARG;
        if (list_off[b + 1] < list_off[b]) return STK_ERR_INVALID_ARG;
    }
    for (int s = 0; s < n_src_box; s++)
        if (src_begin[s] < 0 || src_end[s] < src_begin[s] || src_end[s] > nsrc) return STK_ERR_INVALID_ARG;
    const int nent = list_off[n_trg_box];
    for (int e = 0; e < nent; e++) {
        const int sb = list_ent[e] >> 5, code = list_ent[e] & 31;
        if (list_ent[e] < 0 || sb >= n_src_box || code > 26) return STK_ERR_INVALID_ARG;
    }
    if (nsrc > 0 && (!d_src_coord || !d_src_value)) return STK_ERR_INVALID_ARG;
    if (!d_trg_coord || !d_trg_value) return STK_ERR_INVALID_ARG;
    if ((uk_tvdim_host(ukernel) > 0) != (d_trg_aux != nullptr)) return STK_ERR_INVALID_ARG;
    Workspace &ws = Workspace::thread_local_ws();
    int rc = ws.ensure_device();
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if ((rc = ws.begin(s))) return rc;
    std::vector<WorkItem> items;
    long long pairs = 0;
    build_list_items(n_trg_box, trg_begin, trg_end, list_off, list_ent, src_begin, src_end, items, pairs);
    if (items.empty()) return STK_OK;
    const int sd = uk_sdim_host(ukernel), rs = uk_record_stride(ukernel);
    double *rec = ws.buf<double>(Workspace::kRec, (size_t)std::max(nsrc, 1) * rs);
    int *d_sbeg = ws.buf<int>(Workspace::kSrcBeg, n_src_box);
    int *d_send = ws.buf<int>(Workspace::kSrcEnd, n_src_box);
    int *d_ent = ws.buf<int>(Workspace::kEnt, nent);
    WorkItem *d_items = ws.buf<WorkItem>(Workspace::kItems, items.size());
    if (!rec || !d_sbeg || !d_send || !d_ent || !d_items) return STK_ERR_CUDA;
    STK_CUDA(launch_pack_records(nsrc, nullptr, d_src_coord, d_src_value, sd, nullptr, 0, rs, rec, s));
    STK_CUDA(cudaMemcpyAsync(d_sbeg, src_begin, n_src_box * sizeof(int), cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemcpyAsync(d_send, src_end, n_src_box * sizeof(int), cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemcpyAsync(d_ent, list_ent, nent * sizeof(int), cudaMemcpyHostToDevice, s));
    STK_CUDA(cudaMemcpyAsync(d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, s));
    ListP2PArgs a{};
    a.src_rec = rec;
    a.src_box_begin = d_sbeg;
    a.src_box_end = d_send;
    a.list_ent = d_ent;
    a.items = d_items;
    a.n_items = (int)items.size();
    a.counter = ws.counter();
    a.trg_xyz = d_trg_coord;
    a.trg_out = d_trg_value;
    a.box_centre = nullptr;
    a.period = period;
    a.atomic_out = 0;
    a.trg_aux = d_trg_aux;
    STK_CUDA(launch_list_p2p(ukernel, precision, a, ws.num_sms(), s));
    return ws.end(s);  // queued: no host wait (see direct_device)
}

extern "C" int stk_p2p_lists(int ukernel, int precision, int n_trg_box, const int *trg_begin, const int *trg_end,
                             const int *list_off, const int *list_ent, int n_src_box, const int *src_begin,
                             const int *src_end, int nsrc, const double *d_src_coord, const double *d_src_value,
                             int ntrg, const double *d_trg_coord, double *d_trg_value, double period, void *stream) {
    return p2p_lists(ukernel, precision, n_trg_box, trg_begin, trg_end, list_off, list_ent, n_src_box, src_begin,
                     src_end, nsrc, d_src_coord, d_src_value, ntrg, d_trg_coord, nullptr, d_trg_value, period, stream);
}

extern "C" int stk_p2p_lists_aux(int ukernel, int precision, int n_trg_box, const int *trg_begin, const int *trg_end,
                                 const int *list_off, const int *list_ent, int n_src_box, const int *src_begin,
                                 const int *src_end, int nsrc, const double *d_src_coord, const double *d_src_value,
                                 int ntrg, const double *d_trg_coord, const double *d_trg_aux, double *d_trg_value,
                                 double period, void *stream) {
    return p2p_lists(ukernel, precision, n_trg_box, trg_begin, trg_end, list_off, list_ent, n_src_box, src_begin,
                     src_end, nsrc, d_src_coord, d_src_value, ntrg, d_trg_coord, d_trg_aux, d_trg_value, period,
                     stream);
}

// ---------------------------------------------------------------------------
// the tensor-core GEMM of the mixed M2L (3xTF32 on tcgen05), for direct use and tests
// ---------------------------------------------------------------------------
extern "C" int stk_gemm_3xtf32(int M, int N, int K, const float *d_A, int lda, const float *d_B, int ldb, float *d_C,
                               int ldc, int beta, void *stream) {
    if (M < 0 || N < 0 || K < 0 || (beta != 0 && beta != 1)) return STK_ERR_INVALID_ARG;
    if (M == 0 || N == 0) return STK_OK;
    if (!d_A || !d_B || !d_C || lda < K || ldb < K || ldc < M) return STK_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return STK_ERR_NO_DEVICE;
    }
    if (!umma_available()) return STK_ERR_NOT_SUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    const int la = (K + 3) / 4 * 4;
    float *buf = nullptr;
    int *err = nullptr;
    const size_t na = (size_t)M * la, nb = (size_t)N * la;
    if (cudaMalloc(&buf, sizeof(float) * 2 * (na + nb) + 64) != cudaSuccess) {
        cudaGetLastError();
        return STK_ERR_CUDA;
    }
    err = reinterpret_cast<int *>(buf + 2 * (na + nb));
    float *ah = buf, *al = ah + na, *bh = al + na, *bl = bh + nb;
    // K-major copies padded to a multiple of 4 floats per row, split into hi / lo
    int rc = STK_OK;
    if (cudaMemsetAsync(buf, 0, sizeof(float) * 2 * (na + nb) + 64, s) != cudaSuccess ||
        cudaMemcpy2DAsync(ah, sizeof(float) * la, d_A, sizeof(float) * lda, sizeof(float) * K, M,
                          cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpy2DAsync(bh, sizeof(float) * la, d_B, sizeof(float) * ldb, sizeof(float) * K, N,
                          cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        tf32_split(ah, (long long)na, ah, al, s) != cudaSuccess || tf32_split(bh, (long long)nb, bh, bl, s) != cudaSuccess ||
        umma_gemm_3xtf32(M, N, K, Tf32Split{ah, al, la}, Tf32Split{bh, bl, la}, d_C, ldc, beta, err, s) != cudaSuccess)
        rc = STK_ERR_CUDA;
    int e = 0;
    if (!rc && (cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess))
        rc = STK_ERR_CUDA;
    if (!rc && e) rc = STK_ERR_CUDA;
    cudaStreamSynchronize(s);
    cudaFree(buf);
    cudaGetLastError();
    return rc;
}

// ---------------------------------------------------------------------------
// ker_poten shims
// ---------------------------------------------------------------------------
static thread_local int g_last_ker_status = STK_OK;
extern "C" int stk_ker_last_status(void) { return g_last_ker_status; }

static void ker_shim(int uk, double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt,
                     double *k_out) {
    if (dof != 1) {
        g_last_ker_status = STK_ERR_NOT_SUPPORTED;
        return;
    }
    g_last_ker_status = direct_host(uk, src_cnt, r_src, v_src, trg_cnt, r_trg, k_out, PREC_FP64);
}

#define STK_KER_SHIM(NAME, UK)                                                                                    \
    extern "C" void stk_ker_##NAME(double *r_src, int src_cnt, double *v_src, int dof, double *r_trg, int trg_cnt, \
                                   double *k_out, void *) {                                                       \
        ker_shim(UK, r_src, src_cnt, v_src, dof, r_trg, trg_cnt, k_out);                                          \
    }
STK_KER_SHIM(laplace_p, UK_LAPLACE_P)
STK_KER_SHIM(laplace_pgrad, UK_LAPLACE_PGRAD)
STK_KER_SHIM(laplace_dipolep, UK_LAPLACE_DIPOLEP)
STK_KER_SHIM(laplace_dipolepgrad, UK_LAPLACE_DIPOLEPGRAD)
STK_KER_SHIM(stokes_vel, UK_STOKES_VEL)
STK_KER_SHIM(rpy_u, UK_RPY_U)
STK_KER_SHIM(rpy_ulapu, UK_RPY_ULAPU)
STK_KER_SHIM(stk_ulapu, UK_STK_ULAPU)
STK_KER_SHIM(stokes_regvel, UK_STOKES_REGVEL)
STK_KER_SHIM(stokes_pvel, UK_STOKES_PVEL)
STK_KER_SHIM(stokes_doublepvel, UK_STOKES_DOUBLEPVEL)
STK_KER_SHIM(laplace_pgradgrad, UK_LAPLACE_PGRADGRAD)
STK_KER_SHIM(laplace_dipolepgradgrad, UK_LAPLACE_DIPOLEPGRADGRAD)
STK_KER_SHIM(laplace_quadp, UK_LAPLACE_QUADP)
STK_KER_SHIM(laplace_quadpgradgrad, UK_LAPLACE_QUADPGRADGRAD)
STK_KER_SHIM(stokes_pvelgrad, UK_STOKES_PVELGRAD)
STK_KER_SHIM(stokes_doublepvelgrad, UK_STOKES_DOUBLEPVELGRAD)
STK_KER_SHIM(stokes_pvellaplacian, UK_STOKES_PVELLAPLACIAN)
STK_KER_SHIM(stokes_doublelaplacian, UK_STOKES_DOUBLELAPLACIAN)
STK_KER_SHIM(stokes_traction, UK_STOKES_TRACTION)
STK_KER_SHIM(stokes_doubletraction, UK_STOKES_DOUBLETRACTION)
STK_KER_SHIM(stokes_regftvel, UK_STOKES_REGFTVEL)
STK_KER_SHIM(stokes_regftvelomega, UK_STOKES_REGFTVELOMEGA)
STK_KER_SHIM(stokes_velomega, UK_STOKES_VELOMEGA)
