// stk_noalloc.cu -- a direct-sum entry point that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc / cudaFree during their
// run.  cudaMalloc and cudaFree synchronise the whole device, which stalls a
// caller that keeps several streams busy; some frameworks hand the whole device
// to their own caching allocator, so memory taken behind its back can make it
// fail; and some real-time or embedded hosts forbid run-time allocation
// outright.  stk_ukernel_direct_device keeps a per-thread workspace that grows
// with cudaMalloc; this variant instead works inside one fixed scratch array
// that the library reserves when it is loaded.
//
// Mechanics: the scratch is the file-scope array g_stk_noalloc_scratch below.
// Its host-side name is only a stand-in, so the device address is fetched with
// cudaGetSymbolAddress, once per device, the first time the entry point runs on
// that device (with that device current), and cached.  That first call therefore
// does set-up work and should come before any stream capture; so should the
// first call of each (micro-kernel, precision) pair, whose list-kernel instance
// runs a one-time occupancy query (and, with lazy module loading, its module
// load).  The cached address belongs to the device's primary context: after a
// cudaDeviceReset of that device the entry point must not be used again in the
// process.  Every call shares the array and leaves its contents behind: the
// work counter that must start at zero is cleared by each call, and two calls
// whose work overlaps on the GPU (different streams, or host threads, at the
// same time) race on the array.
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/stkfmm_b200.h"
#include "stk_p2p.cuh"
#include "stk_tree.hpp"

namespace {

// Fixed scratch capacity: 8 MiB, held by every GPU that loads the library.
constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kItemTargets = 64;

static __device__ __align__(256) unsigned char g_stk_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_addr[kNoAllocMaxDevices] = {};

inline size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Device address of the scratch array for the current device.
int noalloc_scratch(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return STK_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kNoAllocMaxDevices) return STK_ERR_NOT_SUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_stk_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return STK_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
    }
    *out = g_noalloc_addr[dev];
    return STK_OK;
}

__host__ __device__ inline int lanes_log2(int m) {
    int glog = 0;
    while (glog < 5 && (m << (glog + 1)) <= kItemTargets) glog++;
    return glog;
}

// Writes the work list of a direct sum (64-target chunks x source chunks of
// `sc` points) into the scratch.  Same decomposition as the allocating path.
__global__ void noalloc_direct_items_kernel(int ntrg, int nsrc, int nchunk, int nsc, int sc,
                                           stk::WorkItem *items, int *sbeg, int *send, int *ent) {
    const int total = nchunk * nsc;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int c = i / nsc, k = i - (i / nsc) * nsc;
        const int t0 = kItemTargets * c;
        const int m = min(kItemTargets, ntrg - t0);
        items[i] = stk::WorkItem{c, t0, m, lanes_log2(m), k, k + 1};
        if (c == 0) {
            sbeg[k] = k * sc;
            send[k] = min(nsrc, (k + 1) * sc);
            ent[k] = (k << 5) | stk::kShiftNone;
        }
    }
}

}  // namespace

extern "C" int stk_ukernel_direct_device_noalloc(int ukernel, int nsrc, const double *d_src_coord,
                                                 const double *d_src_value, int ntrg, const double *d_trg_coord,
                                                 double *d_trg_value, int precision, void *stream) {
    // every micro-kernel the allocating direct sum takes without per-target values
    // (the adjoint kernels, which need them, go through stk_ukernel_direct_aux_device)
    int sdim = 0, tdim = 0;
    if (stk_ukernel_dims(ukernel, &sdim, &tdim) != STK_OK || stk::uk_tvdim_host(ukernel) > 0 || nsrc < 0 || ntrg < 0)
        return STK_ERR_INVALID_ARG;
    if (precision != STK_FP64 && precision != STK_MIXED) return STK_ERR_INVALID_ARG;
    if (nsrc == 0 || ntrg == 0) return STK_OK;
    if (!d_src_coord || !d_src_value || !d_trg_coord || !d_trg_value) return STK_ERR_INVALID_ARG;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return STK_ERR_NO_DEVICE;
    }
    // work decomposition (as the allocating direct path)
    const long long nchunk = (ntrg + kItemTargets - 1) / kItemTargets;
    const long long want_items = (long long)(sms > 0 ? sms : 1) * 64;
    long long nsc = (want_items + nchunk - 1) / nchunk;
    if (nsc < 1) nsc = 1;
    if (nsc > (nsrc / 256 > 1 ? nsrc / 256 : 1)) nsc = nsrc / 256 > 1 ? nsrc / 256 : 1;
    long long sc = (nsrc + nsc - 1) / nsc;
    sc = (sc + 31) / 32 * 32;
    nsc = (nsrc + sc - 1) / sc;
    const long long nitems = nchunk * nsc;
    // scratch layout: counter | items | source-chunk ranges and entries | source records
    const int rs = stk::uk_record_stride(ukernel);
    const size_t off_items = 256;
    const size_t off_sbeg = round_up(off_items + (size_t)nitems * sizeof(stk::WorkItem), 256);
    const size_t off_send = round_up(off_sbeg + (size_t)nsc * sizeof(int), 256);
    const size_t off_ent = round_up(off_send + (size_t)nsc * sizeof(int), 256);
    const size_t off_rec = round_up(off_ent + (size_t)nsc * sizeof(int), 256);
    const size_t need = off_rec + (size_t)nsrc * rs * sizeof(double);
    if (need > kNoAllocScratchBytes) return STK_ERR_SIZE;  // beyond the fixed 8 MiB scratch

    void *base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    unsigned char *s = static_cast<unsigned char *>(base);
    cudaStream_t st = (cudaStream_t)stream;
    stk::WorkItem *items = reinterpret_cast<stk::WorkItem *>(s + off_items);
    int *sbeg = reinterpret_cast<int *>(s + off_sbeg);
    int *send = reinterpret_cast<int *>(s + off_send);
    int *ent = reinterpret_cast<int *>(s + off_ent);
    double *rec = reinterpret_cast<double *>(s + off_rec);

    const int threads = 256;
    const int grid = (int)((nitems + threads - 1) / threads < 1024 ? (nitems + threads - 1) / threads : 1024);
    noalloc_direct_items_kernel<<<grid, threads, 0, st>>>(ntrg, nsrc, (int)nchunk, (int)nsc, (int)sc, items, sbeg,
                                                          send, ent);
    if (cudaGetLastError() != cudaSuccess) return STK_ERR_CUDA;
    if (stk::launch_pack_records(nsrc, nullptr, d_src_coord, d_src_value, sdim, nullptr, 0, rs, rec, st) !=
        cudaSuccess)
        return STK_ERR_CUDA;
    stk::ListP2PArgs a{};
    a.src_rec = rec;
    a.src_box_begin = sbeg;
    a.src_box_end = send;
    a.list_ent = ent;
    a.items = items;
    a.n_items = (int)nitems;
    a.counter = reinterpret_cast<unsigned int *>(s);  // zeroed by the launch itself
    a.trg_xyz = d_trg_coord;
    a.trg_out = d_trg_value;
    a.box_centre = nullptr;
    a.period = 1.0;
    a.atomic_out = nsc > 1 ? 1 : 0;
    if (stk::launch_list_p2p(ukernel, precision, a, sms, st) != cudaSuccess) return STK_ERR_CUDA;
    return STK_OK;
}
