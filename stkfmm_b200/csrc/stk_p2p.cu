// stk_p2p.cu -- sm_100a list P2P kernel: the U/W/X-list and direct-sum hot loop.
//
// Replaces the per-(target box, source box) ker_poten calls that PVFMM's
// PtFMM_Evaluate makes for the U-list (S2T), and the OpenMP target-chunk loop of
// FMMData::evaluateKernel (Lib/src/FMMData.cpp:252-283).
//
// Design (one warp = one work item, persistent warps):
//  * A work item is <= 32 targets of one target box plus a range of its
//    interaction-list entries.  Items are sorted by cost (targets x sources) on
//    the host, largest first, and persistent warps take them from a global
//    counter, so uneven adaptive trees balance themselves.
//  * The warp streams the sources of its list entries through a 32-record
//    shared-memory tile: lane i loads record i with 16-byte vector loads, the
//    next tile is prefetched into registers while the current one is consumed.
//  * Every lane owns one target (or, with fewer than 32 targets, a group of
//    2^glog lanes owns one target and splits the tile); the group is reduced with
//    warp shuffles at the end.
//  * FP64 path: everything in double, r = x_t - (x_s + image shift) exactly as
//    the oracle forms it.
//  * Mixed path: when a source record is staged its coordinates are shifted to
//    the target box's centre in FP64 and rounded to FP32 once; per pair the
//    displacement is an FP32 difference of two centre-relative coordinates, the
//    kernel tensor is FP32 with MUFU rsqrt + one Newton step, and each tile's
//    FP32 partial sum is added into a Kahan-compensated FP32 accumulator.
#include <algorithm>
#include <type_traits>

#include "stk_p2p.cuh"
#include "stk_ukernels.cuh"

namespace stk {

namespace {

constexpr int kWarpsPerCta = 4;
constexpr int kThreads = 32 * kWarpsPerCta;
constexpr unsigned kFull = 0xffffffffu;

template <int UK> struct Rec {
    static constexpr int SDIM = Uk<UK>::SDIM;
    static constexpr int RS = (3 + SDIM + 1) & ~1;   // doubles per global/FP64 record (16-byte multiple)
    static constexpr int RSF = (3 + SDIM + 3) & ~3;  // floats per FP32 shared-memory record
};

// Load N doubles (N even) from 16-byte aligned global memory with double2 loads.
template <int N>
__device__ __forceinline__ void load_rec_global(double (&r)[N], const double *p) {
    static_assert(N % 2 == 0, "record stride must be even");
#pragma unroll
    for (int q = 0; q < N / 2; q++) {
        double2 v = __ldg(reinterpret_cast<const double2 *>(p) + q);
        r[2 * q] = v.x;
        r[2 * q + 1] = v.y;
    }
}

template <int N>
__device__ __forceinline__ void load_rec_shared(double (&r)[N], const double *p) {
#pragma unroll
    for (int q = 0; q < N / 2; q++) {
        double2 v = reinterpret_cast<const double2 *>(p)[q];
        r[2 * q] = v.x;
        r[2 * q + 1] = v.y;
    }
}

template <int N>
__device__ __forceinline__ void load_rec_shared(float (&r)[N], const float *p) {
#pragma unroll
    for (int q = 0; q < N / 4; q++) {
        float4 v = reinterpret_cast<const float4 *>(p)[q];
        r[4 * q] = v.x;
        r[4 * q + 1] = v.y;
        r[4 * q + 2] = v.z;
        r[4 * q + 3] = v.w;
    }
}

template <int UK, bool MIXED>
__global__ void __launch_bounds__(kThreads) list_p2p_kernel(const ListP2PArgs a) {
    using K = Uk<UK>;
    constexpr int SDIM = K::SDIM;
    constexpr int TDIM = K::TDIM;
    constexpr int RS = Rec<UK>::RS;
    using R = typename std::conditional<MIXED, float, double>::type;
    constexpr int SREC = MIXED ? Rec<UK>::RSF : RS;

    __shared__ __align__(16) R tile[kWarpsPerCta][32 * SREC];
    const int lane = threadIdx.x & 31;
    R *my = tile[threadIdx.x >> 5];

    for (;;) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(a.counter, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (it >= a.n_items) break;
        const WorkItem w = a.items[it];
        const int glog = w.glog;
        const int g = 1 << glog;
        const int ti = lane >> glog;
        const int sub = lane & (g - 1);
        const bool active = ti < w.nt;
        const int t = w.t0 + (active ? ti : 0);

        const double xt = a.trg_xyz[3 * (size_t)t + 0];
        const double yt = a.trg_xyz[3 * (size_t)t + 1];
        const double zt = a.trg_xyz[3 * (size_t)t + 2];
        double cx = 0.0, cy = 0.0, cz = 0.0;
        if constexpr (MIXED) {
            // local origin: the target box centre, or the item's first target
            const double *o = a.box_centre ? a.box_centre + 3 * (size_t)w.trg_box : a.trg_xyz + 3 * (size_t)w.t0;
            cx = o[0];
            cy = o[1];
            cz = o[2];
        }
        const R tx = R(xt - cx), ty = R(yt - cy), tz = R(zt - cz);

        R acc[TDIM], comp[TDIM];
#pragma unroll
        for (int k = 0; k < TDIM; k++) acc[k] = comp[k] = R(0);

        // ---- tile iterator over the source records of entries [e0, e1) ----
        int e = w.e0, base = 0, end = 0;
        double shx = 0.0, shy = 0.0, shz = 0.0;
        auto open_entry = [&](int ee) {
            const int ent = a.list_ent[ee];
            const int sb = ent >> 5;
            const int code = ent & 31;
            base = a.src_box_begin[sb];
            end = a.src_box_end[sb];
            shx = (code % 3 - 1) * a.period;
            shy = ((code / 3) % 3 - 1) * a.period;
            shz = (code / 9 - 1) * a.period;
        };
        while (e < w.e1) {
            open_entry(e);
            if (base < end) break;
            e++;
        }
        bool have = e < w.e1;
        double rn[RS];
        if (have && lane < end - base) load_rec_global(rn, a.src_rec + (size_t)(base + lane) * RS);

        while (have) {
            const int n = min(32, end - base);
            // stage this lane's record of the current tile
            if (lane < n) {
                const double sx = rn[0] + shx, sy = rn[1] + shy, sz = rn[2] + shz;
                R *d = my + lane * SREC;
                if constexpr (MIXED) {
                    float4 *d4 = reinterpret_cast<float4 *>(d);
                    float v[SREC];
                    v[0] = float(sx - cx);
                    v[1] = float(sy - cy);
                    v[2] = float(sz - cz);
#pragma unroll
                    for (int q = 0; q < SDIM; q++) v[3 + q] = float(rn[3 + q]);
#pragma unroll
                    for (int q = 3 + SDIM; q < SREC; q++) v[q] = 0.0f;
#pragma unroll
                    for (int q = 0; q < SREC / 4; q++) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                } else {
                    double2 *d2 = reinterpret_cast<double2 *>(d);
                    double v[RS];
                    v[0] = sx;
                    v[1] = sy;
                    v[2] = sz;
#pragma unroll
                    for (int q = 3; q < RS; q++) v[q] = rn[q];
#pragma unroll
                    for (int q = 0; q < RS / 2; q++) d2[q] = make_double2(v[2 * q], v[2 * q + 1]);
                }
            }
            // advance to the next tile and prefetch it
            base += 32;
            if (base >= end) {
                e++;
                while (e < w.e1) {
                    open_entry(e);
                    if (base < end) break;
                    e++;
                }
                have = e < w.e1;
            }
            if (have && lane < end - base) load_rec_global(rn, a.src_rec + (size_t)(base + lane) * RS);
            __syncwarp();

            if (active) {
                if constexpr (MIXED) {
                    R part[TDIM];
#pragma unroll
                    for (int k = 0; k < TDIM; k++) part[k] = R(0);
#pragma unroll 4
                    for (int j = sub; j < n; j += g) {
                        R s[SREC];
                        load_rec_shared(s, my + j * SREC);
                        K::eval(part, tx - s[0], ty - s[1], tz - s[2], s + 3);
                    }
                    // Kahan-compensated accumulation of the tile's partial sum
#pragma unroll
                    for (int k = 0; k < TDIM; k++) {
                        const R y = part[k] - comp[k];
                        const R tt = acc[k] + y;
                        comp[k] = (tt - acc[k]) - y;
                        acc[k] = tt;
                    }
                } else {
#pragma unroll 4
                    for (int j = sub; j < n; j += g) {
                        R s[SREC];
                        load_rec_shared(s, my + j * SREC);
                        K::eval(acc, tx - s[0], ty - s[1], tz - s[2], s + 3);
                    }
                }
            }
            __syncwarp();
        }

        // ---- reduce the lanes that share a target, then accumulate ----
        double out[TDIM];
#pragma unroll
        for (int k = 0; k < TDIM; k++) {
            if constexpr (MIXED) out[k] = double(acc[k]) - double(comp[k]);
            else out[k] = acc[k];
        }
        for (int o = 1; o < g; o <<= 1) {
#pragma unroll
            for (int k = 0; k < TDIM; k++) out[k] += __shfl_xor_sync(kFull, out[k], o);
        }
        if (active && sub == 0) {
            double *dst = a.trg_out + (size_t)t * TDIM;
#pragma unroll
            for (int k = 0; k < TDIM; k++) {
                const double v = K::SCALE * out[k];
                if (a.atomic_out)
                    atomicAdd(dst + k, v);
                else
                    dst[k] += v;
            }
        }
    }
}

template <int UK, bool MIXED>
cudaError_t launch_impl(const ListP2PArgs &a, int num_sms, cudaStream_t stream) {
    static int blocks_per_sm = 0;
    if (blocks_per_sm == 0) {
        cudaError_t err =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, list_p2p_kernel<UK, MIXED>, kThreads, 0);
        if (err != cudaSuccess) return err;
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    long long want = ((long long)a.n_items + kWarpsPerCta - 1) / kWarpsPerCta;
    int grid = (int)std::max(1LL, std::min<long long>((long long)num_sms * blocks_per_sm, want));
    cudaError_t err = cudaMemsetAsync(a.counter, 0, sizeof(unsigned int), stream);
    if (err != cudaSuccess) return err;
    list_p2p_kernel<UK, MIXED><<<grid, kThreads, 0, stream>>>(a);
    return cudaGetLastError();
}

template <int UK>
cudaError_t launch_prec(int prec, const ListP2PArgs &a, int num_sms, cudaStream_t stream) {
    return prec == PREC_MIXED ? launch_impl<UK, true>(a, num_sms, stream) : launch_impl<UK, false>(a, num_sms, stream);
}

__global__ void pack_records_kernel(int n, const int *__restrict__ perm, const double *__restrict__ xyz,
                                    const double *__restrict__ v1, int d1, const double *__restrict__ v2, int d2,
                                    int stride, double *__restrict__ rec) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = perm ? perm[i] : i;
        double *r = rec + (size_t)i * stride;
        r[0] = xyz[3 * (size_t)i + 0];
        r[1] = xyz[3 * (size_t)i + 1];
        r[2] = xyz[3 * (size_t)i + 2];
        int q = 3;
        for (int k = 0; k < d1; k++) r[q++] = v1[(size_t)p * d1 + k];
        for (int k = 0; k < d2; k++) r[q++] = v2[(size_t)p * d2 + k];
        for (; q < stride; q++) r[q] = 0.0;
    }
}

__global__ void scatter_add_kernel(int n, int d, const int *__restrict__ perm, const double *__restrict__ in,
                                   const double *__restrict__ alpha, double *__restrict__ out) {
    const long long total = (long long)n * d;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(idx / d);
        const int k = (int)(idx - (long long)i * d);
        const int p = perm ? perm[i] : i;
        out[(size_t)p * d + k] += (alpha ? alpha[k] : 1.0) * in[idx];
    }
}

}  // namespace

int uk_sdim_host(int uk) { return uk_sdim(uk); }
int uk_tdim_host(int uk) { return uk_tdim(uk); }
double uk_scale_host(int uk) { return uk_scale(uk); }
int uk_record_stride(int uk) { return (3 + uk_sdim(uk) + 1) & ~1; }

cudaError_t launch_list_p2p(int uk, int prec, const ListP2PArgs &a, int num_sms, cudaStream_t stream) {
    if (a.n_items <= 0) return cudaSuccess;
    switch (uk) {
    case UK_LAPLACE_P: return launch_prec<UK_LAPLACE_P>(prec, a, num_sms, stream);
    case UK_LAPLACE_PGRAD: return launch_prec<UK_LAPLACE_PGRAD>(prec, a, num_sms, stream);
    case UK_LAPLACE_DIPOLEP: return launch_prec<UK_LAPLACE_DIPOLEP>(prec, a, num_sms, stream);
    case UK_LAPLACE_DIPOLEPGRAD: return launch_prec<UK_LAPLACE_DIPOLEPGRAD>(prec, a, num_sms, stream);
    case UK_STOKES_VEL: return launch_prec<UK_STOKES_VEL>(prec, a, num_sms, stream);
    case UK_RPY_U: return launch_prec<UK_RPY_U>(prec, a, num_sms, stream);
    case UK_RPY_ULAPU: return launch_prec<UK_RPY_ULAPU>(prec, a, num_sms, stream);
    case UK_STK_ULAPU: return launch_prec<UK_STK_ULAPU>(prec, a, num_sms, stream);
    case UK_STOKES_REGVEL: return launch_prec<UK_STOKES_REGVEL>(prec, a, num_sms, stream);
    case UK_STOKES_PVEL: return launch_prec<UK_STOKES_PVEL>(prec, a, num_sms, stream);
    case UK_STOKES_DOUBLEPVEL: return launch_prec<UK_STOKES_DOUBLEPVEL>(prec, a, num_sms, stream);
    case UK_LAPLACE_SLDL_PGRAD: return launch_prec<UK_LAPLACE_SLDL_PGRAD>(prec, a, num_sms, stream);
    case UK_STOKES_SLDL_PVEL: return launch_prec<UK_STOKES_SLDL_PVEL>(prec, a, num_sms, stream);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pack_records(int n, const int *perm, const double *xyz, const double *v1, int d1,
                                const double *v2, int d2, int stride, double *rec, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const int grid = std::min((n + threads - 1) / threads, 148 * 16);
    pack_records_kernel<<<grid, threads, 0, stream>>>(n, perm, xyz, v1, d1, v2, d2, stride, rec);
    return cudaGetLastError();
}

cudaError_t launch_scatter_add(int n, int d, const int *perm, const double *in, const double *alpha, double *out,
                               cudaStream_t stream) {
    if (n <= 0 || d <= 0) return cudaSuccess;
    const int threads = 256;
    const long long total = (long long)n * d;
    const int grid = (int)std::min<long long>((total + threads - 1) / threads, 148 * 16);
    scatter_add_kernel<<<grid, threads, 0, stream>>>(n, d, perm, in, alpha, out);
    return cudaGetLastError();
}

}  // namespace stk
