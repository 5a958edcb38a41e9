// stk_umma.cu -- sm_100a tensor-core GEMM (tcgen05 / TMEM / TMA) for the
// mixed-precision M2L: C (=|+=) A B to FP32 accuracy from TF32 products.
//
// FP32 accuracy from TF32 tensor cores ("3xTF32"): each operand is split into
// hi = the value rounded to TF32 (to nearest) and lo = the remainder, also
// rounded to TF32, so that both are exact tensor-core inputs and hi + lo carries
// the value to ~2^-24 relative; A B ~ Ah Bh + Ah Bl + Al Bh (the dropped Al Bl is
// ~2^-24 relative).  The tensor core accumulates in FP32 but not with round-to-nearest
// over long sums, which is what kept an earlier library 3xTF32 M2L above the
// 1e-6 bar: here every 32-wide K-block is accumulated in its own TMEM buffer and
// then drained into FP32 registers with ordinary (round-to-nearest) adds, so the
// tensor core only ever sums 12 products (4 K-steps x 3 splits) per output.
//
// Pipeline of one CTA (persistent: 128 x 128 output tiles in turn, each over its whole K range):
//   warp 0  TMA producer: per K-block the four 128 x 32 FP32 tiles Ah, Al, Bh, Bl
//           (128-byte swizzle, K-major) into a 3-stage shared-memory ring;
//   warp 1  TMEM owner and MMA issuer: 12 tcgen05.mma (M = 128, N = 128, K = 8,
//           kind::tf32) per K-block into one of four TMEM accumulators
//           (4 x 128 columns), committed to the stage's "empty" barrier and the
//           accumulator's "full" barrier;
//   warps 2-5 drain: tcgen05.ld of the accumulator (each warp its 32 TMEM lanes =
//           output rows, two 32-column loads per wait), added into 128 FP32
//           registers per thread; the buffer is released to the MMA warp; at the
//           end the rows are written (or added) to C with coalesced column stores.
// What bounds it: per K-block the 12 MMAs read 96 KB of operand tiles from shared
// memory (Ah and Bh twice, Al and Bl once, 16 KB each) and TMA writes 64 KB into
// it, ~200 bytes per clock at the nominal TF32 rate against ~128 that shared
// memory delivers; the tensor pipe runs at ~60% of its rate inside a tile.  Wider
// tiles (N = 256, or M = 256 over a CTA pair) would read each A tile for twice
// the products.
// Every mbarrier wait has an iteration limit: on expiry the kernel records an
// error code, stops issuing work, waits (bounded) for what it issued, frees its
// TMEM and returns.  TMA loads read this GPU's memory only, without multicast.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "stk_umma.cuh"

namespace stk {

namespace {

constexpr int kBM = 128, kBN = 128, kBK = 32;  // output tile, K-block (32 FP32 = one 128-byte swizzle row)
constexpr int kStages = 3;
constexpr int kTileBytes = kBM * kBK * 4;      // 16 KB (A and B tiles are both 128 x 32 FP32)
constexpr int kStageBytes = 4 * kTileBytes;    // Ah, Al, Bh, Bl
constexpr int kThreads = 192;                  // 6 warps
// FP32 accumulators of 128 columns in TMEM (the MMA warp runs up to kAccBufs - 1
// K-blocks ahead of the drain); 4 take all 512 columns, which one CTA per SM allows
// (198 KB of shared memory per CTA).  4 accumulators with two TMEM loads per wait
// measured 2% faster than 2 with one (mixed M2L of the 2M-point RPY PXYZ FMM,
// 17.4 against 17.8 ms).
#ifndef STK_UMMA_ACCBUFS
#define STK_UMMA_ACCBUFS 4
#endif
constexpr int kAccBufs = STK_UMMA_ACCBUFS;
static_assert(kAccBufs == 2 || kAccBufs == 4, "2 or 4 accumulators");
constexpr uint32_t kTmemCols = 128 * kAccBufs;
// TMEM columns per drain load before its wait (32: one load per wait; 64: two)
#ifndef STK_UMMA_LDCOLS
#define STK_UMMA_LDCOLS 64
#endif
constexpr int kLdCols = STK_UMMA_LDCOLS;
constexpr long long kSpinLimit = 1LL << 25;    // ~ a second of polling per wait
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /* barriers */ + 1024 /* alignment */;

struct Bars {
    unsigned long long full[kStages], empty[kStages], accf[kAccBufs], acce[kAccBufs];
    uint32_t tmem;
};

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t a, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
// bounded wait for the phase with the given parity; false when the limit expired
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity) {
    for (long long i = 0; i < kSpinLimit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major tile, rows of 128 bytes, 128-byte swizzle,
// 8-row groups 1024 bytes apart (SBO); sm_100 descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;              // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;    // stride byte offset
    d |= (uint64_t)1 << 46;              // version
    d |= (uint64_t)2 << 61;              // SWIZZLE_128B
    return d;
}

// instruction descriptor: D FP32, A and B TF32, both K-major, M = 128, N = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// One output tile: output rows [0, 128) are rows a_row .. a_row + 127 of A, output
// columns [0, 128) rows b_row .. b_row + 127 of B (tensor-map coordinates), summed
// over k < K (K-blocks of 32; the maps zero-fill beyond their inner extent).
struct TileSpec {
    int a_row, b_row, K;
};

// One GEMM C = A B^T over (gx = ceil(M/128)) x ceil(N/128) tiles.
struct DenseJob {
    int M, N, K, ldc, beta, gx, ntiles;
    float *C;
    __device__ TileSpec tile(int i) const { return {(i % gx) * kBM, (i / gx) * kBN, K}; }
    __device__ void store(int, const TileSpec &t, int row, const float (&acc)[kBN]) const {
        const int m = t.a_row + row;
        if (m >= M) return;
#pragma unroll
        for (int j = 0; j < kBN; j++) {
            const int n = t.b_row + j;
            if (n < N) {
                float *p = C + (size_t)n * ldc + m;
                *p = beta ? *p + acc[j] : acc[j];
            }
        }
    }
};

// Many small GEMMs in one launch: tile i is described by tiles[i].
struct GroupJob {
    const GroupTile *tiles;
    int ntiles;
    float *C, *C_lo;
    __device__ TileSpec tile(int i) const {
        const GroupTile &g = tiles[i];
        return {g.a_row, g.b_row, g.K};
    }
    __device__ void store(int i, const TileSpec &, int row, const float (&acc)[kBN]) const {
        const GroupTile &g = tiles[i];
        if (row >= g.m_store) return;
        const bool valid = row < g.m_valid;
        const int nv = g.n_valid;
        float *c = C + g.c_off + row;
        float *cl = C_lo ? C_lo + g.c_off + row : nullptr;
#pragma unroll
        for (int j = 0; j < kBN; j++) {
            if (j < nv) {
                const float v = valid ? acc[j] : 0.0f;
                if (cl) {
                    float h, l;
                    tf32_split_value(v, h, l);
                    c[(size_t)j * g.ldc] = h;
                    cl[(size_t)j * g.ldc] = l;
                } else {
                    c[(size_t)j * g.ldc] = v;
                }
            }
        }
    }
};

// Persistent: CTA b computes tiles b, b + gridDim.x, ...  The three roles walk the
// same sequence of K-blocks over all of the CTA's tiles; stage, accumulator buffer
// and barrier parities follow the running K-block count g, so the loads and MMAs
// of a tile start while the drain warps still finish the previous one.
template <class Job>
__global__ void __launch_bounds__(kThreads, 1)
    umma_3xtf32_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                       const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl, const Job job,
                       int *err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = saddr(smem_raw);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    uint8_t *tiles = smem_raw + pad;  // kStages x {Ah, Al, Bh, Bl}, 1024-byte aligned
    Bars *bars = reinterpret_cast<Bars *>(tiles + kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(saddr(&bars->full[s]), 1);
            mbar_init(saddr(&bars->empty[s]), 1);
        }
        for (int b = 0; b < kAccBufs; b++) {
            mbar_init(saddr(&bars->accf[b]), 1);
            mbar_init(saddr(&bars->acce[b]), 4);  // one arrival per drain warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // TMEM: kAccBufs 128-column accumulators, owned by warp 1
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&bars->tmem)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = bars->tmem;
    bool ok = true;

    if (warp == 0) {
        // ---- TMA producer ----
        if (lane == 0) {
            long long g = 0;  // K-blocks issued so far
            for (int t = blockIdx.x; t < job.ntiles && ok; t += gridDim.x) {
                const TileSpec ts = job.tile(t);
                const int nkb = (ts.K + kBK - 1) / kBK;
                for (int kb = 0; kb < nkb; kb++, g++) {
                    const int s = (int)(g % kStages);
                    const uint32_t ph = (uint32_t)(g / kStages) & 1u;
                    if (!mbar_wait(saddr(&bars->empty[s]), ph ^ 1u)) {
                        ok = false;
                        break;
                    }
                    const uint32_t fb = saddr(&bars->full[s]);
                    mbar_expect_tx(fb, kStageBytes);
                    const uint32_t st = saddr(tiles + s * kStageBytes);
                    tma_load_2d(st, &mAh, fb, kb * kBK, ts.a_row);
                    tma_load_2d(st + kTileBytes, &mAl, fb, kb * kBK, ts.a_row);
                    tma_load_2d(st + 2 * kTileBytes, &mBh, fb, kb * kBK, ts.b_row);
                    tma_load_2d(st + 3 * kTileBytes, &mBl, fb, kb * kBK, ts.b_row);
                }
            }
            if (!ok) {
                atomicExch(err, 1);
                // let the loads already issued land before the CTA exits
                if (g > 0) mbar_wait(saddr(&bars->full[(g - 1) % kStages]), (uint32_t)((g - 1) / kStages) & 1u);
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            long long g = 0;  // K-blocks committed so far
            for (int t = blockIdx.x; t < job.ntiles && ok; t += gridDim.x) {
                const int nkb = (job.tile(t).K + kBK - 1) / kBK;
                for (int kb = 0; kb < nkb; kb++) {
                    const int s = (int)(g % kStages), b = (int)(g % kAccBufs);
                    if (!mbar_wait(saddr(&bars->acce[b]), ((uint32_t)(g / kAccBufs) & 1u) ^ 1u) ||
                        !mbar_wait(saddr(&bars->full[s]), (uint32_t)(g / kStages) & 1u)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = saddr(tiles + s * kStageBytes);
                    const uint32_t d = tmem + (uint32_t)(b * kBN);
#pragma unroll
                    for (int ks = 0; ks < kBK / 8; ks++) {
                        const uint32_t off = (uint32_t)ks * 32u;  // 8 TF32 = 32 bytes along K
                        const uint64_t ah = smem_desc(st + off), al = smem_desc(st + kTileBytes + off);
                        const uint64_t bh = smem_desc(st + 2 * kTileBytes + off),
                                       bl = smem_desc(st + 3 * kTileBytes + off);
                        // small terms first; the block's first product overwrites the buffer
                        mma_tf32(d, al, bh, ks > 0 ? 1u : 0u);
                        mma_tf32(d, ah, bl, 1u);
                        mma_tf32(d, ah, bh, 1u);
                    }
                    mma_commit(saddr(&bars->empty[s]));  // the stage is free once these MMAs are done
                    mma_commit(saddr(&bars->accf[b]));   // the accumulator is ready
                    g++;
                }
            }
            if (!ok) atomicExch(err, 2);
            // the MMAs issued last must be complete before the TMEM is freed
            if (g > 0) mbar_wait(saddr(&bars->accf[(g - 1) % kAccBufs]), (uint32_t)((g - 1) / kAccBufs) & 1u);
        }
        __syncwarp();
    } else {
        // ---- drain + epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 ----
        const int q = warp & 3;
        const int row = q * 32 + lane;
        long long g = 0;  // K-blocks drained so far
        for (int t = blockIdx.x; t < job.ntiles && ok; t += gridDim.x) {
            const TileSpec ts = job.tile(t);
            const int nkb = (ts.K + kBK - 1) / kBK;
            float acc[kBN];
#pragma unroll
            for (int j = 0; j < kBN; j++) acc[j] = 0.0f;
            for (int kb = 0; kb < nkb; kb++, g++) {
                const int b = (int)(g % kAccBufs);
                // warp-uniform decision: tcgen05.ld below is a warp-wide instruction
                if (!__all_sync(0xffffffffu, mbar_wait(saddr(&bars->accf[b]), (uint32_t)(g / kAccBufs) & 1u))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kBN);
                if constexpr (kLdCols == 64) {
#pragma unroll
                    for (int c = 0; c < kBN / 64; c++) {
                        uint32_t r0[32], r1[32];
                        tmem_ld32_nowait(tb + (uint32_t)(c * 64), r0);
                        tmem_ld32_nowait(tb + (uint32_t)(c * 64 + 32), r1);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            acc[c * 64 + j] += __uint_as_float(r0[j]);
                            acc[c * 64 + 32 + j] += __uint_as_float(r1[j]);
                        }
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < kBN / 32; c++) {
                        uint32_t r[32];
                        tmem_ld32(tb + (uint32_t)(c * 32), r);
#pragma unroll
                        for (int j = 0; j < 32; j++) acc[c * 32 + j] += __uint_as_float(r[j]);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(saddr(&bars->acce[b]));
            }
            if (!ok) {
                if (lane == 0) atomicExch(err, 3);
            } else {
                job.store(t, ts, row, acc);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

__global__ void tf32_split_kernel(const float *__restrict__ x, long long n, float *__restrict__ hi,
                                  float *__restrict__ lo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float h, l;
        tf32_split_value(x[i], h, l);
        hi[i] = h;
        lo[i] = l;
    }
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no libcuda link)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
    });
    return fn;
}

// rows x K FP32, row pitch ld floats; boxes of 128 rows x 32 K, 128-byte swizzle
bool encode(CUtensorMap *m, const float *base, int rows, int K, int ld) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 4};
    const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kBM};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// SMs of the current device (one persistent CTA each; the pipeline's shared memory
// keeps one CTA per SM)
int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

// opt-in to the pipeline's dynamic shared memory, once per kernel instance
template <class Job> cudaError_t smem_attr() {
    static std::once_flag once;
    static cudaError_t e = cudaSuccess;
    std::call_once(once, [] {
        e = cudaFuncSetAttribute(umma_3xtf32_kernel<Job>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes);
    });
    return e;
}

}  // namespace

bool umma_available() {
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return major == 10 && encode_fn() != nullptr;
}

cudaError_t umma_gemm_3xtf32(int M, int N, int K, Tf32Split A, Tf32Split B, float *C, int ldc, int beta, int *err,
                             cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    auto aligned = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!A.hi || !A.lo || !B.hi || !B.lo || !C || !err || A.ld % 4 || B.ld % 4 || A.ld < K || B.ld < K || ldc < M ||
        !aligned(A.hi) || !aligned(A.lo) || !aligned(B.hi) || !aligned(B.lo))
        return cudaErrorInvalidValue;
    CUtensorMap mah, mal, mbh, mbl;
    if (!encode(&mah, A.hi, M, K, A.ld) || !encode(&mal, A.lo, M, K, A.ld) || !encode(&mbh, B.hi, N, K, B.ld) ||
        !encode(&mbl, B.lo, N, K, B.ld))
        return cudaErrorInvalidValue;
    const cudaError_t ae = smem_attr<DenseJob>();
    if (ae != cudaSuccess) return ae;
    const int gx = (M + kBM - 1) / kBM, gy = (N + kBN - 1) / kBN;
    const long long nt = (long long)gx * gy;
    if (nt > 0x7fffffff) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(nt, sm_count());
    umma_3xtf32_kernel<DenseJob><<<grid, kThreads, kSmemBytes, s>>>(
        mah, mal, mbh, mbl, DenseJob{M, N, K, ldc, beta, gx, (int)nt, C}, err);
    return cudaGetLastError();
}

cudaError_t umma_grouped_3xtf32(Tf32Rows A, Tf32Rows B, const GroupTile *tiles, int ntiles, float *C, float *C_lo,
                                int *err, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    auto aligned = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (!A.hi || !A.lo || !B.hi || !B.lo || !tiles || !C || !err || A.ld % 4 || B.ld % 4 || A.k > A.ld ||
        B.k > B.ld || A.k <= 0 || B.k <= 0 || A.rows <= 0 || B.rows <= 0 || !aligned(A.hi) || !aligned(A.lo) ||
        !aligned(B.hi) || !aligned(B.lo))
        return cudaErrorInvalidValue;
    CUtensorMap mah, mal, mbh, mbl;
    if (!encode(&mah, A.hi, A.rows, A.k, A.ld) || !encode(&mal, A.lo, A.rows, A.k, A.ld) ||
        !encode(&mbh, B.hi, B.rows, B.k, B.ld) || !encode(&mbl, B.lo, B.rows, B.k, B.ld))
        return cudaErrorInvalidValue;
    const cudaError_t ae = smem_attr<GroupJob>();
    if (ae != cudaSuccess) return ae;
    umma_3xtf32_kernel<GroupJob><<<std::min(ntiles, sm_count()), kThreads, kSmemBytes, s>>>(
        mah, mal, mbh, mbl, GroupJob{tiles, ntiles, C, C_lo}, err);
    return cudaGetLastError();
}

cudaError_t tf32_split(const float *x, long long n, float *hi, float *lo, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    const long long want = (n + threads - 1) / threads;
    const int grid = (int)(want < 148 * 16 ? want : 148 * 16);
    tf32_split_kernel<<<grid, threads, 0, s>>>(x, n, hi, lo);
    return cudaGetLastError();
}

}  // namespace stk
