// stk_p2p.cu -- sm_100a list P2P kernel: the U/W/X-list and direct-sum hot loop.
//
// Replaces the per-(target box, source box) ker_poten calls that PVFMM's
// PtFMM_Evaluate makes for the U-list (S2T), and the OpenMP target-chunk loop of
// FMMData::evaluateKernel (Lib/src/FMMData.cpp:252-283).
//
// Design (one warp = one work item, persistent warps):
//  * A work item is <= 64 targets of one target box plus a range of its
//    interaction-list entries.  Items are sorted by cost on the host, largest
//    first; persistent warps take them from a global counter, so uneven
//    adaptive trees balance themselves.
//  * Each lane owns two target slots (lane and lane + 32).  With fewer than 64
//    targets, 2^glog consecutive lanes share a target and split the source
//    tile; they are reduced with warp shuffles at the end.
//  * The sources of an item's list entries form one stream: each entry is a
//    segment (its source box's records, with its periodic shift), and the warp
//    walks the concatenated stream in 32-source tiles that cross segment
//    boundaries, so only the last tile of an item is padded (with one tile per
//    entry, padding was ~19% of the evaluated pairs on clustered trees).
//  * Tile staging: lane i copies the raw record of stream position i of the
//    next tile into its own shared-memory slot with cp.async (16-byte
//    asynchronous copies, L2 -> shared) while the current tile is consumed;
//    then it applies the periodic image shift, computes the per-source staged
//    values (Uk<>::stage) and writes one column of the structure-of-arrays
//    tile (one row per component).
//  * FP64 path: one source and two targets per step; r = x_t - (x_s + shift)
//    formed in double exactly as the oracle forms it.
//  * Mixed path: at staging each source coordinate, shifted to the target
//    box's centre c in FP64, is split into FP32 hi + lo parts
//    (x - c = hi + lo to ~2^-48 relative); targets likewise.  Per pair the
//    displacement (t_hi - s_hi) + (t_lo - s_lo) is then accurate to FP32
//    relative precision even for nearly coincident points (t_hi - s_hi is exact
//    by Sterbenz' lemma when the points are close).  The kernel tensor runs in
//    Blackwell packed FP32 (fma.rn.f32x2: two sources per instruction) with
//    MUFU rsqrt + one Newton step; each tile's FP32 partial sums are added into
//    Kahan-compensated FP32 accumulators.
#include <algorithm>
#include <type_traits>

#include "stk_p2p.cuh"
#include "stk_ukernels.cuh"

namespace stk {

namespace {

// Warps per CTA.  Every warp works alone (warp-level synchronisation only), so
// this only sets the granularity in which registers fill an SM: one warp per CTA
// lets the FP64 kernels use every register slot (14 warps per SM at 140
// registers instead of 12 in 4-warp CTAs: the benchmark's FP64 launch 1.1%
// faster); the mixed kernels measured best at 4.
template <bool MIXED> struct Cta {
    static constexpr int warps = MIXED ? 4 : 1;
    static constexpr int threads = 32 * warps;
};
constexpr unsigned kFull = 0xffffffffu;
constexpr double kPadCoord = 1.0e4;  // offset of zero-strength padding sources
constexpr int kShiftNoneCode = 13;   // list-entry shift code of the unshifted source box
constexpr int kMayCoincide = 32;     // segment-table flag above the 5-bit shift code

// Number of staged per-output-point values of a micro-kernel (1 as a dummy
// array size when it has none).
template <class K, class = void> struct NtvOf {
    static constexpr int value = 1;
};
template <class K> struct NtvOf<K, std::void_t<decltype(K::NTV)>> {
    static constexpr int value = K::NTV;
};

template <int UK> struct Rec {
    static constexpr int SDIM = Uk<UK>::SDIM;
    static constexpr int RS = (3 + SDIM + 1) & ~1;  // doubles per global record (16-byte multiple)
};

// Resident CTAs per SM requested from the register allocator (1: no
// constraint; forcing 5 measured slower for the FP64 path and neutral for the
// mixed path).  STK_MINB_OVERRIDE builds tuning variants.
template <int UK, bool MIXED> struct MinBlocks {
#ifdef STK_MINB_OVERRIDE
    static constexpr int value = STK_MINB_OVERRIDE;
#else
    static constexpr int value = 1;
#endif
};

// How the mixed path forms the displacement (STK_MIXED_DISP selects at build time):
//   kDispHiLo: FP32 hi + lo parts of the centre-relative coordinates, 3 FP32
//              operations per coordinate and pair on the FP32 pipe;
//   kDispF64:  centre-relative coordinates kept in FP64 in shared memory, one
//              FP64 subtraction and one FP64->FP32 rounding per coordinate and
//              pair, on the otherwise idle FP64 pipe.
constexpr int kDispHiLo = 0, kDispF64 = 1;
#ifdef STK_MIXED_DISP
constexpr int kMixedDisp = STK_MIXED_DISP;
#else
constexpr int kMixedDisp = kDispHiLo;
#endif
static_assert(kMixedDisp == kDispHiLo || kMixedDisp == kDispF64, "STK_MIXED_DISP must be 0 or 1");

// Unroll of the source loop (tuning builds override it)
#ifndef STK_P2P_UNROLL_MIXED
#define STK_P2P_UNROLL_MIXED 2
#endif
#ifndef STK_P2P_UNROLL_FP64
#define STK_P2P_UNROLL_FP64 2
#endif
#define STK_PRAGMA(x) _Pragma(#x)
#define STK_UNROLL(n) STK_PRAGMA(unroll n)

// Target slots per lane: 2 (a warp holds 64 targets), or 4 for small micro-kernels
// in builds with STK_P2P_TPL4 (twice the targets per staged source pair, the
// host's lanes-per-target doubled to keep every target covered).
#ifndef STK_P2P_TPL4
#define STK_P2P_TPL4 0
#endif
template <class K> struct TargetsPerLane {
    static constexpr int value = (STK_P2P_TPL4 && K::TDIM <= 4 && K::NV <= 8 && K::TV == 0) ? 4 : 2;
};

// Mixed path: the packed FP32 partial sums go into the Kahan accumulators every
// kKahanTiles * g tiles, i.e. after ~32 kKahanTiles sources per lane whatever
// the lanes per target g (STK_KAHAN_TILES overrides; the step costs ~5 FP32
// operations per output, which per 32-source tile was ~7% of the instructions
// when g > 1).
#ifndef STK_KAHAN_TILES
#define STK_KAHAN_TILES 1
#endif
constexpr int kKahanTiles = STK_KAHAN_TILES;

// cp.async (Ampere+ asynchronous global -> shared copy, 16 bytes per lane and
// instruction, L2 only): the next tile's raw source records land in shared memory
// while the current tile is consumed, so no register holds a prefetched record.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's most recent groups are still in flight
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Tiles in flight per warp (STK_P2P_DEPTH builds deeper pipelines where the landing
// zones fit the 48 KB of static shared memory per block).  One tile ahead is the
// default: two measured 0.5% slower on the clustered 1M-point LapPGrad U list
// (3.100 against 3.084 ms mixed, 4.446 against 4.409 ms FP64), so the L2 round
// trip is hidden behind one tile's consumption even for items of 8 targets.
#ifndef STK_P2P_DEPTH
#define STK_P2P_DEPTH 1
#endif
template <int RS> struct StageDepth {
    static constexpr int value = RS <= 10 ? STK_P2P_DEPTH : 1;
};

// FP32 hi part of a double by truncation: the top 24 significant bits (the low
// 29 mantissa bits cleared), so (float)hi is exact and d - hi is exact in FP64.
__device__ __forceinline__ double trunc_to_f32_bits(double d) {
    return __hiloint2double(__double2hiint(d), __double2loint(d) & (int)0xE0000000u);
}

// Shared-memory stride (doubles) of a raw record: an odd number of 16-byte units,
// so the 8 lanes of a quarter-warp reading their own records with 16-byte loads
// hit 8 distinct bank groups.
template <int RS> struct RawStride {
    static constexpr int value = ((RS / 2) & 1) ? RS : RS + 2;
};

template <int UK, bool MIXED>
__global__ void __launch_bounds__(Cta<MIXED>::threads, MinBlocks<UK, MIXED>::value)
    list_p2p_kernel(const ListP2PArgs a) {
    constexpr int kWarpsPerCta = Cta<MIXED>::warps;
    using K = Uk<UK>;
    constexpr int TDIM = K::TDIM;
    constexpr int NV = K::NV;
    constexpr int TV = K::TV;  // per-output-point values (adjoint kernels)
    constexpr int NTV = NtvOf<K>::value;
    constexpr int RS = Rec<UK>::RS;
    constexpr int RSS = RawStride<RS>::value;
    constexpr int TPL = TargetsPerLane<K>::value;
    constexpr bool HILO = MIXED && kMixedDisp == kDispHiLo;
    // shared tile, one row per component: coordinates (FP64, or FP32 hi x3 + lo x3)
    // and staged values (FP64 path: double, mixed path: float)
    constexpr int NCC = HILO ? 6 : 3;
    using CT = typename std::conditional<HILO, float, double>::type;
    using S = typename std::conditional<MIXED, float, double>::type;

    __shared__ __align__(16) CT tcoord[kWarpsPerCta][NCC][32];
    __shared__ __align__(16) S tval[kWarpsPerCta][NV][32];
    constexpr int DEPTH = StageDepth<RS>::value;
    // cp.async landing zones, one record per lane and tile in flight
    __shared__ __align__(16) double traw[kWarpsPerCta][DEPTH][32][RSS];
    // the item's list entries (up to 32 at a time) as segments of one source stream
    __shared__ int sg_end[kWarpsPerCta][32];   // stream position one past the segment
    __shared__ int sg_src[kWarpsPerCta][32];   // first record of the segment minus its stream start
    __shared__ int sg_code[kWarpsPerCta][32];  // periodic shift code
    const int wid = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    CT(*mc)[32] = tcoord[wid];
    S(*mv)[32] = tval[wid];
    int *s_end = sg_end[wid];
    int *s_src = sg_src[wid];
    int *s_code = sg_code[wid];

    for (;;) {
        int it = 0;
        if (lane == 0) it = (int)atomicAdd(a.counter, 1u);
        it = __shfl_sync(kFull, it, 0);
        if (it >= a.n_items) break;
        const WorkItem w = a.items[it];
        // the host sizes glog for 64 slots; 4 slots per lane give twice the lanes per target
        const int glog = TPL == 4 ? min(5, w.glog + 1) : w.glog;
        const int g = 1 << glog;
        const int sub = lane & (g - 1);
        bool act[TPL];
        int tt[TPL];
#pragma unroll
        for (int h = 0; h < TPL; h++) {
            const int ti = (lane + 32 * h) >> glog;
            act[h] = ti < w.nt;
            tt[h] = w.t0 + (act[h] ? ti : 0);
        }

        double c[3] = {0.0, 0.0, 0.0};
        if constexpr (MIXED) {
            // local origin: the target box centre, or the item's first target
            const double *o = a.box_centre ? a.box_centre + 3 * (size_t)w.trg_box : a.trg_xyz + 3 * (size_t)w.t0;
            c[0] = o[0];
            c[1] = o[1];
            c[2] = o[2];
        }
        double xt[TPL][3];
#pragma unroll
        for (int h = 0; h < TPL; h++)
#pragma unroll
            for (int k = 0; k < 3; k++) xt[h][k] = a.trg_xyz[3 * (size_t)tt[h] + k];

        // per-output-point values, staged once per item
        using V = typename std::conditional<MIXED, F2, double>::type;
        V ta[TPL][NTV];
        if constexpr (TV > 0) {
#pragma unroll
            for (int h = 0; h < TPL; h++) {
                double r0[TV], s0[NTV];
#pragma unroll
                for (int q = 0; q < TV; q++) r0[q] = a.trg_aux[(size_t)tt[h] * TV + q];
                K::stage_aux(r0, s0);
#pragma unroll
                for (int q = 0; q < NTV; q++) {
                    if constexpr (MIXED)
                        ta[h][q] = splat((float)s0[q]);
                    else
                        ta[h][q] = s0[q];
                }
            }
        }
        auto eval = [&](auto &u, auto dx, auto dy, auto dz, const auto *sv, const auto *tav) {
            if constexpr (TV > 0)
                K::eval(u, dx, dy, dz, sv, tav);
            else
                K::eval(u, dx, dy, dz, sv);
        };

        // accumulators: FP64 path sums directly; mixed path keeps Kahan sum + compensation
        S acc[TPL][TDIM], cmp[TPL][TDIM];
#pragma unroll
        for (int h = 0; h < TPL; h++)
#pragma unroll
            for (int k = 0; k < TDIM; k++) acc[h][k] = cmp[h][k] = S(0);
        // mixed path: packed FP32 partial sums, added into the Kahan accumulators in steps
        F2 pp[TPL][TDIM];
#pragma unroll
        for (int h = 0; h < TPL; h++)
#pragma unroll
            for (int k = 0; k < TDIM; k++) pp[h][k] = splat(0.0f);
        int kahan_tiles = 0;
        auto kahan_step = [&]() {
            if constexpr (MIXED) {
#pragma unroll
                for (int h = 0; h < TPL; h++)
#pragma unroll
                    for (int k = 0; k < TDIM; k++) {
                        const float y = (pp[h][k].v.x + pp[h][k].v.y) - cmp[h][k];
                        const float t = acc[h][k] + y;
                        cmp[h][k] = (t - acc[h][k]) - y;
                        acc[h][k] = t;
                        pp[h][k] = splat(0.0f);
                    }
            }
            kahan_tiles = 0;
        };
        F2 th[TPL][3], tl[TPL][3];  // hi/lo targets (HILO)
        double tr[TPL][3];          // centre-relative targets (FP64 displacement)
#pragma unroll
        for (int h = 0; h < TPL; h++)
#pragma unroll
            for (int k = 0; k < 3; k++) tr[h][k] = xt[h][k] - c[k];
        if constexpr (HILO) {
#pragma unroll
            for (int h = 0; h < TPL; h++)
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const float hv = (float)tr[h][k];
                    th[h][k] = splat(hv);
                    tl[h][k] = splat((float)(tr[h][k] - (double)hv));
                }
        }

        // ---- the item's sources as one stream: its list entries, 32 at a time, in
        // order, each a segment of its source box's records; tiles of 32 stream
        // positions cross segment boundaries, so only a chunk's last tile is padded ----
        for (int ec = w.e0; ec < w.e1; ec += 32) {
            const int ne = min(32, w.e1 - ec);
            int sz = 0, sbeg = 0, code = kShiftNoneCode;
            if (lane < ne) {
                const int ent = a.list_ent[ec + lane];
                const int sb = ent >> 5;
                code = ent & 31;
                sbeg = a.src_box_begin[sb];
                sz = a.src_box_end[sb] - sbeg;
                // bit 5: the segment may hold a source at a target's position (always,
                // unless the lists guarantee coincidence only in the unshifted own box)
                if (!a.coincident_own_box || sb == w.trg_box || code != kShiftNoneCode) code |= kMayCoincide;
            }
            int incl = sz;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const int total = __shfl_sync(kFull, incl, 31);
            __syncwarp();  // the previous chunk's segment table is no longer read
            s_end[lane] = lane < ne ? incl : 0x7fffffff;
            s_src[lane] = sbeg - (incl - sz);
            s_code[lane] = code;
            __syncwarp();
            if (total == 0) continue;

            // per-lane cursor into the segment table; positions only grow
            int seg = 0;
            // segment of the record in each landing zone, oldest first (registers:
            // every index below is a compile-time constant)
            int zseg[DEPTH];
            // cp.async the record at stream position p into this lane's slot of zone z,
            // or nothing past the stream's end; one commit group per call either way,
            // so every lane counts the same groups
            auto fetch = [&](int p, int z, int &zs) {
                if (p < total) {
                    while (p >= s_end[seg]) seg++;
                    const double *src = a.src_rec + (size_t)(s_src[seg] + p) * RS;
                    double *dst = traw[wid][z][lane];
#pragma unroll
                    for (int q = 0; q < RS / 2; q++) cp_async16(dst + 2 * q, src + 2 * q);
                    zs = seg;
                }
                cp_async_commit();
            };
#pragma unroll
            for (int z = 0; z < DEPTH; z++) fetch(32 * z + lane, z, zseg[z]);
            int p0 = 0, zone = 0;
            while (p0 < total) {
                const int n = min(32, total - p0);
                // ---- stage: lane i turns stream position p0 + i (its landed record)
                // into tile column i, or writes zero-strength padding ----
                cp_async_wait_group<DEPTH - 1>();  // this tile's group; later ones may still fly
                __syncwarp();  // every lane has finished reading the previous tile
                int may_coincide = 0;
                {
                    double v[NV];
                    double x[3];
                    if (lane < n) {
                        const double *raw = traw[wid][zone][lane];
                        double rn[RS];
#pragma unroll
                        for (int q = 0; q < RS / 2; q++) {
                            const double2 t2 = *reinterpret_cast<const double2 *>(raw + 2 * q);
                            rn[2 * q] = t2.x;
                            rn[2 * q + 1] = t2.y;
                        }
                        x[0] = rn[0];
                        x[1] = rn[1];
                        x[2] = rn[2];
                        const int cdf = s_code[zseg[0]];
                        may_coincide = cdf & kMayCoincide;
                        const int cd = cdf & 31;
                        if (cd != kShiftNoneCode) {  // periodic image
                            x[0] += (cd % 3 - 1) * a.period;
                            x[1] += ((cd / 3) % 3 - 1) * a.period;
                            x[2] += (cd / 9 - 1) * a.period;
                        }
                        K::stage(rn + 3, v);
                    } else {
#pragma unroll
                        for (int k = 0; k < 3; k++) x[k] = c[k] + kPadCoord;
#pragma unroll
                        for (int q = 0; q < NV; q++) v[q] = 0.0;
                    }
                    if constexpr (HILO) {
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            const double d = x[k] - c[k];
                            const double hd = trunc_to_f32_bits(d);
                            mc[k][lane] = (float)hd;
                            mc[3 + k][lane] = (float)(d - hd);
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < 3; k++) mc[k][lane] = x[k] - c[k];  // c = 0 on the FP64 path
                    }
#pragma unroll
                    for (int q = 0; q < NV; q++) mv[q][lane] = (S)v[q];
                }
                // ---- prefetch the tile DEPTH ahead into the zone just staged ----
#pragma unroll
                for (int z = 0; z + 1 < DEPTH; z++) zseg[z] = zseg[z + 1];
                fetch(p0 + 32 * DEPTH + lane, zone, zseg[DEPTH - 1]);
                p0 += 32;
                zone = DEPTH > 1 ? (zone + 1 == DEPTH ? 0 : zone + 1) : 0;
                __syncwarp();

                // ---- consume the tile ----
                if constexpr (MIXED) {
                    // sources j, j+1 in one packed pair; entries [n, n+1] are zero-strength padding.
                    // P: F2 (rsqrt masks coincident pairs) or F2U (no source of the tile can sit
                    // at a target's position)
                    auto consume = [&](auto proto) {
                        using P = decltype(proto);
STK_UNROLL(STK_P2P_UNROLL_MIXED)
                        for (int j = 2 * sub; j < n; j += 2 * g) {
                            P sv[NV];
#pragma unroll
                            for (int q = 0; q < NV; q++) sv[q].v = *reinterpret_cast<const float2 *>(&mv[q][j]);
                            P dxyz[TPL][3];
                            if constexpr (HILO) {
                                F2 sh[3], sl[3];
#pragma unroll
                                for (int k = 0; k < 3; k++) {
                                    sh[k].v = *reinterpret_cast<const float2 *>(&mc[k][j]);
                                    sl[k].v = *reinterpret_cast<const float2 *>(&mc[3 + k][j]);
                                }
#pragma unroll
                                for (int h = 0; h < TPL; h++)
#pragma unroll
                                    for (int k = 0; k < 3; k++)
                                        dxyz[h][k].v = ((th[h][k] - sh[k]) + (tl[h][k] - sl[k])).v;
                            } else {
                                double2 sx[3];
#pragma unroll
                                for (int k = 0; k < 3; k++) sx[k] = *reinterpret_cast<const double2 *>(&mc[k][j]);
#pragma unroll
                                for (int h = 0; h < TPL; h++)
#pragma unroll
                                    for (int k = 0; k < 3; k++)
                                        dxyz[h][k].v = make_float2((float)(tr[h][k] - sx[k].x),
                                                                   (float)(tr[h][k] - sx[k].y));
                            }
#pragma unroll
                            for (int h = 0; h < TPL; h++) {
                                P u[TDIM], tv[NTV];
#pragma unroll
                                for (int k = 0; k < TDIM; k++) u[k].v = pp[h][k].v;
#pragma unroll
                                for (int q = 0; q < NTV; q++) tv[q].v = ta[h][q].v;
                                eval(u, dxyz[h][0], dxyz[h][1], dxyz[h][2], sv, tv);
#pragma unroll
                                for (int k = 0; k < TDIM; k++) pp[h][k].v = u[k].v;
                            }
                        }
                    };
                    if (__any_sync(kFull, may_coincide))
                        consume(F2{});
                    else
                        consume(F2U{});
                    // Kahan-compensated accumulation of the partial sums once a lane has
                    // evaluated ~32 sources since the last step (every g tiles)
                    if (++kahan_tiles >= kKahanTiles * g) kahan_step();
                } else {
STK_UNROLL(STK_P2P_UNROLL_FP64)
                    for (int j = sub; j < n; j += g) {
                        double sv[NV];
#pragma unroll
                        for (int q = 0; q < NV; q++) sv[q] = mv[q][j];
                        const double sx = mc[0][j], sy = mc[1][j], sz = mc[2][j];
#pragma unroll
                        for (int h = 0; h < TPL; h++)
                            eval(acc[h], xt[h][0] - sx, xt[h][1] - sy, xt[h][2] - sz, sv, ta[h]);
                    }
                }
            }
        }
        __syncwarp();
        if (kahan_tiles > 0) kahan_step();

        // ---- reduce the lanes that share a target, then accumulate ----
        double o[TPL][TDIM];
#pragma unroll
        for (int h = 0; h < TPL; h++)
#pragma unroll
            for (int k = 0; k < TDIM; k++) {
                if constexpr (MIXED)
                    o[h][k] = double(acc[h][k]) - double(cmp[h][k]);
                else
                    o[h][k] = acc[h][k];
            }
        for (int off = 1; off < g; off <<= 1) {
#pragma unroll
            for (int h = 0; h < TPL; h++)
#pragma unroll
                for (int k = 0; k < TDIM; k++) o[h][k] += __shfl_xor_sync(kFull, o[h][k], off);
        }
        if (sub == 0) {
#pragma unroll
            for (int h = 0; h < TPL; h++) {
                if (!act[h]) continue;
                double *dst = a.trg_out + (size_t)tt[h] * TDIM;
#pragma unroll
                for (int k = 0; k < TDIM; k++) {
                    const double val = K::SCALE * K::comp_scale(k) * o[h][k];
                    if (a.atomic_out)
                        atomicAdd(dst + k, val);
                    else
                        dst[k] += val;
                }
            }
        }
    }
}

template <int UK, bool MIXED>
cudaError_t launch_impl(const ListP2PArgs &a, int num_sms, cudaStream_t stream) {
    static int blocks_per_sm = 0;
    if (blocks_per_sm == 0) {
        cudaError_t err =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, list_p2p_kernel<UK, MIXED>,
                                                          Cta<MIXED>::threads, 0);
        if (err != cudaSuccess) return err;
        if (blocks_per_sm < 1) blocks_per_sm = 1;
    }
    constexpr int kWarpsPerCta = Cta<MIXED>::warps;
    long long want = ((long long)a.n_items + kWarpsPerCta - 1) / kWarpsPerCta;
    int grid = (int)std::max(1LL, std::min<long long>((long long)num_sms * blocks_per_sm, want));
    cudaError_t err = cudaMemsetAsync(a.counter, 0, sizeof(unsigned int), stream);
    if (err != cudaSuccess) return err;
    list_p2p_kernel<UK, MIXED><<<grid, Cta<MIXED>::threads, 0, stream>>>(a);
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
int uk_tvdim_host(int uk) { return uk_tvdim(uk); }
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
    case UK_LAPLACE_SLDL_P: return launch_prec<UK_LAPLACE_SLDL_P>(prec, a, num_sms, stream);
    case UK_LAPLACE_PGRADGRAD: return launch_prec<UK_LAPLACE_PGRADGRAD>(prec, a, num_sms, stream);
    case UK_LAPLACE_DIPOLEPGRADGRAD: return launch_prec<UK_LAPLACE_DIPOLEPGRADGRAD>(prec, a, num_sms, stream);
    case UK_LAPLACE_QUADP: return launch_prec<UK_LAPLACE_QUADP>(prec, a, num_sms, stream);
    case UK_LAPLACE_QUADPGRADGRAD: return launch_prec<UK_LAPLACE_QUADPGRADGRAD>(prec, a, num_sms, stream);
    case UK_STOKES_PVELGRAD: return launch_prec<UK_STOKES_PVELGRAD>(prec, a, num_sms, stream);
    case UK_STOKES_DOUBLEPVELGRAD: return launch_prec<UK_STOKES_DOUBLEPVELGRAD>(prec, a, num_sms, stream);
    case UK_STOKES_PVELLAPLACIAN: return launch_prec<UK_STOKES_PVELLAPLACIAN>(prec, a, num_sms, stream);
    case UK_STOKES_DOUBLELAPLACIAN: return launch_prec<UK_STOKES_DOUBLELAPLACIAN>(prec, a, num_sms, stream);
    case UK_STOKES_TRACTION: return launch_prec<UK_STOKES_TRACTION>(prec, a, num_sms, stream);
    case UK_STOKES_DOUBLETRACTION: return launch_prec<UK_STOKES_DOUBLETRACTION>(prec, a, num_sms, stream);
    case UK_STOKES_REGFTVEL: return launch_prec<UK_STOKES_REGFTVEL>(prec, a, num_sms, stream);
    case UK_STOKES_REGFTVELOMEGA: return launch_prec<UK_STOKES_REGFTVELOMEGA>(prec, a, num_sms, stream);
    case UK_STOKES_VELOMEGA: return launch_prec<UK_STOKES_VELOMEGA>(prec, a, num_sms, stream);
    case UK_REGVEL_ADJ_SRC:
        if (!a.trg_aux) return cudaErrorInvalidValue;
        return launch_prec<UK_REGVEL_ADJ_SRC>(prec, a, num_sms, stream);
    case UK_REGVEL_ADJ_TRG:
        if (!a.trg_aux) return cudaErrorInvalidValue;
        return launch_prec<UK_REGVEL_ADJ_TRG>(prec, a, num_sms, stream);
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
