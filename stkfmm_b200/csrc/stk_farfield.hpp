// stk_farfield.hpp -- KIFMM far field (S2M, M2M, M2L, S2L, L2L, L2T, M2T) on the GPU.
//
// Stands in for the far-field part of PVFMM's PtFMM_Evaluate
// (Lib/src/FMMData.cpp:198), which is not part of the reference tree.  Surfaces
// follow stkfmm::surface (Lib/include/STKFMM/stkfmm_helpers.hpp:46-85) and the
// radii of the reference's operator generator (M2L/SVD_pvfmm.hpp:37-38):
// upward equivalent and downward check at 1.05, upward check and downward
// equivalent at 2.95 times the box half-width, centred on the box.
#pragma once
#include <memory>
#include <vector>

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include "stk_handle.hpp"
#include "stk_kernel_table.hpp"
#include "stk_p2p.cuh"
#include "stk_tree.hpp"

namespace stk {

constexpr double kRad0 = 1.05;  // upward equivalent, downward check
constexpr double kRad1 = 2.95;  // upward check, downward equivalent

// One P2P evaluation over a list, with its work items resident on the device.
struct ListPass {
    int uk = -1;
    int n_items = 0;
    long long pairs = 0;
    DevBuf items, ent, src_beg, src_end, trg_box_centre;
    void reset() {
        uk = -1;
        n_items = 0;
        pairs = 0;
    }
};

// Chunks of one group of columns whose offsets share one padded rank.
struct M2LSeg {
    int group, rank, start, count;
};

// M2L of one complete level (all 8^l boxes present, most of their V lists full):
// boxes grouped by parity type c = (ix & 1) | (iy & 1) << 1 | (iz & 1) << 2, so
// that every target of type c meets the same offsets V_c and every source of
// type c' the same offsets S_c'.  Per source type one GEMM Z = Qs_c'^T Phi_c'
// (all of its offsets at once), per (target type, source type) a gather of Z's
// rows into the targets' order and one GEMM Psi_c += Pv_{c,c'} Zc: no per-pair
// k-vectors, no per-target reduce.
struct M2LDenseLevel {
    int level = 0, n8 = 0;
    DevBuf d_nodes;              // 8 n8 node ids, type-major (type c: [c n8, (c+1) n8))
    DevBuf d_tab;                // per (c, c'): n8 x nq source positions within type c' (-1: no pair)
    std::vector<size_t> tab_off;  // [8 c + c'] start in d_tab
    long long pairs = 0;
};

struct FarField {
    int p = 0, n = 0;      // multipole order, surface points per box
    int ke = 0, kc = 0;    // equivalent density and check potential dims
    int m2x = -1;          // micro-kernel of the translations (k_m2m = k_m2l = k_l2l)
    // K(s r) = s^-1 diag(s^-pot_exp) K(r) diag(s^-den_exp): with densities and check
    // potentials normalised per level and component, the operators of a side-1 box
    // serve every level (all zero for laplace_p / stokes_vel)
    bool scaled = false;
    double pot_exp[4] = {0, 0, 0, 0}, den_exp[4] = {0, 0, 0, 0};
    bool ready = false;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t solver = nullptr;
    // level-independent operators (column-major, FP64)
    DevBuf uc2ue, dc2de;   // (n ke) x (n kc)
    DevBuf m2m;            // [M2M_0 .. M2M_7]: (n ke) x (8 n ke)
    DevBuf l2l;            // [L2L_0; ..; L2L_7]: (8 n ke) x (n ke)
    // compressed M2L: M2L_d = m2l_e C_d m2l_vt
    double m2l_rtol = 0;        // relative singular-value cut of the M2L bases
    int m2l_rank = 0;           // k
    // two-level: per offset slot C_d ~ P_d Q_d^T, P and Q k x r_d (column-major, packed)
    std::vector<int> m2l_r;         // r_d per slot (padded to a multiple of 32)
    std::vector<int> m2l_rt;        // r_d per slot before padding
    std::vector<size_t> m2l_pq_off;  // start of P_d / Q_d in m2l_p / m2l_q
    int m2l_rmax = 1;
    DevBuf m2l_p, m2l_q, m2l_p32, m2l_q32;
    DevBuf m2l_vt;              // V^T: k x (n ke)
    DevBuf m2l_e;               // DC2DE U: (n ke) x k
    std::vector<int> m2l_slot;  // offset code (0..342) -> block, -1 for adjacent offsets
    // periodic (PXY, PXYZ): DC2DE M2C of the root (far images, max |s| >= 2)
    bool periodic = false;
    int m2c_p = 0, m2c_m2x = -1, m2c_pbc = 0, m2c_ff = -1;  // what m2c_op was built for (m2c_ff: far field on)
    DevBuf m2c_op;
    // per-tree data
    DevBuf unit_surf;          // n x 3 points on [-1,1]^3
    DevBuf d_level;            // node levels
    DevBuf ue_xyz, de_xyz;     // every node's surfaces (nodes x n x 3)
    DevBuf uc_xyz, dc_xyz;     // S2M targets (leaves with sources), S2L targets (nodes with X lists)
    DevBuf phi, psi;           // equivalent densities per node (nodes x n x ke)
    DevBuf phi_hat, psi_hat;   // compressed M2L sources / targets (nodes x k)
    DevBuf check, dcheck;      // S2M / S2L check potentials (compact)
    DevBuf rec_surf, rec_pts[2], tmp0, tmp1;
    std::vector<int> s2m_nodes, s2l_nodes;          // compact order (sorted by level)
    std::vector<int> s2m_level_off, s2l_level_off;  // per level start in the compact order
    DevBuf d_s2m_nodes, d_s2l_nodes;
    ListPass s2m[2], s2l[2], m2t, l2t;  // [SL, DL]
    bool fused_src = false;             // S2M / S2L as one SL+DL pass (s2m[0], s2l[0])
    int fused_check_uk = -1;
    ListPass near[2];  // FMM near field per source set: U list + direct W / X entries
    // M2M / L2L per level: the parents (non-leaf nodes) of level l are
    // parents[parent_off[l] .. parent_off[l+1]) in node order
    std::vector<int> parents, parent_off;
    DevBuf d_parents;
    // M2L: V-list pairs grouped by offset in chunks of columns (one batched GEMM)
    int launches = 0;                       // own kernels of the last evaluation (cuBLAS excluded)
    long long m2l_pairs = 0, m2l_cols = 0;  // pairs; columns including chunk padding
    int m2l_chunks = 0, m2l_group_chunks = 1;  // chunks; chunks per group of columns
    DevBuf d_m2l_gsrc;                      // per column: source node, -1 = padding
    DevBuf d_m2l_red_off, d_m2l_red_col;    // per target node: its columns (CSR, offset order)
    DevBuf d_m2l_gstart;                    // per group and target node: first entry in that group
    DevBuf m2l_x, m2l_y, m2l_z;             // one group of columns: k x, k x, rmax x columns (FP64 or FP32)
    DevBuf d_m2l_ptr[5], d_m2l_ptr32[5];    // per chunk: Q_d, X, Z, P_d, Y (FP64 / FP32 views)
    std::vector<M2LSeg> m2l_seg;            // per group of columns and padded rank: chunks in the pointer arrays
    // the mixed path's chunked M2L on the tensor cores (grouped 3xTF32 GEMMs, stk_umma.cu):
    // Q_d^T of every offset as K-major rows (sum_d r_d rows of k4 floats), P_d^T per offset
    // (k rows of rmax floats each, offset after offset), and per group of columns the tiles
    // of both stages (Z = Q_d^T X into split Z, Y = P_d Z)
    bool tcc = false;
    DevBuf tcc_q_hi, tcc_q_lo, tcc_pt_hi, tcc_pt_lo;
    long long tcc_q_rows = 0;
    DevBuf tcc_tiles1, tcc_tiles2;
    std::vector<int> tcc_t1_off, tcc_t2_off;  // per group: its tiles in the arrays above
    double m2l_flops = 0;                   // flops of one M2L (both stages, padded ranks and chunks)
    double m2l_flops_alg = 0;               // the same at the true ranks over the real pairs, plus the
                                            // two basis products (V^T phi, (DC2DE U) psi_hat)
    // complete levels (see M2LDenseLevel); the column chunks above hold the other levels' pairs
    std::vector<std::unique_ptr<M2LDenseLevel>> dense;
    int dn_q[64] = {};                      // offsets of (c, c'): slots q of V_{c,c'}
    std::vector<int> dn_slots[64];
    int dn_rv[8] = {}, dn_rs[8] = {};       // rows of Pv_c (sum of r_d over V_c) and of Qs_c'
    int dn_pstart[64] = {};                 // first column of block (c, c') in Pv_c
    int dn_rcc[64] = {};                    // rows of block (c, c')
    DevBuf dn_pv, dn_qs, dn_pv32, dn_qs32;  // Pv_0..7, Qs_0..7 (k x rows each, packed)
    size_t dn_pv_off[8] = {}, dn_qs_off[8] = {};
    DevBuf dn_rowq, dn_srow;                // per block row: its slot index q, its row in Z_c'
    size_t dn_row_off[64] = {};
    DevBuf dn_phi, dn_psi, dn_z, dn_zc;     // per-level work buffers (FP64 or FP32)
    // mixed path on the tensor cores (stk_umma.cu): 3xTF32 hi / lo operands, K-major
    bool tc = false;
    DevBuf tc_qa_hi, tc_qa_lo;              // Qs_c'^T per source type: dn_rs[c'] rows of k4 floats
    DevBuf tc_pa_hi, tc_pa_lo;              // Pv_c^T per target type: k rows of ceil4(dn_rv[c]) floats
    size_t tc_qa_off[8] = {}, tc_pa_off[8] = {};
    DevBuf tc_b_hi, tc_b_lo;                // per level: Phi operands (8 n8 rows of k4)
    DevBuf tc_z;                            // per level: Z of every source type
    DevBuf tc_zc_hi, tc_zc_lo;              // per stream: the concatenated Zc operand (n8 rows of tc_zc_ld)
    int tc_streams = 0, tc_zc_ld = 0;
    cudaStream_t tc_stream[8] = {};         // target types of the dense M2L run concurrently
    cudaEvent_t tc_ev[8] = {}, tc_fork = nullptr;
    DevBuf tc_err;                          // set by a tensor-core GEMM whose pipeline wait gave up
    // Operators shared through the process-wide cache: the level-independent
    // operators (and the periodic M2C) are built once per (device, translation
    // kernel, p, M2L cut) and aliased by every handle that needs them; each
    // holder keeps the cache entry alive.  `built` is recorded on the stream that
    // built an entry; a handle reusing it makes its stream wait for it.
    std::shared_ptr<FarField> ops_ref, m2c_ref;
    // far field split over a shard group (Stk3DFMM_set_allreduce): this rank's M2L /
    // S2L target nodes; dense levels by parity type (dn_own[c])
    bool split = false;
    bool dn_own[8] = {true, true, true, true, true, true, true, true};
    cudaEvent_t built = nullptr;
    ~FarField();
};

// Precompute the operators for (kernel, p) and the per-tree data; returns a
// stk_status.  Supported: kernels whose translation kernel is laplace_p,
// stokes_vel or stokes_PVel (every STKFMM kernel), free space, PX, PXY, PXYZ.
int farfield_setup(Stk3DFMM *f, KernelData *kd);

// trg_sorted += far field of the sources (values already packed / scaled as the
// near field uses them: d_sl, d_dl in the caller's order).
int farfield_evaluate(Stk3DFMM *f, KernelData *kd, const double *d_sl, const double *d_dl, double *trg_sorted,
                      cudaStream_t s);

// After the evaluation has completed (the caller synchronised): STK_ERR_CUDA, once,
// when a tensor-core M2L GEMM gave up at a pipeline wait, else STK_OK.
int farfield_status(KernelData *kd);

}  // namespace stk
