// stk_handle.hpp -- state behind the opaque Stk3DFMM handle.
#pragma once
#include <functional>
#include <map>
#include <memory>
#include <vector>

#include <cuda_runtime.h>

#include "stk_kernel_table.hpp"
#include "stk_tree.hpp"

namespace stk {

// Owned device allocation (grow-only).
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    // owner of the allocation: share() makes another DevBuf an alias of the same
    // memory (read-only use, e.g. far-field operators shared between handles); the
    // memory is freed with its last owner.  reserve() never writes into memory that
    // another DevBuf shares: it allocates afresh instead.
    std::shared_ptr<void> owner;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release();
    int reserve(size_t n);
    int upload(const void *src, size_t n, cudaStream_t s);
    void share(const DevBuf &o) {
        owner = o.owner;
        ptr = o.ptr;
        bytes = o.bytes;
    }
    bool shared() const { return owner && owner.use_count() > 1; }
};

struct FarField;

// One activated kernel: the reference's impl::FMMData (STKFMM_impl.hpp:19-174).
struct KernelData {
    const KernelInfo *info = nullptr;
    Octree tree;
    bool tree_ready = false;
    bool fused = false;            // SL and DL at the same points: one fused U-list pass
    long long u_pairs[2] = {0, 0}; // exact U-list (target, source point) pairs, SL and DL
    int n_items[2] = {0, 0};
    DevBuf d_xyz[3], d_perm[3], d_beg[3], d_end[3];  // per point set: sorted coords, perm, node ranges
    DevBuf d_centre, d_uent, d_items[2], d_counter;
    DevBuf d_val[2], d_rec[2], d_out_sorted, d_out_user, d_alpha;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // bracket the kernel launches of the last evaluation
    bool timed = false;
    // end of each phase of the last evaluation: 0 U-list P2P, 1 S2M (+ solve),
    // 2 M2M, 3 M2L, 4 S2L (+ solve), 5 L2L, 6 L2T, 7 M2T
    static constexpr int kPhases = 8;
    cudaEvent_t ph[kPhases] = {};
    bool last_far = false;
    int launches = 0;  // own kernels launched by the last evaluation (cuBLAS calls excluded)
    std::unique_ptr<FarField> far;  // KIFMM operators and per-tree far-field data
    bool far_ready = false;
    ~KernelData();
};

}  // namespace stk

struct Stk3DFMM {
    int mult_order = 10, max_pts = 2000, pbc = 0;
    unsigned kernel_comb = 0;
    double origin[3] = {0, 0, 0};
    double len = 1.0, scale_factor = 1.0;
    int precision = 0;
    int device = 0, sms = 1;
    int shard_rank = 0, shard_n = 1;  // target-side work of this handle: shard shard_rank of shard_n
    // collective of the shard group: with it the far field's M2L / S2L are split too
    int (*allreduce)(double *, long long, void *, void *) = nullptr;
    void *allreduce_user = nullptr;
    // periodic far field (the reference's enableFF, STKFMM.hpp:199-200): off, the
    // periodic sum stops two cells away
    bool enable_ff = true;
    cudaStream_t stream = nullptr;
    // host-array evaluations: the caller's target array is uploaded on aux_stream
    // while the P2P kernels run (ev_out joins it before the final scatter)
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t ev_out = nullptr;
    bool points_set = false, sl_dl_same = false;
    int nsl = 0, ndl = 0, ntrg = 0;
    std::vector<double> sl, dl, trg;  // scaled, wrapped coordinates (caller's order)
    // points that refine the octree in place of the largest of sl / dl / trg
    // (FMMData::setupTree's custom tree points, FMMData.cpp:131-135); unit-box
    // coordinates, set by composite FMMs (StkWallFMM), empty otherwise
    std::vector<double> tree_pts;
    std::map<unsigned, std::unique_ptr<stk::KernelData>> pool;
    ~Stk3DFMM();
};

namespace stk {
// before_scatter (optional) runs on the host right before the final scatter into
// d_out_user is queued on s (after every P2P / far-field launch): host-array
// callers upload the target array there, overlapping the kernels.
int near_device(Stk3DFMM *f, KernelData *kd, const double *d_sl, const double *d_dl, double *d_out_user,
                cudaStream_t s, bool far, const std::function<int()> &before_scatter = nullptr);
}
