// stk_p2p.cuh -- host-side interface of the sm_100a P2P kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace stk {

enum Precision : int { PREC_FP64 = 0, PREC_MIXED = 1 };

// One unit of P2P work: up to 64 targets of one target box against source-list
// entries [e0, e1).  A warp has 64 target slots (two per lane); glog =
// log2(slots per target) <= 5: the lanes that share a target split the source
// tile and are reduced with warp shuffles.
struct WorkItem {
    int trg_box;
    int t0;   // first target (leaf-sorted index)
    int nt;   // number of targets (1..64)
    int glog; // lanes per target = 1 << glog
    int e0;   // first list entry
    int e1;   // one past the last list entry
};

// Device-resident description of one list evaluation.
struct ListP2PArgs {
    const double *src_rec;     // source records, RS doubles each: x, y, z, values..., padding
    const int *src_box_begin;  // per source box: first record
    const int *src_box_end;    // per source box: one past the last record
    const int *list_ent;       // per entry: (source box << 5) | periodic shift code (0..26, 13 = none)
    const WorkItem *items;     // cost-sorted work items
    int n_items;
    unsigned int *counter;     // work counter, zero at launch
    const double *trg_xyz;     // targets, 3 doubles each
    double *trg_out;           // outputs, TDIM doubles each, accumulated
    const double *box_centre;  // per target box: local origin for the mixed path (3 doubles)
    double period;             // periodic image length (1 for the unit box)
    int atomic_out;            // 1 when several items may write the same target
    const double *trg_aux;     // per-target values (TV doubles each) of the adjoint kernels, else null
    int coincident_own_box;    // 1: a source can sit at a target's position only in an unshifted
                               // entry of the target's own box (lists of one octree over both
                               // point sets); the mixed path then skips the coincidence mask
                               // elsewhere.  0: every pair is masked.
};

// Record stride (doubles) for a micro-kernel: 3 coordinates + SDIM values,
// rounded up to a 16-byte multiple.
int uk_record_stride(int uk);
int uk_sdim_host(int uk);
int uk_tdim_host(int uk);
int uk_tvdim_host(int uk);  // per-target values read by a micro-kernel (adjoint kernels)
double uk_scale_host(int uk);

// Launch the list kernel for micro-kernel `uk` with the given precision.
cudaError_t launch_list_p2p(int uk, int prec, const ListP2PArgs &a, int num_sms, cudaStream_t stream);

// rec[i] = (xyz[perm[i]], v1[perm[i]] (d1 values), v2[perm[i]] (d2 values), 0 padding)
// perm may be null (identity).  v2 may be null (d2 = 0).  Coordinates are
// multiplied by coord_scale after subtracting coord_shift (per axis).
cudaError_t launch_pack_records(int n, const int *perm, const double *xyz, const double *v1, int d1,
                                const double *v2, int d2, int stride, double *rec, cudaStream_t stream);

// out[perm[i] * d + k] += alpha_k * in[i * d + k]   (alpha per component; perm may be null)
cudaError_t launch_scatter_add(int n, int d, const int *perm, const double *in, const double *alpha,
                               double *out, cudaStream_t stream);

}  // namespace stk
