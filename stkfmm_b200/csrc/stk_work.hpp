// stk_work.hpp -- per-thread device workspace and work-list builders (host C++).
#pragma once
#include <cstddef>
#include <map>
#include <vector>

#include <cuda_runtime.h>

#include "stk_p2p.cuh"

namespace stk {

// Grow-only device buffers, one set per (host thread, device), plus a
// non-blocking stream and the persistent-kernel work counter.  The stateless
// C-ABI calls (direct sums, ker_poten shims, list calls) use it, so they are
// re-entrant across host threads (the reference calls ker_poten from OpenMP
// threads concurrently, Lib/src/FMMData.cpp:275-282).  A workspace is handed
// to the next thread when its thread ends and is never freed before exit.
class Workspace {
  public:
    enum Slot { kRec, kSrcBeg, kSrcEnd, kEnt, kItems, kHostSrc, kHostVal, kHostTrg, kHostOut, kNumSlots };
    static Workspace &thread_local_ws();
    ~Workspace();
    int ensure_device();  // STK_OK, STK_ERR_NO_DEVICE or STK_ERR_CUDA
    // Stream ordering of the workspace's buffers across calls: begin() makes
    // `s` wait for the work that the previous call queued on its stream (which
    // may still read the buffers), end() marks the end of this call's work on
    // `s`.  Calls then return without a host wait.
    int begin(cudaStream_t s);
    int end(cudaStream_t s);
    template <class T> T *buf(int slot, size_t n) { return static_cast<T *>(raw(slot, n * sizeof(T))); }
    unsigned int *counter();
    int num_sms();
    cudaStream_t stream();

  private:
    struct Dev {
        void *ptr[kNumSlots] = {};
        size_t cap[kNumSlots] = {};
        unsigned int *counter = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;  // end of the last call's work on its stream
        bool recorded = false;
        int sms = 0;
    };
    std::map<int, Dev> devs_;
    Dev *cur_ = nullptr;
    void *raw(int slot, size_t bytes);
};

// Direct sum as a list problem: 64-target chunks x source chunks.
void build_direct_items(int ntrg, int nsrc, int num_sms, std::vector<WorkItem> &items, std::vector<int> &src_begin,
                        std::vector<int> &src_end, std::vector<int> &ent);

// Cost-sorted work items for an explicit list; pairs = exact (target, source point) pair count.
// balance_warps > 0: boxes with many sources get smaller target chunks, so that no
// item holds more than ~pairs / (2 balance_warps) pairs.  shard_n > 1: only the items
// of shard shard_rank are kept (partition_lpt over the cost-sorted items), and pairs
// counts those.
void build_list_items(int n_trg_box, const int *trg_begin, const int *trg_end, const int *list_off,
                      const int *list_ent, const int *src_begin, const int *src_end, std::vector<WorkItem> &items,
                      long long &pairs, int balance_warps = 0, int shard_rank = 0, int shard_n = 1);

// Source points of one work item (the sum over its list entries).
long long pair_sources(const WorkItem &w, const int *list_ent, const int *src_begin, const int *src_end);

// Morton order of points inside their own bounding box.
void morton_order(const double *xyz, int n, std::vector<int> &order, std::vector<double> &sorted);

}  // namespace stk
