// stk_work.cpp -- per-thread device workspace and work-list builders.
#include "stk_work.hpp"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>

#include "../../include/stkfmm_b200.h"
#include "stk_tree.hpp"

namespace stk {

namespace {

// Workspaces outlive the threads that used them: when a thread ends (for
// example torch's autograd worker at interpreter shutdown) its workspace goes
// back to this free list, with no CUDA call, and the next new thread reuses it.
// Calling cudaFree from a thread-exit destructor can run after the CUDA runtime
// has been torn down.  The pool itself is never destroyed; its device memory
// is released with the CUDA context when the process ends.
class WorkspacePool {
  public:
    Workspace *acquire() {
        std::lock_guard<std::mutex> lock(mu_);
        if (!free_.empty()) {
            Workspace *w = free_.back();
            free_.pop_back();
            return w;
        }
        return new Workspace();
    }
    void release(Workspace *w) {
        std::lock_guard<std::mutex> lock(mu_);
        free_.push_back(w);
    }

  private:
    std::mutex mu_;
    std::vector<Workspace *> free_;
};

WorkspacePool &pool() {
    static WorkspacePool *p = new WorkspacePool();
    return *p;
}

struct WorkspaceHolder {
    Workspace *ws = pool().acquire();
    ~WorkspaceHolder() { pool().release(ws); }
};

}  // namespace

Workspace &Workspace::thread_local_ws() {
    static thread_local WorkspaceHolder holder;
    return *holder.ws;
}

Workspace::~Workspace() = default;

int Workspace::ensure_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return STK_ERR_NO_DEVICE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return STK_ERR_CUDA;
    Dev &d = devs_[dev];
    cur_ = &d;
    if (!d.stream) {
        if (cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking) != cudaSuccess) return STK_ERR_CUDA;
        if (cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return STK_ERR_CUDA;
        if (cudaMalloc(&d.counter, 64) != cudaSuccess) return STK_ERR_CUDA;
        if (cudaEventCreateWithFlags(&d.done, cudaEventDisableTiming) != cudaSuccess) return STK_ERR_CUDA;
    }
    return STK_OK;
}

int Workspace::begin(cudaStream_t s) {
    if (!cur_) return STK_ERR_CUDA;
    if (cur_->recorded && cudaStreamWaitEvent(s, cur_->done, 0) != cudaSuccess) return STK_ERR_CUDA;
    return STK_OK;
}

int Workspace::end(cudaStream_t s) {
    if (!cur_) return STK_ERR_CUDA;
    if (cudaEventRecord(cur_->done, s) != cudaSuccess) return STK_ERR_CUDA;
    cur_->recorded = true;
    return STK_OK;
}

void *Workspace::raw(int slot, size_t bytes) {
    if (!cur_ || slot < 0 || slot >= kNumSlots) return nullptr;
    if (bytes == 0) bytes = 16;
    if (cur_->cap[slot] < bytes) {
        const size_t want = std::max(bytes, cur_->cap[slot] * 3 / 2);
        if (cur_->ptr[slot]) {
            // the previous contents may still be read by work queued on any stream
            cudaDeviceSynchronize();
            cudaFree(cur_->ptr[slot]);
        }
        cur_->ptr[slot] = nullptr;
        cur_->cap[slot] = 0;
        if (cudaMalloc(&cur_->ptr[slot], want) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cur_->cap[slot] = want;
    }
    return cur_->ptr[slot];
}

unsigned int *Workspace::counter() { return cur_ ? cur_->counter : nullptr; }
int Workspace::num_sms() { return cur_ ? cur_->sms : 1; }
cudaStream_t Workspace::stream() { return cur_ ? cur_->stream : nullptr; }

// A warp has 64 target slots (two per lane); items hold at most kItemTargets targets.
constexpr int kItemTargets = 64;

static inline int lanes_log2(int m) {
    // largest g = 2^glog <= 32 with m * g <= 64 slots
    int glog = 0;
    while (glog < 5 && (m << (glog + 1)) <= kItemTargets) glog++;
    return glog;
}

void build_direct_items(int ntrg, int nsrc, int num_sms, std::vector<WorkItem> &items, std::vector<int> &src_begin,
                        std::vector<int> &src_end, std::vector<int> &ent) {
    const int nchunk = (ntrg + kItemTargets - 1) / kItemTargets;
    // enough items to fill every warp slot several times over, but source
    // chunks of at least 256 points
    const long long want_items = (long long)std::max(num_sms, 1) * 64;
    int nsc = (int)std::max(1LL, (want_items + nchunk - 1) / nchunk);
    nsc = std::min(nsc, std::max(1, nsrc / 256));
    int sc = (nsrc + nsc - 1) / nsc;
    sc = (sc + 31) / 32 * 32;
    nsc = (nsrc + sc - 1) / sc;
    src_begin.resize(nsc);
    src_end.resize(nsc);
    ent.resize(nsc);
    for (int k = 0; k < nsc; k++) {
        src_begin[k] = k * sc;
        src_end[k] = std::min(nsrc, (k + 1) * sc);
        ent[k] = (k << 5) | kShiftNone;
    }
    items.clear();
    items.reserve((size_t)nchunk * nsc);
    // full chunks first (largest cost), the ragged last chunk at the end
    for (int c = 0; c < nchunk; c++) {
        const int t0 = kItemTargets * c;
        const int m = std::min(kItemTargets, ntrg - t0);
        for (int k = 0; k < nsc; k++) items.push_back({c, t0, m, lanes_log2(m), k, k + 1});
    }
}

void build_list_items(int n_trg_box, const int *trg_begin, const int *trg_end, const int *list_off,
                      const int *list_ent, const int *src_begin, const int *src_end, std::vector<WorkItem> &items,
                      long long &pairs, int balance_warps, int shard_rank, int shard_n) {
    items.clear();
    pairs = 0;
    std::vector<long long> box_ns(n_trg_box, 0);
    for (int b = 0; b < n_trg_box; b++) {
        const int nt = trg_end[b] - trg_begin[b];
        if (nt <= 0) continue;
        long long ns = 0;
        for (int e = list_off[b]; e < list_off[b + 1]; e++) {
            const int sb = list_ent[e] >> 5;
            ns += src_end[sb] - src_begin[sb];
        }
        box_ns[b] = ns;
        pairs += (long long)nt * ns;
    }
    // Load balance: no item above ~half of one warp's share of the pairs, so a
    // box with very many sources (a long W list) is not a single long item that
    // finishes after every other warp.  Items keep at least 8 targets (64 slots
    // filled with 8 lanes per target).
    const long long cap = balance_warps > 0 ? std::max(pairs / (2LL * balance_warps), 1LL) : 0;
    std::vector<double> cost;
    for (int b = 0; b < n_trg_box; b++) {
        const int nt = trg_end[b] - trg_begin[b];
        const long long ns = box_ns[b];
        if (nt <= 0 || ns == 0) continue;
        int mmax = kItemTargets;
        while (cap > 0 && mmax > 8 && (long long)mmax * ns > cap) mmax /= 2;
        // Split the box into full mmax-target items, then power-of-two chunks of
        // the remainder (32, 16, 8 targets; the last < 8 targets together): a
        // chunk of m = 2^k targets fills all 64 slots with 64/m lanes per target,
        // so the box costs ~nt/64 warp passes over its sources instead of
        // ceil(nt/64).  Chunks below 8 targets would mostly re-stage sources.
        int t0 = trg_begin[b];
        int left = nt;
        while (left > 0) {
            int m = mmax;
            if (left < mmax) {
                m = 1;
                while (m * 2 <= left) m *= 2;
                if (m < 8) m = left;
            }
            const int glog = lanes_log2(m);
            items.push_back({b, t0, m, glog, list_off[b], list_off[b + 1]});
            cost.push_back((double)ns / (1 << glog) + 64.0 * (list_off[b + 1] - list_off[b]));
            t0 += m;
            left -= m;
        }
    }
    std::vector<int> idx(items.size());
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<WorkItem> sorted;
    sorted.reserve(items.size());
    if (shard_n > 1) {
        // this shard's items: the cost-sorted items dealt to the least-loaded
        // shard in turn (the same deterministic assignment on every shard)
        std::vector<int> owner;
        std::vector<double> sc;
        for (int i : idx) sc.push_back(cost[i]);
        partition_lpt((int)sc.size(), sc.data(), shard_n, owner);
        pairs = 0;
        for (size_t i = 0; i < idx.size(); i++)
            if (owner[i] == shard_rank) {
                const WorkItem &w = items[idx[i]];
                sorted.push_back(w);
                pairs += (long long)w.nt * pair_sources(w, list_ent, src_begin, src_end);
            }
    } else {
        for (size_t i = 0; i < idx.size(); i++) sorted.push_back(items[idx[i]]);
    }
    items.swap(sorted);
}

long long pair_sources(const WorkItem &w, const int *list_ent, const int *src_begin, const int *src_end) {
    long long ns = 0;
    for (int e = w.e0; e < w.e1; e++) {
        const int sb = list_ent[e] >> 5;
        ns += src_end[sb] - src_begin[sb];
    }
    return ns;
}

void morton_order(const double *xyz, int n, std::vector<int> &order, std::vector<double> &sorted) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], xyz[3 * (size_t)i + k]);
            hi[k] = std::max(hi[k], xyz[3 * (size_t)i + k]);
        }
    double span = 0;
    for (int k = 0; k < 3; k++) span = std::max(span, hi[k] - lo[k]);
    const double inv = span > 0 ? 1.0 / (span * (1.0 + 1e-12)) : 0.0;
    std::vector<uint64_t> key(n);
    for (int i = 0; i < n; i++) {
        double u[3];
        for (int k = 0; k < 3; k++) u[k] = std::min(std::max((xyz[3 * (size_t)i + k] - lo[k]) * inv, 0.0), 0.999999999);
        key[i] = morton_key(u[0], u[1], u[2]);
    }
    order.resize(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
    sorted.resize(3 * (size_t)n);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) sorted[3 * (size_t)i + k] = xyz[3 * (size_t)order[i] + k];
}

}  // namespace stk
