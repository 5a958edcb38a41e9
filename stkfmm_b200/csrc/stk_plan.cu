// stk_plan.cu -- a reusable, asynchronous list P2P plan (C ABI stk_p2p_plan_*).
//
// stk_p2p_lists validates a CSR interaction list, builds its cost-sorted work
// items on the host, uploads them and waits for the result on every call.  A
// caller that evaluates the same list many times (PVFMM's list loops call
// ker_poten for the same U/W/X lists at every evaluation; an autograd forward
// and its two adjoint passes share one U list) builds a plan once instead:
// stk_p2p_plan_create validates the list, builds the items and uploads the list
// and the items into device memory owned by the plan; stk_p2p_plan_execute then
// queues the pack and list kernels on the caller's stream and returns without a
// host wait.
#include <algorithm>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/stkfmm_b200.h"
#include "stk_p2p.cuh"
#include "stk_ukernels.cuh"
#include "stk_work.hpp"

struct stk_p2p_plan {
    int device = -1;
    int num_sms = 1;
    int nsrc = 0, ntrg = 0;
    int n_src_box = 0;
    double period = 1.0;
    long long pairs = 0;
    int n_items = 0;
    int *d_sbeg = nullptr, *d_send = nullptr, *d_ent = nullptr;
    stk::WorkItem *d_items = nullptr;
    unsigned int *d_counter = nullptr;
    double *d_rec = nullptr;  // packed source records, grown to the largest record stride used
    size_t rec_cap = 0;       // doubles
    ~stk_p2p_plan() {
        cudaFree(d_sbeg);
        cudaFree(d_send);
        cudaFree(d_ent);
        cudaFree(d_items);
        cudaFree(d_counter);
        cudaFree(d_rec);
    }
};

namespace {

int validate_lists(int n_trg_box, const int *trg_begin, const int *trg_end, const int *list_off,
                   const int *list_ent, int n_src_box, const int *src_begin, const int *src_end, int nsrc,
                   int ntrg) {
    if (n_trg_box < 0 || n_src_box < 0 || nsrc < 0 || ntrg < 0) return STK_ERR_INVALID_ARG;
    if (n_trg_box > 0 && (!trg_begin || !trg_end || !list_off)) return STK_ERR_INVALID_ARG;
    if (n_trg_box > 0 && list_off[0] != 0) return STK_ERR_INVALID_ARG;
    if (n_src_box > 0 && (!src_begin || !src_end)) return STK_ERR_INVALID_ARG;
    for (int b = 0; b < n_trg_box; b++) {
        if (trg_begin[b] < 0 || trg_end[b] < trg_begin[b] || trg_end[b] > ntrg) return STK_ERR_INVALID_ARG;
        if (list_off[b + 1] < list_off[b]) return STK_ERR_INVALID_ARG;
    }
    for (int s = 0; s < n_src_box; s++)
        if (src_begin[s] < 0 || src_end[s] < src_begin[s] || src_end[s] > nsrc) return STK_ERR_INVALID_ARG;
    const int nent = n_trg_box > 0 ? list_off[n_trg_box] : 0;
    if (nent > 0 && !list_ent) return STK_ERR_INVALID_ARG;
    for (int e = 0; e < nent; e++) {
        const int sb = list_ent[e] >> 5, code = list_ent[e] & 31;
        if (list_ent[e] < 0 || sb >= n_src_box || code > 26) return STK_ERR_INVALID_ARG;
    }
    return STK_OK;
}

template <class T> cudaError_t upload(T **dst, const T *src, size_t n) {
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, n * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

extern "C" stk_p2p_plan *stk_p2p_plan_create(int n_trg_box, const int *trg_begin, const int *trg_end,
                                             const int *list_off, const int *list_ent, int n_src_box,
                                             const int *src_begin, const int *src_end, int nsrc, int ntrg,
                                             double period, int *status) {
    int dummy = 0;
    int &st = status ? *status : dummy;
    st = validate_lists(n_trg_box, trg_begin, trg_end, list_off, list_ent, n_src_box, src_begin, src_end, nsrc, ntrg);
    if (st) return nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        st = STK_ERR_NO_DEVICE;
        return nullptr;
    }
    auto *p = new (std::nothrow) stk_p2p_plan();
    if (!p) {
        st = STK_ERR_CUDA;
        return nullptr;
    }
    p->nsrc = nsrc;
    p->ntrg = ntrg;
    p->n_src_box = n_src_box;
    p->period = period;
    std::vector<stk::WorkItem> items;
    if (n_trg_box > 0)
        stk::build_list_items(n_trg_box, trg_begin, trg_end, list_off, list_ent, src_begin, src_end, items, p->pairs);
    p->n_items = (int)items.size();
    const int nent = n_trg_box > 0 ? list_off[n_trg_box] : 0;
    bool ok = cudaGetDevice(&p->device) == cudaSuccess &&
              cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device) == cudaSuccess &&
              cudaMalloc(&p->d_counter, 64) == cudaSuccess && upload(&p->d_sbeg, src_begin, n_src_box) == cudaSuccess &&
              upload(&p->d_send, src_end, n_src_box) == cudaSuccess && upload(&p->d_ent, list_ent, nent) == cudaSuccess &&
              upload(&p->d_items, items.data(), items.size()) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        delete p;
        st = STK_ERR_CUDA;
        return nullptr;
    }
    return p;
}

extern "C" void stk_p2p_plan_destroy(stk_p2p_plan *plan) {
    if (!plan) return;
    int cur = -1;
    cudaGetDevice(&cur);
    const int dev = plan->device;
    if (dev >= 0 && dev != cur) cudaSetDevice(dev);
    cudaDeviceSynchronize();  // work queued on any stream may still read the plan's buffers
    delete plan;
    if (cur >= 0 && dev >= 0 && dev != cur) cudaSetDevice(cur);
}

extern "C" long long stk_p2p_plan_pairs(const stk_p2p_plan *plan) { return plan ? plan->pairs : -1; }

extern "C" int stk_p2p_plan_execute(stk_p2p_plan *plan, int ukernel, int precision, const double *d_src_coord,
                                    const double *d_src_value, const double *d_trg_coord, const double *d_trg_aux,
                                    double *d_trg_value, void *stream) {
    if (!plan || ukernel < 0 || ukernel >= stk::UK_COUNT) return STK_ERR_INVALID_ARG;
    if (precision != stk::PREC_FP64 && precision != stk::PREC_MIXED) return STK_ERR_INVALID_ARG;
    if ((stk::uk_tvdim_host(ukernel) > 0) != (d_trg_aux != nullptr)) return STK_ERR_INVALID_ARG;
    if (plan->n_items == 0) return STK_OK;
    if ((plan->nsrc > 0 && (!d_src_coord || !d_src_value)) || !d_trg_coord || !d_trg_value) return STK_ERR_INVALID_ARG;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != plan->device) return STK_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const int sd = stk::uk_sdim_host(ukernel), rs = stk::uk_record_stride(ukernel);
    const size_t need = (size_t)std::max(plan->nsrc, 1) * rs;
    if (plan->rec_cap < need) {
        // grow the record buffer: earlier executions may still read it on any stream
        if (plan->d_rec) {
            cudaDeviceSynchronize();
            cudaFree(plan->d_rec);
            plan->d_rec = nullptr;
            plan->rec_cap = 0;
        }
        if (cudaMalloc(&plan->d_rec, need * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return STK_ERR_CUDA;
        }
        plan->rec_cap = need;
    }
    if (stk::launch_pack_records(plan->nsrc, nullptr, d_src_coord, d_src_value, sd, nullptr, 0, rs, plan->d_rec, s) !=
        cudaSuccess)
        return STK_ERR_CUDA;
    stk::ListP2PArgs a{};
    a.src_rec = plan->d_rec;
    a.src_box_begin = plan->d_sbeg;
    a.src_box_end = plan->d_send;
    a.list_ent = plan->d_ent;
    a.items = plan->d_items;
    a.n_items = plan->n_items;
    a.counter = plan->d_counter;
    a.trg_xyz = d_trg_coord;
    a.trg_out = d_trg_value;
    a.box_centre = nullptr;
    a.period = plan->period;
    a.atomic_out = 0;
    a.trg_aux = d_trg_aux;
    if (stk::launch_list_p2p(ukernel, precision, a, plan->num_sms, s) != cudaSuccess) return STK_ERR_CUDA;
    return STK_OK;
}
