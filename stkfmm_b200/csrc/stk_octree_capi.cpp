// stk_octree_capi.cpp -- host-only C ABI over the octree and interaction lists.
//
// Exposes the tree that Stk3DFMM_setup_tree builds (stk_tree.hpp) without any
// CUDA call, so list construction can be inspected and tested on a machine
// without a GPU, and so a caller can hand the same lists to stk_p2p_lists.
// This file and stk_tree.cpp are plain C++: besides going into
// libstkfmm_b200.so they are built on their own into libstk_octree.so, which
// a program without a GPU (or that must not map the GPU library) loads.
#include <cstring>
#include <new>
#include <string>

#include "../../include/stkfmm_b200.h"
#include "stk_tree.hpp"

struct stk_octree {
    stk::Octree tree;
};

extern "C" stk_octree *stk_octree_build(const double *tree_pts, int n, int max_pts, int pbc, const double *sl,
                                        int nsl, const double *dl, int ndl, const double *trg, int ntrg) {
    if (n < 0 || nsl < 0 || ndl < 0 || ntrg < 0) return nullptr;
    auto *t = new (std::nothrow) stk_octree();
    if (!t) return nullptr;
    std::string err = t->tree.build(tree_pts, n, max_pts, stk::kMaxDepth, pbc);
    if (err.empty()) err = t->tree.assign(0, sl, nsl);
    if (err.empty()) err = t->tree.assign(1, dl, ndl);
    if (err.empty()) err = t->tree.assign(2, trg, ntrg);
    if (!err.empty()) {
        delete t;
        return nullptr;
    }
    t->tree.build_lists();
    return t;
}

extern "C" void stk_octree_free(stk_octree *t) { delete t; }

extern "C" int stk_octree_sizes(const stk_octree *t, long long *out) {
    if (!t || !out) return STK_ERR_INVALID_ARG;
    const stk::Octree &T = t->tree;
    out[0] = T.num_nodes();
    out[1] = (long long)T.leaves.size();
    out[2] = T.depth();
    out[3] = (long long)T.U.size();
    out[4] = (long long)T.V.size();
    out[5] = (long long)T.W.size();
    out[6] = (long long)T.X.size();
    return STK_OK;
}

extern "C" int stk_octree_nodes(const stk_octree *t, int *level, int *parent, int *first_child, int *ixyz) {
    if (!t) return STK_ERR_INVALID_ARG;
    const stk::Octree &T = t->tree;
    const int nn = T.num_nodes();
    for (int i = 0; i < nn; i++) {
        if (level) level[i] = T.level[i];
        if (parent) parent[i] = T.parent[i];
        if (first_child) first_child[i] = T.first_child[i];
        if (ixyz) {
            ixyz[3 * i + 0] = (int)T.ix[i];
            ixyz[3 * i + 1] = (int)T.iy[i];
            ixyz[3 * i + 2] = (int)T.iz[i];
        }
    }
    return STK_OK;
}

// which: 0 U, 1 V, 2 W, 3 X.  off has num_nodes + 1 entries.
extern "C" int stk_octree_list(const stk_octree *t, int which, int *off, int *ent) {
    if (!t || which < 0 || which > 3) return STK_ERR_INVALID_ARG;
    const stk::Octree &T = t->tree;
    const stk::NodeList &L = which == 0 ? T.U : which == 1 ? T.V : which == 2 ? T.W : T.X;
    if (off) std::memcpy(off, L.off.data(), L.off.size() * sizeof(int));
    if (ent && !L.ent.empty()) std::memcpy(ent, L.ent.data(), L.ent.size() * sizeof(int));
    return STK_OK;
}

// set: 0 SL, 1 DL, 2 targets.  perm has n entries, node_begin / node_end num_nodes.
extern "C" int stk_octree_set(const stk_octree *t, int set, int *perm, int *node_begin, int *node_end) {
    if (!t || set < 0 || set > 2) return STK_ERR_INVALID_ARG;
    const stk::PointSet &P = t->tree.sets[set];
    if (perm && P.n) std::memcpy(perm, P.perm.data(), P.perm.size() * sizeof(int));
    if (node_begin) std::memcpy(node_begin, P.node_begin.data(), P.node_begin.size() * sizeof(int));
    if (node_end) std::memcpy(node_end, P.node_end.data(), P.node_end.size() * sizeof(int));
    return STK_OK;
}

// The shard assignment used by Stk3DFMM_set_shard: items in the given order
// (largest cost first) dealt to the least-loaded part.  Host only.
extern "C" int stk_partition_lpt(int n, const double *cost, int nparts, int *owner) {
    if (n < 0 || nparts < 1 || (n > 0 && (!cost || !owner))) return STK_ERR_INVALID_ARG;
    std::vector<int> o;
    stk::partition_lpt(n, cost, nparts, o);
    if (n) std::memcpy(owner, o.data(), sizeof(int) * n);
    return STK_OK;
}

// Owners of the M2L / S2L target nodes when Stk3DFMM's far field is split over
// nranks ranks (Stk3DFMM_set_allreduce): owner[node] in 0 .. nranks-1.  Host only.
extern "C" int stk_octree_far_owners(const stk_octree *t, int nranks, int *owner) {
    if (!t || nranks < 1 || !owner) return STK_ERR_INVALID_ARG;
    const std::vector<int> o = stk::far_owners(t->tree, nranks);
    if (!o.empty()) std::memcpy(owner, o.data(), sizeof(int) * o.size());
    return STK_OK;
}
