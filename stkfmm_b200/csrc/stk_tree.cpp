// stk_tree.cpp -- adaptive octree and KIFMM interaction lists (host C++).
#include "stk_tree.hpp"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <unordered_set>

namespace stk {

namespace {

inline uint64_t spread3(uint64_t v) {
    v &= 0x1fffffULL;
    v = (v | (v << 32)) & 0x1f00000000ffffULL;
    v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
    v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
    v = (v | (v << 2)) & 0x1249249249249249ULL;
    return v;
}

inline uint64_t interleave(uint64_t x, uint64_t y, uint64_t z) { return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2); }

inline uint32_t quantize(double x) {
    const double s = (double)(1u << kMaxDepth);
    double q = std::floor(x * s);
    if (q < 0) q = 0;
    if (q > s - 1) q = s - 1;
    return (uint32_t)q;
}

// unique key of a node: a marker bit above the 3l Morton bits
inline uint64_t node_key(int l, uint64_t x, uint64_t y, uint64_t z) { return (1ULL << (3 * l)) | interleave(x, y, z); }

}  // namespace

uint64_t morton_key(double x, double y, double z) { return interleave(quantize(x), quantize(y), quantize(z)); }

double Octree::side(int i) const { return std::ldexp(1.0, -level[i]); }

void Octree::corner(int i, double c[3]) const {
    const double h = side(i);
    c[0] = ix[i] * h;
    c[1] = iy[i] * h;
    c[2] = iz[i] * h;
}

void Octree::centre(int i, double c[3]) const {
    const double h = side(i);
    c[0] = (ix[i] + 0.5) * h;
    c[1] = (iy[i] + 0.5) * h;
    c[2] = (iz[i] + 0.5) * h;
}

int Octree::find(int l, int64_t x, int64_t y, int64_t z) const {
    auto it = lookup_.find(node_key(l, (uint64_t)x, (uint64_t)y, (uint64_t)z));
    return it == lookup_.end() ? -1 : it->second;
}

bool Octree::adjacent(int a, int shift, int b) const {
    const int L = std::max(level[a], level[b]);
    const int sa = L - level[a], sb = L - level[b];
    const int64_t n = 1LL << L;
    const int64_t s[3] = {shift % 3 - 1, (shift / 3) % 3 - 1, shift / 9 - 1};
    const uint32_t ac[3] = {ix[a], iy[a], iz[a]};
    const uint32_t bc[3] = {ix[b], iy[b], iz[b]};
    for (int k = 0; k < 3; k++) {
        const int64_t alo = ((int64_t)ac[k] << sa) + s[k] * n, ahi = alo + (1LL << sa);
        const int64_t blo = (int64_t)bc[k] << sb, bhi = blo + (1LL << sb);
        if (alo > bhi || blo > ahi) return false;
    }
    return true;
}

std::string Octree::build(const double *pts, int n, int max_pts, int max_depth, int pbc_) {
    if (n < 0 || (n > 0 && !pts)) return "invalid tree points";
    if (max_pts < 1) return "max_pts must be >= 1";
    if (pbc_ < 0 || pbc_ > 3) return "pbc must be 0..3";
    pbc = pbc_;
    max_depth = std::max(0, std::min(max_depth, kMaxDepth));
    std::vector<uint64_t> keys(n);
    for (int i = 0; i < n; i++) {
        const double *p = pts + 3 * (size_t)i;
        for (int k = 0; k < 3; k++)
            if (!(p[k] >= 0.0 && p[k] < 1.0)) return "tree point outside the unit box after scaling";
        keys[i] = morton_key(p[0], p[1], p[2]);
    }
    std::sort(keys.begin(), keys.end());

    level.assign(1, 0);
    parent.assign(1, -1);
    first_child.assign(1, -1);
    ix.assign(1, 0);
    iy.assign(1, 0);
    iz.assign(1, 0);
    key_lo_.assign(1, 0);
    std::vector<int> pbeg(1, 0), pend(1, n);
    for (size_t i = 0; i < level.size(); i++) {
        const int l = level[i];
        if (pend[i] - pbeg[i] <= max_pts || l >= max_depth) continue;
        first_child[i] = (int)level.size();
        const int cs = 3 * (kMaxDepth - l - 1);
        for (int c = 0; c < 8; c++) {
            const uint64_t lo = key_lo_[i] + ((uint64_t)c << cs);
            const uint64_t hi = lo + (1ULL << cs);
            level.push_back(l + 1);
            parent.push_back((int)i);
            first_child.push_back(-1);
            ix.push_back(2 * ix[i] + (c & 1));
            iy.push_back(2 * iy[i] + ((c >> 1) & 1));
            iz.push_back(2 * iz[i] + ((c >> 2) & 1));
            key_lo_.push_back(lo);
            pbeg.push_back((int)(std::lower_bound(keys.begin() + pbeg[i], keys.begin() + pend[i], lo) - keys.begin()));
            pend.push_back((int)(std::lower_bound(keys.begin() + pbeg[i], keys.begin() + pend[i], hi) - keys.begin()));
        }
    }
    const int nn = (int)level.size();
    max_level = level.back();
    level_begin.assign(max_level + 2, nn);
    for (int i = nn - 1; i >= 0; i--) level_begin[level[i]] = i;
    level_begin[max_level + 1] = nn;
    lookup_.clear();
    lookup_.reserve(nn * 2);
    for (int i = 0; i < nn; i++) lookup_[node_key(level[i], ix[i], iy[i], iz[i])] = i;
    leaves.clear();
    for (int i = 0; i < nn; i++)
        if (first_child[i] < 0) leaves.push_back(i);
    std::sort(leaves.begin(), leaves.end(), [&](int a, int b) { return key_lo_[a] < key_lo_[b]; });
    for (auto &s : sets) s = PointSet();
    U = V = W = X = NodeList();
    return "";
}

std::string Octree::assign(int set, const double *xyz, int n) {
    if (set < 0 || set > 2) return "invalid point set";
    if (n < 0 || (n > 0 && !xyz)) return "invalid points";
    PointSet &ps = sets[set];
    ps.n = n;
    std::vector<uint64_t> keys(n);
    for (int i = 0; i < n; i++) {
        const double *p = xyz + 3 * (size_t)i;
        for (int k = 0; k < 3; k++)
            if (!(p[k] >= 0.0 && p[k] < 1.0)) return "point outside the unit box after scaling";
        keys[i] = morton_key(p[0], p[1], p[2]);
    }
    ps.perm.resize(n);
    std::iota(ps.perm.begin(), ps.perm.end(), 0);
    std::stable_sort(ps.perm.begin(), ps.perm.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    ps.xyz.resize(3 * (size_t)n);
    ps.key.resize(n);
    for (int i = 0; i < n; i++) {
        const int p = ps.perm[i];
        ps.key[i] = keys[p];
        for (int k = 0; k < 3; k++) ps.xyz[3 * (size_t)i + k] = xyz[3 * (size_t)p + k];
    }
    const int nn = num_nodes();
    ps.node_begin.resize(nn);
    ps.node_end.resize(nn);
    for (int i = 0; i < nn; i++) {
        const uint64_t lo = key_lo_[i];
        const uint64_t hi = lo + (1ULL << (3 * (kMaxDepth - level[i])));
        ps.node_begin[i] = (int)(std::lower_bound(ps.key.begin(), ps.key.end(), lo) - ps.key.begin());
        ps.node_end[i] = (int)(std::lower_bound(ps.key.begin(), ps.key.end(), hi) - ps.key.begin());
    }
    return "";
}

namespace {
NodeList to_csr(const std::vector<std::vector<int>> &v) {
    NodeList L;
    L.off.resize(v.size() + 1, 0);
    for (size_t i = 0; i < v.size(); i++) L.off[i + 1] = L.off[i] + (int)v[i].size();
    L.ent.reserve(L.off.back());
    for (auto &x : v) L.ent.insert(L.ent.end(), x.begin(), x.end());
    return L;
}
}  // namespace

void Octree::build_lists() {
    const int nn = num_nodes();
    std::vector<std::vector<int>> Ul(nn), Vl(nn), Wl(nn), Xl(nn);
    const bool per[3] = {pbc >= 1, pbc >= 2, pbc >= 3};

    // Visit the 27 same-level neighbour positions of node b at level l, wrapping
    // periodic axes; calls f(node_or_-1, shift_code, wrapped position).
    auto neighbours = [&](int b, auto &&f) {
        const int l = level[b];
        const int64_t ns = 1LL << l;
        for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    int64_t p[3] = {(int64_t)ix[b] + dx, (int64_t)iy[b] + dy, (int64_t)iz[b] + dz};
                    int s[3] = {0, 0, 0};
                    bool ok = true;
                    for (int k = 0; k < 3; k++) {
                        if (p[k] < 0 || p[k] >= ns) {
                            if (!per[k]) {
                                ok = false;
                                break;
                            }
                            s[k] = p[k] < 0 ? -1 : 1;
                            p[k] -= s[k] * ns;
                        }
                    }
                    if (!ok) continue;
                    f(find(l, p[0], p[1], p[2]), shift_code(s[0], s[1], s[2]), p, l);
                }
    };

    for (int b : leaves) {
        if (trg_count(b) == 0) continue;
        std::unordered_set<long long> seenU, seenW;
        auto addU = [&](int node, int code) {
            if (src_count(node) == 0) return;
            if (seenU.insert((long long)node * 32 + code).second) Ul[b].push_back((node << 5) | code);
        };
        auto addW = [&](int node, int code) {
            if (src_count(node) == 0) return;
            if (seenW.insert((long long)node * 32 + code).second) Wl[b].push_back((node << 5) | code);
        };
        neighbours(b, [&](int node, int code, const int64_t *p, int l) {
            if (node >= 0) {
                if (is_leaf(node)) {
                    addU(node, code);
                    return;
                }
                std::vector<int> stack(1, node);
                while (!stack.empty()) {
                    const int m = stack.back();
                    stack.pop_back();
                    for (int c = first_child[m]; c < first_child[m] + 8; c++) {
                        if (src_count(c) == 0) continue;
                        if (adjacent(c, code, b)) {
                            if (is_leaf(c))
                                addU(c, code);
                            else
                                stack.push_back(c);
                        } else {
                            addW(c, code);
                        }
                    }
                }
            } else {
                // the position is covered by a coarser leaf
                int a = -1;
                for (int ll = l - 1; ll >= 0 && a < 0; ll--)
                    a = find(ll, p[0] >> (l - ll), p[1] >> (l - ll), p[2] >> (l - ll));
                if (a >= 0) addU(a, code);
            }
        });
        std::sort(Ul[b].begin(), Ul[b].end());
        std::sort(Wl[b].begin(), Wl[b].end());
    }

    // V: children of the parent's colleagues that are not adjacent
    for (int b = 1; b < nn; b++) {
        if (trg_count(b) == 0) continue;
        const int P = parent[b];
        neighbours(P, [&](int node, int code, const int64_t *, int) {
            if (node < 0 || is_leaf(node)) return;
            for (int c = first_child[node]; c < first_child[node] + 8; c++) {
                if (src_count(c) == 0) continue;
                if (!adjacent(c, code, b)) Vl[b].push_back((c << 5) | code);
            }
        });
        std::sort(Vl[b].begin(), Vl[b].end());
    }

    // X: the W relation seen from the source side.  For every leaf a with
    // sources, the nodes with targets that are descendants of a's colleagues,
    // not adjacent to a, with a parent adjacent to a, gain a (with the inverse
    // shift).  Walking from the source leaves also covers source leaves that hold
    // no targets, which have no W list of their own.
    for (int a : leaves) {
        if (src_count(a) == 0) continue;
        neighbours(a, [&](int node, int code, const int64_t *, int) {
            if (node < 0 || is_leaf(node)) return;
            std::vector<int> stack(1, node);
            while (!stack.empty()) {
                const int m = stack.back();
                stack.pop_back();
                for (int c = first_child[m]; c < first_child[m] + 8; c++) {
                    if (trg_count(c) == 0) continue;
                    if (adjacent(c, code, a)) {
                        if (!is_leaf(c)) stack.push_back(c);
                    } else {
                        Xl[c].push_back((a << 5) | shift_negate(code));
                    }
                }
            }
        });
    }
    for (auto &x : Xl) {
        std::sort(x.begin(), x.end());
        x.erase(std::unique(x.begin(), x.end()), x.end());
    }

    U = to_csr(Ul);
    V = to_csr(Vl);
    W = to_csr(Wl);
    X = to_csr(Xl);
}

void partition_lpt(int n, const double *cost, int nparts, std::vector<int> &owner) {
    owner.assign(n, 0);
    if (nparts <= 1) return;
    std::vector<double> load(nparts, 0.0);
    for (int i = 0; i < n; i++) {
        int best = 0;
        for (int r = 1; r < nparts; r++)
            if (load[r] < load[best]) best = r;
        owner[i] = best;
        load[best] += cost[i];
    }
}

// Owners of the M2L / S2L target nodes when the far field is split over nranks:
// the nodes of complete levels (all 8^l boxes, l >= 1) by parity type
// ((ix & 1) | (iy & 1) << 1 | (iz & 1) << 2) mod nranks -- the dense M2L splits
// its work by target type -- and every other node, largest first by its V-list
// and X-list size, to the least loaded rank (LPT).  Host only, deterministic.
std::vector<int> far_owners(const Octree &T, int nranks) {
    const int nn = T.num_nodes();
    std::vector<int> owner(nn, 0);
    if (nranks <= 1) return owner;
    std::vector<double> load(nranks, 0.0);
    std::vector<char> done(nn, 0);
    auto cost = [&](int b) { return 1.0 + (T.V.off[b + 1] - T.V.off[b]) + (T.X.off[b + 1] - T.X.off[b]); };
    for (int l = 1; l <= T.depth(); l++) {
        const long long cnt = (long long)T.level_begin[l + 1] - T.level_begin[l];
        if (cnt != (1LL << (3 * l))) continue;
        for (int b = T.level_begin[l]; b < T.level_begin[l + 1]; b++) {
            const int c = (int)((T.ix[b] & 1) | (T.iy[b] & 1) << 1 | (T.iz[b] & 1) << 2);
            owner[b] = c % nranks;
            load[owner[b]] += cost(b);
            done[b] = 1;
        }
    }
    std::vector<int> rest;
    for (int b = 0; b < nn; b++)
        if (!done[b]) rest.push_back(b);
    std::stable_sort(rest.begin(), rest.end(), [&](int a, int b) { return cost(a) > cost(b); });
    for (int b : rest) {
        int best = 0;
        for (int r = 1; r < nranks; r++)
            if (load[r] < load[best]) best = r;
        owner[b] = best;
        load[best] += cost(b);
    }
    return owner;
}

}  // namespace stk
