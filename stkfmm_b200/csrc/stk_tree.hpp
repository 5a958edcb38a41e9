// stk_tree.hpp -- adaptive octree and KIFMM interaction lists (host C++).
//
// Stands in for PVFMM's PtFMM_Tree::Initialize / InitFMM_Tree / SetupFMM
// (called from Lib/src/FMMData.cpp:107-167), which are not part of the
// reference tree.  Rules:
//   * the unit box [0,1)^3 is refined while a node holds more than max_pts of
//     the tree points and its level is below max_depth; refinement always
//     creates all 8 children (FMMData.cpp:111-113 sets max_pts / max_depth);
//   * the tree points are the largest of the SL / DL / target sets, ties going
//     to the targets (FMMData.cpp:123-135);
//   * every point set is sorted in Morton order, so every node owns one
//     contiguous range of each set;
//   * interaction lists follow the standard KIFMM definitions (U: adjacent
//     leaves; V: children of the parent's colleagues that are not adjacent;
//     W: descendants of a leaf's neighbours whose parent is adjacent but which
//     are not; X: the transpose of W), with periodic wrap on the periodic axes
//     recorded as an image shift code per entry.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

namespace stk {

constexpr int kMaxDepth = 20;     // 60-bit Morton keys
constexpr int kShiftNone = 13;    // shift code (sx+1) + 3(sy+1) + 9(sz+1) with sx = sy = sz = 0

inline int shift_code(int sx, int sy, int sz) { return (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1); }
inline int shift_negate(int code) { return 26 - code; }

// Compressed list: entries of node i are ent[off[i] .. off[i+1]); each entry is
// (node << 5) | shift code.
struct NodeList {
    std::vector<int> off;
    std::vector<int> ent;
    size_t size() const { return ent.size(); }
};

struct PointSet {
    int n = 0;
    std::vector<int> perm;           // sorted position -> caller's index
    std::vector<double> xyz;         // sorted coordinates (3 per point)
    std::vector<uint64_t> key;       // sorted Morton keys
    std::vector<int> node_begin;     // per node: first sorted position
    std::vector<int> node_end;       // per node: one past the last
    int count(int node) const { return node_end[node] - node_begin[node]; }
};

class Octree {
  public:
    // Build from tree points (n x 3, already in [0,1) on every axis).  pbc is
    // PAXIS (0 none, 1 x, 2 xy, 3 xyz).  Returns an empty string on success,
    // else an error message.
    std::string build(const double *pts, int n, int max_pts, int max_depth, int pbc);
    // Sort a point set into the tree (0 = SL, 1 = DL, 2 = targets).
    std::string assign(int set, const double *xyz, int n);
    // Build U, V, W, X lists.  Source boxes need SL or DL points; target boxes need targets.
    void build_lists();

    int num_nodes() const { return (int)level.size(); }
    int depth() const { return max_level; }
    bool is_leaf(int i) const { return first_child[i] < 0; }
    double side(int i) const;                       // edge length of node i
    void centre(int i, double c[3]) const;          // centre of node i
    void corner(int i, double c[3]) const;          // lower corner of node i
    int src_count(int i) const { return sets[0].count(i) + sets[1].count(i); }
    int trg_count(int i) const { return sets[2].count(i); }

    // topology
    std::vector<int> level, parent, first_child;
    std::vector<uint32_t> ix, iy, iz;
    std::vector<int> leaves;                        // leaf node ids in Morton order
    std::vector<int> level_begin;                   // nodes are stored level by level
    int max_level = 0;
    int pbc = 0;

    PointSet sets[3];
    NodeList U;   // leaf  -> adjacent leaves            (S2T)
    NodeList V;   // node  -> well-separated same-level  (M2L)
    NodeList W;   // leaf  -> smaller non-adjacent nodes (M2T)
    NodeList X;   // node  -> larger non-adjacent leaves (S2L)

  private:
    std::unordered_map<uint64_t, int> lookup_;
    std::vector<uint64_t> key_lo_;                  // Morton key of each node's lower corner (max depth)
    int find(int l, int64_t x, int64_t y, int64_t z) const;
    bool adjacent(int a, int shift, int b) const;
};

uint64_t morton_key(double x, double y, double z);

// Longest-processing-time assignment: items (in the given order, largest first)
// each go to the part with the smallest load so far; ties to the lowest part.
void partition_lpt(int n, const double *cost, int nparts, std::vector<int> &owner);

// Owners (0 .. nranks-1) of the M2L / S2L target nodes when the far field is split
// over nranks ranks: complete levels by parity type, the other nodes by cost (LPT).
std::vector<int> far_owners(const Octree &T, int nranks);

}  // namespace stk
