// Traversal BVH of the float32 tracer's BVH mode (host-side builder).
//
// A binary BVH over the walls and boxes of a scene, built with the binned
// surface-area heuristic, laid out for per-lane traversal on the GPU: every
// inner node stores the boxes of BOTH children (so one node fetch decides the
// next step), four 16-byte quads per node:
//
//   q0 = {c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y}
//   q1 = {c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y}
//   q2 = {c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z}
//   q3 = {ref0, ref1, 0, 0}   (int32 bit patterns)
//
// A child reference >= 0 is an inner node index; < 0 is a leaf,
// ~((first << 3) | (count - 1)) over the leaf-ordered surface slots, so a leaf
// holds 1..8 surfaces.  Node 0 is the root and always an inner node (a scene
// with one such surface gets a root whose two children are the same leaf).
// This BVH is unrelated to the reference's escape-link BVH (bvh.py), which the
// float64 kernel keeps walking for parity.
#pragma once

#include <cstdint>
#include <vector>

namespace ac {

constexpr int kBvhMaxLeaf = 8;
#ifndef AC_BVH_STACK
#define AC_BVH_STACK 32
#endif
constexpr int kBvhStack = AC_BVH_STACK;   // traversal stack entries; the builder keeps the depth below this

struct TraversalBvh {
    std::vector<float> nodes;      // [num_nodes][16]
    std::vector<int64_t> order;    // surface index per leaf slot
    int32_t depth = 0;             // inner-node levels on the longest root-to-leaf path
    int64_t num_nodes() const { return static_cast<int64_t>(nodes.size() / 16); }
};

// `surfaces`: the surface indices to include; `lo`/`hi`: per-surface AABBs
// [S][3] (indexed by surface); `pad`: absolute padding added to every node
// box on top of rounding the float32 bounds outward.
int build_traversal_bvh(const std::vector<int64_t> &surfaces, const double *lo, const double *hi, int leaf_max,
                        double pad, TraversalBvh *out);

}  // namespace ac
