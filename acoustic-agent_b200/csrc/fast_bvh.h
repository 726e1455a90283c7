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
// Most traversal stack entries per lane; the builder keeps the depth below this.  A launch sizes each lane's
// stack (shared memory) between the scenes' stack_need and this.
constexpr int kBvhStack = AC_BVH_STACK;

// Four-wide variant (`width` 4): the binary tree above collapsed so that every
// inner node holds up to four children -- a node repeatedly replaces its inner
// child of largest surface area by that child's two children -- eight quads
// per node, one 128-byte line:
//
//   q0 = lo.x[0..3]  q1 = hi.x[0..3]  q2 = lo.y[0..3]  q3 = hi.y[0..3]
//   q4 = lo.z[0..3]  q5 = hi.z[0..3]  q6 = ref[0..3]   q7 = {children, 0, 0, 0}
//
// Unused child slots hold a box at (1e30, 1e30, 1e30): a ray reaches it only if
// its distance to all three slab planes were equal and below 1.000001e30, which
// needs every direction component near 1, so no unit-length ray enters it.
// Child references mean what they mean in the binary layout.
constexpr int kBvh4Floats = 32;
constexpr float kBvh4Empty = 1e30f;

struct TraversalBvh {
    std::vector<float> nodes;      // [num_nodes][16] (width 2) or [num_nodes][32] (width 4)
    std::vector<int64_t> order;    // surface index per leaf slot
    int32_t depth = 0;             // inner-node levels of the binary tree on the longest root-to-leaf path
    int32_t width = 2;
    int32_t stack_need = 0;        // traversal stack entries a ray can need at most, the sentinel included
    int64_t num_nodes() const { return static_cast<int64_t>(nodes.size() / (width == 4 ? kBvh4Floats : 16)); }
};

// `surfaces`: the surface indices to include; `lo`/`hi`: per-surface AABBs
// [S][3] (indexed by surface); `pad`: absolute padding added to every node
// box on top of rounding the float32 bounds outward.
// `width` 2 or 4 (see above); a four-wide tree whose stack need would exceed
// the traversal stack stays binary (out->width tells which was built).
int build_traversal_bvh(const std::vector<int64_t> &surfaces, const double *lo, const double *hi, int leaf_max,
                        double pad, TraversalBvh *out, int width = 2);

}  // namespace ac
