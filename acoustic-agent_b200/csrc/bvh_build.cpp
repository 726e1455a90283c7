// Host BVH builder: a restatement of acoustic_agent/bvh.py:8-77 (build_bvh).
//
// Top-down: a node over more than `leaf_size` surfaces splits at n/2 along the
// axis of largest centroid extent (first axis on ties), after a stable sort of
// the surfaces by centroid on that axis.  Leaves list their surfaces in
// ascending index order.  Nodes are emitted in preorder; `escape` is the index
// of the first node after the subtree, which drives the stackless walk of
// steam_rt.py:4481-4506.  The tree must be identical to the reference's so that
// traversal statistics and any order-dependent behaviour match exactly.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "acoustic_rt.h"
#include "common.h"

namespace {

struct Builder {
    const double *lower;
    const double *upper;
    std::vector<double> centroid;
    int64_t leaf_size;
    ac_bvh *out;
    int64_t nodes = 0;
    int64_t prims = 0;
    int64_t leaves = 0;
    int64_t max_depth = 0;

    int64_t append(std::vector<int64_t> &indices, int64_t depth) {
        const int64_t node = nodes++;
        for (int a = 0; a < 3; ++a) {
            double mn = lower[3 * indices[0] + a], mx = upper[3 * indices[0] + a];
            for (size_t k = 1; k < indices.size(); ++k) {
                mn = std::min(mn, lower[3 * indices[k] + a]);
                mx = std::max(mx, upper[3 * indices[k] + a]);
            }
            out->bounds_min[3 * node + a] = mn;
            out->bounds_max[3 * node + a] = mx;
        }
        out->start[node] = -1;
        out->count[node] = 0;
        out->escape[node] = -1;
        max_depth = std::max(max_depth, depth);
        if (static_cast<int64_t>(indices.size()) <= leaf_size) {
            std::vector<int64_t> ordered(indices);
            std::stable_sort(ordered.begin(), ordered.end());
            out->start[node] = prims;
            out->count[node] = static_cast<int64_t>(ordered.size());
            for (int64_t v : ordered) out->primitives[prims++] = v;
            ++leaves;
        } else {
            int axis = 0;
            double best = -1.0;
            for (int a = 0; a < 3; ++a) {
                double mn = centroid[3 * indices[0] + a], mx = mn;
                for (size_t k = 1; k < indices.size(); ++k) {
                    mn = std::min(mn, centroid[3 * indices[k] + a]);
                    mx = std::max(mx, centroid[3 * indices[k] + a]);
                }
                const double extent = mx - mn;
                if (a == 0 || extent > best) {  // np.argmax: first maximum wins
                    best = extent;
                    axis = a;
                }
            }
            std::vector<int64_t> sorted(indices);
            std::stable_sort(sorted.begin(), sorted.end(), [&](int64_t x, int64_t y) {
                return centroid[3 * x + axis] < centroid[3 * y + axis];
            });
            const size_t split = sorted.size() / 2;
            std::vector<int64_t> left(sorted.begin(), sorted.begin() + split);
            std::vector<int64_t> right(sorted.begin() + split, sorted.end());
            append(left, depth + 1);
            append(right, depth + 1);
        }
        out->escape[node] = nodes;
        return node;
    }
};

}  // namespace

extern "C" int ac_bvh_build(const double *bounds_min, const double *bounds_max, int64_t num_surfaces,
                            int32_t leaf_size, ac_bvh *out) {
    if (!bounds_min || !bounds_max || !out || !out->bounds_min || !out->bounds_max || !out->start ||
        !out->count || !out->escape || !out->primitives)
        return ac::fail(AC_ERR_INVALID, "ac_bvh_build: null pointer");
    if (num_surfaces < 1) return ac::fail(AC_ERR_INVALID, "BVH requires at least one surface");
    for (int64_t i = 0; i < 3 * num_surfaces; ++i) {
        if (!std::isfinite(bounds_min[i]) || !std::isfinite(bounds_max[i]))
            return ac::fail(AC_ERR_INVALID, "BVH bounds must be finite");
        if (bounds_max[i] < bounds_min[i])
            return ac::fail(AC_ERR_INVALID, "BVH maximum bounds must not be below minimum bounds");
    }
    Builder b;
    b.lower = bounds_min;
    b.upper = bounds_max;
    b.leaf_size = std::max<int64_t>(1, leaf_size);
    b.out = out;
    b.centroid.resize(3 * num_surfaces);
    for (int64_t i = 0; i < 3 * num_surfaces; ++i) b.centroid[i] = 0.5 * (bounds_min[i] + bounds_max[i]);
    std::vector<int64_t> all(num_surfaces);
    std::iota(all.begin(), all.end(), 0);
    b.append(all, 1);
    out->node_count = b.nodes;
    out->leaf_count = b.leaves;
    out->max_depth = b.max_depth;
    return AC_OK;
}
