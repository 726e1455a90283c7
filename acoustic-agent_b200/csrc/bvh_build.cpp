// Host BVH builder: a restatement of acoustic_agent/bvh.py:8-77 (build_bvh).
//
// Top-down: a node over more than `leaf_size` surfaces splits at n/2 along the
// axis of largest centroid extent (first axis on ties) after a stable sort of
// its surfaces by centroid on that axis.  Leaves list their surfaces in
// ascending index order.  Nodes are emitted in preorder; `escape` is the index
// of the first node after the subtree, which drives the stackless walk of
// steam_rt.py:4481-4506.  The tree must be identical to the reference's so that
// traversal statistics and any order-dependent behaviour match exactly.
//
// A node's stable order is lexicographic: the root sorts arange(S) (ties fall
// back to the surface index) and each child sorts its parent's order stably,
// so the order is (centroid on the node's axis, then on its ancestors' axes,
// most recent first, then the index), a unique key.  The left child is the n/2
// smallest keys in any order, so each node partitions its range in place
// (std::nth_element, linear time) instead of sorting it.  Centroids travel
// with their indices, so a node's range is scanned in order; bounds are read
// only at the leaves, and an inner node's are the union of its children's.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "acoustic_rt.h"
#include "common.h"

namespace {

// min / max that order -0.0 below +0.0, so the result does not depend on the order of the surfaces
inline double lower_of(double a, double b) { return (b < a || (b == a && std::signbit(b))) ? b : a; }
inline double upper_of(double a, double b) { return (b > a || (b == a && !std::signbit(b))) ? b : a; }

struct Item {   // a surface's centroid next to its index, so node ranges are scanned in order
    double c[3];
    int64_t index;
};

struct Builder {
    const double *lower;
    const double *upper;
    std::vector<Item> items;   // each node owns a contiguous range
    int64_t leaf_size;
    ac_bvh *out;
    int64_t nodes = 0;
    int64_t leaves = 0;
    int64_t max_depth = 0;

    void append(int64_t b, int64_t e, int64_t depth, const int *parent_axes, int parent_count) {
        const int64_t node = nodes++;
        const int64_t n = e - b;
        out->start[node] = -1;
        out->count[node] = 0;
        max_depth = std::max(max_depth, depth);
        if (n <= leaf_size) {
            std::sort(items.begin() + b, items.begin() + e,
                      [](const Item &x, const Item &y) { return x.index < y.index; });
            out->start[node] = b;
            out->count[node] = n;
            for (int a = 0; a < 3; ++a) {
                double mn = lower[3 * items[b].index + a], mx = upper[3 * items[b].index + a];
                for (int64_t k = b + 1; k < e; ++k) {
                    mn = lower_of(mn, lower[3 * items[k].index + a]);
                    mx = upper_of(mx, upper[3 * items[k].index + a]);
                }
                out->bounds_min[3 * node + a] = mn;
                out->bounds_max[3 * node + a] = mx;
            }
            for (int64_t k = b; k < e; ++k) out->primitives[k] = items[k].index;
            ++leaves;
            out->escape[node] = nodes;
            return;
        }
        double mn[3], mx[3];   // np.ptp of the centroids, np.argmax: first maximum wins
        for (int a = 0; a < 3; ++a) mn[a] = mx[a] = items[b].c[a];
        for (int64_t k = b + 1; k < e; ++k)
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::min(mn[a], items[k].c[a]);
                mx[a] = std::max(mx[a], items[k].c[a]);
            }
        int axis = 0;
        double best = mx[0] - mn[0];
        for (int a = 1; a < 3; ++a)
            if (mx[a] - mn[a] > best) {
                best = mx[a] - mn[a];
                axis = a;
            }
        int axes[3] = {axis, 0, 0}, count = 1;   // this node's axis, then the ancestors' without repeats
        for (int j = 0; j < parent_count; ++j)
            if (parent_axes[j] != axis) axes[count++] = parent_axes[j];
        auto less = [&axes, count](const Item &x, const Item &y) {
            for (int j = 0; j < count; ++j) {
                const double cx = x.c[axes[j]], cy = y.c[axes[j]];
                if (cx < cy) return true;
                if (cy < cx) return false;
            }
            return x.index < y.index;
        };
        const int64_t split = b + n / 2;
        std::nth_element(items.begin() + b, items.begin() + split, items.begin() + e, less);
        const int64_t left = nodes;
        append(b, split, depth + 1, axes, count);
        const int64_t right = nodes;
        append(split, e, depth + 1, axes, count);
        for (int a = 0; a < 3; ++a) {   // the union of the children's bounds (the min/max over the node's surfaces)
            out->bounds_min[3 * node + a] = lower_of(out->bounds_min[3 * left + a], out->bounds_min[3 * right + a]);
            out->bounds_max[3 * node + a] = upper_of(out->bounds_max[3 * left + a], out->bounds_max[3 * right + a]);
        }
        out->escape[node] = nodes;
    }
};

}  // namespace

extern "C" int ac_bvh_build(const double *bounds_min, const double *bounds_max, int64_t num_surfaces,
                            int32_t leaf_size, ac_bvh *out) {
    if (!bounds_min || !bounds_max || !out || !out->bounds_min || !out->bounds_max || !out->start ||
        !out->count || !out->escape || !out->primitives)
        return ac::fail(AC_ERR_INVALID, "ac_bvh_build: null pointer");
    if (num_surfaces < 1) return ac::fail(AC_ERR_INVALID, "BVH requires at least one surface");
    for (int64_t i = 0; i < 3 * num_surfaces; ++i)
        if (!std::isfinite(bounds_min[i]) || !std::isfinite(bounds_max[i]))
            return ac::fail(AC_ERR_INVALID, "BVH bounds must be finite");
    for (int64_t i = 0; i < 3 * num_surfaces; ++i)
        if (bounds_max[i] < bounds_min[i])
            return ac::fail(AC_ERR_INVALID, "BVH maximum bounds must not be below minimum bounds");
    Builder b;
    b.lower = bounds_min;
    b.upper = bounds_max;
    b.leaf_size = std::max<int64_t>(1, leaf_size);
    b.out = out;
    b.items.resize(num_surfaces);
    for (int64_t i = 0; i < num_surfaces; ++i) {
        for (int a = 0; a < 3; ++a) b.items[i].c[a] = 0.5 * (bounds_min[3 * i + a] + bounds_max[3 * i + a]);
        b.items[i].index = i;
    }
    b.append(0, num_surfaces, 1, nullptr, 0);
    out->node_count = b.nodes;
    out->leaf_count = b.leaves;
    out->max_depth = b.max_depth;
    return AC_OK;
}
