// Binned-SAH builder of the float32 traversal BVH (layout in fast_bvh.h).
#include "fast_bvh.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <limits>

#include "acoustic_rt.h"
#include "common.h"

namespace ac {
namespace {

constexpr int kBins = 16;

struct Box {
    double lo[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                    std::numeric_limits<double>::infinity()};
    double hi[3] = {-std::numeric_limits<double>::infinity(), -std::numeric_limits<double>::infinity(),
                    -std::numeric_limits<double>::infinity()};
    void grow(const double *l, const double *h) {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], l[a]);
            hi[a] = std::max(hi[a], h[a]);
        }
    }
    void grow(const Box &b) { grow(b.lo, b.hi); }
    bool empty() const { return !(lo[0] <= hi[0]); }
    double area() const {
        if (empty()) return 0.0;
        const double dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
};

struct Item {
    double lo[3], hi[3], c[3];
    int64_t surface;
};

class Builder {
  public:
    Builder(std::vector<Item> &items, int leaf_max, double pad, int median_from, TraversalBvh *out)
        : items_(items), leaf_max_(leaf_max), pad_(pad), median_from_(median_from), out_(out) {}

    // Returns the child reference of the subtree over items_[begin, end) and its bounds.
    int32_t build(int64_t begin, int64_t end, int depth, Box *bounds) {
        Box b, cb;
        for (int64_t i = begin; i < end; ++i) {
            b.grow(items_[i].lo, items_[i].hi);
            cb.grow(items_[i].c, items_[i].c);
        }
        *bounds = b;
        const int64_t n = end - begin;
        if (n <= leaf_max_) return leaf(begin, end);
        int64_t mid = -1;
        if (depth < median_from_) mid = sah_split(begin, end, cb);
        if (mid < 0) mid = median_split(begin, end, cb);
        const int64_t node = out_->num_nodes();
        out_->nodes.resize(out_->nodes.size() + 16, 0.0f);
        out_->depth = std::max(out_->depth, depth + 1);
        Box lb, rb;
        const int32_t left = build(begin, mid, depth + 1, &lb);
        const int32_t right = build(mid, end, depth + 1, &rb);
        write_node(node, lb, left, rb, right);
        return static_cast<int32_t>(node);
    }

    void write_root_pair(int32_t ref, const Box &b) {   // one leaf under the root, twice
        out_->nodes.assign(16, 0.0f);
        out_->depth = 1;
        write_node(0, b, ref, b, ref);
    }

  private:
    int32_t leaf(int64_t begin, int64_t end) {
        const int64_t first = static_cast<int64_t>(out_->order.size());
        for (int64_t i = begin; i < end; ++i) out_->order.push_back(items_[i].surface);
        return ~static_cast<int32_t>((first << 3) | (end - begin - 1));
    }

    // Binned SAH over the centroids: the split position, or -1 when no bin boundary separates them.
    int64_t sah_split(int64_t begin, int64_t end, const Box &cb) {
        double best = std::numeric_limits<double>::infinity();
        int best_axis = -1, best_bin = -1;
        for (int axis = 0; axis < 3; ++axis) {
            const double extent = cb.hi[axis] - cb.lo[axis];
            if (!(extent > 0.0)) continue;
            std::array<Box, kBins> bins;
            std::array<int64_t, kBins> counts{};
            const double scale = kBins / extent;
            for (int64_t i = begin; i < end; ++i) {
                const int k = bin_of(items_[i].c[axis], cb.lo[axis], scale);
                bins[k].grow(items_[i].lo, items_[i].hi);
                ++counts[k];
            }
            std::array<double, kBins> right_area{};
            std::array<int64_t, kBins> right_count{};
            Box acc;
            int64_t cnt = 0;
            for (int k = kBins - 1; k > 0; --k) {
                acc.grow(bins[k]);
                cnt += counts[k];
                right_area[k] = acc.area();
                right_count[k] = cnt;
            }
            Box left;
            int64_t lcnt = 0;
            for (int k = 0; k < kBins - 1; ++k) {
                left.grow(bins[k]);
                lcnt += counts[k];
                if (lcnt == 0 || right_count[k + 1] == 0) continue;
                const double cost = left.area() * lcnt + right_area[k + 1] * right_count[k + 1];
                if (cost < best) {
                    best = cost;
                    best_axis = axis;
                    best_bin = k;
                }
            }
        }
        if (best_axis < 0) return -1;
        const double extent = cb.hi[best_axis] - cb.lo[best_axis];
        const double scale = kBins / extent;
        const double lo = cb.lo[best_axis];
        Item *first = items_.data() + begin, *last = items_.data() + end;
        Item *m = std::partition(first, last, [&](const Item &it) {
            return bin_of(it.c[best_axis], lo, scale) <= best_bin;
        });
        const int64_t mid = m - items_.data();
        return (mid > begin && mid < end) ? mid : -1;
    }

    int64_t median_split(int64_t begin, int64_t end, const Box &cb) {
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (cb.hi[a] - cb.lo[a] > cb.hi[axis] - cb.lo[axis]) axis = a;
        const int64_t mid = begin + (end - begin) / 2;
        std::nth_element(items_.data() + begin, items_.data() + mid, items_.data() + end,
                         [axis](const Item &x, const Item &y) {
                             return x.c[axis] < y.c[axis] || (x.c[axis] == y.c[axis] && x.surface < y.surface);
                         });
        return mid;
    }

    static int bin_of(double v, double lo, double scale) {
        const int k = static_cast<int>((v - lo) * scale);
        return std::min(std::max(k, 0), kBins - 1);
    }

    // float32 bounds rounded outward, then padded
    float down(double v) const {
        float f = static_cast<float>(v - pad_);
        if (static_cast<double>(f) > v - pad_) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
        return f;
    }
    float up(double v) const {
        float f = static_cast<float>(v + pad_);
        if (static_cast<double>(f) < v + pad_) f = std::nextafter(f, std::numeric_limits<float>::infinity());
        return f;
    }

    void write_node(int64_t node, const Box &l, int32_t lref, const Box &r, int32_t rref) {
        float *q = out_->nodes.data() + 16 * node;
        q[0] = down(l.lo[0]); q[1] = up(l.hi[0]); q[2] = down(l.lo[1]); q[3] = up(l.hi[1]);
        q[4] = down(r.lo[0]); q[5] = up(r.hi[0]); q[6] = down(r.lo[1]); q[7] = up(r.hi[1]);
        q[8] = down(l.lo[2]); q[9] = up(l.hi[2]); q[10] = down(r.lo[2]); q[11] = up(r.hi[2]);
        std::memcpy(q + 12, &lref, 4);
        std::memcpy(q + 13, &rref, 4);
        q[14] = 0.0f;
        q[15] = 0.0f;
    }

    std::vector<Item> &items_;
    int leaf_max_;
    double pad_;
    int median_from_;
    TraversalBvh *out_;
};

// Collapse of the binary layout into the four-wide one (fast_bvh.h).
class Collapser {
  public:
    explicit Collapser(const std::vector<float> &bin) : bin_(bin) {}

    struct Child {
        float box[6];   // lo.x, hi.x, lo.y, hi.y, lo.z, hi.z
        int32_t ref;
    };

    // Wide node for binary node `b`; returns its index.  `need`: stack entries a ray can need from here down.
    int32_t collapse(int32_t b, std::vector<float> &wide, int32_t *need) {
        std::vector<Child> kids = {child(b, 0), child(b, 1)};
        while (kids.size() < 4) {
            int pick = -1;
            double area = -1.0;
            for (size_t k = 0; k < kids.size(); ++k) {
                if (kids[k].ref < 0) continue;
                const float *q = kids[k].box;
                const double dx = q[1] - q[0], dy = q[3] - q[2], dz = q[5] - q[4];
                const double a = dx * dy + dy * dz + dz * dx;
                if (a > area) { area = a; pick = static_cast<int>(k); }
            }
            if (pick < 0) break;
            const int32_t inner = kids[pick].ref;
            kids[pick] = child(inner, 0);
            kids.insert(kids.begin() + pick + 1, child(inner, 1));
        }
        const int32_t node = static_cast<int32_t>(wide.size() / kBvh4Floats);
        wide.resize(wide.size() + kBvh4Floats, 0.0f);
        int32_t refs[4];
        int32_t below = 0;
        for (size_t k = 0; k < 4; ++k) {
            if (k >= kids.size()) { refs[k] = ~0; continue; }
            if (kids[k].ref >= 0) {
                int32_t sub = 0;
                refs[k] = collapse(kids[k].ref, wide, &sub);
                below = std::max(below, sub);
            } else {
                refs[k] = kids[k].ref;
            }
        }
        float *q = wide.data() + static_cast<size_t>(node) * kBvh4Floats;
        for (int k = 0; k < 4; ++k) {
            for (int f = 0; f < 6; ++f)
                q[4 * f + k] = k < static_cast<int>(kids.size()) ? kids[k].box[f] : kBvh4Empty;
            std::memcpy(q + 24 + k, &refs[k], 4);
        }
        const int32_t count = static_cast<int32_t>(kids.size());
        std::memcpy(q + 28, &count, 4);
        // a visit pushes at most (children - 1) entries before descending into one child
        *need = count - 1 + below;
        return node;
    }

  private:
    Child child(int32_t b, int side) const {
        const float *q = bin_.data() + 16 * static_cast<size_t>(b);
        Child c;
        const float *xy = q + 4 * side;
        c.box[0] = xy[0]; c.box[1] = xy[1]; c.box[2] = xy[2]; c.box[3] = xy[3];
        c.box[4] = q[8 + 2 * side]; c.box[5] = q[9 + 2 * side];
        std::memcpy(&c.ref, q + 12 + side, 4);
        return c;
    }

    const std::vector<float> &bin_;
};

}  // namespace

int build_traversal_bvh(const std::vector<int64_t> &surfaces, const double *lo, const double *hi, int leaf_max,
                        double pad, TraversalBvh *out, int width) {
    if (width != 2 && width != 4) return fail(AC_ERR_INVALID, "BVH width %d is not 2 or 4", width);
    *out = TraversalBvh{};
    if (leaf_max < 1 || leaf_max > kBvhMaxLeaf)
        return fail(AC_ERR_INVALID, "BVH leaf size %d is outside 1..%d", leaf_max, kBvhMaxLeaf);
    if (surfaces.empty()) return AC_OK;
    if (surfaces.size() >= (size_t{1} << 27)) return fail(AC_ERR_CAPACITY, "too many surfaces for the float32 BVH");
    std::vector<Item> items(surfaces.size());
    for (size_t k = 0; k < surfaces.size(); ++k) {
        const int64_t si = surfaces[k];
        Item &it = items[k];
        for (int a = 0; a < 3; ++a) {
            it.lo[a] = lo[3 * si + a];
            it.hi[a] = hi[3 * si + a];
            it.c[a] = 0.5 * (it.lo[a] + it.hi[a]);
        }
        it.surface = si;
    }
    // Surface-area splits down to `median_from` levels, median splits below, so the
    // depth stays within the traversal stack whatever the geometry:
    // depth <= median_from + ceil(log2(n)) <= kBvhStack - 1.
    int log2n = 0;
    while ((int64_t{1} << log2n) < static_cast<int64_t>(items.size())) ++log2n;
    const int median_from = std::max(0, kBvhStack - 1 - log2n);
    Builder builder(items, leaf_max, pad, median_from, out);
    Box rb;
    const int32_t root = builder.build(0, static_cast<int64_t>(items.size()), 0, &rb);
    if (root < 0) builder.write_root_pair(root, rb);   // everything fits one leaf
    else if (root != 0) return fail(AC_ERR_INVALID, "internal: BVH root is not node 0");
    if (out->depth > kBvhStack - 1) return fail(AC_ERR_CAPACITY, "float32 BVH depth %d exceeds the traversal stack", out->depth);
    out->stack_need = out->depth + 1;   // one push per inner level on a path, plus the sentinel entry
    if (width == 4) {
        std::vector<float> wide;
        int32_t need = 0;
        Collapser(out->nodes).collapse(0, wide, &need);
        if (need <= kBvhStack - 1) {   // else keep the binary layout, whose need is bounded by its depth
            out->nodes.swap(wide);
            out->width = 4;
            out->stack_need = need + 1;
        }
    }
    return AC_OK;
}

}  // namespace ac
