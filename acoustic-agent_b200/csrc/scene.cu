// Scene upload: the reference's float64 surface SoA (steam_rt.py:834-924) is
// validated, given a BVH if it has none (bvh.py:8-77 restated in
// bvh_build.cpp), and packed into 16-byte aligned quads, once in float32 for
// the production kernel and once in float64 for the parity kernel.  One device
// allocation per precision; the handle owns both.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "fast_bvh.h"
#include "scene_internal.h"

namespace {

template <typename T>
inline T tag_value(int tag);
template <>
inline float tag_value<float>(int tag) {
    float f;
    std::memcpy(&f, &tag, sizeof(f));
    return f;
}
template <>
inline double tag_value<double>(int tag) { return static_cast<double>(tag); }

struct Offsets {
    size_t prims_linear, prims_leaf, nodes, mats, corners, normals, wall_clusters, walls, polys, box_clusters,
        box_bounds, boxes, edges, bvh_nodes, bvh_prims, total;  // elements
};

// Scenes with more walls + boxes than this trace in BVH mode unless the caller chooses;
// with at most kAutoHybridWalls walls (one room) in hybrid mode.  Measured on B200:
// U room (8 walls, 20 boxes) hybrid 11.4 ms < BVH 11.8 < scan 12.3; 8-room apartment
// (52 walls, 374 boxes) BVH 5.1 ms < hybrid 6.3 < scan 9.6.
constexpr int64_t kAutoBvhSurfaces = 16;
constexpr int64_t kAutoHybridWalls = 16;
// Float32 BVH node boxes are padded by this much (metres) beyond the surface bounds.
constexpr double kBvhPad = 1e-4;
// Surfaces per BVH leaf unless the caller chooses: one surface per leaf measured
// fastest on B200 for rooms of 30 to 430 surfaces (deeper tree, fewer tests).
constexpr int kDefaultBvhLeaf = 1;
// Children per inner node of the float32 traversal BVH unless the caller chooses.
#ifndef AC_DEFAULT_BVH_WIDTH
#define AC_DEFAULT_BVH_WIDTH 2
#endif
constexpr int kDefaultBvhWidth = AC_DEFAULT_BVH_WIDTH;

inline size_t round4(size_t v) { return (v + 3) & ~static_cast<size_t>(3); }

// Float32 scan lists: walls and boxes in clusters of up to 32 (leaves of a BVH
// over each kind's bounds, preorder), horizontal polygons as a flat list.
struct FastLists {
    std::vector<int64_t> wall_slots, box_slots, polys;                    // surface index per slot
    std::vector<std::array<int64_t, 2>> wall_clusters, box_clusters;      // {first slot, count}
    std::vector<std::array<double, 6>> wall_cluster_bounds, box_cluster_bounds;
    bool use_bvh = false;                                                 // BVH or hybrid mode
    bool hybrid = false;                                                  // walls stay in the scan
    ac::TraversalBvh bvh;                                                 // walls and boxes (hybrid: boxes)
};

int cluster_kind(const ac_scene_desc *d, const double *blo, const double *bhi, int64_t kind, int leaf,
                 std::vector<int64_t> &slots, std::vector<std::array<int64_t, 2>> &clusters,
                 std::vector<std::array<double, 6>> &bounds) {
    std::vector<int64_t> members;
    for (int64_t i = 0; i < d->num_surfaces; ++i)
        if (d->kinds[i] == kind) members.push_back(i);
    if (members.empty()) return AC_OK;
    const int64_t M = static_cast<int64_t>(members.size());
    std::vector<double> lo(3 * M), hi(3 * M);
    for (int64_t k = 0; k < M; ++k)
        for (int a = 0; a < 3; ++a) {
            lo[3 * k + a] = blo[3 * members[k] + a];
            hi[3 * k + a] = bhi[3 * members[k] + a];
        }
    const size_t cap = 2 * static_cast<size_t>(M);
    std::vector<double> nmin(3 * cap), nmax(3 * cap);
    std::vector<int64_t> nstart(cap), ncount(cap), nesc(cap), nprims(M);
    ac_bvh b{nmin.data(), nmax.data(), nstart.data(), ncount.data(), nesc.data(), nprims.data(), 0, 0, 0};
    const int rc = ac_bvh_build(lo.data(), hi.data(), M, leaf, &b);
    if (rc != AC_OK) return rc;
    for (int64_t k = 0; k < M; ++k) slots.push_back(members[nprims[k]]);
    for (int64_t n = 0; n < b.node_count; ++n) {
        if (ncount[n] <= 0) continue;
        clusters.push_back({nstart[n], ncount[n]});
        bounds.push_back({nmin[3 * n], nmin[3 * n + 1], nmin[3 * n + 2], nmax[3 * n], nmax[3 * n + 1], nmax[3 * n + 2]});
    }
    return AC_OK;
}

Offsets layout(size_t S, size_t P, size_t N, size_t C, const FastLists *f) {
    Offsets o{};
    size_t off = 0;
    o.prims_linear = off;  off += round4(S * ac::kPrimStride);
    o.prims_leaf = off;    off += round4(P * ac::kPrimStride);
    o.nodes = off;         off += round4(N * ac::kNodeStride);
    o.mats = off;          off += round4(S * ac::kMatStride);
    o.corners = off;       off += round4(C * 2);
    o.normals = off;       off += round4(S * 3);
    o.wall_clusters = off; off += round4(f ? f->wall_clusters.size() * ac::kClusterStride : 0);
    o.walls = off;         off += round4(f ? f->wall_slots.size() * 8 : 0);
    o.polys = off;         off += round4(f ? f->polys.size() * 4 : 0);
    o.box_clusters = off;  off += round4(f ? f->box_clusters.size() * ac::kClusterStride : 0);
    o.box_bounds = off;    off += round4(f ? f->box_slots.size() * 8 : 0);
    o.boxes = off;         off += round4(f ? f->box_slots.size() * ac::kPrimStride : 0);
    o.edges = off;         off += round4(f ? C * 4 : 0);
    off = (off + 31) & ~static_cast<size_t>(31);   // BVH nodes start on a 128-byte line
    o.bvh_nodes = off;     off += round4(f && f->use_bvh ? f->bvh.nodes.size() : 0);
    o.bvh_prims = off;     off += round4(f && f->use_bvh ? f->bvh.order.size() * ac::kPrimStride : 0);
    o.total = off;
    return o;
}

// Padded per-surface AABBs (steam_rt.py:234-262), used when the caller passes none.
void surface_bounds(const ac_scene_desc *d, std::vector<double> &lo, std::vector<double> &hi) {
    const int64_t S = d->num_surfaces;
    lo.assign(3 * S, 0.0);
    hi.assign(3 * S, 0.0);
    double cx0 = 0, cx1 = 0, cy0 = 0, cy1 = 0;
    for (int64_t c = 0; c < d->num_corners; ++c) {
        const double x = d->corners[2 * c], y = d->corners[2 * c + 1];
        if (c == 0 || x < cx0) cx0 = x;
        if (c == 0 || x > cx1) cx1 = x;
        if (c == 0 || y < cy0) cy0 = y;
        if (c == 0 || y > cy1) cy1 = y;
    }
    for (int64_t i = 0; i < S; ++i) {
        double l[3], h[3];
        if (d->kinds[i] == AC_KIND_WALL) {
            const double ax = d->wall_a[2 * i], ay = d->wall_a[2 * i + 1];
            const double bx = ax + d->wall_delta[2 * i], by = ay + d->wall_delta[2 * i + 1];
            l[0] = std::min(ax, bx); l[1] = std::min(ay, by); l[2] = d->wall_z[2 * i];
            h[0] = std::max(ax, bx); h[1] = std::max(ay, by); h[2] = d->wall_z[2 * i + 1];
        } else if (d->kinds[i] == AC_KIND_BOX) {
            const double ex = std::fabs(d->box_axis_u[2 * i]) * d->box_half[2 * i] +
                              std::fabs(d->box_axis_v[2 * i]) * d->box_half[2 * i + 1];
            const double ey = std::fabs(d->box_axis_u[2 * i + 1]) * d->box_half[2 * i] +
                              std::fabs(d->box_axis_v[2 * i + 1]) * d->box_half[2 * i + 1];
            l[0] = d->box_center[2 * i] - ex; l[1] = d->box_center[2 * i + 1] - ey; l[2] = d->box_z[2 * i];
            h[0] = d->box_center[2 * i] + ex; h[1] = d->box_center[2 * i + 1] + ey; h[2] = d->box_z[2 * i + 1];
        } else {
            l[0] = cx0; l[1] = cy0; l[2] = d->z_values[i];
            h[0] = cx1; h[1] = cy1; h[2] = d->z_values[i];
        }
        for (int a = 0; a < 3; ++a) {
            lo[3 * i + a] = l[a] - 2.0e-6;
            hi[3 * i + a] = h[a] + 2.0e-6;
        }
    }
}

template <typename T>
void pack_record(const ac_scene_desc *d, int64_t si, T *rec) {
    std::fill(rec, rec + ac::kPrimStride, T(0));
    const int kind = static_cast<int>(d->kinds[si]);
    if (kind == AC_KIND_WALL) {
        rec[0] = T(d->wall_a[2 * si]);
        rec[1] = T(d->wall_a[2 * si + 1]);
        rec[2] = T(d->wall_delta[2 * si]);
        rec[3] = T(d->wall_delta[2 * si + 1]);
        rec[4] = T(d->wall_z[2 * si]);
        rec[5] = T(d->wall_z[2 * si + 1]);
        rec[6] = T(d->normals[3 * si]);
        rec[7] = T(d->normals[3 * si + 1]);
        rec[8] = T(d->normals[3 * si + 2]);
    } else if (kind == AC_KIND_BOX) {
        rec[0] = T(d->box_center[2 * si]);
        rec[1] = T(d->box_center[2 * si + 1]);
        rec[2] = T(d->box_axis_u[2 * si]);
        rec[3] = T(d->box_axis_u[2 * si + 1]);
        rec[4] = T(d->box_axis_v[2 * si]);
        rec[5] = T(d->box_axis_v[2 * si + 1]);
        rec[6] = T(d->box_half[2 * si]);
        rec[7] = T(d->box_half[2 * si + 1]);
        rec[8] = T(d->box_z[2 * si]);
        rec[9] = T(d->box_z[2 * si + 1]);
    } else {
        rec[0] = T(d->z_values[si]);
        rec[1] = T(d->normals[3 * si]);
        rec[2] = T(d->normals[3 * si + 1]);
        rec[3] = T(d->normals[3 * si + 2]);
    }
    rec[11] = tag_value<T>(static_cast<int>(si) * 4 + kind);
}

template <typename T>
int pack_and_upload(const ac_scene_desc *d, const ac_bvh &bvh, const FastLists *f, const double *bounds_lo,
                    const double *bounds_hi, ac_scene_s *s, void **storage, size_t *bytes, ac::SceneDev<T> *view) {
    const size_t S = static_cast<size_t>(d->num_surfaces);
    const size_t N = static_cast<size_t>(bvh.node_count);
    const size_t P = S;
    const size_t C = static_cast<size_t>(d->num_corners);
    const Offsets o = layout(S, P, N, C, f);
    std::vector<T> host(o.total, T(0));
    if (f) {
        auto put_clusters = [&](size_t base, const std::vector<std::array<int64_t, 2>> &cl,
                                const std::vector<std::array<double, 6>> &cb) {
            for (size_t c = 0; c < cl.size(); ++c) {
                T *cp = host.data() + base + c * ac::kClusterStride;
                for (int a = 0; a < 3; ++a) {
                    cp[a] = T(cb[c][a]);
                    cp[4 + a] = T(cb[c][3 + a]);
                }
                cp[3] = tag_value<T>(static_cast<int>(cl[c][0]));
                cp[7] = tag_value<T>(static_cast<int>(cl[c][1]));
            }
        };
        put_clusters(o.wall_clusters, f->wall_clusters, f->wall_cluster_bounds);
        put_clusters(o.box_clusters, f->box_clusters, f->box_cluster_bounds);
        for (size_t k = 0; k < f->wall_slots.size(); ++k) {
            const int64_t si = f->wall_slots[k];
            T *w = host.data() + o.walls + 8 * k;
            w[0] = T(d->wall_a[2 * si]);
            w[1] = T(d->wall_a[2 * si + 1]);
            w[2] = T(d->wall_delta[2 * si]);
            w[3] = T(d->wall_delta[2 * si + 1]);
            w[4] = T(d->wall_z[2 * si]);
            w[5] = T(d->wall_z[2 * si + 1]);
            w[6] = tag_value<T>(static_cast<int>(si) * 4 + AC_KIND_WALL);
        }
        for (size_t k = 0; k < f->polys.size(); ++k) {
            const int64_t si = f->polys[k];
            T *pp = host.data() + o.polys + 4 * k;
            pp[0] = T(d->z_values[si]);
            pp[1] = tag_value<T>(static_cast<int>(si) * 4 + AC_KIND_HORIZONTAL);
        }
        for (size_t k = 0; k < f->box_slots.size(); ++k) {
            const int64_t si = f->box_slots[k];
            pack_record<T>(d, si, host.data() + o.boxes + k * ac::kPrimStride);
            T *bb = host.data() + o.box_bounds + 8 * k;
            for (int a = 0; a < 3; ++a) {
                bb[a] = T(bounds_lo[3 * si + a]);
                bb[4 + a] = T(bounds_hi[3 * si + a]);
            }
            bb[3] = tag_value<T>(static_cast<int>(si) * 4 + AC_KIND_BOX);
        }
        // Polygon edges for the even-odd test: {x_i, y_i, y_j, (x_j - x_i) / (y_j - y_i)} with j the
        // previous corner (steam_rt.py:4259-4274); an edge the reference skips gets y_j = y_i.
        for (size_t i = 0; i < C; ++i) {
            const size_t j = (i + C - 1) % C;
            const double xi = d->corners[2 * i], yi = d->corners[2 * i + 1];
            const double xj = d->corners[2 * j], yj = d->corners[2 * j + 1];
            T *e = host.data() + o.edges + 4 * i;
            const bool skip = std::fabs(yj - yi) <= 1e-12;
            e[0] = T(xi);
            e[1] = T(yi);
            e[2] = skip ? T(yi) : T(yj);
            e[3] = skip ? T(0) : T((xj - xi) / (yj - yi));
        }
        if (f->use_bvh) {
            std::copy(f->bvh.nodes.begin(), f->bvh.nodes.end(), host.begin() + o.bvh_nodes);
            for (size_t k = 0; k < f->bvh.order.size(); ++k)
                pack_record<T>(d, f->bvh.order[k], host.data() + o.bvh_prims + k * ac::kPrimStride);
        }
    }
    for (size_t si = 0; si < S; ++si) pack_record<T>(d, static_cast<int64_t>(si), host.data() + o.prims_linear + si * ac::kPrimStride);
    for (size_t k = 0; k < P; ++k)
        pack_record<T>(d, bvh.primitives[k], host.data() + o.prims_leaf + k * ac::kPrimStride);
    for (size_t n = 0; n < N; ++n) {
        T *np = host.data() + o.nodes + n * ac::kNodeStride;
        for (int a = 0; a < 3; ++a) {
            np[a] = T(bvh.bounds_min[3 * n + a]);
            np[4 + a] = T(bvh.bounds_max[3 * n + a]);
        }
        np[3] = tag_value<T>(static_cast<int>(bvh.escape[n]));
        const int64_t start = bvh.count[n] > 0 ? bvh.start[n] : 0;
        np[7] = tag_value<T>(static_cast<int>(start | (bvh.count[n] << 24)));
    }
    for (size_t si = 0; si < S; ++si) {
        T *m = host.data() + o.mats + si * ac::kMatStride;
        for (int b = 0; b < 6; ++b) m[b] = T(d->reflection[6 * si + b]);
        m[6] = T(d->scattering[si]);
    }
    for (size_t c = 0; c < 2 * C; ++c) host[o.corners + c] = T(d->corners[c]);
    for (size_t k = 0; k < 3 * S; ++k) host[o.normals + k] = T(d->normals[k]);

    *bytes = o.total * sizeof(T);
    void *dev = nullptr;
    // Stream-ordered allocation on the legacy default stream: unlike cudaMalloc/cudaFree it does not
    // wait for the whole device, so uploading or destroying a scene does not stall work that other
    // (non-blocking) streams have in flight.  The upload is complete when this function returns.
    cudaError_t err = cudaMallocAsync(&dev, *bytes, cudaStreamLegacy);
    if (err != cudaSuccess) return ac::fail(AC_ERR_NOMEM, "scene allocation of %zu bytes failed: %s", *bytes, cudaGetErrorString(err));
    err = cudaMemcpyAsync(dev, host.data(), *bytes, cudaMemcpyHostToDevice, cudaStreamLegacy);
    if (err == cudaSuccess) err = cudaStreamSynchronize(cudaStreamLegacy);
    if (err != cudaSuccess) {
        cudaFreeAsync(dev, cudaStreamLegacy);
        return ac::fail(AC_ERR_CUDA, "scene upload failed: %s", cudaGetErrorString(err));
    }
    *storage = dev;
    const T *base = static_cast<const T *>(dev);
    view->prims_linear = base + o.prims_linear;
    view->prims_leaf = base + o.prims_leaf;
    view->nodes = base + o.nodes;
    view->mats = base + o.mats;
    view->corners = base + o.corners;
    view->normals = base + o.normals;
    view->num_surfaces = static_cast<int32_t>(S);
    view->num_nodes = static_cast<int32_t>(N);
    view->num_corners = static_cast<int32_t>(C);
    view->num_leaf_prims = static_cast<int32_t>(P);
    if (f) {
        const float *fbase = reinterpret_cast<const float *>(dev);
        s->fast.wall_clusters = fbase + o.wall_clusters;
        s->fast.walls = fbase + o.walls;
        s->fast.polys = fbase + o.polys;
        s->fast.box_clusters = fbase + o.box_clusters;
        s->fast.box_bounds = fbase + o.box_bounds;
        s->fast.boxes = fbase + o.boxes;
        s->fast.edges = fbase + o.edges;
        s->fast.num_wall_clusters = static_cast<int32_t>(f->wall_clusters.size());
        s->fast.num_polys = static_cast<int32_t>(f->polys.size());
        s->fast.num_box_clusters = static_cast<int32_t>(f->box_clusters.size());
        s->fast.num_edges = static_cast<int32_t>(C);
        s->num_clusters = static_cast<int64_t>(f->wall_clusters.size() + f->box_clusters.size());
        if (f->use_bvh) {
            // BVH mode: walls and boxes come from the traversal BVH, only polygons stay in the scan;
            // hybrid mode: boxes from the BVH, walls and polygons in the scan
            s->fast.bvh_nodes = reinterpret_cast<const float4 *>(fbase + o.bvh_nodes);
            s->fast.bvh_prims = fbase + o.bvh_prims;
            s->fast.num_bvh_nodes = static_cast<int32_t>(f->bvh.num_nodes());
            s->fast.bvh_width = f->bvh.width;
            if (!f->hybrid) s->fast.num_wall_clusters = 0;
            s->fast.num_box_clusters = 0;
        }
    }
    return AC_OK;
}

bool finite_all(const double *p, size_t n) {
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

}  // namespace

extern "C" int ac_scene_create(const ac_scene_desc *d, ac_scene_t *out) {
    ac::NvtxRange nvtx_range("ac_scene_create");
    if (!d || !out) return ac::fail(AC_ERR_INVALID, "ac_scene_create: null argument");
    *out = nullptr;
    const int64_t S = d->num_surfaces;
    if (S < 1) return ac::fail(AC_ERR_INVALID, "scene needs at least one surface");
    if (S >= (1 << 22)) return ac::fail(AC_ERR_CAPACITY, "scene has %lld surfaces; the limit is 4194303", (long long)S);
    if (!d->kinds || !d->wall_a || !d->wall_delta || !d->wall_z || !d->z_values || !d->box_center || !d->box_axis_u ||
        !d->box_axis_v || !d->box_half || !d->box_z || !d->normals || !d->reflection || !d->scattering)
        return ac::fail(AC_ERR_INVALID, "scene description has a null surface array");
    bool has_horizontal = false;
    for (int64_t i = 0; i < S; ++i) {
        if (d->kinds[i] < 0 || d->kinds[i] > 2) return ac::fail(AC_ERR_INVALID, "surface %lld has unknown kind %lld", (long long)i, (long long)d->kinds[i]);
        has_horizontal |= d->kinds[i] == AC_KIND_HORIZONTAL;
    }
    if (has_horizontal && (d->num_corners < 3 || !d->corners))
        return ac::fail(AC_ERR_INVALID, "horizontal surfaces need a room polygon of at least 3 corners");
    const size_t s2 = 2 * static_cast<size_t>(S);
    if (!finite_all(d->wall_a, s2) || !finite_all(d->wall_delta, s2) || !finite_all(d->wall_z, s2) ||
        !finite_all(d->z_values, S) || !finite_all(d->box_center, s2) || !finite_all(d->box_axis_u, s2) ||
        !finite_all(d->box_axis_v, s2) || !finite_all(d->box_half, s2) || !finite_all(d->box_z, s2) ||
        !finite_all(d->normals, 3 * S) || !finite_all(d->reflection, 6 * S) || !finite_all(d->scattering, S) ||
        (d->num_corners > 0 && !finite_all(d->corners, 2 * static_cast<size_t>(d->num_corners))))
        return ac::fail(AC_ERR_INVALID, "scene arrays must be finite");

    // BVH: given, or built here from the padded surface bounds.
    std::vector<double> bmin, bmax;
    std::vector<int64_t> bstart, bcount, besc, bprims;
    ac_bvh bvh{};
    if (d->bvh_node_count > 0) {
        if (!d->bvh_bounds_min || !d->bvh_bounds_max || !d->bvh_start || !d->bvh_count || !d->bvh_escape || !d->bvh_primitives)
            return ac::fail(AC_ERR_INVALID, "BVH arrays missing");
        bvh.bounds_min = const_cast<double *>(d->bvh_bounds_min);
        bvh.bounds_max = const_cast<double *>(d->bvh_bounds_max);
        bvh.start = const_cast<int64_t *>(d->bvh_start);
        bvh.count = const_cast<int64_t *>(d->bvh_count);
        bvh.escape = const_cast<int64_t *>(d->bvh_escape);
        bvh.primitives = const_cast<int64_t *>(d->bvh_primitives);
        bvh.node_count = d->bvh_node_count;
        int64_t leaves = 0;
        for (int64_t n = 0; n < d->bvh_node_count; ++n) leaves += d->bvh_count[n] > 0;
        bvh.leaf_count = leaves;
    } else {
        if (!d->surface_bounds_min || !d->surface_bounds_max)
            return ac::fail(AC_ERR_INVALID, "surface bounds required to build the BVH");
        const size_t cap = 2 * static_cast<size_t>(S);
        bmin.resize(3 * cap); bmax.resize(3 * cap); bstart.resize(cap); bcount.resize(cap); besc.resize(cap); bprims.resize(S);
        bvh.bounds_min = bmin.data(); bvh.bounds_max = bmax.data(); bvh.start = bstart.data(); bvh.count = bcount.data();
        bvh.escape = besc.data(); bvh.primitives = bprims.data();
        const int rc = ac_bvh_build(d->surface_bounds_min, d->surface_bounds_max, S, 4, &bvh);
        if (rc != AC_OK) return rc;
    }
    // Structural checks: the kernel walks escape links and reads leaf slots.
    int32_t max_leaf = 0;
    for (int64_t n = 0; n < bvh.node_count; ++n) {
        if (bvh.escape[n] <= n || bvh.escape[n] > bvh.node_count)
            return ac::fail(AC_ERR_INVALID, "BVH node %lld has an invalid escape link", (long long)n);
        if (bvh.count[n] < 0 || bvh.count[n] > 255)
            return ac::fail(AC_ERR_INVALID, "BVH leaf %lld holds %lld primitives (limit 255)", (long long)n, (long long)bvh.count[n]);
        if (bvh.count[n] > 0 && (bvh.start[n] < 0 || bvh.start[n] + bvh.count[n] > S || bvh.start[n] >= (1 << 24)))
            return ac::fail(AC_ERR_INVALID, "BVH leaf %lld addresses primitives out of range", (long long)n);
        max_leaf = std::max<int32_t>(max_leaf, static_cast<int32_t>(bvh.count[n]));
        if (!std::isfinite(bvh.bounds_min[3 * n]) || !std::isfinite(bvh.bounds_max[3 * n]))
            return ac::fail(AC_ERR_INVALID, "BVH bounds must be finite");
    }
    for (int64_t k = 0; k < S; ++k)
        if (bvh.primitives[k] < 0 || bvh.primitives[k] >= S)
            return ac::fail(AC_ERR_INVALID, "BVH primitive slot %lld references surface %lld", (long long)k, (long long)bvh.primitives[k]);

    int ndev = 0;
    AC_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (d->device < 0 || d->device >= ndev) return ac::fail(AC_ERR_UNSUPPORTED, "CUDA device %d is not available", d->device);
    AC_CUDA_TRY(cudaSetDevice(d->device));

    ac_scene_s *s = new (std::nothrow) ac_scene_s();
    if (!s) return ac::fail(AC_ERR_NOMEM, "out of host memory");
    s->device = d->device;
    s->num_surfaces = S;
    s->num_corners = d->num_corners;
    s->node_count = bvh.node_count;
    s->leaf_count = bvh.leaf_count;
    s->max_leaf = max_leaf;
    s->max_reflection = 0.0;
    s->max_scattering = -1e300;
    s->min_scattering = 1e300;
    for (int64_t i = 0; i < 6 * S; ++i) s->max_reflection = std::max(s->max_reflection, std::fabs(d->reflection[i]));
    for (int64_t i = 0; i < S; ++i) {
        s->max_scattering = std::max(s->max_scattering, d->scattering[i]);
        s->min_scattering = std::min(s->min_scattering, d->scattering[i]);
    }
    // Cluster BVH for the float32 scan: leaves of `cluster_size` surfaces.
    std::vector<double> slo, shi;
    const double *blo = d->surface_bounds_min, *bhi = d->surface_bounds_max;
    if (!blo || !bhi) {
        surface_bounds(d, slo, shi);
        blo = slo.data();
        bhi = shi.data();
    }
    s->cluster_size = d->cluster_size > 0 ? std::min(d->cluster_size, ac::kMaxCluster) : ac::kMaxCluster;
    FastLists lists;
    for (int64_t i = 0; i < S; ++i)
        if (d->kinds[i] == AC_KIND_HORIZONTAL) lists.polys.push_back(i);
    int rc = cluster_kind(d, blo, bhi, AC_KIND_WALL, s->cluster_size, lists.wall_slots, lists.wall_clusters,
                          lists.wall_cluster_bounds);
    if (rc == AC_OK)
        rc = cluster_kind(d, blo, bhi, AC_KIND_BOX, s->cluster_size, lists.box_slots, lists.box_clusters,
                          lists.box_cluster_bounds);
    if (rc == AC_OK) {
        if (d->traversal < AC_TRAVERSAL_AUTO || d->traversal > AC_TRAVERSAL_HYBRID) {
            rc = ac::fail(AC_ERR_INVALID, "unknown traversal %d", d->traversal);
        } else {
            int64_t walls = 0, boxes = 0;
            for (int64_t i = 0; i < S; ++i) {
                walls += d->kinds[i] == AC_KIND_WALL;
                boxes += d->kinds[i] == AC_KIND_BOX;
            }
            // AUTO: a single room's few walls are cheapest in lockstep, its furniture in a BVH
            lists.hybrid = d->traversal == AC_TRAVERSAL_HYBRID ||
                           (d->traversal == AC_TRAVERSAL_AUTO && walls + boxes > kAutoBvhSurfaces &&
                            walls <= kAutoHybridWalls && boxes > 0);
            std::vector<int64_t> members;
            for (int64_t i = 0; i < S; ++i)
                if (d->kinds[i] == AC_KIND_BOX || (d->kinds[i] == AC_KIND_WALL && !lists.hybrid)) members.push_back(i);
            lists.use_bvh = !members.empty() &&
                            (d->traversal == AC_TRAVERSAL_BVH || lists.hybrid ||
                             (d->traversal == AC_TRAVERSAL_AUTO && static_cast<int64_t>(members.size()) > kAutoBvhSurfaces));
            if (!lists.use_bvh) lists.hybrid = false;   // no boxes: plain scan
            if (lists.use_bvh)
                rc = ac::build_traversal_bvh(members, blo, bhi, d->bvh_leaf > 0 ? d->bvh_leaf : kDefaultBvhLeaf, kBvhPad,
                                             &lists.bvh, d->bvh_width > 0 ? d->bvh_width : kDefaultBvhWidth);
        }
    }
    if (rc != AC_OK) {
        delete s;
        return rc;
    }
    s->traversal = lists.hybrid ? AC_TRAVERSAL_HYBRID : (lists.use_bvh ? AC_TRAVERSAL_BVH : AC_TRAVERSAL_SCAN);
    s->bvh_depth = lists.use_bvh ? lists.bvh.depth : 0;
    s->bvh_nodes = lists.use_bvh ? lists.bvh.num_nodes() : 0;
    s->bvh_width = lists.use_bvh ? lists.bvh.width : 0;
    s->bvh_stack_need = lists.use_bvh ? lists.bvh.stack_need : 0;
    rc = pack_and_upload<float>(d, bvh, &lists, blo, bhi, s, &s->storage_f32, &s->bytes_f32, &s->f32);
    if (rc == AC_OK)
        rc = pack_and_upload<double>(d, bvh, nullptr, blo, bhi, s, &s->storage_f64, &s->bytes_f64, &s->f64);
    if (rc != AC_OK) {
        if (s->storage_f32) cudaFreeAsync(s->storage_f32, cudaStreamLegacy);
        delete s;
        return rc;
    }
    *out = s;
    return AC_OK;
}

namespace ac {

int note_scene_use(ac_scene_s *scene, void *stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    AC_CUDA_TRY(cudaStreamIsCapturing(stream, &capture));
    if (capture != cudaStreamCaptureStatusNone) return AC_OK;
    std::lock_guard<std::mutex> guard(scene->use_lock);
    cudaEvent_t event = nullptr;
    for (const auto &use : scene->uses)
        if (use.first == stream) event = use.second;
    if (!event) {
        AC_CUDA_TRY(cudaEventCreateWithFlags(&event, cudaEventDisableTiming));
        scene->uses.emplace_back(stream, event);
    }
    AC_CUDA_TRY(cudaEventRecord(event, stream));
    return AC_OK;
}

}  // namespace ac

extern "C" int ac_scene_destroy(ac_scene_t s) {
    ac::NvtxRange nvtx_range("ac_scene_destroy");
    if (!s) return AC_OK;
    cudaSetDevice(s->device);
    // The frees go on the legacy stream after every recorded last use, so work
    // still queued on other streams reads the scene before its memory returns
    // to the pool.  Work captured into a CUDA graph is the graph owner's to
    // finish before destroying the scene.
    {
        std::lock_guard<std::mutex> guard(s->use_lock);
        for (const auto &use : s->uses) {
            cudaStreamWaitEvent(cudaStreamLegacy, use.second, 0);
            cudaEventDestroy(use.second);   // released once its last record completes
        }
        s->uses.clear();
    }
    if (s->storage_f32) cudaFreeAsync(s->storage_f32, cudaStreamLegacy);
    if (s->storage_f64) cudaFreeAsync(s->storage_f64, cudaStreamLegacy);
    delete s;
    return AC_OK;
}

extern "C" int ac_scene_get_info(ac_scene_t s, ac_scene_info *info) {
    if (!s || !info) return ac::fail(AC_ERR_INVALID, "ac_scene_get_info: null argument");
    info->num_surfaces = s->num_surfaces;
    info->num_corners = s->num_corners;
    info->node_count = s->node_count;
    info->leaf_count = s->leaf_count;
    info->device_bytes = static_cast<int64_t>(s->bytes_f32 + s->bytes_f64);
    info->device = s->device;
    info->max_leaf = s->max_leaf;
    info->num_clusters = s->num_clusters;
    info->traversal = s->traversal;
    info->bvh_depth = s->bvh_depth;
    info->bvh_nodes = s->bvh_nodes;
    info->bvh_width = s->bvh_width;
    info->bvh_stack_need = s->bvh_stack_need;
    return AC_OK;
}
