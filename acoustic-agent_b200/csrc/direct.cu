// Direct-path occlusion and transmission on the GPU: the ray-casting part of
// simulate_direct (acoustic_agent/steam_rt.py:1315-1350) for a batch of
// (source, listener) pairs of one scene, in float64.
//
// The reference runs these queries through its Python surface objects
// (RoomRayScene.closest_hit / any_hit, steam_rt.py:320-352), whose tests equal
// the Numba kernel's except that a horizontal polygon also accepts a point
// within 1e-8 of its outline (geometry.py:194-235).  The queries here use the
// float64 kernel's surface records and tests plus that outline rule, a linear
// scan (the reference's BVH only prunes candidates, so it finds the same
// hits), ties to the lower surface index, and any-hit as t < distance - 1e-6.
// Compiled with -fmad=false like the other float64 parity code.
//
// One warp per query.  The volumetric samples (_volumetric_occlusion,
// :4215-4240) are spread over the lanes, each testing its two legs against
// every surface; the closest hits (the blocking surface and the transmission
// walk of _transmission, :3437-3462) are warp-cooperative, lanes taking
// surfaces lane, lane + 32, ... and a shuffle reduction picking the nearest.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "scene_internal.h"

namespace ac {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr double kMiss = 1e30;

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// geometry.py:224-235 _point_on_boundary (tolerance 1e-8).
__device__ bool on_outline(double x, double y, const double *corners, int n) {
    for (int i = 0; i < n; ++i) {
        const int j = i + 1 < n ? i + 1 : 0;
        const double ax = __ldg(corners + 2 * i), ay = __ldg(corners + 2 * i + 1);
        const double abx = __ldg(corners + 2 * j) - ax, aby = __ldg(corners + 2 * j + 1) - ay;
        const double denom = abx * abx + aby * aby;
        if (denom <= 1e-8) continue;
        double t = ((x - ax) * abx + (y - ay) * aby) / denom;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        const double ex = ax + t * abx - x, ey = ay + t * aby - y;
        if (sqrt(ex * ex + ey * ey) <= 1e-8) return true;
    }
    return false;
}

// The reference's Python intersect() of surface `si`: t, or kMiss.
__device__ double surface_t(const SceneDev<double> &sc, int si, const double *o, const double *d) {
    const double *rec = sc.prims_linear + static_cast<size_t>(si) * kPrimStride;
    const int kind = rec_tag(rec) & 3;
    if (kind == 1) {
        if (fabs(d[2]) <= 1e-12) return kMiss;
        const double z = __ldg(rec);
        const double t = (z - o[2]) / d[2];
        if (t <= 1e-6) return kMiss;
        const double px = o[0] + t * d[0], py = o[1] + t * d[1];
        return (point_in_polygon(px, py, sc.corners, sc.num_corners) || on_outline(px, py, sc.corners, sc.num_corners))
                   ? t
                   : kMiss;
    }
    double n[3];
    return surface_hit(rec, kind, o, d, sc.corners, sc.num_corners, n);
}

// RoomRayScene.any_hit: some surface at _EPS < t < max_distance - _EPS (one lane).
__device__ bool lane_any_hit(const SceneDev<double> &sc, const double *o, const double *d, double max_distance) {
    const double limit = max_distance - 1e-6;
    for (int si = 0; si < sc.num_surfaces; ++si)
        if (surface_t(sc, si, o, d) < limit) return true;
    return false;
}

// RoomRayScene.closest_hit, warp-cooperative: the nearest surface, ties to the
// lower index; -1 (and t = kMiss) when nothing is hit.  Every lane gets the result.
__device__ int warp_closest(const SceneDev<double> &sc, const double *o, const double *d, double &t_out) {
    const int lane = threadIdx.x & 31;
    double best_t = kMiss;
    int best = -1;
    for (int si = lane; si < sc.num_surfaces; si += 32) {
        const double t = surface_t(sc, si, o, d);
        if (t < best_t) {   // a lane visits its surfaces in increasing index: equal t keeps the lower one
            best_t = t;
            best = si;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double ot = __shfl_xor_sync(kFull, best_t, off);
        const int os = __shfl_xor_sync(kFull, best, off);
        if (os >= 0 && (best < 0 || ot < best_t || (ot == best_t && os < best))) {
            best_t = ot;
            best = os;
        }
    }
    t_out = best_t;
    return best;
}

__global__ void __launch_bounds__(128) direct_kernel(const ac_direct_query *queries, int num_queries,
                                                     const __grid_constant__ SceneDev<double> sc,
                                                     const __grid_constant__ ac_direct_tables tables,
                                                     ac_direct_result *results) {
    const int lane = threadIdx.x & 31;
    const int w = static_cast<int>((blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5);
    if (w >= num_queries) return;   // uniform per warp
    const ac_direct_query q = queries[w];
    const double *s = q.source;
    const double *l = q.listener;
    // steam_rt.py:1323-1331
    const double dx = s[0] - l[0], dy = s[1] - l[1], dz = s[2] - l[2];
    const double distance = sqrt(dx * dx + dy * dy + dz * dz);
    double occlusion = 1.0;
    double tr[6] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
    int blocking = -1;
    if (q.occlusion && distance > 1e-6) {
        const double dir[3] = {dx / distance, dy / distance, dz / distance};
        double t;
        const int si = warp_closest(sc, l, dir, t);
        blocking = (si >= 0 && t < distance - 1e-6) ? si : -1;
        if (q.volumetric) {
            // _volumetric_occlusion: sample points around the source; a point counts if the source sees
            // it, and is visible if the listener sees it too
            int visible = 0, valid = 0;
            for (int k = lane; k < tables.num_samples; k += 32) {
                double p[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) p[a] = __ldg(tables.unit_samples + 3 * k + a) * q.radius + s[a];
                const double sl[3] = {p[0] - s[0], p[1] - s[1], p[2] - s[2]};
                const double sd = sqrt(sl[0] * sl[0] + sl[1] * sl[1] + sl[2] * sl[2]);
                if (sd > 1e-9) {
                    const double sdir[3] = {sl[0] / sd, sl[1] / sd, sl[2] / sd};
                    if (lane_any_hit(sc, s, sdir, sd)) continue;
                }
                const double ll[3] = {p[0] - l[0], p[1] - l[1], p[2] - l[2]};
                const double ld = sqrt(ll[0] * ll[0] + ll[1] * ll[1] + ll[2] * ll[2]);
                ++valid;
                if (ld <= 1e-9) {
                    ++visible;
                } else {
                    const double m = ld > 1e-9 ? ld : 1e-9;
                    const double ldir[3] = {ll[0] / m, ll[1] / m, ll[2] / m};
                    if (!lane_any_hit(sc, l, ldir, ld)) ++visible;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                visible += __shfl_xor_sync(kFull, visible, off);
                valid += __shfl_xor_sync(kFull, valid, off);
            }
            occlusion = valid ? static_cast<double>(visible) / static_cast<double>(valid) : 0.0;
        } else {
            occlusion = blocking >= 0 ? 0.0 : 1.0;
        }
        if (occlusion < 1.0) {
            if (!q.transmission) {
#pragma unroll
                for (int b = 0; b < 6; ++b) tr[b] = 0.0;
            } else {
                // _transmission: alternate closest hits from the listener and from the source, multiplying
                // in each newly named surface's transmission, until the two walks meet
                const double back[3] = {(l[0] - s[0]) / distance, (l[1] - s[1]) / distance, (l[2] - s[2]) / distance};
                double reached[2] = {0.0, 0.0};
                int seen[AC_DIRECT_MAX_LAYERS];
                int num_seen = 0;
                int current = 0;
                const int iterations = 2 * q.max_layers + 2;
                for (int it = 0; it < iterations; ++it) {
                    const double *e = current ? s : l;
                    const double *dd = current ? back : dir;
                    const double md = reached[current];
                    const double origin[3] = {e[0] + md * dd[0], e[1] + md * dd[1], e[2] + md * dd[2]};
                    double th;
                    const int hit = warp_closest(sc, origin, dd, th);
                    const double absolute = md + th;
                    if (hit < 0 || absolute >= distance) break;
                    const int group = __ldg(tables.surface_group + hit);
                    bool known = false;
                    for (int j = 0; j < num_seen; ++j) known = known || seen[j] == group;
                    if (!known) {
#pragma unroll
                        for (int b = 0; b < 6; ++b) {
                            double v = __ldg(tables.transmission + 6 * hit + b);
                            v = v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v);
                            tr[b] = tr[b] * v;
                        }
                        seen[num_seen++] = group;
                        if (num_seen >= q.max_layers) break;
                    }
                    reached[current] = absolute + 1e-2;
                    if (reached[current] >= distance || (0.0 + reached[0]) + reached[1] >= distance) break;
                    current = 1 - current;
                }
            }
        }
    }
    if (lane == 0) {
        ac_direct_result r;
        r.occlusion = occlusion;
#pragma unroll
        for (int b = 0; b < 6; ++b) r.transmission[b] = tr[b];
        r.occlusion_surface = blocking;
        r.reserved = 0;
        results[w] = r;
    }
}

}  // namespace
}  // namespace ac

extern "C" int ac_direct_workspace_size(int32_t num_queries, size_t *bytes) {
    if (!bytes || num_queries < 0) return ac::fail(AC_ERR_INVALID, "ac_direct_workspace_size: bad argument");
    *bytes = ac::align256(static_cast<size_t>(num_queries) * sizeof(ac_direct_query));
    return AC_OK;
}

extern "C" int ac_direct(ac_scene_t scene, const ac_direct_query *queries, int32_t num_queries,
                         const ac_direct_tables *tables, ac_direct_result *results, void *workspace,
                         size_t workspace_bytes, void *host_staging, void *stream_ptr) {
    ac::NvtxRange nvtx_range("ac_direct");
    if (!scene || !tables || num_queries < 0 || (num_queries > 0 && (!queries || !results)))
        return ac::fail(AC_ERR_INVALID, "ac_direct: null argument");
    if (num_queries > (1 << 26)) return ac::fail(AC_ERR_CAPACITY, "ac_direct: %d queries is too many", num_queries);
    bool any_volumetric = false, any_transmission = false;
    for (int32_t i = 0; i < num_queries; ++i) {
        const ac_direct_query &q = queries[i];
        for (int a = 0; a < 3; ++a)
            if (!std::isfinite(q.source[a]) || !std::isfinite(q.listener[a]))
                return ac::fail(AC_ERR_INVALID, "ac_direct: query %d has a non-finite position", i);
        if (!std::isfinite(q.radius)) return ac::fail(AC_ERR_INVALID, "ac_direct: query %d radius", i);
        if (q.max_layers < 1 || q.max_layers > AC_DIRECT_MAX_LAYERS)
            return ac::fail(AC_ERR_INVALID, "ac_direct: query %d max_layers %d outside 1..%d", i, q.max_layers,
                            AC_DIRECT_MAX_LAYERS);
        any_volumetric = any_volumetric || (q.occlusion && q.volumetric);
        any_transmission = any_transmission || (q.occlusion && q.transmission);
    }
    if (any_volumetric && (tables->num_samples < 1 || !tables->unit_samples))
        return ac::fail(AC_ERR_INVALID, "ac_direct: volumetric queries need the unit sample table");
    if (any_transmission && (!tables->transmission || !tables->surface_group))
        return ac::fail(AC_ERR_INVALID, "ac_direct: transmission needs the surface transmission and group tables");
    if (num_queries == 0) return AC_OK;
    int current = 0;
    AC_CUDA_TRY(cudaGetDevice(&current));
    if (current != scene->device)
        return ac::fail(AC_ERR_INVALID, "ac_direct: the scene lives on device %d, the caller is on %d", scene->device,
                        current);
    size_t need = 0;
    ac_direct_workspace_size(num_queries, &need);
    if (!workspace || workspace_bytes < need)
        return ac::fail(AC_ERR_CAPACITY, "ac_direct workspace too small: %zu < %zu", workspace_bytes, need);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t bytes = static_cast<size_t>(num_queries) * sizeof(ac_direct_query);
    if (host_staging) {
        std::memcpy(host_staging, queries, bytes);
        AC_CUDA_TRY(cudaMemcpyAsync(workspace, host_staging, bytes, cudaMemcpyHostToDevice, stream));
    } else {
        AC_CUDA_TRY(cudaMemcpyAsync(workspace, queries, bytes, cudaMemcpyHostToDevice, stream));
        AC_CUDA_TRY(cudaStreamSynchronize(stream));  // pageable source must stay alive
    }
    ac_direct_tables t = *tables;
    if (!any_volumetric) t.num_samples = 0;
    const int blocks = static_cast<int>((static_cast<int64_t>(num_queries) * 32 + 127) / 128);
    ac::direct_kernel<<<blocks, 128, 0, stream>>>(static_cast<const ac_direct_query *>(workspace), num_queries,
                                                  scene->f64, t, results);
    AC_CUDA_TRY(cudaGetLastError());
    return ac::note_scene_use(scene, stream_ptr);
}
