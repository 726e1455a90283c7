// Float32 production tracer for sm_100a: warp-uniform scene scan.
//
// Same per-ray algorithm as trace_kernel.cuh (steam_rt.py:4708-4850), but the
// intersection queries are organised for SIMT instead of restating the
// reference's per-thread escape-link walk:
//
//   * a warp always works on ONE scene.  All 32 lanes step through the
//     scene's surface clusters (leaves of a BVH built with 8 surfaces per leaf,
//     in preorder) together; each lane tests its own ray against the cluster's
//     AABB with its current best t, and the warp skips the cluster when no lane
//     needs it (__any_sync).  Inside a cluster every lane tests the same surface
//     at the same time, so the surface-kind branch is uniform and each record is
//     one broadcast load;
//   * primitive tests compute only t, with reciprocal multiplies; the normal is
//     evaluated once, for the winning surface (boxes re-run the slab test);
//   * the shadow query runs the same scan with an early exit once every lane
//     that needs it has found a blocker;
//   * lanes refill the moment their ray ends from the warp's current range of
//     (job, ray) work items; all jobs that share a scene form one range, so the
//     eight channels of an array trace as one stream.  A warp moves to another
//     scene only when its lanes are idle.
//
// The closest hit is the minimum t with ties to the lower surface index, as in
// the reference.  When no surface is hit in BVH mode the lane falls back to the
// reference's escape-link walk, which reproduces its rule that a missed ray
// returns the lowest visited surface with t = 1e30 (steam_rt.py:4501).
#pragma once

#include "trace_kernel.cuh"

namespace ac {

// Cluster record: {lo.x, lo.y, lo.z, first slot} {hi.x, hi.y, hi.z, count}
constexpr int kClusterStride = 8;

struct FastScene {
    const float *clusters;       // [NC][8]
    const float *prims;          // [P][12] surface records in cluster-slot order
    const float *boxes;          // [P][8] world AABB per slot {lo.xyz, 0, hi.xyz, 0} (used for boxes)
    const float *edges;          // [C][4] {x_i, y_i, y_j (or y_i if skipped), (x_j-x_i)/(y_j-y_i)}
    int32_t num_clusters;
    int32_t num_edges;
};

// One group = the jobs that share a scene; chunks never straddle groups.
struct FastGroup {
    SceneDev<float> scene;
    FastScene fast;
    int32_t first_job;
    int32_t num_jobs;
};

struct FastChunk {
    int64_t begin;
    int64_t end;
    int32_t group;
    int32_t pad;
};

struct FastTable {
    const Job<float> *jobs;
    const int64_t *ray_begin;      // [num_jobs + 1]
    const FastGroup *groups;
    const FastChunk *chunks;
    int64_t num_chunks;
    int32_t num_jobs;
    int32_t chunk_rays;            // single-job launches: rays per chunk
    unsigned long long *chunk_counter;
};

struct FRay {
    float o[3];
    float d[3];
    float inv[3];
};

__device__ __forceinline__ float safe_inv(float d) {
    const float m = fabsf(d) < 1e-20f ? copysignf(1e-20f, d) : d;
    return __frcp_rn(m);
}

__device__ __forceinline__ void make_ray(FRay &r, const float *o, const float *d) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        r.o[a] = o[a];
        r.d[a] = d[a];
        r.inv[a] = safe_inv(d[a]);
    }
}

// Conservative slab test: could any point of the box be hit before max_t?
__device__ __forceinline__ bool cluster_overlaps(const FRay &r, const Quad<float> &lo, const Quad<float> &hi,
                                                 float max_t) {
    float enter = 0.0f, exit_ = max_t * 1.000001f + 1e-5f;
    const float los[3] = {lo.x, lo.y, lo.z}, his[3] = {hi.x, hi.y, hi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float t0 = (los[a] - r.o[a]) * r.inv[a];
        const float t1 = (his[a] - r.o[a]) * r.inv[a];
        enter = fmaxf(enter, fminf(t0, t1));
        exit_ = fminf(exit_, fmaxf(t0, t1));
    }
    return enter <= exit_;
}

__device__ __forceinline__ bool point_in_polygon_fast(float x, float y, const float *edges, int n) {
    bool inside = false;
    for (int i = 0; i < n; ++i) {
        const Quad<float> e = ldq(edges + 4 * i);  // uniform across the warp
        if ((e.y > y) != (e.z > y)) {
            if (x < e.x + (y - e.y) * e.w) inside = !inside;
        }
    }
    return inside;
}

// t of one surface for one ray (1e30 = miss); steam_rt.py:4361-4392 restated with reciprocals.
__device__ __forceinline__ float surface_t(const float *rec, int kind, const FRay &r, const FastScene &fs) {
    if (kind == 0) {
        const Quad<float> A = ldq(rec), B = ldq(rec + 4);
        const float det = A.z * r.d[1] - A.w * r.d[0];
        if (fabsf(det) > 1e-12f) {
            const float inv = __frcp_rn(det);
            const float relx = r.o[0] - A.x, rely = r.o[1] - A.y;
            const float t = (relx * A.w - rely * A.z) * inv;
            const float u = (relx * r.d[1] - rely * r.d[0]) * inv;
            const float z = r.o[2] + t * r.d[2];
            if (t > 1e-6f && u >= -1e-6f && u <= 1.000001f && z >= B.x - 1e-6f && z <= B.y + 1e-6f) return t;
        }
        return 1e30f;
    }
    if (kind == 2) {
        const Quad<float> A = ldq(rec), B = ldq(rec + 4), C = ldq(rec + 8);
        const float relx = r.o[0] - A.x, rely = r.o[1] - A.y;
        const float ox = relx * A.z + rely * A.w;
        const float oy = relx * B.x + rely * B.y;
        const float dx = r.d[0] * A.z + r.d[1] * A.w;
        const float dy = r.d[0] * B.x + r.d[1] * B.y;
        float t_min = -1e30f, t_max = 1e30f;
        if (fabsf(dx) <= 1e-12f) {
            if (ox < -B.z || ox > B.z) return 1e30f;
        } else {
            const float ix = __frcp_rn(dx);
            const float a = (-B.z - ox) * ix, b = (B.z - ox) * ix;
            t_min = fminf(a, b);
            t_max = fmaxf(a, b);
        }
        if (fabsf(dy) <= 1e-12f) {
            if (oy < -B.w || oy > B.w) return 1e30f;
        } else {
            const float iy = __frcp_rn(dy);
            const float a = (-B.w - oy) * iy, b = (B.w - oy) * iy;
            t_min = fmaxf(t_min, fminf(a, b));
            t_max = fminf(t_max, fmaxf(a, b));
        }
        if (fabsf(r.d[2]) <= 1e-12f) {
            if (r.o[2] < C.x || r.o[2] > C.y) return 1e30f;
        } else {
            const float a = (C.x - r.o[2]) * r.inv[2], b = (C.y - r.o[2]) * r.inv[2];
            t_min = fmaxf(t_min, fminf(a, b));
            t_max = fminf(t_max, fmaxf(a, b));
        }
        if (t_min > t_max || t_max <= 1e-6f) return 1e30f;
        const float t = t_min > 1e-6f ? t_min : t_max;
        return t < 1e29f ? t : 1e30f;
    }
    const Quad<float> A = ldq(rec);
    if (fabsf(r.d[2]) > 1e-12f) {
        const float t = (A.x - r.o[2]) * r.inv[2];
        if (t > 1e-6f) {
            const float px = r.o[0] + t * r.d[0];
            const float py = r.o[1] + t * r.d[1];
            if (point_in_polygon_fast(px, py, fs.edges, fs.num_edges)) return t;
        }
    }
    return 1e30f;
}

// Warp-uniform closest hit.  Every lane of the warp must call it; `active`
// lanes carry a ray.  Returns the winning surface index (-1: none) and its slot.
__device__ __forceinline__ int closest_scan(const FastScene &fs, const FRay &r, bool active, float &best_t,
                                            int &best_slot) {
    const unsigned full = 0xFFFFFFFFu;
    best_t = 1e30f;
    int best = -1;
    best_slot = -1;
    for (int c = 0; c < fs.num_clusters; ++c) {
        const float *cp = fs.clusters + kClusterStride * c;
        const Quad<float> lo = ldq(cp), hi = ldq(cp + 4);
        const bool pass = active && cluster_overlaps(r, lo, hi, best_t);
        if (!__any_sync(full, pass)) continue;
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
        for (int k = 0; k < count; ++k) {
            const float *rec = fs.prims + static_cast<size_t>(first + k) * kPrimStride;
            const int tag = __float_as_int(__ldg(rec + 11));
            bool test = pass;
            if ((tag & 3) == 2) {
                // Boxes: cheap world-AABB check first; the warp skips the box if no lane needs it.
                const float *bb = fs.boxes + static_cast<size_t>(first + k) * 8;
                test = pass && cluster_overlaps(r, ldq(bb), ldq(bb + 4), best_t);
                if (!__any_sync(full, test)) continue;
            }
            if (test) {
                const float t = surface_t(rec, tag & 3, r, fs);
                const int si = tag >> 2;
                if (t < best_t || (t == best_t && t < 1e30f && si < best)) {
                    best_t = t;
                    best = si;
                    best_slot = first + k;
                }
            }
        }
    }
    return best;
}

// Warp-uniform shadow query: is a surface hit before max_t?  Lanes with
// `active` false (or that already found a blocker) ride along.
__device__ __forceinline__ bool shadow_scan(const FastScene &fs, const FRay &r, bool active, float max_t) {
    const unsigned full = 0xFFFFFFFFu;
    bool blocked = false;
    for (int c = 0; c < fs.num_clusters; ++c) {
        const bool searching = active && !blocked;
        if (!__any_sync(full, searching)) break;
        const float *cp = fs.clusters + kClusterStride * c;
        const Quad<float> lo = ldq(cp), hi = ldq(cp + 4);
        const bool pass = searching && cluster_overlaps(r, lo, hi, max_t);
        if (!__any_sync(full, pass)) continue;
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
        for (int k = 0; k < count; ++k) {
            const float *rec = fs.prims + static_cast<size_t>(first + k) * kPrimStride;
            const int tag = __float_as_int(__ldg(rec + 11));
            bool test = pass && !blocked;
            if ((tag & 3) == 2) {
                const float *bb = fs.boxes + static_cast<size_t>(first + k) * 8;
                test = test && cluster_overlaps(r, ldq(bb), ldq(bb + 4), max_t);
                if (!__any_sync(full, test)) continue;
            }
            if (test) {
                if (surface_t(rec, tag & 3, r, fs) < max_t) blocked = true;
            }
        }
    }
    return blocked;
}

// Normal of the winning surface, oriented against the ray.
__device__ __forceinline__ void winner_normal(const FastScene &fs, int slot, const FRay &r, float *n) {
    const float *rec = fs.prims + static_cast<size_t>(slot) * kPrimStride;
    const int kind = __float_as_int(__ldg(rec + 11)) & 3;
    if (kind == 0) {
        n[0] = __ldg(rec + 6); n[1] = __ldg(rec + 7); n[2] = __ldg(rec + 8);
    } else if (kind == 2) {
        const Quad<float> A = ldq(rec), B = ldq(rec + 4), C = ldq(rec + 8);
        float bn[3] = {0.0f, 0.0f, 1.0f};
        box_hit(A, B, C, r.o, r.d, bn);
        n[0] = bn[0]; n[1] = bn[1]; n[2] = bn[2];
    } else {
        n[0] = __ldg(rec + 1); n[1] = __ldg(rec + 2); n[2] = __ldg(rec + 3);
    }
    if (n[0] * r.d[0] + n[1] * r.d[1] + n[2] * r.d[2] > 0.0f) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
}

// The reference's escape-link walk, kept out of line: only rays that miss
// every surface in BVH mode take it.
static __device__ __noinline__ int2 fallback_walk(const SceneDev<float> sc, float ox, float oy, float oz, float dx,
                                                  float dy, float dz) {
    const float o[3] = {ox, oy, oz}, d[3] = {dx, dy, dz};
    float n[3], t;
    const int surf = closest_hit(sc, true, o, d, t, n);
    return make_int2(surf, __float_as_int(t));
}

struct FastLane {
    float o[3];
    float d[3];
    float acc[kBands];
    double path;
    int64_t ray;
    int job;
    int bounce;
    int queries;
    int shadows;
};

__device__ __forceinline__ int find_job_range(const int64_t *prefix, int lo, int hi, int64_t g) {
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <bool kSingle>
__global__ void __launch_bounds__(256) trace_fast_kernel(const __grid_constant__ Job<float> single,
                                                         const __grid_constant__ FastScene single_fast,
                                                         const __grid_constant__ FastTable table) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const unsigned lanes_below = (1u << lane_id) - 1u;

    // Warp-uniform work state.
    int group = -1;
    int64_t next = 0, end = 0;
    int64_t pending = -1;           // chunk of another scene, taken but not started
    bool exhausted = false;
    const int64_t num_chunks = kSingle ? (single.num_rays + table.chunk_rays - 1) / table.chunk_rays : table.num_chunks;

    FastLane s;
    bool has = false;
    s.job = 0;

    while (true) {
        // ---- refill lanes from the warp's range; take more chunks of the same scene as needed
        unsigned need = __ballot_sync(full, !has);
        while (need && pending < 0 && !exhausted) {
            if (next >= end) {
                long long c = 0;
                if (lane_id == 0) c = static_cast<long long>(atomicAdd(table.chunk_counter, 1ull));
                c = __shfl_sync(full, c, 0);
                if (c >= num_chunks) { exhausted = true; break; }
                int64_t cb, ce;
                int cg;
                if (kSingle) {
                    cb = c * table.chunk_rays;
                    ce = min(cb + static_cast<int64_t>(table.chunk_rays), single.num_rays);
                    cg = 0;
                } else {
                    const FastChunk ch = table.chunks[c];
                    cb = ch.begin; ce = ch.end; cg = ch.group;
                }
                if (group >= 0 && cg != group) {
                    if (!__any_sync(full, has)) {
                        group = cg; next = cb; end = ce;  // idle warp: switch scenes now
                    } else {
                        pending = c;
                        break;
                    }
                } else {
                    group = cg; next = cb; end = ce;
                }
            }
            const int take = static_cast<int>(min(static_cast<int64_t>(__popc(need)), end - next));
            // the `take` lowest needing lanes get rays next .. next+take-1
            const int rank = __popc(need & lanes_below);
            if (!has && rank < take) {
                const int64_t g = next + rank;
                int j = 0;
                int64_t ri = g;
                if (!kSingle) {
                    const FastGroup &grp = table.groups[group];
                    j = find_job_range(table.ray_begin, grp.first_job, grp.first_job + grp.num_jobs - 1, g);
                    ri = g - __ldg(table.ray_begin + j);
                }
                const Job<float> &job = kSingle ? single : table.jobs[j];
                s.job = j;
                s.ray = ri;
                s.bounce = 0;
                s.queries = 0;
                s.shadows = 0;
                s.path = 0.0;
                s.o[0] = job.lst[0]; s.o[1] = job.lst[1]; s.o[2] = job.lst[2];
                initial_direction(job, ri, s.d);
#pragma unroll
                for (int b = 0; b < kBands; ++b) s.acc[b] = 1.0f;
                has = true;
                if (job.num_bounces <= 0) {
                    atomicAdd(job.counters + 1, 1ull);
                    has = false;
                }
            }
            next += take;
            need = __ballot_sync(full, !has);
        }
        if (!__any_sync(full, has)) {
            if (pending >= 0) {
                const FastChunk ch = table.chunks[pending];
                group = ch.group; next = ch.begin; end = ch.end;
                pending = -1;
                continue;
            }
            if (exhausted || next >= end) {
                if (exhausted) break;
                continue;
            }
        }

        const FastScene &fs = kSingle ? single_fast : table.groups[group].fast;
        const Job<float> &job = kSingle ? single : table.jobs[s.job];

        // ---- closest hit (all lanes)
        FRay ray;
        make_ray(ray, s.o, s.d);
        float t;
        int slot;
        int surf = closest_scan(fs, ray, has, t, slot);
        if (has && surf < 0 && job.use_bvh) {
            // Missed everything: the reference's BVH walk reports the lowest visited surface.
            const int2 fb = fallback_walk(job.scene, s.o[0], s.o[1], s.o[2], s.d[0], s.d[1], s.d[2]);
            surf = fb.x;
            t = __int_as_float(fb.y);
            slot = -1;
        }
        float n[3] = {0.0f, 0.0f, 1.0f};
        bool finished = false, alive_at_end = false, count_hit = false;
        bool need_shadow = false;
        float hx = 0.0f, hy = 0.0f, hz = 0.0f, dist = 0.0f, facing = 0.0f;
        float sd[3] = {0.0f, 0.0f, 0.0f};
        if (has) {
            s.queries += 1;
            bool dead = surf < 0 || t <= job.listener_radius || s.path > job.max_path_length;
            if (!dead && s.bounce > 0) {
                if (sphere_before(s.o, s.d, job.lst, job.listener_radius, t)) dead = true;
                else if (job.source_distance > job.source_radius &&
                         sphere_before(s.o, s.d, job.src, job.source_radius, t))
                    dead = true;
            }
            if (dead) {
                finished = true;
            } else {
                count_hit = true;
                if (slot >= 0) {
                    winner_normal(fs, slot, ray, n);
                } else {
                    n[0] = __ldg(job.scene.normals + 3 * surf);
                    n[1] = __ldg(job.scene.normals + 3 * surf + 1);
                    n[2] = __ldg(job.scene.normals + 3 * surf + 2);
                    if (n[0] * s.d[0] + n[1] * s.d[1] + n[2] * s.d[2] > 0.0f) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
                }
                if (job.ray_surfaces) job.ray_surfaces[s.ray * job.num_bounces + s.bounce] = surf;
                hx = s.o[0] + t * s.d[0] + 1e-2f * n[0];
                hy = s.o[1] + t * s.d[1] + 1e-2f * n[1];
                hz = s.o[2] + t * s.d[2] + 1e-2f * n[2];
                const float tsx = job.src[0] - hx, tsy = job.src[1] - hy, tsz = job.src[2] - hz;
                dist = sqrtf(tsx * tsx + tsy * tsy + tsz * tsz);
                if (dist > job.irradiance_min_distance) {
                    const float inv = 1.0f / dist;
                    sd[0] = tsx * inv; sd[1] = tsy * inv; sd[2] = tsz * inv;
                    facing = n[0] * sd[0] + n[1] * sd[1] + n[2] * sd[2];
                    need_shadow = facing > 0.0f;
                }
            }
        }

        // ---- per-surface hit counters: one atomic per distinct (job, surface) in the warp
        const unsigned counting = __ballot_sync(full, count_hit);
        if (count_hit) {
            warp_count(counting, (static_cast<unsigned long long>(s.job) << 32) | static_cast<unsigned>(surf), 1u,
                       job.hit_counts + surf);
        }

        // ---- shadow ray toward the source (all lanes; those not needing it ride along)
        FRay shadow;
        const float h[3] = {hx, hy, hz};
        make_ray(shadow, h, sd);
        const bool occluded = shadow_scan(fs, shadow, need_shadow, dist - 1e-6f);

        if (has && !finished) {
            const Quad<float> m0 = ldq(job.scene.mats + static_cast<size_t>(surf) * kMatStride);
            const Quad<float> m1 = ldq(job.scene.mats + static_cast<size_t>(surf) * kMatStride + 4);
            const float refl[kBands] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y};
            const float scat = m1.z;
            if (need_shadow) {
                s.shadows += 1;
                if (!occluded) {
                    const float diffuse = static_cast<float>(1.0 / kPi) * scat * facing;
                    float half[3];
                    normalize3(sd[0] - s.d[0], sd[1] - s.d[1], sd[2] - s.d[2], half);
                    float cos_half = half[0] * n[0] + half[1] * n[1] + half[2] * n[2];
                    cos_half = cos_half > 0.0f ? cos_half : 0.0f;
                    const float specular = ((job.specular_exponent + 2.0f) * static_cast<float>(1.0 / (8.0 * kPi))) *
                                           (1.0f - scat) * __powf(cos_half, job.specular_exponent);
                    const float dmax = fmaxf(dist, job.irradiance_min_distance);
                    const float distance_term = static_cast<float>(1.0 / (4.0 * kPi)) / (dmax * dmax);
                    const float source_cosine = -(job.fwd[0] * sd[0] + job.fwd[1] * sd[1] + job.fwd[2] * sd[2]);
                    const float gain_base = fabsf((1.0f - job.dipole_weight) + job.dipole_weight * source_cosine);
                    const float source_gain = job.dipole_power == 1.0f ? gain_base : __powf(gain_base, job.dipole_power);
                    const double rel_delay =
                        (s.path + static_cast<double>(t) + static_cast<double>(dist)) / job.speed_of_sound -
                        job.direct_delay;
                    const double q = floor(rel_delay / job.bin_duration);
                    if (q >= 0.0 && q < static_cast<double>(job.num_bins)) {
                        const int bin = static_cast<int>(q);
                        const float common = job.ray_scale * source_gain * distance_term * (diffuse + specular);
                        long long esum = 0;
#pragma unroll
                        for (int b = 0; b < kBands; ++b) {
                            const float e = common * refl[b] * s.acc[b];
                            const long long qe = quantize(e, job.energy_scale);
                            add_fixed(job.echogram_fx + 2 * (static_cast<size_t>(b) * job.num_bins + bin), qe);
                            if (job.ambisonic_fx) {
                                float d0[3];
                                initial_direction(job, s.ray, d0);
                                unsigned long long *a =
                                    job.ambisonic_fx + 2 * (static_cast<size_t>(b) * 4 * job.num_bins + bin);
                                const size_t stride = 2 * static_cast<size_t>(job.num_bins);
                                add_fixed(a, qe);
                                add_fixed(a + stride, quantize(e * d0[0], job.energy_scale));
                                add_fixed(a + 2 * stride, quantize(e * d0[1], job.energy_scale));
                                add_fixed(a + 3 * stride, quantize(e * d0[2], job.energy_scale));
                            }
                            esum += qe;
                        }
                        atomicAdd(job.contrib_counts + surf, 1ull);
                        add_fixed(job.surface_energy_fx + 2 * static_cast<size_t>(surf), esum);
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kBands; ++b) s.acc[b] *= refl[b];
            s.path += static_cast<double>(t);
            s.o[0] = hx; s.o[1] = hy; s.o[2] = hz;
            bool use_diffuse;
            int sample;
            if (job.rng_mode == 0) {
                const size_t k = static_cast<size_t>(s.bounce) * job.num_rays + s.ray;
                use_diffuse = job.diffuse_random[k] < scat;
                sample = use_diffuse ? job.diffuse_indices[k] : 0;
            } else {
                const u32x4 rr = trace_draw(job.seed, job.stream_key, static_cast<uint32_t>(s.ray),
                                            static_cast<uint32_t>(s.bounce) + 1u);
                use_diffuse = u01_53(rr.x, rr.y) < static_cast<double>(scat);
                sample = static_cast<int>(below(rr.z, static_cast<uint32_t>(job.num_bank)));
            }
            if (use_diffuse) {
                const float *bs = job.diffuse_bank + 3 * sample;
                diffuse_direction(__ldg(bs), __ldg(bs + 1), __ldg(bs + 2), n[0], n[1], n[2], s.d);
            } else {
                const float dot = s.d[0] * n[0] + s.d[1] * n[1] + s.d[2] * n[2];
                normalize3(s.d[0] - 2.0f * dot * n[0], s.d[1] - 2.0f * dot * n[1], s.d[2] - 2.0f * dot * n[2], s.d);
            }
            s.bounce += 1;
            if (s.path > job.max_path_length) {
                finished = true;
            } else if (s.bounce >= job.num_bounces) {
                finished = true;
                alive_at_end = true;
            }
        }

        // ---- ray completion statistics, one atomic per distinct job in the warp
        const unsigned ending = __ballot_sync(full, finished);
        if (finished) {
            const unsigned grp = __match_any_sync(ending, static_cast<unsigned>(s.job));
            const unsigned q_sum = __reduce_add_sync(grp, static_cast<unsigned>(s.queries));
            const unsigned q_max = __reduce_max_sync(grp, static_cast<unsigned>(s.queries));
            const unsigned sh_sum = __reduce_add_sync(grp, static_cast<unsigned>(s.shadows));
            const unsigned alive_sum = __reduce_add_sync(grp, alive_at_end ? 1u : 0u);
            if (lane_id == __ffs(grp) - 1) {
                atomicMax(job.counters + 0, static_cast<unsigned long long>(q_max));
                if (alive_sum) atomicAdd(job.counters + 1, static_cast<unsigned long long>(alive_sum));
                atomicAdd(job.counters + 2, static_cast<unsigned long long>(q_sum));
                if (sh_sum) atomicAdd(job.counters + 3, static_cast<unsigned long long>(sh_sum));
            }
            if (job.ray_surfaces)
                for (int b = s.bounce; b < job.num_bounces; ++b) job.ray_surfaces[s.ray * job.num_bounces + b] = -1;
            has = false;
        }
    }
}

}  // namespace ac
