// Float32 production tracer for sm_100a: warp-uniform scene scan.
//
// Specialised at compile time on (single job, Philox stream, ambisonics,
// visual-path candidates), so no variant carries the state or the branches
// of an option it does not use.
//
// Same per-ray algorithm as trace_kernel.cuh (steam_rt.py:4708-4850), but the
// intersection queries are organised for SIMT instead of restating the
// reference's per-thread escape-link walk.  A warp always works on ONE scene;
// its surfaces are kept in three kind-separated lists:
//
//   * walls (2-D segments with a z range) and horizontal polygons are tested by
//     every lane in lockstep: all lanes read the same record (one broadcast
//     load) and the code path is uniform.  Walls are grouped in clusters of up
//     to 32 with an AABB the warp skips when no lane's ray can reach it;
//   * boxes (oriented furniture proxies) are grouped in clusters of up to 32.
//     Each lane first builds a 32-bit candidate mask from cheap world-AABB
//     tests done in lockstep, then all lanes pop their OWN next candidate
//     together -- same instructions, different box -- so the warp runs as many
//     exact box tests as the busiest lane needs, not the union over lanes;
//   * primitive tests compute only t, with reciprocal multiplies; the normal is
//     evaluated once, for the winning surface (boxes re-run the slab test);
//   * the shadow query tests boxes first (the likely blockers) and stops once
//     every lane that needs it has found a blocker;
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

#include "common.h"
#include "fast_bvh.h"
#include "trace_kernel.cuh"

namespace ac {

// Resident 256-thread blocks per SM the register allocation targets.
#ifndef AC_FAST_MIN_BLOCKS
#define AC_FAST_MIN_BLOCKS 3
#endif

// Cluster record: {lo.x, lo.y, lo.z, first} {hi.x, hi.y, hi.z, count}, count <= 32
constexpr int kClusterStride = 8;
constexpr int kMaxCluster = 32;

struct FastScene {
    const float *wall_clusters;  // [NWC][8]
    const float *walls;          // [NW][8]  {ax, ay, sx, sy} {z0, z1, tag, 0}
    const float *polys;          // [NP][4]  {z, tag, 0, 0}
    const float *box_clusters;   // [NBC][8]
    const float *box_bounds;     // [NB][8]  world AABB {lo.xyz, tag} {hi.xyz, 0}
    const float *boxes;          // [NB][12] box records (trace_kernel.cuh layout)
    const float *edges;          // [C][4]   {x_i, y_i, y_j (or y_i if skipped), (x_j-x_i)/(y_j-y_i)}
    int32_t num_wall_clusters;
    int32_t num_polys;
    int32_t num_box_clusters;
    int32_t num_edges;
    const float4 *bvh_nodes;     // BVH mode: [N][4] (width 2) or [N][8] (width 4) traversal BVH over walls and
                                 // boxes (fast_bvh.h); else null
    const float *bvh_prims;      // BVH mode: [P][12] surface records in leaf order
    int32_t num_bvh_nodes;       // 0: scan mode
    int32_t bvh_width;           // 2 or 4
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

// Continuous batching (ac_service_*): a ring of job slots in device memory that
// the host appends to while a persistent launch runs.  A slot is written once
// per job before the job is published and not rewritten while a launch that
// may hold it in L1 runs (each launch takes at most half a ring of sequence
// numbers); the slot stride keeps slots on separate cache lines.
struct alignas(256) ServiceSlot {
    Job<float> job;
    FastScene fast;
    float *echogram;             // float32 outputs the finishing warp converts the fixed-point sums into
    float *surface_energy;
    int64_t seq;                 // the job's sequence number
    int64_t num_chunks;
    uint64_t scene_id;           // jobs with equal ids share a scene (no lane drain between them)
    int64_t chunk_rays;
    int64_t ray_offset;          // rays of every job submitted before this one (a launch's warps start on
                                 // the job that holds their share of the published rays)
};

struct ServiceSlotState {        // device, zeroed by the host before the slot is published
    unsigned long long chunks_taken;
    unsigned long long rays_finished;
};

// Host-mapped control block.
struct ServiceControl {
    long long published;         // host: jobs below this sequence number are in the ring
    long long pad[15];
    long long done[1];           // [capacity] device: done[slot] = seq once that job's outputs are final
};

struct FastTable {
    const Job<float> *jobs;
    const int64_t *ray_begin;      // [num_jobs + 1]
    const FastGroup *groups;
    const FastChunk *chunks;       // group by group
    int64_t num_chunks;
    int32_t num_jobs;
    int32_t chunk_rays;            // single-job launches: rays per chunk
    unsigned long long *chunk_counter;   // single-job launches: next chunk
    // Batched launches: one chunk queue per scene group.  A warp starts on the
    // group that holds its share of the rays and stays on it until the group's
    // chunks run out, then takes the following groups' (wrapping), so a warp
    // drains its lanes for a change of scene about once per group it visits,
    // not at every group boundary of one shared queue.
    unsigned long long *group_next;      // [num_groups] chunks taken from each group
    const int64_t *group_chunk_begin;    // [num_groups + 1] first chunk of each group
    const int64_t *group_ray_begin;      // [num_groups + 1] first ray (over all jobs) of each group
    int32_t num_groups;
    int32_t reserved;
    // Service launches (continuous batching): the ring, its per-slot state and the control block.
    const ServiceSlot *slots;
    ServiceSlotState *slot_state;
    ServiceControl *control;             // host-mapped
    unsigned long long *low_water;       // device: jobs below it have no chunks left
    unsigned long long *published_copy;  // device: the published count as last read from the host
    unsigned long long *refresh_at;      // device: %globaltimer time at which the copy is read again
    unsigned long long *launch_words;    // device, this launch's own: [0] warps alive, [16] warps waiting for
                                         // work, [32] %globaltimer time at which a warp last began to wait,
                                         // [48] nonzero once the launch is closing
    int64_t window_first;                // this launch takes jobs from this sequence number
    int64_t window_end;                  // to below this one only
    int64_t idle_ns;                     // and ends once its warps found no work for this long
    int64_t mask;                        // ring capacity - 1
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    return now;
}

// Service launches: the published job count.  One warp of the whole grid at a time reads the host-mapped
// word (at most once per `kRefreshNs`) and raises a device copy of it; the others read the copy.  The
// acquire/release pair carries the host's slot writes to the reading warp through the copy.
constexpr unsigned long long kServiceRefreshNs = 2000;

__device__ __forceinline__ long long service_published(const FastTable &t) {
    const unsigned long long now = global_ns();
    const unsigned long long due = *reinterpret_cast<volatile unsigned long long *>(t.refresh_at);
    if (now >= due && atomicCAS(t.refresh_at, due, now + kServiceRefreshNs) == due) {
        long long pub;
        asm volatile("ld.acquire.sys.global.s64 %0, [%1];" : "=l"(pub) : "l"(&t.control->published) : "memory");
        asm volatile("red.release.gpu.global.max.u64 [%0], %1;" ::"l"(t.published_copy),
                     "l"(static_cast<unsigned long long>(pub)) : "memory");
        return pub;
    }
    unsigned long long pub;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(pub) : "l"(t.published_copy) : "memory");
    return static_cast<long long>(pub);
}

enum ServiceTake : int { kTakeChunk = 1, kTakeNone = 0, kTakeEnd = -1 };
constexpr unsigned long long kServiceRetryNs = 4000;   // a warp with live lanes asks for work this often

// Service launches, lane 0 of a warp: the next chunk (seq, chunk index) from job `queue` onward.
//  * kTakeChunk: a chunk was taken.
//  * kTakeNone (only when `may_wait` is false, i.e. some lanes of the warp still trace rays): nothing to
//    take right now; the warp carries on with its live lanes and asks again later.  A warp never sleeps
//    while it holds rays.
//  * kTakeEnd: the launch should end for this warp -- the whole launch has had nothing to trace for
//    `idle_ns` (every warp alive is waiting, the latest for longer than that), or the launch's window of
//    sequence numbers is used up.  The first warp to find the launch idle marks it closing, and from then
//    on no warp of it takes work, so the launch ends whole: it never shrinks to the few warps that happened
//    to find a job arriving as the others left, while the host, seeing it alive, starts no other.  Jobs
//    published meanwhile go to the next launch.
// Every wait is bounded: the idle deadline, and a poll cap.
__device__ __forceinline__ int service_take(const FastTable &t, bool may_wait, int64_t &queue, int64_t &published,
                                            int64_t *seq_out, int64_t *chunk_out) {
    unsigned long long *const alive = t.launch_words, *const waiting = t.launch_words + 16,
                              *const last_wait = t.launch_words + 32, *const closing = t.launch_words + 48;
    if (*reinterpret_cast<volatile unsigned long long *>(closing)) return kTakeEnd;
    unsigned long long idle_from = 0;
    unsigned sleep_ns = 256;
    bool rescanned = false, counted = false;   // counted: this warp is in the launch's waiting count
    auto leave = [&](int result) {
        if (counted) atomicAdd(waiting, ~0ull);   // -1
        return result;
    };
#pragma unroll 1
    for (int polls = 0; polls < (1 << 22); ++polls) {
        if (queue < published && queue < t.window_end) {
            const ServiceSlot &sl = t.slots[queue & t.mask];
            ServiceSlotState *st = t.slot_state + (queue & t.mask);
            const int64_t chunks = sl.num_chunks;
            if (static_cast<int64_t>(*reinterpret_cast<volatile unsigned long long *>(&st->chunks_taken)) < chunks) {
                const int64_t k = static_cast<int64_t>(atomicAdd(&st->chunks_taken, 1ull));
                if (k < chunks) {
                    *seq_out = queue;
                    *chunk_out = k;
                    return leave(kTakeChunk);
                }
            }
            // no chunks left here: raise the low-water mark past it if it points here, then move on
            atomicCAS(t.low_water, static_cast<unsigned long long>(queue), static_cast<unsigned long long>(queue + 1));
            ++queue;
            idle_from = 0;
            continue;
        }
        // caught up with the published jobs (or this launch's window): older jobs may still hold chunks
        // (other warps' jobs), so rescan them once from the low-water mark
        if (!rescanned) {
            rescanned = true;
            const int64_t low = max(static_cast<int64_t>(*reinterpret_cast<volatile unsigned long long *>(t.low_water)),
                                    t.window_first);
            if (low < queue) {
                queue = low;
                continue;
            }
        }
        if (queue >= t.window_end) return leave(kTakeEnd);
        if (*reinterpret_cast<volatile unsigned long long *>(closing)) return leave(kTakeEnd);
        const long long pub = service_published(t);
        if (pub > published) {
            published = pub;
            rescanned = false;
            continue;
        }
        if (!may_wait) return kTakeNone;
        // nothing to trace: wait for the host to publish more, until the whole launch has been idle for the
        // idle limit
        const unsigned long long now = global_ns();
        if (!counted) {
            counted = true;
            atomicAdd(waiting, 1ull);
            atomicMax(last_wait, now);
        }
        if (idle_from == 0) idle_from = now;
        const unsigned long long limit = static_cast<unsigned long long>(t.idle_ns);
        if (now - idle_from > limit &&
            *reinterpret_cast<volatile unsigned long long *>(waiting) >=
                *reinterpret_cast<volatile unsigned long long *>(alive) &&
            now - *reinterpret_cast<volatile unsigned long long *>(last_wait) > limit) {
            atomicExch(closing, 1ull);   // the launch is idle: it ends whole
            return leave(kTakeEnd);
        }
        __nanosleep(sleep_ns);
        if (sleep_ns < 32768) sleep_ns <<= 1;
    }
    return leave(kTakeEnd);
}

// Service launches, whole warp: `n` more rays of the job in `slot` have finished in this warp.  Every lane's
// sums and counters for those rays were added before this call; after the warp barrier lane 0's fence
// orders them (cumulatively) before the count, so the warp that completes the count sees every ray's sums.
// Returns true on the warp that counted the job's last ray.
__device__ __forceinline__ bool service_count(const FastTable &t, int slot, unsigned long long n, int lane_id) {
    __syncwarp();
    unsigned long long before = 0;
    if (lane_id == 0) {
        __threadfence();
        before = atomicAdd(&t.slot_state[slot].rays_finished, n);
    }
    before = __shfl_sync(0xFFFFFFFFu, before, 0);
    return before + n == static_cast<unsigned long long>(t.slots[slot].job.num_rays);
}

// Service launches: the job in `slot` has finished its last ray; every lane of the warp converts its
// fixed-point sums to the float32 outputs, then lane 0 flags it done to the host.  The sums were added at L2
// by atomics of all warps before they counted their rays finished (service_count fences first); they are
// read around L1 here.
__device__ __forceinline__ void service_finish(const FastTable &t, int slot, int lane_id) {
    __threadfence();
    const ServiceSlot &sl = t.slots[slot];
    const Job<float> &job = sl.job;
    const double inv = 1.0 / job.energy_scale;
    const int64_t nb = static_cast<int64_t>(kBands) * job.num_bins;
    for (int64_t i = lane_id; i < nb; i += 32) {
        const double v = ldexp(static_cast<double>(static_cast<long long>(__ldcg(job.echogram_fx + 2 * i + 1))), 32) +
                         static_cast<double>(__ldcg(job.echogram_fx + 2 * i));
        sl.echogram[i] = static_cast<float>(v * inv);
    }
    if (sl.surface_energy) {
        for (int64_t i = lane_id; i < job.scene.num_surfaces; i += 32) {
            const double v =
                ldexp(static_cast<double>(static_cast<long long>(__ldcg(job.surface_energy_fx + 2 * i + 1))), 32) +
                static_cast<double>(__ldcg(job.surface_energy_fx + 2 * i));
            sl.surface_energy[i] = static_cast<float>(v * inv);
        }
    }
    __syncwarp();
    if (lane_id == 0) {
        __threadfence_system();
        asm volatile("st.release.sys.global.s64 [%0], %1;" ::"l"(&t.control->done[slot]), "l"(sl.seq) : "memory");
    }
}

// Node boxes are culled with the ray's slab planes as one fused multiply-add
// each (t = v * inv - o * inv); measured 2-4 % faster than (v - o) * inv on the
// U room and the 8-room apartment, with identical results (node boxes are
// padded, so the culling stays conservative under either rounding).
#ifndef AC_WARP_DEPOSIT
#define AC_WARP_DEPOSIT 0
#endif
#ifndef AC_FMA_SLAB
#define AC_FMA_SLAB 1
#endif

struct FRay {
    float o[3];
    float d[3];
    float inv[3];
#if AC_FMA_SLAB
    float oi[3];   // o * inv: a slab plane's t is then one fused multiply-add
#endif
};

// Approximate reciprocal (MUFU, ~1 ulp): the float32 path needs no correctly rounded division.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ float safe_inv(float d) {
    const float m = fabsf(d) < 1e-20f ? copysignf(1e-20f, d) : d;
    return rcp_approx(m);
}

__device__ __forceinline__ void make_ray(FRay &r, const float *o, const float *d) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        r.o[a] = o[a];
        r.d[a] = d[a];
        r.inv[a] = safe_inv(d[a]);
#if AC_FMA_SLAB
        r.oi[a] = o[a] * r.inv[a];
#endif
    }
}

// t of the plane x_a = v along the ray (conservative box culling only: node boxes are padded)
__device__ __forceinline__ float slab_t(const FRay &r, int a, float v) {
#if AC_FMA_SLAB
    return fmaf(v, r.inv[a], -r.oi[a]);
#else
    return (v - r.o[a]) * r.inv[a];
#endif
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
#pragma unroll 1
    for (int i = 0; i < n; ++i) {
        const Quad<float> e = ldq(edges + 4 * i);  // uniform across the warp
        if ((e.y > y) != (e.z > y)) {
            if (x < e.x + (y - e.y) * e.w) inside = !inside;
        }
    }
    return inside;
}

// Wall t (steam_rt.py:4366-4377 with a reciprocal); 1e30 = miss.
__device__ __forceinline__ float wall_t(const Quad<float> &A, const Quad<float> &B, const FRay &r) {
    const float det = A.z * r.d[1] - A.w * r.d[0];
    if (fabsf(det) > 1e-12f) {
        const float inv = rcp_approx(det);
        const float relx = r.o[0] - A.x, rely = r.o[1] - A.y;
        const float t = (relx * A.w - rely * A.z) * inv;
        const float u = (relx * r.d[1] - rely * r.d[0]) * inv;
        const float z = r.o[2] + t * r.d[2];
        if (t > 1e-6f && u >= -1e-6f && u <= 1.000001f && z >= B.x - 1e-6f && z <= B.y + 1e-6f) return t;
    }
    return 1e30f;
}

// Oriented box t (steam_rt.py:4277-4358, slabs with reciprocals); 1e30 = miss.
__device__ __forceinline__ float box_t(const float *rec, const FRay &r) {
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
        const float ix = rcp_approx(dx);
        const float a = (-B.z - ox) * ix, b = (B.z - ox) * ix;
        t_min = fminf(a, b);
        t_max = fmaxf(a, b);
    }
    if (fabsf(dy) <= 1e-12f) {
        if (oy < -B.w || oy > B.w) return 1e30f;
    } else {
        const float iy = rcp_approx(dy);
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

__device__ __forceinline__ void take(float t, int si, float &best_t, int &best) {
    if (t < best_t || (t == best_t && t < 1e30f && si < best)) {
        best_t = t;
        best = si;
    }
}

// Scene query of the warp's lanes; every lane of the warp must call it.
//
// Closest-hit mode (best_t starts at 1e30): the minimum t over all surfaces,
// ties to the lower surface index.  Any-hit mode (best_t starts at the shadow
// ray's length): a lane stops as soon as it finds any surface closer than
// that.  Both modes use the same update rule, so the code exists once:
// `best` is the surface found (-1: none) and best_t its t.  The mode is a
// lane's own: lanes of one warp may run closest-hit and shadow queries together.
__device__ __forceinline__ void scene_scan(const FastScene &fs, const FRay &r, bool active, bool any_hit,
                                           float &best_t, int &best) {
    const unsigned full = 0xFFFFFFFFu;
    best = -1;
    // Walls, in lockstep.
#pragma unroll 1
    for (int c = 0; c < fs.num_wall_clusters; ++c) {
        const bool searching = active && !(any_hit && best >= 0);
        if (!__any_sync(full, searching)) return;
        const float *cp = fs.wall_clusters + kClusterStride * c;
        const Quad<float> lo = ldq(cp), hi = ldq(cp + 4);
        const bool pass = searching && cluster_overlaps(r, lo, hi, best_t);
        if (!__any_sync(full, pass)) continue;
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
#pragma unroll 1
        for (int k = 0; k < count; ++k) {
            const float *w = fs.walls + static_cast<size_t>(first + k) * 8;
            const Quad<float> A = ldq(w), B = ldq(w + 4);
            if (pass) take(wall_t(A, B, r), __float_as_int(B.z) >> 2, best_t, best);
        }
    }
    // Horizontal polygons (floor, ceiling), in lockstep.
#pragma unroll 1
    for (int k = 0; k < fs.num_polys; ++k) {
        const Quad<float> P = ldq(fs.polys + 4 * k);
        const float t = (P.x - r.o[2]) * r.inv[2];
        const int si = __float_as_int(P.y) >> 2;
        const bool cand = active && !(any_hit && best >= 0) && fabsf(r.d[2]) > 1e-12f && t > 1e-6f &&
                          (t < best_t || (t == best_t && si < best));
        if (__any_sync(full, cand)) {
            const float px = r.o[0] + t * r.d[0], py = r.o[1] + t * r.d[1];
            if (cand && point_in_polygon_fast(px, py, fs.edges, fs.num_edges)) take(t, si, best_t, best);
        }
    }
    // Boxes: per-lane candidate masks from world AABBs, then per-lane candidates in lockstep.
#pragma unroll 1
    for (int c = 0; c < fs.num_box_clusters; ++c) {
        const bool searching = active && !(any_hit && best >= 0);
        if (!__any_sync(full, searching)) return;
        const float *cp = fs.box_clusters + kClusterStride * c;
        const Quad<float> lo = ldq(cp), hi = ldq(cp + 4);
        const bool pass = searching && cluster_overlaps(r, lo, hi, best_t);
        if (!__any_sync(full, pass)) continue;
        const int first = __float_as_int(lo.w), count = __float_as_int(hi.w);
        unsigned mask = 0u;
#pragma unroll 1
        for (int k = 0; k < count; ++k) {
            const float *bb = fs.box_bounds + static_cast<size_t>(first + k) * 8;
            if (pass && cluster_overlaps(r, ldq(bb), ldq(bb + 4), best_t)) mask |= 1u << k;
        }
        while (__any_sync(full, mask != 0u)) {
            if (mask) {
                const int k = __ffs(mask) - 1;
                mask &= mask - 1u;
                const float *rec = fs.boxes + static_cast<size_t>(first + k) * kPrimStride;
                take(box_t(rec, r), __float_as_int(__ldg(rec + 11)) >> 2, best_t, best);
                if (any_hit && best >= 0) mask = 0u;
            }
        }
    }
}

// Slab test of one child box of a traversal-BVH node, with the scan's margin on max_t.
__device__ __forceinline__ bool child_box(const FRay &r, float lx, float hx, float ly, float hy, float lz, float hz,
                                          float max_t, float &enter) {
    const float x0 = slab_t(r, 0, lx), x1 = slab_t(r, 0, hx);
    const float y0 = slab_t(r, 1, ly), y1 = slab_t(r, 1, hy);
    const float z0 = slab_t(r, 2, lz), z1 = slab_t(r, 2, hz);
    enter = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.0f));
    const float exit_ = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), max_t));
    return enter <= exit_;
}

// Per-lane descent of the traversal BVH (BVH mode), organised "while-while"
// (Aila and Laine, "Understanding the efficiency of ray traversal on GPUs",
// HPG 2009): a lane descends inner nodes -- nearer child first, the farther
// one on a short stack in local memory -- until it holds a leaf, then keeps
// descending while other lanes of the warp still look for theirs, so leaves
// are tested by as many lanes at once as possible.  The builder bounds the
// depth by kBvhStack - 1; the stack holds one sentinel plus one entry per
// inner level.  Same update rule as the scan, so closest-hit and
// any-hit modes work as there.
constexpr int kBvhDone = static_cast<int>(0x80000000u);  // below every leaf reference

// The per-lane traversal stack.  In shared memory (AC_SMEM_STACK, the
// default): entry-major, [entries][256] words per block in the launch's
// dynamic shared memory, so the lanes of a warp hit 32 different banks
// whatever their stack depths, and stack traffic stays out of L1, where the
// scene's nodes and surfaces live.  The launch picks `entries` (a tuned
// knob: fewer entries leave more of the SM's on-chip memory to L1) no lower
// than the stack_need of any BVH scene it traces, which bounds every push.
// Otherwise in local memory (a per-thread array of kBvhStack).
#ifndef AC_SMEM_STACK
#define AC_SMEM_STACK 1
#endif
constexpr int kStackStride = 256;   // threads per block at most

struct LaneStack {
#if AC_SMEM_STACK
    int *base;
    __device__ __forceinline__ int &operator[](int i) { return base[i * kStackStride]; }
#else
    int entries[kBvhStack];
    __device__ __forceinline__ int &operator[](int i) { return entries[i]; }
#endif
};

// Host: the traversal stack entries of a float32 launch, from the requested count (0: kBvhStack) and the
// largest stack_need among the launch's BVH scenes (0: none has a BVH, the launch needs no stack).
inline int launch_stack_entries(int requested, int need, int *entries) {
    *entries = 0;
    if (requested < 0 || requested > kBvhStack)
        return fail(AC_ERR_INVALID, "stack_entries %d is outside 0..%d", requested, kBvhStack);
    if (need <= 0) return AC_OK;
    const int n = requested > 0 ? requested : kBvhStack;
    if (n < need)
        return fail(AC_ERR_INVALID, "stack_entries %d is below the %d a BVH scene of the launch needs", n, need);
    *entries = n;
    return AC_OK;
}

// Host: dynamic shared memory of a float32 launch with `entries` stack entries per lane.
inline size_t stack_smem_bytes(int entries) {
    return AC_SMEM_STACK ? static_cast<size_t>(entries) * kStackStride * sizeof(int) : 0;
}

__device__ __forceinline__ LaneStack lane_stack() {
#if AC_SMEM_STACK
    extern __shared__ int stack_words[];
    return LaneStack{stack_words + threadIdx.x};
#else
    return LaneStack{};
#endif
}

__device__ __forceinline__ void bvh_traverse(const FastScene &fs, const FRay &r, bool any_hit, float &best_t,
                                             int &best) {
    LaneStack stack = lane_stack();
    stack[0] = kBvhDone;
    int sp = 1;
    int node = 0;      // next node to visit (>= 0 inner, < 0 leaf, kBvhDone finished)
    int leaf = 0;      // a leaf waiting to be tested (< 0), 0 = none
#pragma unroll 1
    while (node != kBvhDone || leaf < 0) {
#pragma unroll 1
        while (node >= 0) {
            const float4 *np = fs.bvh_nodes + 4 * static_cast<size_t>(node);
            const float4 a = __ldg(np), b = __ldg(np + 1), c = __ldg(np + 2), k = __ldg(np + 3);
            const float max_t = best_t * 1.000001f + 1e-5f;
            float e0, e1;
            const bool h0 = child_box(r, a.x, a.y, a.z, a.w, c.x, c.y, max_t, e0);
            const bool h1 = child_box(r, b.x, b.y, b.z, b.w, c.z, c.w, max_t, e1);
            const int k0 = __float_as_int(k.x), k1 = __float_as_int(k.y);
            if (h0 && h1) {
                const bool swap = e1 < e0;
                node = swap ? k1 : k0;
                stack[sp++] = swap ? k0 : k1;
            } else if (h0 || h1) {
                node = h0 ? k0 : k1;
            } else {
                node = stack[--sp];
            }
            if (node < 0 && node != kBvhDone && leaf == 0) {   // park the leaf, keep descending
                leaf = node;
                node = stack[--sp];
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;   // every lane holds a leaf: test them
        }
#pragma unroll 1
        while (leaf < 0) {
            const int code = ~leaf;
            const int first = code >> 3, count = (code & 7) + 1;
#pragma unroll 1
            for (int i = 0; i < count; ++i) {
                const float *rec = fs.bvh_prims + static_cast<size_t>(first + i) * kPrimStride;
                const int tag = __float_as_int(__ldg(rec + 11));
                const float tt = (tag & 3) == 0 ? wall_t(ldq(rec), ldq(rec + 4), r) : box_t(rec, r);
                take(tt, tag >> 2, best_t, best);
            }
            if (any_hit && best >= 0) return;
            leaf = 0;
            if (node < 0 && node != kBvhDone) {   // the next stop is a leaf too
                leaf = node;
                node = stack[--sp];
            }
        }
    }
}

// Four-wide descent (width 4 layout of fast_bvh.h), organised like bvh_traverse:
// a node fetch tests all its children; the hit ones are ordered by entry
// distance, the nearest is taken next and the others pushed farthest first;
// leaves are parked so that lanes test them together.  The builder keeps the
// stack a ray can need below kBvhStack.
__device__ __forceinline__ void cswap(float &ea, int &ra, float &eb, int &rb) {
    if (eb < ea) {
        const float e = ea; ea = eb; eb = e;
        const int r = ra; ra = rb; rb = r;
    }
}

__device__ __forceinline__ void bvh4_traverse(const FastScene &fs, const FRay &r, bool any_hit, float &best_t,
                                              int &best) {
    LaneStack stack = lane_stack();
    stack[0] = kBvhDone;
    int sp = 1;
    int node = 0;
    int leaf = 0;
#pragma unroll 1
    while (node != kBvhDone || leaf < 0) {
#pragma unroll 1
        while (node >= 0) {
            const float4 *np = fs.bvh_nodes + 8 * static_cast<size_t>(node);
            const float4 lx = __ldg(np), hx = __ldg(np + 1), ly = __ldg(np + 2), hy = __ldg(np + 3);
            const float4 lz = __ldg(np + 4), hz = __ldg(np + 5), rf = __ldg(np + 6);
            const float max_t = best_t * 1.000001f + 1e-5f;
            float e0, e1, e2, e3;
            const bool h0 = child_box(r, lx.x, hx.x, ly.x, hy.x, lz.x, hz.x, max_t, e0);
            const bool h1 = child_box(r, lx.y, hx.y, ly.y, hy.y, lz.y, hz.y, max_t, e1);
            const bool h2 = child_box(r, lx.z, hx.z, ly.z, hy.z, lz.z, hz.z, max_t, e2);
            const bool h3 = child_box(r, lx.w, hx.w, ly.w, hy.w, lz.w, hz.w, max_t, e3);
            // misses sort last (+inf); a five-comparator network orders the four by entry distance
            const float inf = __int_as_float(0x7f800000);
            float d0 = h0 ? e0 : inf, d1 = h1 ? e1 : inf, d2 = h2 ? e2 : inf, d3 = h3 ? e3 : inf;
            int r0 = __float_as_int(rf.x), r1 = __float_as_int(rf.y), r2 = __float_as_int(rf.z), r3 = __float_as_int(rf.w);
            cswap(d0, r0, d1, r1);
            cswap(d2, r2, d3, r3);
            cswap(d0, r0, d2, r2);
            cswap(d1, r1, d3, r3);
            cswap(d1, r1, d2, r2);
            const int hits = static_cast<int>(h0) + static_cast<int>(h1) + static_cast<int>(h2) + static_cast<int>(h3);
            if (hits >= 4) stack[sp++] = r3;
            if (hits >= 3) stack[sp++] = r2;
            if (hits >= 2) stack[sp++] = r1;
            node = hits >= 1 ? r0 : stack[--sp];
            if (node < 0 && node != kBvhDone && leaf == 0) {   // park the leaf, keep descending
                leaf = node;
                node = stack[--sp];
            }
            if (!__any_sync(__activemask(), leaf == 0)) break;   // every lane holds a leaf: test them
        }
#pragma unroll 1
        while (leaf < 0) {
            const int code = ~leaf;
            const int first = code >> 3, count = (code & 7) + 1;
#pragma unroll 1
            for (int i = 0; i < count; ++i) {
                const float *rec = fs.bvh_prims + static_cast<size_t>(first + i) * kPrimStride;
                const int tag = __float_as_int(__ldg(rec + 11));
                const float tt = (tag & 3) == 0 ? wall_t(ldq(rec), ldq(rec + 4), r) : box_t(rec, r);
                take(tt, tag >> 2, best_t, best);
            }
            if (any_hit && best >= 0) return;
            leaf = 0;
            if (node < 0 && node != kBvhDone) {   // the next stop is a leaf too
                leaf = node;
                node = stack[--sp];
            }
        }
    }
}

// The closest-hit / any-hit query of one ray: the lockstep scan (walls and
// boxes in scan mode, horizontal polygons always) and, in BVH mode, the
// per-lane BVH descent over walls and boxes.  Every lane must call it.
__device__ __forceinline__ void scene_query(const FastScene &fs, const FRay &r, bool active, bool any_hit,
                                            float &best_t, int &best) {
    scene_scan(fs, r, active, any_hit, best_t, best);
    if (fs.num_bvh_nodes > 0 && active && !(any_hit && best >= 0)) {
        if (fs.bvh_width == 4) bvh4_traverse(fs, r, any_hit, best_t, best);
        else bvh_traverse(fs, r, any_hit, best_t, best);
    }
}

// Normal of the winning surface, oriented against the ray.
__device__ __forceinline__ void winner_normal(const SceneDev<float> &sc, int si, const FRay &r, float t, float *n) {
    const float *rec = sc.prims_linear + static_cast<size_t>(si) * kPrimStride;
    const int kind = __float_as_int(__ldg(rec + 11)) & 3;
    if (kind == 0) {
        n[0] = __ldg(rec + 6); n[1] = __ldg(rec + 7); n[2] = __ldg(rec + 8);
    } else if (kind == 2) {
        // Face of the box the hit point lies on: the box-frame axis where the
        // point is closest to the face, relative to the half extent.
        const Quad<float> A = ldq(rec), B = ldq(rec + 4), C = ldq(rec + 8);
        const float px = r.o[0] + t * r.d[0] - A.x, py = r.o[1] + t * r.d[1] - A.y, pz = r.o[2] + t * r.d[2];
        const float lx = px * A.z + py * A.w, ly = px * B.x + py * B.y;
        const float hz = 0.5f * (C.y - C.x), lz = pz - 0.5f * (C.x + C.y);
        const float ex = fabsf(fabsf(lx) - B.z), ey = fabsf(fabsf(ly) - B.w), ez = fabsf(fabsf(lz) - hz);
        if (ex <= ey && ex <= ez) {
            const float sg = lx >= 0.0f ? 1.0f : -1.0f;
            n[0] = sg * A.z; n[1] = sg * A.w; n[2] = 0.0f;
        } else if (ey <= ez) {
            const float sg = ly >= 0.0f ? 1.0f : -1.0f;
            n[0] = sg * B.x; n[1] = sg * B.y; n[2] = 0.0f;
        } else {
            n[0] = 0.0f; n[1] = 0.0f; n[2] = lz >= 0.0f ? 1.0f : -1.0f;
        }
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

// Float32 unit vector with the reference's zero-length rule (|v| <= 1e-12 -> 0), via rsqrt.
__device__ __forceinline__ void normalize3f(float x, float y, float z, float *out) {
    const float n2 = x * x + y * y + z * z;
    if (n2 <= 1e-24f) { out[0] = 0.0f; out[1] = 0.0f; out[2] = 0.0f; return; }
    const float inv = rsqrtf(n2);
    out[0] = x * inv; out[1] = y * inv; out[2] = z * inv;
}

// steam_rt.py:4564-4582 in float32 with rsqrt normalisation.
__device__ __forceinline__ void diffuse_direction_f(float s0, float s1, float s2, float nx, float ny, float nz,
                                                    float *out) {
    float hx = 1.0f, hy = 0.0f;
    if (fabsf(nx) >= 0.9f) { hx = 0.0f; hy = 1.0f; }
    float t[3];
    normalize3f(hy * nz, -hx * nz, hx * ny - hy * nx, t);
    const float bx = ny * t[2] - nz * t[1];
    const float by = nz * t[0] - nx * t[2];
    const float bz = nx * t[1] - ny * t[0];
    normalize3f(s0 * t[0] + s1 * bx + s2 * nx, s0 * t[1] + s1 * by + s2 * ny, s0 * t[2] + s1 * bz + s2 * nz, out);
}


// A lane's ray in registers; its band energies, counters and ray number, which only the shading and the
// completion use, live in shared memory (LaneShared) so that they hold no registers during the traversal.
struct FastLane {
    float o[3];
    float d[3];
    float d0[3];  // initial direction (ambisonic coefficients)
    double path;
    int job;
    int bounce;
    int vslot;    // visual-candidate slot, -1 for none
};

// Per-lane shared state, entry-major ([entry][256]) so that a warp's lanes hit 32 different banks.
struct LaneShared {
    float acc[kBands][kStackStride];     // band energies
    int queries[kStackStride];           // closest-hit queries of the ray so far
    int shadows[kStackStride];           // shadow queries
    long long ray[kStackStride];         // ray number within its job
};

__device__ __forceinline__ int find_job_range(const int64_t *prefix, int lo, int hi, int64_t g) {
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <bool kSingle, bool kPhilox, bool kAmb, bool kVisual, bool kService = false>
__global__ void __launch_bounds__(256, AC_FAST_MIN_BLOCKS) trace_fast_kernel(const __grid_constant__ Job<float> single,
                                                         const __grid_constant__ FastScene single_fast,
                                                         const __grid_constant__ FastTable table) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const unsigned lanes_below = (1u << lane_id) - 1u;

    // Warp-uniform work state, kept in shared memory between iterations: each iteration loads it into locals
    // for the refill and stores it back before the rays are traced, so it holds no registers (nor spill
    // slots) during the traversal.  Every lane stores the same values.
    struct WarpWork {
        long long next, end;   // rays next .. end - 1 of the current chunk are not handed out yet
        long long pending;     // chunk of another scene, taken but not started (-1: none)
        int group;             // the scene group (service launches: the slot) the warp's lanes trace
        int queue;             // batched launches: the group queue this warp takes chunks from
        int exhausted;
    };
    __shared__ WarpWork warp_work[8];
    volatile WarpWork &ww = warp_work[threadIdx.x >> 5];
    ww.next = 0; ww.end = 0; ww.pending = -1; ww.group = -1; ww.queue = 0; ww.exhausted = 0;
    const int64_t num_chunks = kSingle ? (single.num_rays + table.chunk_rays - 1) / table.chunk_rays : table.num_chunks;
    // Service launches: the warp's job-ring state lives in shared memory and is read where it is used, so it
    // holds no registers across the traversal (every lane stores the same values).
    struct ServiceWarp {
        long long queue, published;            // next job to take chunks from, jobs seen published
        long long pending_begin, pending_end;  // the ray range of a chunk of another scene, taken but not started
        unsigned long long retry_at;           // lane 0: next ask while lanes are live
        unsigned long long count_n;            // finished rays of job count_slot not yet added to its count
        int cur_slot;                          // the job of the chunk being handed out
        int count_slot;
    };
    __shared__ ServiceWarp service_warps[kService ? 8 : 1];
    volatile ServiceWarp &sw = service_warps[kService ? (threadIdx.x >> 5) : 0];
    volatile long long &svc_queue = sw.queue;
    volatile long long &svc_published = sw.published;
    volatile int &cur_slot = sw.cur_slot;
    volatile unsigned long long &retry_at = sw.retry_at;
    volatile int &count_slot = sw.count_slot;
    volatile unsigned long long &count_n = sw.count_n;
    volatile long long &pending_begin = sw.pending_begin;
    volatile long long &pending_end = sw.pending_end;
    if (kService) {
        svc_queue = 0; svc_published = 0; cur_slot = 0; retry_at = 0; count_slot = -1; count_n = 0;
        pending_begin = 0; pending_end = 0;
        __syncwarp();
    }
    if (kService) {
        long long pub = 0;
        if (lane_id == 0)
            asm volatile("ld.acquire.sys.global.s64 %0, [%1];" : "=l"(pub) : "l"(&table.control->published) : "memory");
        pub = __shfl_sync(full, pub, 0);
        const long long low = max(static_cast<long long>(*reinterpret_cast<volatile unsigned long long *>(table.low_water)),
                                  static_cast<long long>(table.window_first));
        const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
        const int64_t warp = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        svc_published = pub;
        svc_queue = low;
        if (lane_id == 0) atomicAdd(table.launch_words, 1ull);   // this warp is alive in the launch
        const int64_t last = min(static_cast<int64_t>(pub), table.window_end) - 1;
        if (last > low) {
            // start on the job that holds this warp's share of the published rays
            const ServiceSlot &a = table.slots[low & table.mask];
            const ServiceSlot &b = table.slots[last & table.mask];
            const int64_t r0 = a.ray_offset;
            const int64_t at = r0 + static_cast<int64_t>((static_cast<double>(warp) + 0.5) / static_cast<double>(warps) *
                                                         static_cast<double>(b.ray_offset + b.job.num_rays - r0));
            int64_t lo = low, hi = last;
            while (lo < hi) {   // last job whose first ray is at or before `at`
                const int64_t mid = (lo + hi + 1) >> 1;
                if (table.slots[mid & table.mask].ray_offset <= at) lo = mid; else hi = mid - 1;
            }
            svc_queue = lo;
        }
    } else if (!kSingle) {
        const int64_t warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
        const int64_t warp = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
        const int64_t total = __ldg(table.group_ray_begin + table.num_groups);
        const int64_t at = static_cast<int64_t>((static_cast<double>(warp) + 0.5) / static_cast<double>(warps) *
                                                static_cast<double>(total));
        int lo = 0, hi = table.num_groups - 1;
        while (lo < hi) {   // last group whose first ray is at or before `at`
            const int mid = (lo + hi + 1) >> 1;
            if (__ldg(table.group_ray_begin + mid) <= at) lo = mid; else hi = mid - 1;
        }
        ww.queue = lo;
    }

    FastLane s;
    __shared__ LaneShared lane_shared;
    volatile float *const lane_acc = &lane_shared.acc[0][threadIdx.x];          // [b * kStackStride]
    volatile int &lane_queries = lane_shared.queries[threadIdx.x];
    volatile int &lane_shadows = lane_shared.shadows[threadIdx.x];
    volatile long long &lane_ray = lane_shared.ray[threadIdx.x];
    bool has = false;
    s.job = 0;

    while (true) {
        int group = ww.group, queue = ww.queue;
        int64_t next = ww.next, end = ww.end, pending = ww.pending;
        bool exhausted = ww.exhausted != 0;
        auto save = [&]() {   // after every lane has read the old values
            __syncwarp();
            ww.group = group; ww.queue = queue; ww.next = next; ww.end = end; ww.pending = pending;
            ww.exhausted = exhausted ? 1 : 0;
        };
        // ---- refill lanes from the warp's range; take more chunks of the same scene as needed
        unsigned need = __ballot_sync(full, !has);
        while (need && pending < 0 && !exhausted) {
            if (next >= end) {
                long long c = 0;
                if (kService) {
                    const bool live = __any_sync(full, has);
                    long long seq = -1, chunk = 0;
                    int got = kTakeNone;
                    int64_t wq = svc_queue, wp = svc_published;
                    if (lane_id == 0 && (!live || global_ns() >= retry_at)) {   // live warps ask every few us
                        int64_t sq = 0, ck = 0;
                        got = service_take(table, !live, wq, wp, &sq, &ck);
                        if (got == kTakeChunk) { seq = sq; chunk = ck; }
                        if (got == kTakeNone) retry_at = global_ns() + kServiceRetryNs;
                    }
                    got = __shfl_sync(full, got, 0);
                    seq = __shfl_sync(full, seq, 0);
                    chunk = __shfl_sync(full, chunk, 0);
                    wq = __shfl_sync(full, static_cast<long long>(wq), 0);
                    wp = __shfl_sync(full, static_cast<long long>(wp), 0);
                    svc_queue = wq;
                    svc_published = wp;
                    if (got == kTakeEnd) {
                        if (lane_id == 0) atomicAdd(table.launch_words, ~0ull);   // takes no more work
                        exhausted = true;
                        break;
                    }
                    if (got == kTakeNone) break;   // nothing now: trace the live lanes, ask again later
                    const int slot = static_cast<int>(seq & table.mask);
                    const ServiceSlot &sl = table.slots[slot];
                    const int64_t cb = chunk * sl.chunk_rays;
                    const int64_t ce = min(cb + sl.chunk_rays, sl.job.num_rays);
                    if (group >= 0 && sl.scene_id != table.slots[group].scene_id) {   // (group: a slot index)
                        if (!__any_sync(full, has)) {
                            group = slot; cur_slot = slot; next = cb; end = ce;   // idle warp: switch scenes now
                        } else {
                            pending = slot; pending_begin = cb; pending_end = ce;
                            break;
                        }
                    } else {
                        if (group < 0) group = slot;
                        cur_slot = slot; next = cb; end = ce;
                    }
                } else if (kSingle) {
                    if (lane_id == 0) c = static_cast<long long>(atomicAdd(table.chunk_counter, 1ull));
                    c = __shfl_sync(full, c, 0);
                    if (c >= num_chunks) { exhausted = true; break; }
                } else {
                    // this warp's group queue, then the following groups' until one has chunks left
                    int probes = 0;
                    while (true) {
                        if (lane_id == 0) {
                            c = -1;
                            const int64_t first = __ldg(table.group_chunk_begin + queue);
                            const int64_t count = __ldg(table.group_chunk_begin + queue + 1) - first;
                            const unsigned long long taken =
                                *reinterpret_cast<volatile unsigned long long *>(table.group_next + queue);
                            if (static_cast<int64_t>(taken) < count) {
                                const int64_t k = static_cast<int64_t>(atomicAdd(table.group_next + queue, 1ull));
                                if (k < count) c = first + k;
                            }
                        }
                        c = __shfl_sync(full, c, 0);
                        if (c >= 0 || ++probes >= table.num_groups) break;
                        queue = queue + 1 == table.num_groups ? 0 : queue + 1;
                    }
                    if (c < 0) { exhausted = true; break; }
                }
                if constexpr (!kService) {
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
            }
            const int take = static_cast<int>(min(static_cast<int64_t>(__popc(need)), end - next));
            // the `take` lowest needing lanes get rays next .. next+take-1
            const int rank = __popc(need & lanes_below);
            if (!has && rank < take) {
                const int64_t g = next + rank;
                int j = 0;
                int64_t ri = g;
                if (kService) {
                    j = cur_slot;
                } else if (!kSingle) {
                    const FastGroup &grp = table.groups[group];
                    j = find_job_range(table.ray_begin, grp.first_job, grp.first_job + grp.num_jobs - 1, g);
                    ri = g - __ldg(table.ray_begin + j);
                }
                const Job<float> &job = kSingle ? single : (kService ? table.slots[j].job : table.jobs[j]);
                s.job = j;
                lane_ray = ri;
                s.bounce = 0;
                lane_queries = 0;
                lane_shadows = 0;
                s.path = 0.0;
                if (kVisual) {
                    s.vslot = visual_slot(job, ri);
                    if (s.vslot >= 0) job.visual_rays[s.vslot] = static_cast<int32_t>(ri);
                }
                s.o[0] = job.lst[0]; s.o[1] = job.lst[1]; s.o[2] = job.lst[2];
                if (kPhilox) {
                    const double3 v = philox_direction(job.seed, job.stream_key, job.num_rays, ri);
                    s.d[0] = static_cast<float>(v.x); s.d[1] = static_cast<float>(v.y); s.d[2] = static_cast<float>(v.z);
                } else {
                    s.d[0] = job.directions[3 * ri]; s.d[1] = job.directions[3 * ri + 1];
                    s.d[2] = job.directions[3 * ri + 2];
                }
                if (kAmb) { s.d0[0] = s.d[0]; s.d0[1] = s.d[1]; s.d0[2] = s.d[2]; }
#pragma unroll
                for (int b = 0; b < kBands; ++b) lane_acc[b * kStackStride] = 1.0f;
                has = true;
                if (job.num_bounces <= 0) {   // the host refuses such jobs in service launches
                    atomicAdd(job.counters + 1, 1ull);
                    has = false;
                }
            }
            next += take;
            need = __ballot_sync(full, !has);
        }
        if (!__any_sync(full, has)) {
            if (pending >= 0) {
                if (kService) {
                    group = static_cast<int>(pending); cur_slot = group; next = pending_begin; end = pending_end;
                } else {
                    const FastChunk ch = table.chunks[pending];
                    group = ch.group; next = ch.begin; end = ch.end;
                }
                pending = -1;
                save();
                continue;
            }
            if (exhausted || next >= end) {
                if (exhausted) break;
                save();
                continue;
            }
        }
        save();

        const FastScene &fs = kSingle ? single_fast : (kService ? table.slots[group].fast : table.groups[group].fast);
        const Job<float> &job = kSingle ? single : (kService ? table.slots[s.job].job : table.jobs[s.job]);

        // ---- two queries per bounce through one copy of the scan: phase 0 finds the
        // closest hit, phase 1 casts the shadow ray toward the source.
        FRay ray;
        make_ray(ray, s.o, s.d);
        float t = 1e30f;
        int surf = -1;
        float n[3] = {0.0f, 0.0f, 1.0f};
        bool finished = false, alive_at_end = false, count_hit = false;
        bool need_shadow = false, occluded = false;
        float hx = 0.0f, hy = 0.0f, hz = 0.0f, dist = 0.0f, facing = 0.0f, inv_dist = 0.0f;
        float sd[3] = {0.0f, 0.0f, 0.0f};
        FRay query = ray;
        bool query_active = has;
        float limit = 1e30f;
#pragma unroll 1
        for (int phase = 0; phase < 2; ++phase) {
            float found_t = limit;
            int found = -1;
            scene_query(fs, query, query_active, phase == 1, found_t, found);
            if (phase == 1) {
                occluded = found >= 0;
                break;
            }
            t = found_t;
            surf = found;
            bool from_walk = false;
            if (has && surf < 0 && job.use_bvh) {
                // Missed everything: the reference's BVH walk reports the lowest visited surface.
                const int2 fb = fallback_walk(job.scene, s.o[0], s.o[1], s.o[2], s.d[0], s.d[1], s.d[2]);
                surf = fb.x;
                t = __int_as_float(fb.y);
                from_walk = true;
            }
            if (has) {
                lane_queries += 1;
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
                    if (!from_walk) {
                        winner_normal(job.scene, surf, ray, t, n);
                    } else {
                        n[0] = __ldg(job.scene.normals + 3 * surf);
                        n[1] = __ldg(job.scene.normals + 3 * surf + 1);
                        n[2] = __ldg(job.scene.normals + 3 * surf + 2);
                        if (n[0] * s.d[0] + n[1] * s.d[1] + n[2] * s.d[2] > 0.0f) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
                    }
                    if (job.ray_surfaces) job.ray_surfaces[lane_ray * job.num_bounces + s.bounce] = surf;
                    hx = s.o[0] + t * s.d[0] + 1e-2f * n[0];
                    hy = s.o[1] + t * s.d[1] + 1e-2f * n[1];
                    hz = s.o[2] + t * s.d[2] + 1e-2f * n[2];
                    if (kVisual && s.vslot >= 0) visual_hit(job, s.vslot, s.bounce, hx, hy, hz, surf);
                    const float tsx = job.src[0] - hx, tsy = job.src[1] - hy, tsz = job.src[2] - hz;
                    const float d2 = tsx * tsx + tsy * tsy + tsz * tsz;
                    const float inv = rsqrtf(fmaxf(d2, 1e-30f));
                    dist = d2 * inv;
                    if (dist > job.irradiance_min_distance) {
                        inv_dist = inv;
                        sd[0] = tsx * inv; sd[1] = tsy * inv; sd[2] = tsz * inv;
                        facing = n[0] * sd[0] + n[1] * sd[1] + n[2] * sd[2];
                        need_shadow = facing > 0.0f;
                    }
                }
            }
            // per-surface hit counters: one atomic per distinct (job, surface) in the warp.  The
            // lanes of a warp trace jobs of one scene group of at most 1024 consecutive jobs
            // (surfaces < 2^22), so (job mod 1024, surface) is a 32-bit key -- cheaper to match
            // than a 64-bit one.
            const unsigned counting = __ballot_sync(full, count_hit);
            if (count_hit) {
                // service launches: lanes may hold jobs of any ring slots, so the key is the full slot
                const unsigned same =
                    kService ? __match_any_sync(counting, (static_cast<unsigned long long>(s.job) << 32) |
                                                              static_cast<unsigned>(surf))
                             : __match_any_sync(counting, ((static_cast<unsigned>(s.job) & 1023u) << 22) |
                                                              static_cast<unsigned>(surf));
                if (lane_id == __ffs(same) - 1)
                    atomicAdd(job.hit_counts + surf, static_cast<unsigned long long>(__popc(same)));
            }
            const float h[3] = {hx, hy, hz};
            make_ray(query, h, sd);
            query_active = need_shadow;
            limit = dist - 1e-6f;
        }

        if (has && !finished) {
            const Quad<float> m0 = ldq(job.scene.mats + static_cast<size_t>(surf) * kMatStride);
            const Quad<float> m1 = ldq(job.scene.mats + static_cast<size_t>(surf) * kMatStride + 4);
            const float refl[kBands] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y};
            const float scat = m1.z;
            if (need_shadow) {
                lane_shadows += 1;
                if (!occluded) {
                    const float diffuse = static_cast<float>(1.0 / kPi) * scat * facing;
                    float half[3];
                    normalize3f(sd[0] - s.d[0], sd[1] - s.d[1], sd[2] - s.d[2], half);
                    float cos_half = half[0] * n[0] + half[1] * n[1] + half[2] * n[2];
                    cos_half = cos_half > 0.0f ? cos_half : 0.0f;
                    const float specular = ((job.specular_exponent + 2.0f) * static_cast<float>(1.0 / (8.0 * kPi))) *
                                           (1.0f - scat) * __powf(cos_half, job.specular_exponent);
                    // dist > irradiance_min_distance here, so max(dist, min) = dist
                    const float distance_term = static_cast<float>(1.0 / (4.0 * kPi)) * (inv_dist * inv_dist);
                    const float source_cosine = -(job.fwd[0] * sd[0] + job.fwd[1] * sd[1] + job.fwd[2] * sd[2]);
                    const float gain_base = fabsf((1.0f - job.dipole_weight) + job.dipole_weight * source_cosine);
                    const float source_gain = job.dipole_power == 1.0f ? gain_base : __powf(gain_base, job.dipole_power);
                    // reciprocal multiplies (the float32 path needs no correctly rounded division here)
                    const double rel_delay =
                        (s.path + static_cast<double>(t) + static_cast<double>(dist)) * job.inv_speed_of_sound -
                        job.direct_delay;
                    const double q = floor(rel_delay * job.inv_bin_duration);
                    if (q >= 0.0 && q < static_cast<double>(job.num_bins)) {
                        const int bin = static_cast<int>(q);
                        const float common = job.ray_scale * source_gain * distance_term * (diffuse + specular);
                        long long esum = 0;
                        float energy_sum = 0.0f;
#if AC_WARP_DEPOSIT
                        // lanes depositing into the same (job, bin) add their quanta in the warp first and one of
                        // them issues the two atomics of each band (quanta are non-negative and below 2^62, so
                        // their 16-bit pieces sum exactly in 32 bits)
                        const unsigned dep_mask = __activemask();
                        const unsigned dep_same =
                            kService ? __match_any_sync(dep_mask, (static_cast<unsigned long long>(s.job) << 32) |
                                                                      static_cast<unsigned>(bin))
                                     : __match_any_sync(dep_mask, ((static_cast<unsigned>(s.job) & 1023u) << 21) |
                                                                      static_cast<unsigned>(bin));
                        const bool dep_alone = kAmb || __popc(dep_same) == 1;
                        const bool dep_leader = lane_id == __ffs(dep_same) - 1;
#endif
#pragma unroll
                        for (int b = 0; b < kBands; ++b) {
                            const float e = common * refl[b] * lane_acc[b * kStackStride];
                            if (kVisual) energy_sum += e;
                            const long long qe = quantize(e, job.energy_scale);
#if AC_WARP_DEPOSIT
                            if (dep_alone) {
                                add_fixed(job.echogram_fx + 2 * (static_cast<size_t>(b) * job.num_bins + bin), qe);
                            } else {
                                const unsigned long long uq = static_cast<unsigned long long>(qe);
                                const unsigned l0 = __reduce_add_sync(dep_same, static_cast<unsigned>(uq & 0xFFFFu));
                                const unsigned l1 =
                                    __reduce_add_sync(dep_same, static_cast<unsigned>((uq >> 16) & 0xFFFFu));
                                const unsigned h0 =
                                    __reduce_add_sync(dep_same, static_cast<unsigned>((uq >> 32) & 0xFFFFu));
                                const unsigned h1 = __reduce_add_sync(dep_same, static_cast<unsigned>(uq >> 48));
                                if (dep_leader) {
                                    unsigned long long *w =
                                        job.echogram_fx + 2 * (static_cast<size_t>(b) * job.num_bins + bin);
                                    const unsigned long long lo = static_cast<unsigned long long>(l0) +
                                                                  (static_cast<unsigned long long>(l1) << 16);
                                    const unsigned long long hi = static_cast<unsigned long long>(h0) +
                                                                  (static_cast<unsigned long long>(h1) << 16);
                                    if (lo) atomicAdd(w, lo);
                                    if (hi) atomicAdd(w + 1, hi);
                                }
                            }
#else
                            add_fixed(job.echogram_fx + 2 * (static_cast<size_t>(b) * job.num_bins + bin), qe);
#endif
                            if (kAmb) {
                                const float *d0 = s.d0;
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
                        if (kVisual && s.vslot >= 0)
                            visual_contribution(job, s.vslot, s.bounce, energy_sum,
                                                static_cast<float>(s.path + static_cast<double>(t) +
                                                                   static_cast<double>(dist)));
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kBands; ++b) lane_acc[b * kStackStride] *= refl[b];
            s.path += static_cast<double>(t);
            s.o[0] = hx; s.o[1] = hy; s.o[2] = hz;
            bool use_diffuse;
            int sample;
            if (!kPhilox) {
                const size_t k = static_cast<size_t>(s.bounce) * job.num_rays + lane_ray;
                use_diffuse = job.diffuse_random[k] < scat;
                sample = use_diffuse ? job.diffuse_indices[k] : 0;
            } else {
                const u32x4 rr = trace_draw(job.seed, job.stream_key, static_cast<uint32_t>(lane_ray),
                                            static_cast<uint32_t>(s.bounce) + 1u);
                use_diffuse = u01_53(rr.x, rr.y) < static_cast<double>(scat);
                sample = static_cast<int>(below(rr.z, static_cast<uint32_t>(job.num_bank)));
            }
            if (use_diffuse) {
                const float *bs = job.diffuse_bank + 3 * sample;
                diffuse_direction_f(__ldg(bs), __ldg(bs + 1), __ldg(bs + 2), n[0], n[1], n[2], s.d);
            } else {
                const float dot = s.d[0] * n[0] + s.d[1] * n[1] + s.d[2] * n[2];
                normalize3f(s.d[0] - 2.0f * dot * n[0], s.d[1] - 2.0f * dot * n[1], s.d[2] - 2.0f * dot * n[2], s.d);
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
            const unsigned q_sum = __reduce_add_sync(grp, static_cast<unsigned>(lane_queries));
            const unsigned q_max = __reduce_max_sync(grp, static_cast<unsigned>(lane_queries));
            const unsigned sh_sum = __reduce_add_sync(grp, static_cast<unsigned>(lane_shadows));
            const unsigned alive_sum = __reduce_add_sync(grp, alive_at_end ? 1u : 0u);
            if (lane_id == __ffs(grp) - 1) {
                atomicMax(job.counters + 0, static_cast<unsigned long long>(q_max));
                if (alive_sum) atomicAdd(job.counters + 1, static_cast<unsigned long long>(alive_sum));
                atomicAdd(job.counters + 2, static_cast<unsigned long long>(q_sum));
                if (sh_sum) atomicAdd(job.counters + 3, static_cast<unsigned long long>(sh_sum));
            }
            if (job.ray_surfaces)
                for (int b = s.bounce; b < job.num_bounces; ++b) job.ray_surfaces[lane_ray * job.num_bounces + b] = -1;
            has = false;
        }
        if (kService) {
            // The warp counts its finished rays per job and adds them to the job's count once it holds no
            // more of that job's rays (or a ray of another job finishes first): one fence per run of a job
            // through the warp instead of one per iteration in which a ray ends.
            int cs = count_slot;
            unsigned long long cn = count_n;
            unsigned rest = ending;
            while (rest) {
                const int j = __shfl_sync(full, s.job, __ffs(rest) - 1);
                const unsigned grp = __ballot_sync(full, finished && s.job == j);
                rest &= ~grp;
                if (j != cs) {
                    if (cn && service_count(table, cs, cn, lane_id)) service_finish(table, cs, lane_id);
                    cs = j;
                    cn = 0;
                }
                cn += static_cast<unsigned long long>(__popc(grp));
            }
            if (cn && !__any_sync(full, has && s.job == cs) && !(cur_slot == cs && ww.next < ww.end)) {
                if (service_count(table, cs, cn, lane_id)) service_finish(table, cs, lane_id);
                cs = -1;
                cn = 0;
            }
            __syncwarp();   // every lane has read the old values
            count_slot = cs;
            count_n = cn;
        }
    }
    if (kService) {
        const int cs = count_slot;
        const unsigned long long cn = count_n;
        if (cn && service_count(table, cs, cn, lane_id)) service_finish(table, cs, lane_id);
    }
}

}  // namespace ac
