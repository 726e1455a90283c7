// Six-band listener-space path tracer for sm_100a.
//
// One template serves both precisions:
//   T = float   production path (compiled with FMA contraction, like any FP32 CUDA code)
//   T = double  parity path, compiled with -fmad=false so every multiply and add
//               rounds separately, as in the reference's Numba float64 tracer.
//
// Algorithm (per ray, per bounce) follows acoustic_agent/steam_rt.py:4708-4850;
// intersection routines follow steam_rt.py:4258-4583.  What differs is the
// execution model:
//   * persistent blocks; each lane pulls a new ray the moment its ray ends
//     (warp-aggregated atomic on a work counter), so lanes never idle while
//     the warp's other rays finish;
//   * many jobs (scene, source, listener, outputs) may share one launch; a
//     lane maps its global ray index to (job, ray) through a prefix table;
//   * the echogram is accumulated as exact fixed point (energy * 2^s rounded
//     per deposit to int64, summed as two 32-bit halves), so the result is
//     bit-identical for any schedule;
//   * per-surface hit counters are aggregated per warp (match_any) before
//     the atomic, removing the same-address contention of one atomic per
//     bounce per ray;
//   * the shadow ray is an any-hit query that stops at the first blocker
//     closer than the source: the reference's "closest hit, then compare
//     with the source distance" gives the same boolean.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "philox.cuh"

namespace ac {

constexpr int kBands = 6;
constexpr double kPi = 3.141592653589793;

// Per-surface record: three quads (12 values of T).
//  wall       : {ax, ay, sx, sy} {z0, z1, nx, ny} {nz, 0, 0, tag}
//  horizontal : {z, nx, ny, nz}  {0, 0, 0, 0}     {0, 0, 0, tag}
//  box        : {cx, cy, ux, uy} {vx, vy, hw, hd} {z0, z1, 0, tag}
// tag = surface_index * 4 + kind.  For float the tag is stored as int bits.
constexpr int kPrimStride = 12;
// BVH node: {lo.x, lo.y, lo.z, escape} {hi.x, hi.y, hi.z, start + (count << 24)}
constexpr int kNodeStride = 8;
// Material row: {r0, r1, r2, r3} {r4, r5, scattering, 0}
constexpr int kMatStride = 8;

template <typename T>
struct Quad {
    T x, y, z, w;
};

__device__ __forceinline__ Quad<float> ldq(const float *p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Quad<double> ldq(const double *p) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return {a.x, a.y, b.x, b.y};
}

__host__ __device__ __forceinline__ int tag_bits(float v) {
#ifdef __CUDA_ARCH__
    return __float_as_int(v);
#else
    int i;
    __builtin_memcpy(&i, &v, sizeof(i));
    return i;
#endif
}
__host__ __device__ __forceinline__ int tag_bits(double v) { return static_cast<int>(v); }

template <typename T>
struct Consts;
template <>
struct Consts<float> {
    // steam_rt_cuda.py:21 and :397 (FP32 epsilons of the reference CUDA backend)
    static constexpr float bvh_eps = 1e-5f;
    static constexpr float axis_eps = 1e-12f;
};
template <>
struct Consts<double> {
    // steam_rt.py:44 and :4412 (Numba float64)
    static constexpr double bvh_eps = 2.0e-6;
    static constexpr double axis_eps = 1e-15;
};

template <typename T>
struct SceneDev {
    const T *prims_linear;  // [S][12] surface order
    const T *prims_leaf;    // [P][12] BVH leaf-slot order
    const T *nodes;         // [N][8]
    const T *mats;          // [S][8]
    const T *corners;       // [C][2]
    const T *normals;       // [S][3]
    int32_t num_surfaces;
    int32_t num_nodes;
    int32_t num_corners;
    int32_t num_leaf_prims;
};

template <typename T>
struct Job {
    SceneDev<T> scene;
    T src[3];
    T lst[3];
    T fwd[3];
    T listener_radius;
    T source_radius;
    T irradiance_min_distance;
    T specular_exponent;
    T dipole_weight;
    T dipole_power;
    T ray_scale;        // 4*pi / num_rays
    T source_distance;  // |listener - source|
    double speed_of_sound;
    double direct_delay;
    double bin_duration;
    double max_path_length;
    double energy_scale;
    double inv_speed_of_sound;
    double inv_bin_duration;
    int64_t num_rays;
    int64_t ray_begin;  // first global work index of this job
    int32_t num_bounces;
    int32_t num_bins;
    int32_t use_bvh;
    int32_t render_ambisonics;
    int32_t rng_mode;
    int32_t num_bank;
    uint64_t seed;
    uint64_t stream_key;
    const T *directions;           // [R,3]  reference stream
    const T *diffuse_random;       // [B,R]
    const int32_t *diffuse_indices;// [B,R]
    const T *diffuse_bank;         // [K,3]
    unsigned long long *echogram_fx;   // [6,bins,2] fixed point (sum of low halves, sum of high halves)
    unsigned long long *ambisonic_fx;  // [6,4,bins,2] or null
    unsigned long long *hit_counts;    // [S]
    unsigned long long *contrib_counts;// [S]
    unsigned long long *surface_energy_fx; // [S,2]
    unsigned long long *counters;      // [8]
    int32_t *ray_surfaces;             // [R,B] or null
    // visual-path candidates (steam_rt.py:4718-4731): slot = ray / stride for rays with ray % stride == 0
    int32_t visual_limit;              // 0: none
    int32_t visual_stride;
    T *visual_hit_points;              // [L,B,3]
    int32_t *visual_surfaces;          // [L,B]
    int32_t *visual_rays;              // [L]
    int32_t *visual_orders;            // [L]
    T *visual_distances;               // [L]
    T *visual_gains;                   // [L]
};

// Visual slot of a ray, -1 for none (steam_rt.py:4726-4731).
template <typename T>
__device__ __forceinline__ int visual_slot(const Job<T> &job, int64_t ray) {
    if (job.visual_limit <= 0 || ray % job.visual_stride != 0) return -1;
    const int64_t slot = ray / job.visual_stride;
    return slot < job.visual_limit ? static_cast<int>(slot) : -1;
}

// A hit of a candidate ray (steam_rt.py:4765-4769).
template <typename T>
__device__ __forceinline__ void visual_hit(const Job<T> &job, int slot, int bounce, T hx, T hy, T hz, int surf) {
    const size_t k = static_cast<size_t>(slot) * job.num_bounces + bounce;
    job.visual_hit_points[3 * k] = hx;
    job.visual_hit_points[3 * k + 1] = hy;
    job.visual_hit_points[3 * k + 2] = hz;
    job.visual_surfaces[k] = surf;
}

// The strongest contribution of a candidate ray so far (steam_rt.py:4821-4824).
template <typename T>
__device__ __forceinline__ void visual_contribution(const Job<T> &job, int slot, int bounce, T energy_sum,
                                                    T distance) {
    const T g = job.visual_gains[slot];
    if (energy_sum > g * g) {
        job.visual_orders[slot] = bounce + 1;
        job.visual_distances[slot] = distance;
        job.visual_gains[slot] = sqrt(energy_sum > T(0) ? energy_sum : T(0));
    }
}

// ---------------------------------------------------------------------------
// Intersection routines (steam_rt.py:4259-4426)

template <typename T>
__device__ __forceinline__ bool point_in_polygon(T x, T y, const T *corners, int n) {
    bool inside = false;
    int j = n - 1;
    for (int i = 0; i < n; ++i) {
        const T xi = __ldg(corners + 2 * i), yi = __ldg(corners + 2 * i + 1);
        const T xj = __ldg(corners + 2 * j), yj = __ldg(corners + 2 * j + 1);
        if ((yi > y) != (yj > y)) {
            const T denom = yj - yi;
            if (fabs(denom) > T(1e-12)) {
                const T x_cross = (xj - xi) * (y - yi) / denom + xi;
                if (x < x_cross) inside = !inside;
            }
        }
        j = i;
    }
    return inside;
}

// steam_rt.py:4277-4358: oriented box slab test in the box frame.
template <typename T>
__device__ __forceinline__ T box_hit(const Quad<T> &A, const Quad<T> &B, const Quad<T> &C, const T *o, const T *d,
                                     T *n) {
    const T relx = o[0] - A.x;
    const T rely = o[1] - A.y;
    const T ox = relx * A.z + rely * A.w;
    const T oy = relx * B.x + rely * B.y;
    const T oz = o[2];
    const T dx = d[0] * A.z + d[1] * A.w;
    const T dy = d[0] * B.x + d[1] * B.y;
    const T dz = d[2];
    T t_min = T(-1.0e30), t_max = T(1.0e30);
    T nx = 0, ny = 0, nz = 0, ex = 0, ey = 0, ez = 0;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        T oo, dd, lo, hi, ax, ay, az;
        if (axis == 0) { oo = ox; dd = dx; lo = -B.z; hi = B.z; ax = A.z; ay = A.w; az = T(0); }
        else if (axis == 1) { oo = oy; dd = dy; lo = -B.w; hi = B.w; ax = B.x; ay = B.y; az = T(0); }
        else { oo = oz; dd = dz; lo = C.x; hi = C.y; ax = T(0); ay = T(0); az = T(1); }
        if (fabs(dd) <= T(1.0e-12)) {
            if (oo < lo || oo > hi) return T(1.0e30);
            continue;
        }
        T enter, exit_, enx, eny, enz, oux, ouy, ouz;
        if (dd > T(0)) {
            enter = (lo - oo) / dd; exit_ = (hi - oo) / dd;
            enx = -ax; eny = -ay; enz = -az; oux = ax; ouy = ay; ouz = az;
        } else {
            enter = (hi - oo) / dd; exit_ = (lo - oo) / dd;
            enx = ax; eny = ay; enz = az; oux = -ax; ouy = -ay; ouz = -az;
        }
        if (enter > t_min) { t_min = enter; nx = enx; ny = eny; nz = enz; }
        if (exit_ < t_max) { t_max = exit_; ex = oux; ey = ouy; ez = ouz; }
        if (t_min > t_max) return T(1.0e30);
    }
    if (t_max <= T(1e-6)) return T(1.0e30);
    if (t_min > T(1e-6)) { n[0] = nx; n[1] = ny; n[2] = nz; return t_min; }
    n[0] = ex; n[1] = ey; n[2] = ez;
    return t_max;
}

// steam_rt.py:4361-4392.  Returns t (1e30 = miss); writes the hit normal
// (the surface normal for walls and polygons, the slab normal for boxes).
template <typename T>
__device__ __forceinline__ T surface_hit(const T *rec, int kind, const T *o, const T *d, const T *corners,
                                         int num_corners, T *n) {
    T t = T(1e30);
    if (kind == 0) {
        const Quad<T> A = ldq(rec), B = ldq(rec + 4);
        const T nz = __ldg(rec + 8);
        n[0] = B.z; n[1] = B.w; n[2] = nz;
        const T sx = A.z, sy = A.w;
        const T det = sx * d[1] - sy * d[0];
        if (fabs(det) > T(1e-12)) {
            const T relx = o[0] - A.x;
            const T rely = o[1] - A.y;
            const T cand = (relx * sy - rely * sx) / det;
            const T u = (relx * d[1] - rely * d[0]) / det;
            const T z = o[2] + cand * d[2];
            if (cand > T(1e-6) && u >= T(-1e-6) && u <= T(1.0 + 1e-6) && z >= B.x - T(1e-6) && z <= B.y + T(1e-6))
                t = cand;
        }
    } else if (kind == 2) {
        const Quad<T> A = ldq(rec), B = ldq(rec + 4), C = ldq(rec + 8);
        T bn[3];
        const T cand = box_hit(A, B, C, o, d, bn);
        if (cand > T(1e-6) && cand < T(1.0e29)) {
            t = cand;
            n[0] = bn[0]; n[1] = bn[1]; n[2] = bn[2];
        } else {
            n[0] = T(0); n[1] = T(0); n[2] = T(1);
        }
    } else {
        const Quad<T> A = ldq(rec);
        n[0] = A.y; n[1] = A.z; n[2] = A.w;
        if (fabs(d[2]) > T(1e-12)) {
            const T cand = (A.x - o[2]) / d[2];
            const T px = o[0] + cand * d[0];
            const T py = o[1] + cand * d[1];
            if (cand > T(1e-6) && point_in_polygon(px, py, corners, num_corners)) t = cand;
        }
    }
    return t;
}

// steam_rt.py:4406-4426
template <typename T>
__device__ __forceinline__ bool ray_aabb(const T *o, const T *d, const Quad<T> &lo, const Quad<T> &hi, T max_distance) {
    T enter = T(0);
    T exit_ = max_distance + Consts<T>::bvh_eps;
    const T los[3] = {lo.x, lo.y, lo.z}, his[3] = {hi.x, hi.y, hi.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const T v = d[a];
        if (fabs(v) <= Consts<T>::axis_eps) {
            if (o[a] < los[a] || o[a] > his[a]) return false;
            continue;
        }
        T first = (los[a] - o[a]) / v;
        T second = (his[a] - o[a]) / v;
        if (first > second) { const T tmp = first; first = second; second = tmp; }
        if (first > enter) enter = first;
        if (second < exit_) exit_ = second;
        if (enter > exit_) return false;
    }
    return exit_ > T(1e-6);
}

template <typename T>
__device__ __forceinline__ int rec_tag(const T *rec) { return tag_bits(__ldg(rec + 11)); }

// Closest hit: steam_rt.py:4429-4478 (linear) and :4481-4506 (escape-link walk).
// The BVH walk keeps the reference's tie rule, including its side effect that a
// ray missing every visited surface returns the lowest visited index with t=1e30.
template <typename T>
__device__ __forceinline__ int closest_hit(const SceneDev<T> &sc, bool use_bvh, const T *o, const T *d, T &t_out,
                                           T *n_out) {
    T best_t = T(1e30);
    int best = -1;
    T bn[3] = {T(0), T(0), T(0)};
    T n[3];
    if (use_bvh) {
        int node = 0;
        while (node < sc.num_nodes) {
            const T *np = sc.nodes + static_cast<size_t>(node) * kNodeStride;
            const Quad<T> lo = ldq(np), hi = ldq(np + 4);
            if (!ray_aabb(o, d, lo, hi, best_t)) {
                node = tag_bits(lo.w);
                continue;
            }
            const int sc_bits = tag_bits(hi.w);
            const int count = static_cast<int>(static_cast<unsigned>(sc_bits) >> 24);
            if (count > 0) {
                const int start = sc_bits & 0xFFFFFF;
                for (int k = 0; k < count; ++k) {
                    const T *rec = sc.prims_leaf + static_cast<size_t>(start + k) * kPrimStride;
                    const int tag = rec_tag(rec);
                    const int si = tag >> 2;
                    const T t = surface_hit(rec, tag & 3, o, d, sc.corners, sc.num_corners, n);
                    if (t < best_t || (t == best_t && (best < 0 || si < best))) {
                        best_t = t; best = si; bn[0] = n[0]; bn[1] = n[1]; bn[2] = n[2];
                    }
                }
            }
            ++node;
        }
        if (best >= 0 && best_t == T(1e30)) {
            bn[0] = __ldg(sc.normals + 3 * best);
            bn[1] = __ldg(sc.normals + 3 * best + 1);
            bn[2] = __ldg(sc.normals + 3 * best + 2);
        }
    } else {
        for (int si = 0; si < sc.num_surfaces; ++si) {
            const T *rec = sc.prims_linear + static_cast<size_t>(si) * kPrimStride;
            const T t = surface_hit(rec, rec_tag(rec) & 3, o, d, sc.corners, sc.num_corners, n);
            if (t < best_t) { best_t = t; best = si; bn[0] = n[0]; bn[1] = n[1]; bn[2] = n[2]; }
        }
    }
    if (best >= 0) {
        const T dot = bn[0] * d[0] + bn[1] * d[1] + bn[2] * d[2];
        if (dot > T(0)) { bn[0] = -bn[0]; bn[1] = -bn[1]; bn[2] = -bn[2]; }
    }
    t_out = best_t;
    n_out[0] = bn[0]; n_out[1] = bn[1]; n_out[2] = bn[2];
    return best;
}

// Shadow query: is any surface hit strictly closer than max_t?  Equivalent to the
// reference's `closest t < distance - EPS` test (steam_rt.py:4794).
template <typename T>
__device__ __forceinline__ bool any_hit(const SceneDev<T> &sc, bool use_bvh, const T *o, const T *d, T max_t) {
    T n[3];
    if (use_bvh) {
        int node = 0;
        while (node < sc.num_nodes) {
            const T *np = sc.nodes + static_cast<size_t>(node) * kNodeStride;
            const Quad<T> lo = ldq(np), hi = ldq(np + 4);
            if (!ray_aabb(o, d, lo, hi, max_t)) {
                node = tag_bits(lo.w);
                continue;
            }
            const int sc_bits = tag_bits(hi.w);
            const int count = static_cast<int>(static_cast<unsigned>(sc_bits) >> 24);
            if (count > 0) {
                const int start = sc_bits & 0xFFFFFF;
                for (int k = 0; k < count; ++k) {
                    const T *rec = sc.prims_leaf + static_cast<size_t>(start + k) * kPrimStride;
                    const T t = surface_hit(rec, rec_tag(rec) & 3, o, d, sc.corners, sc.num_corners, n);
                    if (t < max_t) return true;
                }
            }
            ++node;
        }
        return false;
    }
    for (int si = 0; si < sc.num_surfaces; ++si) {
        const T *rec = sc.prims_linear + static_cast<size_t>(si) * kPrimStride;
        const T t = surface_hit(rec, rec_tag(rec) & 3, o, d, sc.corners, sc.num_corners, n);
        if (t < max_t) return true;
    }
    return false;
}

template <typename T>
__device__ __forceinline__ bool sphere_before(const T *o, const T *d, const T *c, T radius, T max_distance) {
    const T ox = o[0] - c[0], oy = o[1] - c[1], oz = o[2] - c[2];
    const T b = ox * d[0] + oy * d[1] + oz * d[2];
    const T cc = ox * ox + oy * oy + oz * oz - radius * radius;
    const T disc = b * b - cc;
    if (disc < T(0)) return false;
    const T root = -b - sqrt(disc > T(0) ? disc : T(0));
    return root >= T(0) && root < max_distance;
}

template <typename T>
__device__ __forceinline__ void normalize3(T x, T y, T z, T *out) {
    const T n = sqrt(x * x + y * y + z * z);
    if (n <= T(1e-12)) { out[0] = T(0); out[1] = T(0); out[2] = T(0); return; }
    out[0] = x / n; out[1] = y / n; out[2] = z / n;
}

// steam_rt.py:4564-4582: cosine-bank sample rotated into the hemisphere of n.
template <typename T>
__device__ __forceinline__ void diffuse_direction(T s0, T s1, T s2, T nx, T ny, T nz, T *out) {
    T hx = T(1), hy = T(0), hz = T(0);
    if (fabs(nx) >= T(0.9)) { hx = T(0); hy = T(1); }
    T t[3];
    normalize3(hy * nz - hz * ny, hz * nx - hx * nz, hx * ny - hy * nx, t);
    const T bx = ny * t[2] - nz * t[1];
    const T by = nz * t[0] - nx * t[2];
    const T bz = nx * t[1] - ny * t[0];
    normalize3(s0 * t[0] + s1 * bx + s2 * nx, s0 * t[1] + s1 * by + s2 * ny, s0 * t[2] + s1 * bz + s2 * nz, out);
}

template <typename T>
__device__ __forceinline__ T t_pow(T x, T y);
template <>
__device__ __forceinline__ float t_pow<float>(float x, float y) { return powf(x, y); }
template <>
__device__ __forceinline__ double t_pow<double>(double x, double y) { return pow(x, y); }

__device__ __forceinline__ long long quantize(float e, double scale) { return __double2ll_rn(static_cast<double>(e) * scale); }
__device__ __forceinline__ long long quantize(double e, double scale) { return __double2ll_rn(e * scale); }

// Exact fixed-point accumulation without returning atomics.  A signed 64-bit
// quantum q is split into its low 32 bits (unsigned, < 2^32) and its high part
// (q >> 32, signed); acc[0] sums the low parts and acc[1] the high parts, both
// with fire-and-forget reductions.  The accumulated value is
// acc[1] * 2^32 + acc[0], exact and independent of the order of the additions
// as long as fewer than 2^32 quanta reach one accumulator (the launcher
// requires num_rays * num_bounces < 2^32).
__device__ __forceinline__ void add_fixed(unsigned long long *acc, long long q) {
    if (q == 0) return;
    const unsigned long long lo = static_cast<unsigned long long>(q) & 0xFFFFFFFFull;
    const long long hi = q >> 32;
    if (lo) atomicAdd(acc, lo);
    if (hi) atomicAdd(acc + 1, static_cast<unsigned long long>(hi));
}

// Jittered Fibonacci-sphere direction of ray `ri` drawn from the counter-based
// stream (steam_rt.py:3959-3968 layout, jitter from Philox).  The angle is kept
// in turns and reduced before sincospi, so no large-argument trigonometry runs;
// explicitly rounded operations keep the result independent of FMA contraction.
static __device__ __noinline__ double3 philox_direction(uint64_t seed, uint64_t key, int64_t num_rays, int64_t ri) {
    const u32x4 r = trace_draw(seed, key, static_cast<uint32_t>(ri), 0u);
    // jitter U(-0.02, 0.02) rad, expressed in turns
    const double jitter = __dmul_rn(__dadd_rn(-0.02, __dmul_rn(0.04, u01_53(r.x, r.y))), kInvTwoPi);
    const double i = static_cast<double>(ri) + 0.5;
    const double z = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(2.0, i), static_cast<double>(num_rays)));
    double rr = __dsub_rn(1.0, __dmul_rn(z, z));
    rr = __dsqrt_rn(rr < 0.0 ? 0.0 : (rr > 1.0 ? 1.0 : rr));
    const double turns = __dadd_rn(__dmul_rn(i, kGoldenTurns), jitter);
    const double frac = __dsub_rn(turns, floor(turns));
    double s, c;
    sincospi(__dmul_rn(2.0, frac), &s, &c);
    return make_double3(__dmul_rn(c, rr), __dmul_rn(s, rr), z);
}

// Initial direction of ray `ri` of a job.
template <typename T>
__device__ __forceinline__ void initial_direction(const Job<T> &job, int64_t ri, T *d) {
    if (job.rng_mode == 0) {
        d[0] = job.directions[3 * ri];
        d[1] = job.directions[3 * ri + 1];
        d[2] = job.directions[3 * ri + 2];
        return;
    }
    const double3 v = philox_direction(job.seed, job.stream_key, job.num_rays, ri);
    d[0] = static_cast<T>(v.x);
    d[1] = static_cast<T>(v.y);
    d[2] = static_cast<T>(v.z);
}

// ---------------------------------------------------------------------------
// Work distribution

struct BatchTable {
    const void *jobs;          // Job<T>[num_jobs]
    const int64_t *ray_begin;  // [num_jobs + 1] prefix of num_rays
    int32_t num_jobs;
    int32_t pad;
    int64_t total_rays;
    unsigned long long *work_counter;
};

__device__ __forceinline__ int find_job(const int64_t *prefix, int num_jobs, int64_t g) {
    int lo = 0, hi = num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Warp-cooperative add of `value` into counter[key] for lanes in `mask` with
// equal keys: one atomic per distinct key.
__device__ __forceinline__ void warp_count(unsigned mask, unsigned long long key, unsigned value,
                                           unsigned long long *target) {
    const unsigned group = __match_any_sync(mask, key);
    const unsigned total = __reduce_add_sync(group, value);
    const int leader = __ffs(group) - 1;
    if ((threadIdx.x & 31) == leader) atomicAdd(target, static_cast<unsigned long long>(total));
}

template <typename T>
struct Lane {
    T o[3];
    T d[3];
    T d0[3];
    T acc[kBands];
    double path;
    int64_t ray;
    int job;
    int bounce;
    int queries;
    int shadows;
    int vslot;   // visual-candidate slot, -1 for none
};

template <typename T, bool kSingle>
__global__ void __launch_bounds__(256) trace_kernel(const __grid_constant__ Job<T> single,
                                                    const __grid_constant__ BatchTable table) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane_id = threadIdx.x & 31;
    const unsigned lanes_below = (1u << lane_id) - 1u;
    unsigned long long *work_counter = kSingle ? single.counters + 4 : table.work_counter;
    const int64_t total = kSingle ? single.num_rays : table.total_rays;
    const Job<T> *jobs = static_cast<const Job<T> *>(table.jobs);

    Lane<T> s;
    bool has = false;
    bool drained = false;
    s.job = 0;

    while (true) {
        // Refill: every lane without a ray takes the next global index.
        const unsigned need = __ballot_sync(full, !has && !drained);
        if (need) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane_id == leader) base = atomicAdd(work_counter, static_cast<unsigned long long>(__popc(need)));
            base = __shfl_sync(full, base, leader);
            if (!has && !drained) {
                const int64_t g = static_cast<int64_t>(base) + __popc(need & lanes_below);
                if (g < total) {
                    int j = 0;
                    int64_t ri = g;
                    if (!kSingle) {
                        j = find_job(table.ray_begin, table.num_jobs, g);
                        ri = g - __ldg(table.ray_begin + j);
                    }
                    const Job<T> &job = kSingle ? single : jobs[j];
                    s.job = j;
                    s.ray = ri;
                    s.bounce = 0;
                    s.queries = 0;
                    s.shadows = 0;
                    s.path = 0.0;
                    s.vslot = visual_slot(job, ri);
                    if (s.vslot >= 0) job.visual_rays[s.vslot] = static_cast<int32_t>(ri);
                    s.o[0] = job.lst[0]; s.o[1] = job.lst[1]; s.o[2] = job.lst[2];
                    initial_direction(job, ri, s.d);
                    s.d0[0] = s.d[0]; s.d0[1] = s.d[1]; s.d0[2] = s.d[2];
#pragma unroll
                    for (int b = 0; b < kBands; ++b) s.acc[b] = T(1);
                    has = job.num_bounces > 0;
                    if (!has) {
                        // zero-bounce job: the ray is alive by definition (loop never runs)
                        atomicAdd(job.counters + 1, 1ull);
                    }
                } else {
                    drained = true;
                }
            }
        }
        if (!__any_sync(full, has)) {
            if (__all_sync(full, drained || has)) break;
            continue;
        }

        int count_surface = -1;   // surface to count as hit this iteration
        bool finished = false;
        bool alive_at_end = false;
        if (has) {
            const Job<T> &job = kSingle ? single : jobs[s.job];
            const SceneDev<T> &sc = job.scene;
            const bool bvh = job.use_bvh != 0;
            T t, n[3];
            const int surf = closest_hit(sc, bvh, s.o, s.d, t, n);
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
                count_surface = surf;
                if (job.ray_surfaces)
                    job.ray_surfaces[s.ray * job.num_bounces + s.bounce] = surf;
                const T hx = s.o[0] + t * s.d[0] + T(1e-2) * n[0];
                const T hy = s.o[1] + t * s.d[1] + T(1e-2) * n[1];
                const T hz = s.o[2] + t * s.d[2] + T(1e-2) * n[2];
                if (s.vslot >= 0) visual_hit(job, s.vslot, s.bounce, hx, hy, hz, surf);
                const T tsx = job.src[0] - hx, tsy = job.src[1] - hy, tsz = job.src[2] - hz;
                const T dist = sqrt(tsx * tsx + tsy * tsy + tsz * tsz);
                const Quad<T> m0 = ldq(sc.mats + static_cast<size_t>(surf) * kMatStride);
                const Quad<T> m1 = ldq(sc.mats + static_cast<size_t>(surf) * kMatStride + 4);
                const T refl[kBands] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y};
                const T scat = m1.z;
                if (dist > job.irradiance_min_distance) {
                    const T sd[3] = {tsx / dist, tsy / dist, tsz / dist};
                    const T facing = n[0] * sd[0] + n[1] * sd[1] + n[2] * sd[2];
                    if (facing > T(0)) {
                        const T h[3] = {hx, hy, hz};
                        s.shadows += 1;
                        const bool occluded = any_hit(sc, bvh, h, sd, dist - T(1e-6));
                        if (!occluded) {
                            const T diffuse = T(1.0 / kPi) * scat * facing;
                            T half[3];
                            normalize3(sd[0] - s.d[0], sd[1] - s.d[1], sd[2] - s.d[2], half);
                            T cos_half = half[0] * n[0] + half[1] * n[1] + half[2] * n[2];
                            cos_half = cos_half > T(0) ? cos_half : T(0);
                            const T specular = ((job.specular_exponent + T(2.0)) / T(8.0 * kPi)) * (T(1.0) - scat) *
                                               t_pow(cos_half, job.specular_exponent);
                            const T dmax = dist > job.irradiance_min_distance ? dist : job.irradiance_min_distance;
                            const T inv = T(1.0) / dmax;
                            const T distance_term = T(1.0 / (4.0 * kPi)) * (inv * inv);
                            const T source_cosine = -(job.fwd[0] * sd[0] + job.fwd[1] * sd[1] + job.fwd[2] * sd[2]);
                            const T source_gain =
                                t_pow(fabs((T(1.0) - job.dipole_weight) + job.dipole_weight * source_cosine),
                                      job.dipole_power);
                            const double rel_delay =
                                (s.path + static_cast<double>(t) + static_cast<double>(dist)) / job.speed_of_sound -
                                job.direct_delay;
                            const double q = floor(rel_delay / job.bin_duration);
                            if (q >= 0.0 && q < static_cast<double>(job.num_bins)) {
                                const int bin = static_cast<int>(q);
                                const T common = job.ray_scale * source_gain * distance_term * (diffuse + specular);
                                long long esum = 0;
                                T energy_sum = T(0);
#pragma unroll
                                for (int b = 0; b < kBands; ++b) {
                                    const T e = common * refl[b] * s.acc[b];
                                    energy_sum += e;
                                    const long long qe = quantize(e, job.energy_scale);
                                    add_fixed(job.echogram_fx + 2 * (static_cast<size_t>(b) * job.num_bins + bin), qe);
                                    if (job.ambisonic_fx) {
                                        unsigned long long *a =
                                            job.ambisonic_fx + 2 * (static_cast<size_t>(b) * 4 * job.num_bins + bin);
                                        const size_t stride = 2 * static_cast<size_t>(job.num_bins);
                                        add_fixed(a, qe);
                                        add_fixed(a + stride, quantize(e * s.d0[0], job.energy_scale));
                                        add_fixed(a + 2 * stride, quantize(e * s.d0[1], job.energy_scale));
                                        add_fixed(a + 3 * stride, quantize(e * s.d0[2], job.energy_scale));
                                    }
                                    esum += qe;
                                }
                                atomicAdd(job.contrib_counts + surf, 1ull);
                                add_fixed(job.surface_energy_fx + 2 * static_cast<size_t>(surf), esum);
                                if (s.vslot >= 0)
                                    visual_contribution(job, s.vslot, s.bounce, energy_sum,
                                                        static_cast<T>((s.path + static_cast<double>(t)) +
                                                                       static_cast<double>(dist)));
                            }
                        }
                    }
                }
#pragma unroll
                for (int b = 0; b < kBands; ++b) s.acc[b] *= refl[b];
                s.path += static_cast<double>(t);
                s.o[0] = hx; s.o[1] = hy; s.o[2] = hz;
                // Diffuse vs specular continuation (steam_rt.py:4835-4845).
                bool use_diffuse;
                int sample;
                if (job.rng_mode == 0) {
                    const size_t k = static_cast<size_t>(s.bounce) * job.num_rays + s.ray;
                    use_diffuse = job.diffuse_random[k] < scat;
                    sample = use_diffuse ? job.diffuse_indices[k] : 0;
                } else {
                    const u32x4 r = trace_draw(job.seed, job.stream_key, static_cast<uint32_t>(s.ray),
                                               static_cast<uint32_t>(s.bounce) + 1u);
                    use_diffuse = u01_53(r.x, r.y) < static_cast<double>(scat);
                    sample = static_cast<int>(below(r.z, static_cast<uint32_t>(job.num_bank)));
                }
                if (use_diffuse) {
                    const T *bs = job.diffuse_bank + 3 * sample;
                    diffuse_direction(__ldg(bs), __ldg(bs + 1), __ldg(bs + 2), n[0], n[1], n[2], s.d);
                } else {
                    const T dot = s.d[0] * n[0] + s.d[1] * n[1] + s.d[2] * n[2];
                    normalize3(s.d[0] - T(2.0) * dot * n[0], s.d[1] - T(2.0) * dot * n[1],
                               s.d[2] - T(2.0) * dot * n[2], s.d);
                }
                s.bounce += 1;
                if (s.path > job.max_path_length) {
                    finished = true;
                } else if (s.bounce >= job.num_bounces) {
                    finished = true;
                    alive_at_end = true;
                }
            }
        }

        // Per-surface hit counters, one atomic per (job, surface) per warp.
        const unsigned counting = __ballot_sync(full, count_surface >= 0);
        if (count_surface >= 0) {
            const Job<T> &job = kSingle ? single : jobs[s.job];
            warp_count(counting, (static_cast<unsigned long long>(s.job) << 32) | static_cast<unsigned>(count_surface),
                       1u, job.hit_counts + count_surface);
        }
        // Ray completion: bounce statistics per job.
        const unsigned ending = __ballot_sync(full, finished);
        if (finished) {
            const Job<T> &job = kSingle ? single : jobs[s.job];
            const unsigned group = __match_any_sync(ending, static_cast<unsigned>(s.job));
            const unsigned q_sum = __reduce_add_sync(group, static_cast<unsigned>(s.queries));
            const unsigned q_max = __reduce_max_sync(group, static_cast<unsigned>(s.queries));
            const unsigned sh_sum = __reduce_add_sync(group, static_cast<unsigned>(s.shadows));
            const unsigned alive_sum = __reduce_add_sync(group, alive_at_end ? 1u : 0u);
            if (lane_id == __ffs(group) - 1) {
                atomicMax(job.counters + 0, static_cast<unsigned long long>(q_max));
                if (alive_sum) atomicAdd(job.counters + 1, static_cast<unsigned long long>(alive_sum));
                atomicAdd(job.counters + 2, static_cast<unsigned long long>(q_sum));
                if (sh_sum) atomicAdd(job.counters + 3, static_cast<unsigned long long>(sh_sum));
            }
            if (job.ray_surfaces) {
                // bounces never reached read -1, like the reference's visual-path slots
                for (int b = s.bounce; b < job.num_bounces; ++b) job.ray_surfaces[s.ray * job.num_bounces + b] = -1;
            }
            has = false;
        }
    }
}

}  // namespace ac
