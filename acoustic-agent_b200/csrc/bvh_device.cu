// GPU build of the reference's BVH (acoustic_agent/bvh.py:8-77, build_bvh).
//
// The reference splits every node of more than `leaf_size` surfaces at n/2
// after a stable argsort of its surfaces by centroid on the axis of largest
// centroid extent (np.ptp, np.argmax: first axis on ties), emits nodes in
// preorder with escape links, and lists each leaf's surfaces in ascending
// index order.
//
// Two facts make it a parallel build with the same tree:
//  * the shape is data-independent: a node of n surfaces has children of n/2
//    and n - n/2, so node numbers, escapes, depths and leaf slots follow from
//    the counts alone and the host plans them;
//  * a node's stable order is lexicographic.  The root sorts arange(S), so
//    ties fall back to the surface index; a child sorts its parent's order
//    stably, so its order is (centroid on its axis, then on its parent's axis,
//    ..., surface index).  Repeated axes add nothing, so the key of a node is
//    at most three centroid words, most recent axis first, then the index: a
//    unique key.  Which surfaces form the left child is then "the n/2 smallest
//    keys", and the order inside a child never matters (leaves sort by index).
//
// Large nodes (more than 1,024 or 2,048 surfaces) are split level by level by one
// cooperative kernel: per level a reduction gives each node's centroid
// extents, a radix select over the 8-bit digits of the composite key
// finds the node's median (k = n/2) and surfaces are scattered to the two
// halves.  Steps are separated by a grid barrier whose waits are bounded.
// Each remaining subtree of at most 1,024 or 2,048 surfaces is built by one CTA in
// shared memory: per level, a bitonic sort of all its surfaces by (segment,
// composite key) and a split of every internal segment at its half.  Surface
// bounds are read once, at the leaves; every inner node's bounds are the union
// of its children's, filled deepest level first (min and max do not depend on
// the order they are taken in).
//
// Centroid keys map -0.0 to +0.0 (numpy compares them equal); bounds keep the
// sign of zero and take the smaller/larger of -0.0 and +0.0 as -0.0/+0.0.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

#include "acoustic_rt.h"
#include "common.h"

namespace acbvh {

// Surfaces per shared-memory subtree: 1024 (four CTAs per SM) for scenes of 2,049 to 2^18 - 1 surfaces, where the
// extra cooperative level costs less than the larger subtrees' sorts; 2048 (two CTAs per SM) otherwise.
constexpr int kSmallMax = 2048;
constexpr int kSmallMid = 1024;
constexpr int64_t kSmallMidBelow = int64_t{1} << 18;
constexpr int kChunk = 1024;           // surfaces per block work item in the large-node levels
constexpr int kTopThreads = 256;
constexpr int kItems = kChunk / kTopThreads;   // surfaces per thread in a chunk's scatter
constexpr int kSmallThreads = 512;
constexpr int kMaxPasses = 28;         // 3 centroid words x 8 digits + 4 index digits
constexpr long long kSpinLimit = 1ll << 23;
constexpr unsigned long long kSign = 0x8000000000000000ull;
constexpr uint32_t kNoChain = 0x3Fu;   // three empty axis slots

struct LevelPlan {
    int32_t seg_begin, seg_end, chunk_begin, chunk_end;
};
struct BigSeg {
    int64_t start;
    int32_t count, node, parent, depth;
};
struct Chunk {
    int32_t seg, begin, end, pad;
};
struct SmallRoot {
    int64_t start;
    int32_t count, node, parent, depth, buf, pad;
};
struct LevelTab {   // the (at most two) node counts found at one depth and their subtree sizes
    int64_t c0, n0, c1, n1;
};
// The median search of one node after some passes: the digits of the median's key found so far and its rank
// among the keys that share them.  Resolved once that rank is 0: the keys below the prefix are the left half.
struct Select {
    unsigned long long pw[4];
    long long kk;
    int32_t resolved, rw, rs, pad;
};
struct SegState {
    unsigned long long cmax[3], cmin_c[3];   // centroid keys; min kept as max of the complement
    int32_t chain, first_pass;               // axis order; digits shared by the node's min and max key
    int32_t left_fill, right_fill;
    Select sel[2];                           // the median search after an even / odd number of passes
};

struct TopArgs {
    const unsigned long long *ckey;   // [3][S] centroid sort keys
    int32_t *perm0, *perm1;
    int64_t S;
    const LevelPlan *levels;
    int32_t num_levels;
    const BigSeg *bigs;
    const Chunk *chunks;
    const LevelTab *tab;
    SegState *state;
    unsigned *hist;                   // [3][big segments][256], one per pass modulo 3
    int64_t num_bigs;
    unsigned *bar;                    // grid barrier: count, generation
    int32_t *unresolved;              // [levels][kMaxPasses + 1]
    int64_t *out_start, *out_count, *out_escape;
    int32_t *status;
};

struct SmallArgs {
    const double *lo, *hi;
    const unsigned long long *ckey;
    const int32_t *perm0, *perm1;
    int64_t S;
    int32_t leaf;
    const SmallRoot *roots;
    const LevelTab *tab;
    const SegState *state;
    double *out_min, *out_max;
    int64_t *out_start, *out_count, *out_escape, *out_prims;
    int32_t *status;
};

__device__ __forceinline__ unsigned long long order_key(double v) {
    const unsigned long long u = static_cast<unsigned long long>(__double_as_longlong(v));
    return (u & kSign) ? ~u : (u | kSign);
}
__device__ __forceinline__ unsigned long long sort_key(double v) { return order_key(v == 0.0 ? 0.0 : v); }
__device__ __forceinline__ double key_value(unsigned long long k) {
    return __longlong_as_double(static_cast<long long>((k & kSign) ? (k & ~kSign) : ~k));
}
__device__ __forceinline__ int64_t subtree_nodes(const LevelTab *tab, int depth, int64_t count) {
    const LevelTab t = tab[depth];
    return count == t.c0 ? t.n0 : t.n1;
}
// The axis order of a node whose parent's order is `parent`: `axis` first, then the parent's axes without it.
__device__ __forceinline__ uint32_t push_axis(uint32_t parent, int axis) {
    uint32_t out = static_cast<uint32_t>(axis), slot = 1;
    for (int j = 0; j < 3; ++j) {
        const uint32_t a = (parent >> (2 * j)) & 3u;
        if (a == 3u) break;
        if (a != static_cast<uint32_t>(axis)) out |= a << (2 * slot++);
    }
    for (; slot < 3; ++slot) out |= 3u << (2 * slot);
    return out;
}
// np.argmax over np.ptp of the centroids: first maximum wins.
__device__ __forceinline__ int widest_axis(const unsigned long long cmax[3], const unsigned long long cmin_c[3]) {
    int axis = 0;
    double best = key_value(cmax[0]) - key_value(~cmin_c[0]);
    for (int a = 1; a < 3; ++a) {
        const double e = key_value(cmax[a]) - key_value(~cmin_c[a]);
        if (e > best) {
            best = e;
            axis = a;
        }
    }
    return axis;
}

// ---------------------------------------------------------------- keys ----

__global__ void bvh_keys_kernel(const double *__restrict__ lo, const double *__restrict__ hi, int64_t S,
                                unsigned long long *__restrict__ ckey, int32_t *__restrict__ perm0,
                                int32_t *__restrict__ status) {
    int bad = 0;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < S;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        for (int a = 0; a < 3; ++a) {
            const double l = lo[3 * i + a], h = hi[3 * i + a];
            if (!isfinite(l) || !isfinite(h)) bad |= AC_BVH_STATUS_NONFINITE;
            else if (h < l) bad |= AC_BVH_STATUS_ORDER;
            ckey[a * S + i] = sort_key(0.5 * (l + h));   // bvh.py:27, centroids = 0.5 * (lower + upper)
        }
        perm0[i] = static_cast<int32_t>(i);
    }
    if (bad) atomicOr(status, bad);
}

// ------------------------------------------------------- large nodes -----

__device__ __forceinline__ int32_t ld_status(const int32_t *p) { return *reinterpret_cast<const volatile int32_t *>(p); }

// A surface index read back from a permutation buffer; one outside [0, S) is a defect, flagged and skipped.
__device__ __forceinline__ bool bad_index(int32_t i, int64_t S, int32_t *status) {
    if (static_cast<uint32_t>(i) < static_cast<uint64_t>(S)) return false;
    atomicOr(status, AC_BVH_STATUS_INTERNAL);
    return true;
}

// Grid-wide barrier of a cooperative launch over `blocks` arrivals.  A wait
// gives up after `poll_limit` polls, flags AC_BVH_STATUS_TIMEOUT and every
// block then leaves the kernel.
__device__ bool grid_barrier(unsigned *bar, int32_t *status, int *ok_flag, unsigned blocks = 0,
                             long long poll_limit = kSpinLimit) {
    if (blocks == 0) blocks = gridDim.x;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == blocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long polls = 0;
            while (*gen == g) {
                if (++polls > poll_limit || (ld_status(status) & AC_BVH_STATUS_TIMEOUT)) {
                    atomicOr(status, AC_BVH_STATUS_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (ld_status(status) & AC_BVH_STATUS_TIMEOUT) ok = 0;
        *ok_flag = ok;
    }
    __syncthreads();
    return *reinterpret_cast<volatile int *>(ok_flag) != 0;
}

// The barrier alone, for tests of its bounded wait: `expected` arrivals awaited by the launch's blocks.
__global__ void bvh_barrier_probe_kernel(unsigned *bar, int32_t *status, unsigned expected, long long poll_limit) {
    __shared__ int ok_flag;
    grid_barrier(bar, status, &ok_flag, expected, poll_limit);
}

struct PassDigit {
    int w, sh;   // word (0..2 centroid words in the node's axis order, 3 = surface index) and bit shift
};
__device__ __forceinline__ int chain_words(uint32_t chain) {
    int n = 0;
    while (n < 3 && ((chain >> (2 * n)) & 3u) != 3u) ++n;
    return n;
}
__device__ __forceinline__ PassDigit pass_digit(int nwc, int p) {
    if (p < 8 * nwc) return {p >> 3, 56 - 8 * (p & 7)};
    return {3, 24 - 8 * (p - 8 * nwc)};
}
__device__ __forceinline__ unsigned long long key_word(const unsigned long long *ckey, int64_t S, uint32_t chain,
                                                       int w, int32_t i) {
    if (w == 3) return static_cast<unsigned long long>(static_cast<uint32_t>(i));
    const int axis = static_cast<int>((chain >> (2 * w)) & 3u);
    return ckey[axis * S + i];
}

// One pass's digit choice from the node's histogram: every block of the node computes it from the same counts.
__device__ Select select_digit(const Select &prev, const unsigned *hist, PassDigit d, unsigned *scan_s,
                               Select *sel_s, int *found_s, int32_t *status) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned h = __ldcg(hist + tid);
    unsigned incl = h;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) scan_s[warp] = incl;
    if (tid == 0) *found_s = 0;
    __syncthreads();
    unsigned base = 0;
    for (int w = 0; w < warp; ++w) base += scan_s[w];
    incl += base;
    const unsigned excl = incl - h;
    if (d.sh >= 0 && h > 0 && static_cast<long long>(excl) <= prev.kk && prev.kk < static_cast<long long>(incl)) {
        Select s = prev;
        s.pw[d.w] |= static_cast<unsigned long long>(tid) << d.sh;
        s.kk = prev.kk - static_cast<long long>(excl);
        s.rw = d.w;
        s.rs = d.sh;
        s.resolved = s.kk == 0 ? 1 : 0;
        *sel_s = s;
        *found_s = 1;
    }
    __syncthreads();
    Select out = *sel_s;
    if (!*found_s) {   // cannot happen with unique keys; stop this node's search
        out = prev;
        out.resolved = 1;
        if (tid == 0) atomicOr(status, AC_BVH_STATUS_INTERNAL);
    }
    __syncthreads();
    return out;
}

__global__ void __launch_bounds__(kTopThreads) bvh_top_kernel(TopArgs A) {
    __shared__ unsigned hist_s[256];
    __shared__ unsigned long long red[kTopThreads / 32][6];
    __shared__ unsigned scan_s[kTopThreads / 32];
    __shared__ Select sel_s;
    __shared__ unsigned wsum_s[kTopThreads / 32][2], base_s[2];
    __shared__ int ok_flag, found_flag;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (ld_status(A.status) & (AC_BVH_STATUS_NONFINITE | AC_BVH_STATUS_ORDER)) return;   // uniform: set before launch

    for (int lvl = 0; lvl < A.num_levels; ++lvl) {
        const LevelPlan lv = A.levels[lvl];
        const int32_t *src = (lvl & 1) ? A.perm1 : A.perm0;
        int32_t *dst = (lvl & 1) ? A.perm0 : A.perm1;

        // 1. centroid extents of every node of the level (bounds come bottom-up at the end)
        for (int c = lv.chunk_begin + blockIdx.x; c < lv.chunk_end; c += gridDim.x) {
            const Chunk ch = A.chunks[c];
            unsigned long long acc[6];
#pragma unroll
            for (int j = 0; j < 6; ++j) acc[j] = 0ull;
            for (int q = ch.begin + tid; q < ch.end; q += kTopThreads) {
                const int32_t i = __ldcg(src + q);
                if (bad_index(i, A.S, A.status)) continue;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const unsigned long long k = A.ckey[a * A.S + i];
                    acc[a] = max(acc[a], k);
                    acc[3 + a] = max(acc[3 + a], ~k);
                }
            }
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                unsigned long long v = acc[j];
                for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
                if (lane == 0) red[warp][j] = v;
            }
            __syncthreads();
            if (tid < 6) {
                unsigned long long v = red[0][tid];
                for (int w = 1; w < kTopThreads / 32; ++w) v = max(v, red[w][tid]);
                SegState *st = A.state + ch.seg;
                atomicMax(tid < 3 ? &st->cmax[tid] : &st->cmin_c[tid - 3], v);
            }
            __syncthreads();
        }
        if (!grid_barrier(A.bar, A.status, &ok_flag)) return;

        // 2. radix select of each node's median over 8-bit digits.  Pass p applies the digit choice of pass
        // p - 1 (every block of a node from the same histogram; the node's first block keeps the result in
        // sel[(p - 1) & 1]) and counts the digits of pass p, so one grid barrier ends a pass.  Pass 0 chooses
        // the node's axis and starts after the bytes its smallest and largest keys share.
        int final_pass = -1;
        for (int p = 0; p <= kMaxPasses; ++p) {
            for (int c = lv.chunk_begin + blockIdx.x; c < lv.chunk_end; c += gridDim.x) {
                const Chunk ch = A.chunks[c];
                const BigSeg seg = A.bigs[ch.seg];
                SegState *st = A.state + ch.seg;
                const bool first = ch.begin == seg.start;
                uint32_t chain;
                int first_pass;
                Select cur;
                if (p == 0) {
                    unsigned long long cmax[3], cmin_c[3];
                    for (int a = 0; a < 3; ++a) {
                        cmax[a] = __ldcg(&st->cmax[a]);
                        cmin_c[a] = __ldcg(&st->cmin_c[a]);
                    }
                    const uint32_t parent_chain =
                        seg.parent >= 0 ? static_cast<uint32_t>(__ldcg(&A.state[seg.parent].chain)) : kNoChain;
                    const int axis = widest_axis(cmax, cmin_c);
                    chain = push_axis(parent_chain, axis);
                    // every key of the node lies in [min, max]: the bytes they share are the median's too
                    const unsigned long long kmin = ~cmin_c[axis], diff = kmin ^ cmax[axis];
                    first_pass = diff == 0ull ? 8 : __clzll(static_cast<long long>(diff)) / 8;
                    cur.pw[0] = first_pass == 0 ? 0ull : first_pass == 8 ? kmin
                                                                          : (kmin & (~0ull << (64 - 8 * first_pass)));
                    cur.pw[1] = cur.pw[2] = cur.pw[3] = 0ull;
                    cur.kk = seg.count / 2;
                    cur.resolved = 0;
                    cur.rw = cur.rs = cur.pad = 0;
                    if (first && tid == 0) {
                        st->chain = static_cast<int32_t>(chain);
                        st->first_pass = first_pass;
                        st->sel[1] = cur;
                        A.out_start[seg.node] = -1;
                        A.out_count[seg.node] = 0;
                        A.out_escape[seg.node] = seg.node + subtree_nodes(A.tab, seg.depth, seg.count);
                    }
                } else {
                    chain = static_cast<uint32_t>(__ldcg(&st->chain));
                    first_pass = __ldcg(&st->first_pass);
                    const Select *prevp = &st->sel[(p - 2) & 1];
                    Select prev;
                    for (int j = 0; j < 4; ++j) prev.pw[j] = __ldcg(&prevp->pw[j]);
                    prev.kk = __ldcg(&prevp->kk);
                    prev.resolved = __ldcg(&prevp->resolved);
                    prev.rw = __ldcg(&prevp->rw);
                    prev.rs = __ldcg(&prevp->rs);
                    prev.pad = 0;
                    cur = prev;
                    if (!prev.resolved) {   // block-uniform
                        const PassDigit d = pass_digit(chain_words(chain), p - 1 + first_pass);
                        cur = select_digit(prev, A.hist + (static_cast<int64_t>((p - 1) % 3) * A.num_bigs + ch.seg) * 256,
                                           d, scan_s, &sel_s, &found_flag, A.status);
                    }
                    if (first && tid == 0) {
                        st->sel[(p - 1) & 1] = cur;
                        if (!cur.resolved) atomicAdd(&A.unresolved[lvl * (kMaxPasses + 1) + p - 1], 1);
                    }
                    if (first) A.hist[(static_cast<int64_t>((p + 1) % 3) * A.num_bigs + ch.seg) * 256 + tid] = 0u;
                }
                if (cur.resolved || p == kMaxPasses) continue;   // block-uniform
                const int nwc = chain_words(chain);
                const PassDigit d = pass_digit(nwc, p + first_pass);
                if (d.sh < 0) continue;   // past the key's last digit: the next choice flags it
                const unsigned long long hm = d.sh >= 56 ? 0ull : (~0ull << (d.sh + 8));
                const int before = d.w == 3 ? nwc : d.w;
                hist_s[tid] = 0u;
                __syncthreads();
                for (int q0 = ch.begin + tid; q0 < ch.end; q0 += 4 * kTopThreads) {
                    int32_t ii[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {   // four independent index loads in flight
                        const int q = q0 + u * kTopThreads;
                        ii[u] = q < ch.end ? __ldcg(src + q) : -1;
                        if (ii[u] >= 0 && bad_index(ii[u], A.S, A.status)) ii[u] = -1;
                    }
                    unsigned long long W[4];
                    bool match[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        match[u] = ii[u] >= 0;
                        W[u] = match[u] ? key_word(A.ckey, A.S, chain, d.w, ii[u]) : 0ull;
                    }
                    for (int j = 0; j < before; ++j) {
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (match[u]) match[u] = key_word(A.ckey, A.S, chain, j, ii[u]) == cur.pw[j];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
                        if (match[u] && (W[u] & hm) == (cur.pw[d.w] & hm))
                            atomicAdd(&hist_s[(W[u] >> d.sh) & 255u], 1u);
                }
                __syncthreads();
                const unsigned h = hist_s[tid];
                if (h) atomicAdd(&A.hist[(static_cast<int64_t>(p % 3) * A.num_bigs + ch.seg) * 256 + tid], h);
                __syncthreads();
            }
            if (!grid_barrier(A.bar, A.status, &ok_flag)) return;
            // grid-uniform: every count of pass p - 1 landed before the barrier
            if (p >= 1 && (__ldcg(&A.unresolved[lvl * (kMaxPasses + 1) + p - 1]) == 0 || p == kMaxPasses)) {
                final_pass = p - 1;
                break;
            }
        }

        // 3. scatter: keys below the median's to the left half, the rest to the right half.  A block places a
        // whole chunk with one pair of atomics: each thread holds its kItems surfaces, the block scans the counts.
        for (int c = lv.chunk_begin + blockIdx.x; c < lv.chunk_end; c += gridDim.x) {
            const Chunk ch = A.chunks[c];
            SegState *st = A.state + ch.seg;
            const BigSeg seg = A.bigs[ch.seg];
            const uint32_t chain = static_cast<uint32_t>(__ldcg(&st->chain));
            const int nwc = chain_words(chain);
            const Select *fin = &st->sel[final_pass & 1];
            if (!__ldcg(&fin->resolved) && tid == 0) atomicOr(A.status, AC_BVH_STATUS_INTERNAL);
            const int rw = __ldcg(&fin->rw), rs = __ldcg(&fin->rs);
            unsigned long long pw[4];
            for (int j = 0; j < 4; ++j) pw[j] = __ldcg(&fin->pw[j]);
            const int64_t half = seg.count / 2;
            int32_t ii[kItems];
            bool valid[kItems], left[kItems];
            unsigned nl = 0, nr = 0;
#pragma unroll
            for (int u = 0; u < kItems; ++u) {
                const int q = ch.begin + u * kTopThreads + tid;
                ii[u] = q < ch.end ? __ldcg(src + q) : 0;
                valid[u] = q < ch.end && !bad_index(ii[u], A.S, A.status);
                left[u] = false;
                if (valid[u]) {
                    const int words = rw == 3 ? nwc + 1 : rw + 1;
                    for (int j = 0; j < words; ++j) {
                        const int w = j < nwc ? j : 3;
                        const unsigned long long W = key_word(A.ckey, A.S, chain, w, ii[u]);
                        if (w == rw) {
                            left[u] = (W & (~0ull << rs)) < pw[w];
                            break;
                        }
                        if (W != pw[w]) {
                            left[u] = W < pw[w];
                            break;
                        }
                    }
                    nl += left[u] ? 1u : 0u;
                    nr += left[u] ? 0u : 1u;
                }
            }
            unsigned il = nl, ir = nr;   // inclusive scans within the warp
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned vl = __shfl_up_sync(0xffffffffu, il, o), vr = __shfl_up_sync(0xffffffffu, ir, o);
                if (lane >= o) {
                    il += vl;
                    ir += vr;
                }
            }
            if (lane == 31) {
                wsum_s[warp][0] = il;
                wsum_s[warp][1] = ir;
            }
            __syncthreads();
            if (tid == 0) {
                unsigned tl = 0, tr = 0;
                for (int w = 0; w < kTopThreads / 32; ++w) {
                    const unsigned a = wsum_s[w][0], b = wsum_s[w][1];
                    wsum_s[w][0] = tl;
                    wsum_s[w][1] = tr;
                    tl += a;
                    tr += b;
                }
                base_s[0] = tl ? static_cast<unsigned>(atomicAdd(&st->left_fill, static_cast<int>(tl))) : 0u;
                base_s[1] = tr ? static_cast<unsigned>(atomicAdd(&st->right_fill, static_cast<int>(tr))) : 0u;
            }
            __syncthreads();
            int64_t pl = static_cast<int64_t>(base_s[0]) + wsum_s[warp][0] + (il - nl);
            int64_t pr = half + static_cast<int64_t>(base_s[1]) + wsum_s[warp][1] + (ir - nr);
#pragma unroll
            for (int u = 0; u < kItems; ++u) {
                if (!valid[u]) continue;
                const int64_t pos = left[u] ? pl++ : pr++;
                if (left[u] ? pos < half : pos < seg.count) dst[seg.start + pos] = ii[u];
                else atomicOr(A.status, AC_BVH_STATUS_INTERNAL);
            }
            __syncthreads();   // wsum_s and base_s are reused by the next chunk
        }
        if (!grid_barrier(A.bar, A.status, &ok_flag)) return;
    }
}

// ------------------------------------------------------- small subtrees ----

struct Entry {
    uint16_t start, count;
    int32_t node;
    uint32_t chain;
};

constexpr int kMaxSubtreeLevels = 32;

// Shared-memory state of one subtree of at most N surfaces (N a power of two, at most 4096).
template <int N>
struct SmallSmem {
    static constexpr int kCapacity = N;
    unsigned long long key[3][N];
    int32_t gidx[N];
    uint16_t lp[N];        // position -> slot, sorted every level
    uint16_t segslot[N];   // slot -> start of its segment (0xFFFF: padding)
    uint16_t cnt_at[N];    // segment start -> count
    uint8_t chain_at[N];   // segment start -> axis order
    uint8_t split_at[N];   // segment start -> depth at which it was split
    Entry inner[N];        // every internal node of the subtree, level after level (at most n - 1)
    unsigned long long part[kSmallThreads / 32][6];
    int level_begin[kMaxSubtreeLevels + 2];
    int nnext;
};

template <class M>
__device__ __forceinline__ bool slot_less(const M &m, int a, int b) {
    const unsigned sa = m.segslot[a], sb = m.segslot[b];
    if (sa != sb) return sa < sb;
    if (sa == 0xFFFFu) return a < b;
    const uint32_t chain = m.chain_at[sa];
    for (int j = 0; j < 3; ++j) {
        const uint32_t axis = (chain >> (2 * j)) & 3u;
        if (axis == 3u) break;
        const unsigned long long ka = m.key[axis][a], kb = m.key[axis][b];
        if (ka != kb) return ka < kb;
    }
    return m.gidx[a] < m.gidx[b];
}

// A leaf of the positions [s, s + c): its surfaces in ascending index order (bvh.py:48) and its bounds.
template <class M>
__device__ void emit_leaf(M &m, const SmallArgs &A, const SmallRoot &r, int s, int c, int64_t node) {
    for (int x = s + 1; x < s + c; ++x) {   // insertion sort of the leaf's slots by surface index
        const uint16_t v = m.lp[x];
        int y = x - 1;
        while (y >= s && m.gidx[m.lp[y]] > m.gidx[v]) {
            m.lp[y + 1] = m.lp[y];
            --y;
        }
        m.lp[y + 1] = v;
    }
    unsigned long long mx[3] = {0ull, 0ull, 0ull}, mn_c[3] = {0ull, 0ull, 0ull};
    for (int x = s; x < s + c; ++x) {
        const int64_t g = m.gidx[m.lp[x]];
        A.out_prims[r.start + x] = g;
        for (int a = 0; a < 3; ++a) {
            mx[a] = max(mx[a], order_key(A.hi[3 * g + a]));
            mn_c[a] = max(mn_c[a], ~order_key(A.lo[3 * g + a]));
        }
    }
    for (int a = 0; a < 3; ++a) {
        A.out_min[3 * node + a] = key_value(~mn_c[a]);
        A.out_max[3 * node + a] = key_value(mx[a]);
    }
    A.out_start[node] = r.start + s;
    A.out_count[node] = c;
    A.out_escape[node] = node + 1;
}

// An inner node's bounds: the union of its two children's (the min and max over its surfaces, in any order).
__device__ __forceinline__ void union_children(double *out_min, double *out_max, int64_t node, int64_t left,
                                               int64_t right) {
    for (int a = 0; a < 3; ++a) {
        const unsigned long long lmin = min(order_key(out_min[3 * left + a]), order_key(out_min[3 * right + a]));
        const unsigned long long umax = max(order_key(out_max[3 * left + a]), order_key(out_max[3 * right + a]));
        out_min[3 * node + a] = key_value(lmin);
        out_max[3 * node + a] = key_value(umax);
    }
}

// Axis and key order of an internal node from its centroid key extents, and its record (bounds come later).
template <class M>
__device__ __forceinline__ void finish_inner(M &m, const SmallArgs &A, Entry &en, int depth,
                                             const unsigned long long cmax[3], const unsigned long long cmin_c[3]) {
    const uint32_t chain = push_axis(en.chain, widest_axis(cmax, cmin_c));
    en.chain = chain;
    m.chain_at[en.start] = static_cast<uint8_t>(chain);
    m.cnt_at[en.start] = en.count;
    m.split_at[en.start] = static_cast<uint8_t>(depth);
    const int64_t node = en.node;
    A.out_start[node] = -1;
    A.out_count[node] = 0;
    A.out_escape[node] = node + subtree_nodes(A.tab, depth, en.count);
}

// Internal nodes of a level number at most n / 2 (each holds two or more surfaces); all of them at most n - 1.
template <class M>
__device__ __forceinline__ void push_entry(M &m, int32_t *status, const Entry &e) {
    const int at = atomicAdd(&m.nnext, 1);
    if (at < M::kCapacity) m.inner[at] = e;
    else atomicOr(status, AC_BVH_STATUS_INTERNAL);
}

template <int N>
__global__ void __launch_bounds__(kSmallThreads) bvh_small_kernel(SmallArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SmallSmem<N> &m = *reinterpret_cast<SmallSmem<N> *>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int kWarps = kSmallThreads / 32;
    if (ld_status(A.status) != 0) return;
    const SmallRoot r = A.roots[blockIdx.x];
    const int n = r.count;
    int p2 = 1;
    while (p2 < n) p2 <<= 1;
    const int32_t *src = r.buf ? A.perm1 : A.perm0;
    for (int q = tid; q < N; q += kSmallThreads) {
        m.chain_at[q] = static_cast<uint8_t>(kNoChain);
        m.split_at[q] = 0xFF;
        if (q < p2) {
            m.lp[q] = static_cast<uint16_t>(q);
            if (q < n) {
                int32_t g = src[r.start + q];
                if (bad_index(g, A.S, A.status)) g = 0;
                m.gidx[q] = g;
                for (int a = 0; a < 3; ++a) m.key[a][q] = A.ckey[a * A.S + g];
                m.segslot[q] = 0;
            } else {
                m.segslot[q] = 0xFFFFu;
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t parent_chain = r.parent >= 0 ? static_cast<uint32_t>(A.state[r.parent].chain) : kNoChain;
        m.inner[0] = Entry{0, static_cast<uint16_t>(n), r.node, parent_chain};
        m.level_begin[0] = 0;
        m.level_begin[1] = n > A.leaf ? 1 : 0;
        if (n <= A.leaf) emit_leaf(m, A, r, 0, n, r.node);
    }
    __syncthreads();
    int lev = 0;
    for (; lev < kMaxSubtreeLevels; ++lev) {
        const int b = m.level_begin[lev], e = m.level_begin[lev + 1], ncur = e - b;
        if (ncur <= 0) break;
        const int depth = r.depth + lev;
        // 1. centroid extents of every internal node: a thread per node, or warps per node while they are few
        if (ncur >= kWarps) {
            for (int x = b + tid; x < e; x += kSmallThreads) {
                Entry &en = m.inner[x];
                unsigned long long cmax[3] = {0ull, 0ull, 0ull}, cmin_c[3] = {0ull, 0ull, 0ull};
                for (int q = en.start; q < en.start + en.count; ++q) {
                    const int slot = m.lp[q];
                    for (int a = 0; a < 3; ++a) {
                        const unsigned long long k = m.key[a][slot];
                        cmax[a] = max(cmax[a], k);
                        cmin_c[a] = max(cmin_c[a], ~k);
                    }
                }
                finish_inner(m, A, en, depth, cmax, cmin_c);
            }
        } else {
            const int g = kWarps / ncur;
            unsigned long long acc[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
            if (warp / g < ncur) {
                const Entry en = m.inner[b + warp / g];
                for (int q = en.start + (warp % g) * 32 + lane; q < en.start + en.count; q += g * 32) {
                    const int slot = m.lp[q];
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const unsigned long long k = m.key[a][slot];
                        acc[a] = max(acc[a], k);
                        acc[3 + a] = max(acc[3 + a], ~k);
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                unsigned long long v = acc[j];
                for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
                if (lane == 0) m.part[warp][j] = v;
            }
            __syncthreads();
            if (tid < ncur) {
                unsigned long long v[6];
                for (int j = 0; j < 6; ++j) {
                    v[j] = m.part[tid * g][j];
                    for (int w = 1; w < g; ++w) v[j] = max(v[j], m.part[tid * g + w][j]);
                }
                finish_inner(m, A, m.inner[b + tid], depth, v, v + 3);
            }
        }
        if (tid == 0) m.nnext = e;
        __syncthreads();
        // 2. bitonic sort of all positions by (segment, key in the segment's axis order, surface index).
        // Warp w owns pairs [w*ppw, (w+1)*ppw), i.e. positions [2*w*ppw, 2*(w+1)*ppw) while the stride j is at
        // most ppw: such stages need only the warp's own barrier.
        const int pairs = p2 >> 1;
        const int ppw = max(1, pairs / kWarps);
        for (int k = 2; k <= p2; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int rr = lane; rr < ppw; rr += 32) {
                    const int i = warp * ppw + rr;
                    if (i >= pairs) break;
                    const int lo = ((i & ~(j - 1)) << 1) | (i & (j - 1));
                    const int hi = lo | j;
                    const int a = m.lp[lo], bb = m.lp[hi];
                    const bool up = (lo & k) == 0;
                    if (slot_less(m, bb, a) == up) {
                        m.lp[lo] = static_cast<uint16_t>(bb);
                        m.lp[hi] = static_cast<uint16_t>(a);
                    }
                }
                const int next_j = j > 1 ? j >> 1 : k;
                const bool last = k == p2 && j == 1;
                if (!last && j <= ppw && next_j <= ppw) __syncwarp();
                else __syncthreads();
            }
        }
        // 3. the right halves of the split segments become segments of their own
        for (int q = tid; q < n; q += kSmallThreads) {
            const int slot = m.lp[q];
            const unsigned s0 = m.segslot[slot];
            if (m.split_at[s0] == static_cast<uint8_t>(depth)) {
                const unsigned half = s0 + m.cnt_at[s0] / 2u;
                if (static_cast<unsigned>(q) >= half) m.segslot[slot] = static_cast<uint16_t>(half);
            }
        }
        __syncthreads();
        // 4. children: leaves are written now, internal ones form the next level
        for (int x = b + tid; x < e; x += kSmallThreads) {
            const Entry en = m.inner[x];
            const int lc = en.count / 2, rc = en.count - lc;
            const int64_t lnode = en.node + 1;
            const int64_t rnode = lnode + subtree_nodes(A.tab, depth + 1, lc);
            if (lc <= A.leaf) emit_leaf(m, A, r, en.start, lc, lnode);
            else push_entry(m, A.status, Entry{en.start, static_cast<uint16_t>(lc), static_cast<int32_t>(lnode), en.chain});
            if (rc <= A.leaf) emit_leaf(m, A, r, en.start + lc, rc, rnode);
            else push_entry(m, A.status, Entry{static_cast<uint16_t>(en.start + lc), static_cast<uint16_t>(rc),
                                               static_cast<int32_t>(rnode), en.chain});
        }
        __syncthreads();
        if (tid == 0) m.level_begin[lev + 2] = min(m.nnext, N);
        __syncthreads();
    }
    if (lev == kMaxSubtreeLevels && tid == 0) atomicOr(A.status, AC_BVH_STATUS_INTERNAL);
    // 5. bounds of the internal nodes, deepest level first, from their children's
    for (int l = lev - 1; l >= 0; --l) {
        const int depth = r.depth + l;
        for (int x = m.level_begin[l] + tid; x < m.level_begin[l + 1]; x += kSmallThreads) {
            const Entry en = m.inner[x];
            const int64_t left = static_cast<int64_t>(en.node) + 1;
            union_children(A.out_min, A.out_max, en.node, left, left + subtree_nodes(A.tab, depth + 1, en.count / 2));
        }
        __syncthreads();
    }
}

// Bounds of the large nodes, deepest level first, once every subtree below them has its own.
__global__ void __launch_bounds__(512) bvh_big_bounds_kernel(const LevelPlan *levels, int32_t num_levels,
                                                             const BigSeg *bigs, const LevelTab *tab, double *out_min,
                                                             double *out_max, const int32_t *status) {
    if (ld_status(status) != 0) return;
    for (int l = num_levels - 1; l >= 0; --l) {
        const LevelPlan lv = levels[l];
        for (int g = lv.seg_begin + threadIdx.x; g < lv.seg_end; g += blockDim.x) {
            const BigSeg seg = bigs[g];
            const int64_t left = static_cast<int64_t>(seg.node) + 1;
            union_children(out_min, out_max, seg.node, left, left + subtree_nodes(tab, seg.depth + 1, seg.count / 2));
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- plan ------

struct Info {
    int64_t nodes, leaves, height;
};

struct Plan {
    std::vector<LevelPlan> levels;
    std::vector<BigSeg> bigs;
    std::vector<Chunk> chunks;
    std::vector<SmallRoot> smalls;
    std::vector<LevelTab> tab;   // indexed by depth (root depth 1)
    Info root{};
    size_t max_items = 1;        // largest chunk or segment count of one level (cooperative grid bound)

    std::map<int64_t, Info> memo;
    int64_t leaf = 4;
    int64_t small_max = kSmallMax;   // surfaces per shared-memory subtree for this scene

    Info info(int64_t c) {
        auto it = memo.find(c);
        if (it != memo.end()) return it->second;
        Info out{1, 1, 1};
        if (c > leaf) {
            const Info a = info(c / 2), b = info(c - c / 2);
            out = Info{1 + a.nodes + b.nodes, a.leaves + b.leaves, 1 + std::max(a.height, b.height)};
        }
        memo.emplace(c, out);
        return out;
    }

    void walk(int64_t start, int64_t count, int64_t node, int depth, int parent, int buf,
              std::vector<std::vector<BigSeg>> &by_level, std::vector<std::vector<int>> &parent_level_index) {
        if (count > small_max) {
            const int lvl = depth - 1;
            if (static_cast<int>(by_level.size()) <= lvl) {
                by_level.resize(lvl + 1);
                parent_level_index.resize(lvl + 1);
            }
            const int id = static_cast<int>(by_level[lvl].size());
            by_level[lvl].push_back(BigSeg{start, static_cast<int32_t>(count), static_cast<int32_t>(node), parent, depth});
            const int64_t l = count / 2;
            // children refer to their parent by its index within the parent's level; remapped below
            walk(start, l, node + 1, depth + 1, id, buf ^ 1, by_level, parent_level_index);
            walk(start + l, count - l, node + 1 + info(l).nodes, depth + 1, id, buf ^ 1, by_level, parent_level_index);
        } else {
            smalls.push_back(SmallRoot{start, static_cast<int32_t>(count), static_cast<int32_t>(node), parent, depth, buf, 0});
        }
    }

    void build(int64_t S, int64_t leaf_size) {
        leaf = leaf_size;
        small_max = (S > kSmallMax && S < kSmallMidBelow) ? kSmallMid : kSmallMax;
        root = info(S);
        // level table: the counts at each depth (at most two, consecutive)
        tab.assign(static_cast<size_t>(root.height) + 2, LevelTab{-1, 0, -1, 0});
        std::vector<int64_t> vals{S};
        for (int d = 1; d <= root.height; ++d) {
            std::sort(vals.begin(), vals.end());
            vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
            LevelTab t{-1, 0, -1, 0};
            if (!vals.empty()) t.c0 = vals[0], t.n0 = info(vals[0]).nodes;
            if (vals.size() > 1) t.c1 = vals[1], t.n1 = info(vals[1]).nodes;
            tab[d] = t;
            std::vector<int64_t> next;
            for (int64_t c : vals)
                if (c > leaf) {
                    next.push_back(c / 2);
                    next.push_back(c - c / 2);
                }
            vals.swap(next);
        }
        std::vector<std::vector<BigSeg>> by_level;
        std::vector<std::vector<int>> unused;
        walk(0, S, 0, 1, -1, 0, by_level, unused);
        // flatten level by level; parents become global indices
        std::vector<int> offset(by_level.size() + 1, 0);
        for (size_t l = 0; l < by_level.size(); ++l) offset[l + 1] = offset[l] + static_cast<int>(by_level[l].size());
        for (size_t l = 0; l < by_level.size(); ++l) {
            LevelPlan lp{offset[l], offset[l + 1], static_cast<int32_t>(chunks.size()), 0};
            for (size_t k = 0; k < by_level[l].size(); ++k) {
                BigSeg b = by_level[l][k];
                if (b.parent >= 0) b.parent += offset[l - 1];
                const int gid = offset[l] + static_cast<int>(k);
                bigs.push_back(b);
                for (int64_t q = b.start; q < b.start + b.count; q += kChunk)
                    chunks.push_back(Chunk{gid, static_cast<int32_t>(q),
                                           static_cast<int32_t>(std::min<int64_t>(q + kChunk, b.start + b.count)), 0});
            }
            lp.chunk_end = static_cast<int32_t>(chunks.size());
            levels.push_back(lp);
            max_items = std::max<size_t>(max_items, std::max<size_t>(lp.chunk_end - lp.chunk_begin, lp.seg_end - lp.seg_begin));
        }
        for (SmallRoot &s : smalls)
            if (s.parent >= 0) s.parent += offset[s.depth - 2];
    }
};

struct Layout {
    size_t ckey, perm0, perm1, state, hist, bar, unresolved, plan, total;
    size_t levels, bigs, chunks, smalls, tab, plan_bytes;
};

size_t up256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

Layout layout(const Plan &p, int64_t S) {
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += up256(bytes);
        return at;
    };
    L.ckey = take(3 * static_cast<size_t>(S) * sizeof(unsigned long long));
    L.perm0 = take(static_cast<size_t>(S) * sizeof(int32_t));
    L.perm1 = take(static_cast<size_t>(S) * sizeof(int32_t));
    const size_t zero_begin = off;
    L.state = take(std::max<size_t>(1, p.bigs.size()) * sizeof(SegState));
    L.hist = take(3 * std::max<size_t>(1, p.bigs.size()) * 256 * sizeof(unsigned));
    L.bar = take(2 * sizeof(unsigned));
    L.unresolved = take(std::max<size_t>(1, p.levels.size()) * (kMaxPasses + 1) * sizeof(int32_t));
    (void)zero_begin;
    // the plan, copied from the host in one piece
    size_t po = 0;
    auto ptake = [&](size_t bytes) {
        const size_t at = po;
        po += (bytes + 15) & ~static_cast<size_t>(15);
        return at;
    };
    L.levels = ptake(p.levels.size() * sizeof(LevelPlan));
    L.bigs = ptake(p.bigs.size() * sizeof(BigSeg));
    L.chunks = ptake(p.chunks.size() * sizeof(Chunk));
    L.smalls = ptake(p.smalls.size() * sizeof(SmallRoot));
    L.tab = ptake(p.tab.size() * sizeof(LevelTab));
    L.plan_bytes = po;
    L.plan = take(po);
    L.total = off;
    return L;
}

int check_args(int64_t S, int32_t leaf) {
    if (S < 1) return ac::fail(AC_ERR_INVALID, "BVH requires at least one surface");
    if (S >= (int64_t{1} << 30)) return ac::fail(AC_ERR_CAPACITY, "ac_bvh_build_device: %lld surfaces (limit 2^30 - 1)", (long long)S);
    if (leaf < 1 || leaf > 255) return ac::fail(AC_ERR_INVALID, "ac_bvh_build_device: leaf size %d outside 1..255", leaf);
    return AC_OK;
}

}  // namespace acbvh

extern "C" int ac_bvh_device_workspace_size(int64_t num_surfaces, int32_t leaf_size, size_t *workspace_bytes,
                                            size_t *staging_bytes, int64_t *node_count) {
    using namespace acbvh;
    if (!workspace_bytes) return ac::fail(AC_ERR_INVALID, "ac_bvh_device_workspace_size: null argument");
    const int rc = check_args(num_surfaces, leaf_size);
    if (rc != AC_OK) return rc;
    Plan p;
    p.build(num_surfaces, leaf_size);
    const Layout L = layout(p, num_surfaces);
    *workspace_bytes = L.total;
    if (staging_bytes) *staging_bytes = L.plan_bytes;
    if (node_count) *node_count = p.root.nodes;
    return AC_OK;
}

extern "C" int ac_bvh_build_device(const double *bounds_min, const double *bounds_max, int64_t num_surfaces,
                                   int32_t leaf_size, ac_bvh *out, int32_t *status, void *workspace,
                                   size_t workspace_bytes, void *host_staging, void *stream_ptr) {
    using namespace acbvh;
    ac::NvtxRange nvtx_range("ac_bvh_build_device");
    if (!bounds_min || !bounds_max || !out || !status || !out->bounds_min || !out->bounds_max || !out->start ||
        !out->count || !out->escape || !out->primitives)
        return ac::fail(AC_ERR_INVALID, "ac_bvh_build_device: null pointer");
    int rc = check_args(num_surfaces, leaf_size);
    if (rc != AC_OK) return rc;
    const int64_t S = num_surfaces;
    Plan p;
    p.build(S, leaf_size);
    const Layout L = layout(p, S);
    if (!workspace || workspace_bytes < L.total)
        return ac::fail(AC_ERR_CAPACITY, "ac_bvh_build_device workspace too small: %zu < %zu", workspace_bytes, L.total);
    if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
        return ac::fail(AC_ERR_INVALID, "ac_bvh_build_device: workspace must be 256-byte aligned");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    unsigned char *ws = static_cast<unsigned char *>(workspace);

    std::vector<unsigned char> blob_vec;
    unsigned char *blob = static_cast<unsigned char *>(host_staging);
    if (!blob) {
        blob_vec.resize(std::max<size_t>(1, L.plan_bytes));
        blob = blob_vec.data();
    }
    auto put = [&](size_t at, const void *src, size_t bytes) {
        if (bytes) std::memcpy(blob + at, src, bytes);
    };
    put(L.levels, p.levels.data(), p.levels.size() * sizeof(LevelPlan));
    put(L.bigs, p.bigs.data(), p.bigs.size() * sizeof(BigSeg));
    put(L.chunks, p.chunks.data(), p.chunks.size() * sizeof(Chunk));
    put(L.smalls, p.smalls.data(), p.smalls.size() * sizeof(SmallRoot));
    put(L.tab, p.tab.data(), p.tab.size() * sizeof(LevelTab));

    AC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int32_t), stream));
    AC_CUDA_TRY(cudaMemsetAsync(ws + L.state, 0, L.plan - L.state, stream));
    AC_CUDA_TRY(cudaMemcpyAsync(ws + L.plan, blob, L.plan_bytes, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));   // the pageable plan must outlive the copy

    auto *ckey = reinterpret_cast<unsigned long long *>(ws + L.ckey);
    auto *perm0 = reinterpret_cast<int32_t *>(ws + L.perm0);
    auto *perm1 = reinterpret_cast<int32_t *>(ws + L.perm1);
    const LevelTab *tab = reinterpret_cast<const LevelTab *>(ws + L.plan + L.tab);
    auto *state = reinterpret_cast<SegState *>(ws + L.state);

    int device = 0, sms = 0;
    AC_CUDA_TRY(cudaGetDevice(&device));
    AC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    {
        const int64_t want = (S + 255) / 256;
        const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t{8} * sms)));
        bvh_keys_kernel<<<blocks, 256, 0, stream>>>(bounds_min, bounds_max, S, ckey, perm0, status);
        AC_CUDA_TRY(cudaGetLastError());
    }
    if (!p.levels.empty()) {
        int coop = 0, occ = 0;
        AC_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
        if (!coop) return ac::fail(AC_ERR_UNSUPPORTED, "ac_bvh_build_device: the device has no cooperative launch");
        AC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, bvh_top_kernel, kTopThreads, 0));
        if (occ < 1) return ac::fail(AC_ERR_UNSUPPORTED, "ac_bvh_build_device: the top-level kernel does not fit an SM");
        const int grid = static_cast<int>(std::min<size_t>(p.max_items, static_cast<size_t>(occ) * sms));
        TopArgs ta{};
        ta.ckey = ckey;
        ta.perm0 = perm0;
        ta.perm1 = perm1;
        ta.S = S;
        ta.levels = reinterpret_cast<const LevelPlan *>(ws + L.plan + L.levels);
        ta.num_levels = static_cast<int32_t>(p.levels.size());
        ta.bigs = reinterpret_cast<const BigSeg *>(ws + L.plan + L.bigs);
        ta.chunks = reinterpret_cast<const Chunk *>(ws + L.plan + L.chunks);
        ta.tab = tab;
        ta.state = state;
        ta.hist = reinterpret_cast<unsigned *>(ws + L.hist);
        ta.num_bigs = static_cast<int64_t>(p.bigs.size());
        ta.bar = reinterpret_cast<unsigned *>(ws + L.bar);
        ta.unresolved = reinterpret_cast<int32_t *>(ws + L.unresolved);
        ta.out_start = out->start;
        ta.out_count = out->count;
        ta.out_escape = out->escape;
        ta.status = status;
        void *args[] = {&ta};
        AC_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void *>(bvh_top_kernel), dim3(grid),
                                                dim3(kTopThreads), args, 0, stream));
    }
    {
        static_assert(sizeof(SmallSmem<kSmallMax>) <= 227 * 1024, "subtree state must fit shared memory");
        const bool mid = p.small_max == kSmallMid;
        const size_t smem = mid ? sizeof(SmallSmem<kSmallMid>) : sizeof(SmallSmem<kSmallMax>);
        AC_CUDA_TRY(cudaFuncSetAttribute(mid ? bvh_small_kernel<kSmallMid> : bvh_small_kernel<kSmallMax>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        SmallArgs sa{};
        sa.lo = bounds_min;
        sa.hi = bounds_max;
        sa.ckey = ckey;
        sa.perm0 = perm0;
        sa.perm1 = perm1;
        sa.S = S;
        sa.leaf = leaf_size;
        sa.roots = reinterpret_cast<const SmallRoot *>(ws + L.plan + L.smalls);
        sa.tab = tab;
        sa.state = state;
        sa.out_min = out->bounds_min;
        sa.out_max = out->bounds_max;
        sa.out_start = out->start;
        sa.out_count = out->count;
        sa.out_escape = out->escape;
        sa.out_prims = out->primitives;
        sa.status = status;
        if (mid)
            bvh_small_kernel<kSmallMid><<<static_cast<unsigned>(p.smalls.size()), kSmallThreads, smem, stream>>>(sa);
        else
            bvh_small_kernel<kSmallMax><<<static_cast<unsigned>(p.smalls.size()), kSmallThreads, smem, stream>>>(sa);
        AC_CUDA_TRY(cudaGetLastError());
    }
    if (!p.levels.empty()) {
        bvh_big_bounds_kernel<<<1, 512, 0, stream>>>(reinterpret_cast<const LevelPlan *>(ws + L.plan + L.levels),
                                                     static_cast<int32_t>(p.levels.size()),
                                                     reinterpret_cast<const BigSeg *>(ws + L.plan + L.bigs), tab,
                                                     out->bounds_min, out->bounds_max, status);
        AC_CUDA_TRY(cudaGetLastError());
    }
    out->node_count = p.root.nodes;
    out->leaf_count = p.root.leaves;
    out->max_depth = p.root.height;
    return AC_OK;
}

extern "C" int ac_bvh_barrier_probe(int32_t blocks, int32_t expected_blocks, int64_t poll_limit, void *workspace,
                                    int32_t *status, void *stream_ptr) {
    using namespace acbvh;
    if (!workspace || !status) return ac::fail(AC_ERR_INVALID, "ac_bvh_barrier_probe: null pointer");
    if (blocks < 1 || blocks > 64 || expected_blocks < 1 || poll_limit < 1 || poll_limit > (int64_t{1} << 26))
        return ac::fail(AC_ERR_INVALID, "ac_bvh_barrier_probe: blocks 1..64, expected >= 1, poll limit 1..2^26");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    AC_CUDA_TRY(cudaMemsetAsync(workspace, 0, 2 * sizeof(unsigned), stream));
    AC_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int32_t), stream));
    bvh_barrier_probe_kernel<<<blocks, 32, 0, stream>>>(static_cast<unsigned *>(workspace), status,
                                                        static_cast<unsigned>(expected_blocks), poll_limit);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}
