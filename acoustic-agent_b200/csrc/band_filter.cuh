// The crossover recursion of bandlimit_band_signals (acoustic_agent/steam_rt.py
// :3070-3083, :4131-4212) as a systolic warp: lane (unit, chain, stage) runs one
// biquad section of an eight-pole low-pass and passes its float32 output one
// lane up; section s runs kSkew samples behind section s-1.  A "unit" is one
// band of one signal: bands 1-4 need two chains (the low-pass at the upper and
// lower crossover, subtracted), bands 0 and 5 one.  Four units per warp.
//
// Included by every translation unit that band-limits signals; each of them is
// compiled with -fmad=false, so the float64 arithmetic rounds operation by
// operation like the reference's.
#pragma once

#include <cuda_runtime.h>

namespace ac {
namespace {

// One section of an eight-pole low-pass (steam_rt.py:4131-4146):
//     y0 = b0*x0 + b1*x1 + b2*x2 - a1*y1 - a2*y2, evaluated left to right.
// The input part ((b0*x0 + b1*x1) + b2*x2) does not depend on y, so it is
// computed one sample ahead (`feed`); the per-sample recursion (`step`) is then
// only (S - a1*y1) - a2*y2.  Same operations in the same order as the reference.
struct Section {
    double b0, b1, b2, a1, a2, x1, x2, y1, y2;

    __device__ __forceinline__ double feed(double in) {
        const double v = b0 * in + b1 * x1 + b2 * x2;
        x2 = x1;
        x1 = in;
        return v;
    }

    __device__ __forceinline__ float step(double v) {
        const double y0 = v - a1 * y1 - a2 * y2;
        y2 = y1;
        y1 = y0;
        return static_cast<float>(y0);
    }
};

#ifndef AC_SYNTH_PREFETCH
#define AC_SYNTH_PREFETCH 16
#endif
#ifndef AC_SYNTH_SKEW
#define AC_SYNTH_SKEW 4
#endif
constexpr int kPrefetch = AC_SYNTH_PREFETCH;
constexpr int kSkew = AC_SYNTH_SKEW;  // iterations between consecutive sections
constexpr int kLag = kSkew * 3;  // section 3 runs kLag samples behind section 0
static_assert(kSkew >= 3 && kLag + 2 <= kPrefetch, "the prefetch window must hold the lagged input");
static_assert(kPrefetch >= 2, "section 0 reads its input two samples ahead");

// Lane (unit, chain, stage): section `stage` works on sample it - kSkew*stage.
// The float32 output it produces at iteration it is shuffled one lane up at
// iteration it + 1 and consumed there at it + kSkew - 1 (as the input part of
// its step at it + kSkew); the outputs are formed two iterations late and
// written once per chunk of kPrefetch iterations.  So no instruction waits on
// a shuffle issued in its own iteration, no store or bounds test sits in the
// per-sample loop, and only the section's own y dependency is carried from one
// iteration to the next.
//
// The body is branch-free: before a section's first real sample its input is
// +0.0, and a section whose inputs and state are all +0.0 produces exactly +0.0
// and keeps its state at +0.0 (every product is +0.0 or -0.0 and the sums come
// out +0.0), so the steps while the pipeline fills change nothing.
// The per-lane recursion of one warp.  `x` / `out_row` / `n_len` belong to the
// lane's unit (band of one RIR); `co` points at the lane's section
// coefficients.  `iterations` (the longest unit of the warp + kLag + 2) is
// warp-uniform: every lane runs every iteration, so the shuffles stay full-warp.
__device__ __forceinline__ void filter_units(const double *x, float *out_row, int n_len, bool valid_unit, int band,
                                             const double *co, int iterations) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int stage = lane & 3;
    const int chain = (lane >> 2) & 1;
    int cutoff;
    bool active;
    if (band == 0) { cutoff = 0; active = chain == 0; }
    else if (band == 5) { cutoff = 4; active = chain == 0; }
    else { cutoff = chain == 0 ? band : band - 1; active = true; }
    active = active && valid_unit;
    co += cutoff * 20 + stage * 5;
    Section sec{co[0], co[1], co[2], co[3], co[4], 0.0, 0.0, 0.0, 0.0};
    const bool emits = stage == 3 && chain == 0 && active;
    const bool is_first = stage == 0;
    const int mode = band == 0 ? 0 : (band == 5 ? 2 : 1);

    double ahead[kPrefetch], prev[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
        ahead[u] = (valid_unit && u < n_len) ? __ldg(x + u) : 0.0;
        prev[u] = 0.0;
    }
    // q[d]: the value the previous section produced at iteration it - 1 - d (received through the
    // shuffle issued one iteration after it was produced, so no shuffle result is used in the
    // iteration that receives it); q[kSkew - 3] is this section's input two iterations ahead.
    float q[kSkew - 2];
#pragma unroll
    for (int i = 0; i < kSkew - 2; ++i) q[i] = 0.0f;
    float y1f = 0.0f, y2f = 0.0f;   // this lane's float outputs of iterations it - 1 and it - 2
    float lower2 = 0.0f;            // the lower chain's output of iteration it - 2
    // input parts of the first two samples (their inputs are ahead[0], ahead[1] for section 0 and +0.0 for the
    // later sections); each iteration then forms the input part two samples ahead, so that its dependent
    // chain (conversion, products, sums) has a whole iteration to complete before the recursion needs it
    double v = sec.feed(is_first ? ahead[0] : 0.0);
    double v_next = sec.feed(is_first ? ahead[1] : 0.0);
    for (int base = 0; base < iterations; base += kPrefetch) {
        double next[kPrefetch];
        float emitted[kPrefetch];   // this chunk's outputs, written after the chunk (off the recursion's path)
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            const int m = base + kPrefetch + u;
            next[u] = (valid_unit && m < n_len) ? __ldg(x + m) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            const int it = base + u;
            const float y = sec.step(v);   // the recursion: the only chain carried from one iteration to the next
            // exchange the outputs of the previous iteration, already rounded to float32
            const float sent = __shfl_up_sync(full, y1f, 1);
            const float lower = __shfl_down_sync(full, y1f, 4);
#pragma unroll
            for (int i = kSkew - 3; i > 0; --i) q[i] = q[i - 1];
            q[0] = sent;
            // input part of iteration it + 2: section 0 reads the prefetched signal, later sections the
            // value their predecessor produced at it + 2 - kSkew, received at it - 1 (q[kSkew - 3])
            const double in_2 = is_first ? (u + 2 < kPrefetch ? ahead[u + 2] : next[u + 2 - kPrefetch])
                                         : static_cast<double>(q[kSkew - 3]);
            v = v_next;
            v_next = sec.feed(in_2);
            // output of iteration it - 2; x[it - 2 - kLag] is still in registers from the prefetch
            const int k = u - 2 - kLag;
            const double x_n = k >= 0 ? ahead[k] : prev[k + kPrefetch];
            const float band5 = static_cast<float>(x_n - static_cast<double>(y2f));
            emitted[u] = mode == 0 ? y2f : (mode == 2 ? band5 : y2f - lower2);
            lower2 = lower;
            y2f = y1f;
            y1f = y;
        }
        // iteration base + u produced output sample base + u - 2 - kLag
        const int first = base - 2 - kLag;
        if (emits) {
            if (first >= 0 && first + kPrefetch <= n_len) {
#pragma unroll
                for (int u = 0; u < kPrefetch; ++u) out_row[first + u] = emitted[u];
            } else {
#pragma unroll
                for (int u = 0; u < kPrefetch; ++u)
                    if (first + u >= 0 && first + u < n_len) out_row[first + u] = emitted[u];
            }
        }
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            prev[u] = ahead[u];
            ahead[u] = next[u];
        }
    }
}

}  // namespace
}  // namespace ac
