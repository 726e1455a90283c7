// Late reverberation on the GPU: the sixteen-line FDN impulse response and the
// hybrid late tail of acoustic_agent/steam_rt.py:2235-2640.
//
// ac_fdn_impulse restates _fdn_impulse_kernel (:2235-2327) so that every output
// sample is bit-identical to the reference's float64 kernel: this file is
// compiled with -fmad=false and every expression keeps the reference's
// operation order.  The network is sequential in time, but its feedback runs
// through delay lines of at least AC_FDN_MIN_DELAY samples, so nothing a
// sample computes is needed by the next hundred samples except each biquad's
// own state.  A biquad's state recursion ((S - a1*y1) - a2*y2) is three
// dependent float64 operations per sample; a sample needs 96 absorptive
// sections, and one warp issuing three of them per lane is bound by the
// float64 issue rate, so the sections are spread one per lane.  One
// 192-thread block renders one impulse response:
//
//   warps 0-3 (the lines): lane 6j + b of warp w runs absorptive section
//     (band) b of line 4w + j, kLineSkew steps behind band b - 1, whose
//     output reaches it by a shuffle; the input part of each biquad is
//     computed a step ahead, so only its three-operation recursion is on the
//     per-sample path.  Lanes 24-31 idle.  Band 5 of sample m runs at step m + kLineLag and is
//     stored to a shared ring.  Each warp fetches its four delay lines one
//     32-sample block ahead by cp.async.
//   warp 4 (the mix): one block behind, lane i takes sample i of the block
//     from the ring and, in registers, sums its sixteen line outputs in line
//     order, runs the Hadamard butterfly and writes the sixteen delay lines
//     (global memory, L2-resident; coalesced per line), and runs the four
//     all-pass stages (their delays exceed 32, so a block's samples are
//     independent).
//   warp 5 (the tone): two blocks behind, the six tone sections as a
//     systolic chain over lanes 0-5, kToneSkew steps apart.
//
// The six warps meet at one named barrier per block.  A delay-line value
// written by the mix warp is visible to the line warps two barriers later,
// which is why the delays must be at least 128 samples (see check_fdn).
//
// ac_late_tail restates the rest of _render_parametric_fdn_late_reverb
// (:2588-2640): bandlimit_band_signals of the impulse (the systolic crossover
// filter of band_filter.cuh, bit-identical), then one block per (RIR, band)
// measures the traced power at the anchor (_late_tail_start_power,
// :2473-2497), scales the FDN band to the target energy and writes the
// equal-power crossfade.  Its sums run in a fixed order but not numpy's
// pairwise order, so scales agree with the reference to about 1e-15 relative.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "band_filter.cuh"
#include "common.h"

namespace ac {
namespace {

constexpr int kLines = AC_FDN_LINES;
constexpr int kBlk = 32;                   // samples per block
constexpr int kLineSkew = 2;               // steps between consecutive absorptive sections of a line
constexpr int kLineWarps = 4;              // line warps, four lines each
constexpr int kLinesPerWarp = kLines / kLineWarps;
constexpr int kLineLag = 5 * kLineSkew;        // band 5 of sample m runs at step m + kLineLag
constexpr int kRing = 4 * kBlk;            // samples of line outputs kept for the output warp
constexpr int kRowStride = kLines + 1;     // doubles per ring row: column reads without bank conflicts
constexpr int kToneSkew = 2;               // steps between consecutive tone sections
constexpr int kToneLag = 5 * kToneSkew;    // tone section 5 finishes sample g - kToneLag at step g
constexpr int kStageRow = kLines + 1;      // staged inputs: one padded row of 16 lines per sample
constexpr int kStageBlock = kBlk * kStageRow;
constexpr int kStageDoubles = 2 * kStageBlock;
constexpr int kFixedSmem = (kStageDoubles + kRing * kRowStride + 3 * kBlk) * static_cast<int>(sizeof(double));
constexpr int kFdnThreads = 32 * (kLineWarps + 2);
// Warp 1 writes the delay-line values of sample block b between barriers b+1
// and b+2; warp 0's prefetch after barrier j-1 reads samples up to 32j + 63,
// whose delayed sources must lie in blocks <= j - 3: delays of 128 or more.
static_assert(AC_FDN_MIN_DELAY >= 4 * kBlk, "a prefetched delay-line value must be visible to warp 0");

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct FdnJobDev {
    double absorptive[kLines][6][5];
    double tone[6][5];
    int32_t delays[kLines];
    int32_t line_start[kLines];     // offset of each delay line within this job's lines
    int32_t allpass[AC_FDN_ALLPASS];
    int32_t allpass_start[AC_FDN_ALLPASS];  // offsets of the all-pass rings in shared memory
    int32_t num_samples;
    int32_t preroll;
    double *out;
    int64_t pool;                   // offset of this job's delay lines in the workspace pool (doubles)
};

// y = b0*x + b1*x1 + b2*x2 - a1*y1 - a2*y2, left to right, all in float64
// (the absorptive and tone sections of steam_rt.py:2261-2275 / :2312-2325).
// feed() is the input part ((b0*x + b1*x1) + b2*x2), which does not depend on
// y and is computed one sample ahead; step() is the recursion
// (v - a1*y1) - a2*y2.  Same operations in the same order as run().
struct Biquad {
    double b0, b1, b2, a1, a2, x1, x2, y1, y2;

    __device__ __forceinline__ void load(const double *c) {
        b0 = c[0]; b1 = c[1]; b2 = c[2]; a1 = c[3]; a2 = c[4];
        x1 = x2 = y1 = y2 = 0.0;
    }

    __device__ __forceinline__ double feed(double x) {
        const double v = b0 * x + b1 * x1 + b2 * x2;
        x2 = x1;
        x1 = x;
        return v;
    }

    __device__ __forceinline__ double step(double v) {
        const double y = v - a1 * y1 - a2 * y2;
        y2 = y1;
        y1 = y;
        return y;
    }
};

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// The six warps of a block meet here once per sample block.
__device__ __forceinline__ void block_barrier() { asm volatile("bar.sync 1, %0;" ::"n"(kFdnThreads) : "memory"); }

// Block k's delay-line inputs for lines first .. first + 3: lane i fetches
// sample 32k + i of each into row i of the stage; advance the positions by
// one block.
__device__ __forceinline__ void prefetch_block(const double *lines, const int *line_start, const int *delays,
                                               int first, int *pos, double *stage, int lane) {
#pragma unroll
    for (int j = 0; j < kLinesPerWarp; ++j) {
        const int l = first + j;
        cp_async8(stage + lane * kStageRow + l, lines + line_start[l] + pos[j]);
        const int p = pos[j] + kBlk;
        pos[j] = p >= delays[l] ? p - delays[l] : p;
    }
    cp_async_commit();
}

__device__ void fdn_lines(const FdnJobDev &job, const double *lines, double *stage, double *rows, const int *s_start,
                          const int *s_delay, int iterations) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int first = (threadIdx.x >> 5) * kLinesPerWarp;
    const bool valid = lane < 6 * kLinesPerWarp;
    const int line = first + (valid ? lane / 6 : 0);
    const int band = valid ? lane % 6 : 0;
    Biquad sec;
    sec.load(job.absorptive[line][band]);
    if (!valid) sec.b0 = sec.b1 = sec.b2 = sec.a1 = sec.a2 = 0.0;
    const bool stores = valid && band == 5;
    int pos[kLinesPerWarp];
#pragma unroll
    for (int j = 0; j < kLinesPerWarp; ++j) pos[j] = lane;  // every delay exceeds 32
    // band b works on sample n - kLineSkew * b at step n; its input is band b - 1's output of step
    // n - kLineSkew, which arrives by a shuffle issued at step n - kLineSkew and is fed (the input part
    // of the biquad) one step ahead, at step n - 1
    static_assert(kLineSkew == 2, "the shuffle is consumed one step after it is issued");
    double received = 0.0;   // band b - 1's output of the previous step
    double carry = 0.0;      // band b - 1's input for the first step of the next block
    double v = 0.0;          // input part for the current step
    prefetch_block(lines, s_start, s_delay, first, pos, stage, lane);
    for (int k = 0; k < iterations; ++k) {
        prefetch_block(lines, s_start, s_delay, first, pos, stage + ((k + 1) & 1) * kStageBlock, lane);
        cp_async_wait<1>();
        __syncwarp();
        const double *in = stage + (k & 1) * kStageBlock + line;
        v = sec.feed(band == 0 ? in[0] : carry);
        const int m0 = k * kBlk - kLineLag;
        // fully unrolled, so that band 0's staged reads are issued well ahead of their use
#pragma unroll
        for (int t = 0; t < kBlk; ++t) {
            const double y = sec.step(v);                      // the only chain carried between steps
            const double next_in = band == 0 ? in[((t + 1) & (kBlk - 1)) * kStageRow] : received;
            received = __shfl_up_sync(full, y, 1);
            if (t + 1 < kBlk) v = sec.feed(next_in);          // the next block's first input is fed after its fetch
            else carry = next_in;
            // band 5 of sample m0 + t; the ring slots written while m0 + t < 0 (zeros) are
            // rewritten with their real samples before the mix warp reads them
            if (stores) rows[((m0 + t) & (kRing - 1)) * kRowStride + line] = y;
        }
        __syncwarp();
        block_barrier();
    }
    cp_async_wait<0>();
}

__device__ void fdn_mix(const FdnJobDev &job, double *lines, const double *rows, double *tone_in, double *ap,
                        const int *s_start, const int *s_delay, int blocks, int iterations) {
    const int lane = threadIdx.x & 31;
    int apos[AC_FDN_ALLPASS];
#pragma unroll
    for (int s = 0; s < AC_FDN_ALLPASS; ++s) apos[s] = 0;
    int wpos[kLines];   // delay-line position of this lane's sample in the current block
#pragma unroll
    for (int l = 0; l < kLines; ++l) wpos[l] = lane;
    for (int k = 0; k < iterations; ++k) {
        block_barrier();
        if (k == 0 || k > blocks) continue;
        const int base = (k - 1) * kBlk;  // samples base .. base + 31 are complete in the ring
        const int m = base + lane;
        const double *row = rows + (m & (kRing - 1)) * kRowStride;
        double d[kLines];
#pragma unroll
        for (int l = 0; l < kLines; ++l) d[l] = row[l];
        // output: the line outputs summed in line order, over the line count (steam_rt.py:2297-2300)
        double v = 0.0;
#pragma unroll
        for (int l = 0; l < kLines; ++l) v += d[l];
        v /= static_cast<double>(kLines);
        // feedback: unnormalised Hadamard butterfly, strides 1, 2, 4, 8, written back with gain 0.25
        // and the unit impulse at sample 0 (steam_rt.py:2279-2295)
#pragma unroll
        for (int stride = 1; stride < kLines; stride *= 2)
#pragma unroll
            for (int a = 0; a < kLines; ++a)
                if ((a & stride) == 0) {
                    const double first = d[a], second = d[a + stride];
                    d[a] = first + second;
                    d[a + stride] = first - second;
                }
        const double injection = m == 0 ? 1.0 : 0.0;
#pragma unroll
        for (int l = 0; l < kLines; ++l) {
            lines[s_start[l] + wpos[l]] = injection + 0.25 * d[l];
            const int p = wpos[l] + kBlk;
            wpos[l] = p >= s_delay[l] ? p - s_delay[l] : p;
        }
#pragma unroll
        for (int s = 0; s < AC_FDN_ALLPASS; ++s) {
            const int D = job.allpass[s];
            double *ring = ap + job.allpass_start[s];
            int idx = apos[s] + lane;
            idx = idx >= D ? idx - D : idx;
            const double previous = ring[idx];
            const double internal = v + 0.5 * previous;
            ring[idx] = internal;
            v = previous - 0.5 * internal;
            const int p = apos[s] + kBlk;
            apos[s] = p >= D ? p - D : p;
        }
        tone_in[((k - 1) & 1) * kBlk + lane] = v;
    }
}

__device__ void fdn_tone(const FdnJobDev &job, const double *tone_in, double *tone_out, int blocks, int iterations,
                         int total) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    Biquad tone;
    tone.load(job.tone[lane < 6 ? lane : 0]);
    if (lane >= 6) tone.b0 = tone.b1 = tone.b2 = tone.a1 = tone.a2 = 0.0;
    static_assert(kToneSkew == 2, "the shuffle is consumed one step after it is issued");
    // Tone section `lane` works on sample g - kToneSkew * lane at step g; its input is the previous
    // section's output of step g - kToneSkew, fed one step ahead like the line sections.
    double received = 0.0, carry = 0.0, v = 0.0;
    const int preroll = job.preroll;
    double *out = job.out;
    // section 5 stages its output of step base + t in tone_out[t]; the warp writes the block out after it
    const bool last_section = lane == 5;
    auto flush = [&](int base, int count) {
        __syncwarp();
        const int m = base + lane - kToneLag;
        if (lane < count && m >= preroll && m < total) out[m - preroll] = tone_out[lane];
        __syncwarp();
    };
    for (int k = 0; k < iterations; ++k) {
        block_barrier();
        if (k < 2 || k > blocks + 1) continue;
        const int base = (k - 2) * kBlk;
        const double *in = tone_in + ((k - 2) & 1) * kBlk;
        v = tone.feed(lane == 0 ? in[0] : carry);
#pragma unroll
        for (int t = 0; t < kBlk; ++t) {
            const double y = tone.step(v);
            const double next_in = lane == 0 ? in[(t + 1) & (kBlk - 1)] : received;
            received = __shfl_up_sync(full, y, 1);
            if (t + 1 < kBlk) v = tone.feed(next_in);
            else carry = next_in;
            if (last_section) tone_out[t] = y;
        }
        flush(base, kBlk);
    }
    // drain: inputs past the last sample are zero
    v = tone.feed(lane == 0 ? 0.0 : carry);
    for (int t = 0; t < kToneLag; ++t) {
        const double y = tone.step(v);
        const double next_in = lane == 0 ? 0.0 : received;
        received = __shfl_up_sync(full, y, 1);
        v = tone.feed(next_in);
        if (last_section) tone_out[t] = y;
    }
    flush(blocks * kBlk, kToneLag);
}

__global__ void __launch_bounds__(kFdnThreads) fdn_kernel(const FdnJobDev *jobs, double *pool) {
    extern __shared__ __align__(16) double smem[];
    double *stage = smem;
    double *rows = stage + kStageDoubles;
    double *tone_in = rows + kRing * kRowStride;
    double *tone_out = tone_in + 2 * kBlk;
    double *ap = tone_out + kBlk;
    __shared__ int s_start[kLines], s_delay[kLines];
    const FdnJobDev &job = jobs[blockIdx.x];
    const int total = job.preroll + job.num_samples;
    const int blocks = (total + kBlk - 1) / kBlk;
    // every warp passes the block barrier `iterations` times: the lines finish block b in iteration b + 1,
    // the mix takes it in iteration b + 1 and the tone in iteration b + 2
    const int iterations = blocks + 2;
    const int ap_total = job.allpass_start[AC_FDN_ALLPASS - 1] + job.allpass[AC_FDN_ALLPASS - 1];
    for (int i = threadIdx.x; i < ap_total; i += blockDim.x) ap[i] = 0.0;
    if (threadIdx.x < kLines) {
        s_start[threadIdx.x] = job.line_start[threadIdx.x];
        s_delay[threadIdx.x] = job.delays[threadIdx.x];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    if (warp < kLineWarps)
        fdn_lines(job, pool + job.pool, stage, rows, s_start, s_delay, iterations);
    else if (warp == kLineWarps)
        fdn_mix(job, pool + job.pool, rows, tone_in, ap, s_start, s_delay, blocks, iterations);
    else
        fdn_tone(job, tone_in, tone_out, blocks, iterations, total);
}

// ---- the hybrid tail ------------------------------------------------------

struct LateJobDev {
    const double *traced;
    const double *fdn;
    float *out;
    float *component;
    double *stats;
    float *bands;     // workspace: [6, N] band-limited FDN
    double rt60[6];
    int32_t start[6];
    int32_t end[6];
    int32_t anchor[6];
    int32_t changed_from;
    int32_t num_samples;
    int32_t bin_samples;
    int32_t rate_index;
};

// bandlimit_band_signals(np.repeat(raw_fdn[None, :], 6, axis=0)): every band
// filters the same impulse.  Unit = job * 6 + band, four per warp.
__global__ void __launch_bounds__(32) late_band_kernel(const LateJobDev *jobs, int num_units, int longest,
                                                       const __grid_constant__ ac_synth_batch_config cfg) {
    const int lane = threadIdx.x & 31;
    const int unit = blockIdx.x * 4 + (lane >> 3);
    const bool valid_unit = unit < num_units;
    const LateJobDev &job = jobs[valid_unit ? unit / 6 : 0];
    const int band = valid_unit ? unit % 6 : 0;
    const int n_len = valid_unit ? job.num_samples : 0;
    filter_units(job.fdn, job.bands + static_cast<int64_t>(band) * job.num_samples, n_len, valid_unit, band,
                 cfg.crossover[job.rate_index], longest + kLag + 2);
}

constexpr int kMixThreads = 256;

// Sum of one value per thread over the block, in a fixed order; every thread gets the total.
__device__ double block_sum(double v, double *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double total = 0.0;
    for (int w = 0; w < kMixThreads / 32; ++w) total += scratch[w];
    return total;
}

constexpr double kLn10 = 2.302585092994046;  // the float64 nearest ln(10)

// _late_tail_start_power (steam_rt.py:2473-2497) for one band; every thread gets the result.
__device__ double start_power(const double *x, int n_len, int anchor, double rt60, int fs, int bs, double *scratch,
                              double *bin_energy, int *found_bins, double *found_energy) {
    anchor = anchor < 0 ? 0 : (anchor > n_len ? n_len : anchor);
    const int hi = anchor + bs < n_len ? anchor + bs : n_len;
    double acc = 0.0;
    for (int n = anchor + threadIdx.x; n < hi; n += blockDim.x) acc += x[n] * x[n];
    const double here = block_sum(acc, scratch);
    const double measured = hi > anchor ? here / static_cast<double>(hi - anchor) : 0.0;
    if (anchor <= 0) return measured;
    const int nb = (anchor + bs - 1) / bs;
    __shared__ int s_found;
    if (threadIdx.x == 0) s_found = 0;
    __syncthreads();
    // the last five bins with energy above 1e-18, newest first, a block of bins at a time
    for (int top = nb - 1; top >= 0; top -= kMixThreads) {
        const int i = top - static_cast<int>(threadIdx.x);
        double e = 0.0;
        if (i >= 0) {
            const int end = (i + 1) * bs < anchor ? (i + 1) * bs : anchor;
            for (int n = i * bs; n < end; ++n) e += x[n] * x[n];
        }
        bin_energy[threadIdx.x] = e;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int t = 0; t < kMixThreads && s_found < 5 && top - t >= 0; ++t) {
                if (bin_energy[t] > 1e-18) {
                    found_bins[s_found] = top - t;
                    found_energy[s_found] = bin_energy[t];
                    ++s_found;
                }
            }
        }
        __syncthreads();
        if (s_found >= 5) break;
    }
    const int count = s_found;
    if (count == 0) return measured;
    // median of the decayed estimates (np.median: the middle value, or the mean of the two middle ones)
    const double decay = 6.0 * kLn10 / (rt60 > 0.1 ? rt60 : 0.1);
    double est[5];
    for (int j = 0; j < count; ++j) {
        const double centre = (static_cast<double>(found_bins[j]) + 0.5) * bs;
        double elapsed = (static_cast<double>(anchor) - centre) / static_cast<double>(fs > 1 ? fs : 1);
        elapsed = elapsed > 0.0 ? elapsed : 0.0;
        est[j] = (found_energy[j] / bs) * exp(-decay * elapsed);
    }
    for (int a = 1; a < count; ++a)
        for (int b = a; b > 0 && est[b - 1] > est[b]; --b) {
            const double t = est[b];
            est[b] = est[b - 1];
            est[b - 1] = t;
        }
    const double median = (count & 1) ? est[count / 2] : (est[count / 2 - 1] + est[count / 2]) / 2.0;
    return measured > median ? measured : median;
}

__global__ void __launch_bounds__(kMixThreads) late_mix_kernel(const LateJobDev *jobs,
                                                               const __grid_constant__ ac_synth_batch_config cfg) {
    __shared__ double scratch[kMixThreads / 32];
    __shared__ double bin_energy[kMixThreads];
    __shared__ int found_bins[5];
    __shared__ double found_energy[5];
    const LateJobDev &job = jobs[blockIdx.x / 6];
    const int band = blockIdx.x % 6;
    const int N = job.num_samples;
    const int fs = cfg.sample_rates[job.rate_index];
    const double *x = job.traced + static_cast<int64_t>(band) * N;
    const float *f = job.bands + static_cast<int64_t>(band) * N;
    const double rt60 = job.rt60[band];
    const int s = job.start[band], e = job.end[band];
    double scale = 1.0, power = 0.0, fdn_energy = 0.0;
    if (rt60 > 0.0) {
        const int anchor = job.anchor[band];
        power = start_power(x, N, anchor, rt60, fs, job.bin_samples, scratch, bin_energy, found_bins, found_energy);
        const double decay = 6.0 * kLn10 / (rt60 > 0.1 ? rt60 : 0.1);
        double target = 0.0, unit = 0.0;
        for (int k = threadIdx.x; k < N - anchor; k += blockDim.x) {
            target += power * exp(-decay * static_cast<double>(k) / static_cast<double>(fs));
            const double v = static_cast<double>(f[anchor + k]);
            unit += v * v;
        }
        target = block_sum(target, scratch);
        unit = block_sum(unit, scratch);
        scale = target > 0.0 ? sqrt(target / (unit > 1e-24 ? unit : 1e-24)) : 0.0;
        double acc = 0.0;
        for (int n = s + threadIdx.x; n < N; n += blockDim.x) {
            const double v = static_cast<double>(f[n]) * scale;
            acc += v * v;
        }
        fdn_energy = block_sum(acc, scratch);
    }
    // equal-power crossfade: alpha = np.linspace(1, 0, ramp, endpoint=False) = k * (-1 / ramp) + 1
    const int ramp = e - s > 1 ? e - s : 1;
    const double step = -1.0 / static_cast<double>(ramp);
    float *out = job.out + static_cast<int64_t>(band) * N;
    float *comp = job.component + static_cast<int64_t>(band) * N;
    double traced_tail = 0.0, rendered_tail = 0.0, comp_energy = 0.0;
    int changed = 0;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const double t = x[n];
        double o = t;
        double c = 0.0;
        if (n >= s) {
            double w = 1.0;
            if (n < s + ramp) {
                const double alpha = static_cast<double>(n - s) * step + 1.0;
                if (n < e) o = o * sqrt(alpha);
                w = sqrt(1.0 - alpha);
            }
            c = (static_cast<double>(f[n]) * scale) * w;
            traced_tail += t * t;
        }
        if (n >= e) o = 0.0;
        o = o + c;
        out[n] = static_cast<float>(o);
        comp[n] = static_cast<float>(c);
        if (n >= s) rendered_tail += o * o;
        comp_energy += c * c;
        if (n >= job.changed_from && !(fabs(o - t) <= 1e-12 + 1e-7 * fabs(t))) changed = 1;
    }
    traced_tail = block_sum(traced_tail, scratch);
    rendered_tail = block_sum(rendered_tail, scratch);
    comp_energy = block_sum(comp_energy, scratch);
    changed = __syncthreads_or(changed);
    if (threadIdx.x == 0) {
        double *st = job.stats + band * AC_LATE_STATS;
        st[AC_LATE_SCALE] = scale;
        st[AC_LATE_POWER] = power;
        st[AC_LATE_FDN_ENERGY] = fdn_energy;
        st[AC_LATE_TRACED_TAIL] = traced_tail;
        st[AC_LATE_RENDERED_TAIL] = rendered_tail;
        st[AC_LATE_COMPONENT] = comp_energy;
        st[AC_LATE_CHANGED] = changed ? 1.0 : 0.0;
        st[7] = 0.0;
    }
}

// ---- host side -------------------------------------------------------------

struct FdnLayout {
    size_t jobs, pool, total;
    int64_t pool_doubles;
    int max_allpass_doubles;
};

int check_fdn(const ac_fdn_job *jobs, int32_t num_jobs, bool need_buffers, FdnLayout *out) {
    if (num_jobs < 0 || (num_jobs > 0 && !jobs)) return fail(AC_ERR_INVALID, "fdn: null argument");
    if (num_jobs > (1 << 24)) return fail(AC_ERR_CAPACITY, "fdn batch of %d jobs is too large", num_jobs);
    FdnLayout l{};
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_fdn_job &job = jobs[j];
        int64_t lines = 0;
        for (int i = 0; i < kLines; ++i) {
            if (job.delays[i] < AC_FDN_MIN_DELAY || job.delays[i] > (1 << 26))
                return fail(AC_ERR_INVALID, "fdn job %d: delay %d of line %d outside [%d, 2^26]", j, job.delays[i], i,
                            AC_FDN_MIN_DELAY);
            lines += job.delays[i];
        }
        if (lines > 0x7FFFFFFF) return fail(AC_ERR_CAPACITY, "fdn job %d: delay lines too long", j);
        int ap = 0;
        for (int s = 0; s < AC_FDN_ALLPASS; ++s) {
            if (job.allpass_delays[s] <= kBlk || job.allpass_delays[s] > AC_FDN_MAX_ALLPASS)
                return fail(AC_ERR_INVALID, "fdn job %d: all-pass delay %d outside [%d, %d]", j, job.allpass_delays[s],
                            kBlk + 1, AC_FDN_MAX_ALLPASS);
            ap += job.allpass_delays[s];
        }
        if (job.num_samples < 0 || job.preroll < 0 ||
            static_cast<int64_t>(job.num_samples) + job.preroll > (int64_t{1} << 30))
            return fail(AC_ERR_INVALID, "fdn job %d: bad length (%d + %d)", j, job.preroll, job.num_samples);
        if (need_buffers && job.num_samples > 0 && !job.out) return fail(AC_ERR_INVALID, "fdn job %d: null output", j);
        for (int i = 0; i < kLines * 6 * 5; ++i)
            if (!std::isfinite((&job.absorptive[0][0][0])[i]))
                return fail(AC_ERR_INVALID, "fdn job %d: non-finite absorptive coefficient", j);
        for (int i = 0; i < 6 * 5; ++i)
            if (!std::isfinite((&job.tone[0][0])[i])) return fail(AC_ERR_INVALID, "fdn job %d: non-finite tone coefficient", j);
        l.pool_doubles += lines;
        l.max_allpass_doubles = std::max(l.max_allpass_doubles, ap);
    }
    size_t off = 0;
    l.jobs = off; off = align256(off + static_cast<size_t>(num_jobs) * sizeof(FdnJobDev));
    l.pool = off; off = align256(off + static_cast<size_t>(l.pool_doubles) * sizeof(double));
    l.total = off;
    *out = l;
    return AC_OK;
}

std::mutex g_smem_mutex;
int g_smem_set[64] = {0};

// Opt the FDN kernel into the dynamic shared memory it needs on this device.
int ensure_fdn_smem(int bytes) {
    int dev = 0;
    AC_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_smem_mutex);
    const int slot = dev & 63;
    if (g_smem_set[slot] >= bytes) return AC_OK;
    AC_CUDA_TRY(cudaFuncSetAttribute(fdn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    g_smem_set[slot] = bytes;
    return AC_OK;
}

struct LateLayout {
    size_t jobs, bands, total;
    int64_t band_floats;
    int longest;
};

int check_late(const ac_late_tail_job *jobs, int32_t num_jobs, const ac_synth_batch_config *cfg, bool need_buffers,
               LateLayout *out) {
    if (num_jobs < 0 || (num_jobs > 0 && !jobs) || !cfg) return fail(AC_ERR_INVALID, "late tail: null argument");
    if (cfg->num_rates < 1 || cfg->num_rates > AC_SYNTH_MAX_RATES)
        return fail(AC_ERR_INVALID, "late tail: num_rates must be 1..%d", AC_SYNTH_MAX_RATES);
    if (num_jobs > (1 << 24)) return fail(AC_ERR_CAPACITY, "late tail batch of %d jobs is too large", num_jobs);
    LateLayout l{};
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_late_tail_job &job = jobs[j];
        const int N = job.num_samples;
        if (N < 1 || N > (1 << 28)) return fail(AC_ERR_INVALID, "late tail job %d: num_samples %d", j, N);
        if (job.bin_samples < 1) return fail(AC_ERR_INVALID, "late tail job %d: bin_samples must be positive", j);
        if (job.rate_index < 0 || job.rate_index >= cfg->num_rates || cfg->sample_rates[job.rate_index] < 1)
            return fail(AC_ERR_INVALID, "late tail job %d: bad rate_index %d", j, job.rate_index);
        for (int b = 0; b < 6; ++b) {
            if (job.start[b] < 0 || job.start[b] >= N || job.end[b] <= job.start[b] || job.end[b] > N)
                return fail(AC_ERR_INVALID, "late tail job %d band %d: crossfade [%d, %d) outside [0, %d)", j, b,
                            job.start[b], job.end[b], N);
            if (job.anchor[b] < 0 || job.anchor[b] > N)
                return fail(AC_ERR_INVALID, "late tail job %d band %d: anchor %d outside [0, %d]", j, b, job.anchor[b], N);
            if (!std::isfinite(job.rt60[b])) return fail(AC_ERR_INVALID, "late tail job %d: non-finite rt60", j);
        }
        if (job.changed_from < 0) return fail(AC_ERR_INVALID, "late tail job %d: negative changed_from", j);
        if (need_buffers && (!job.traced || !job.fdn || !job.out || !job.fdn_component || !job.stats))
            return fail(AC_ERR_INVALID, "late tail job %d: null buffer", j);
        l.band_floats += static_cast<int64_t>(align256(6 * static_cast<size_t>(N) * sizeof(float)) / sizeof(float));
        l.longest = std::max(l.longest, N);
    }
    size_t off = 0;
    l.jobs = off;  off = align256(off + static_cast<size_t>(num_jobs) * sizeof(LateJobDev));
    l.bands = off; off = align256(off + static_cast<size_t>(l.band_floats) * sizeof(float));
    l.total = off;
    *out = l;
    return AC_OK;
}

}  // namespace
}  // namespace ac

extern "C" int ac_fdn_workspace_size(const ac_fdn_job *jobs, int32_t num_jobs, size_t *bytes) {
    if (!bytes) return ac::fail(AC_ERR_INVALID, "ac_fdn_workspace_size: null argument");
    ac::FdnLayout l;
    const int rc = ac::check_fdn(jobs, num_jobs, false, &l);
    if (rc != AC_OK) return rc;
    *bytes = l.total;
    return AC_OK;
}

extern "C" int ac_fdn_impulse(const ac_fdn_job *jobs, int32_t num_jobs, void *workspace, size_t workspace_bytes,
                              void *host_staging, void *stream_ptr) {
    ac::NvtxRange nvtx_range("ac_fdn_impulse");
    ac::FdnLayout l;
    const int rc = ac::check_fdn(jobs, num_jobs, true, &l);
    if (rc != AC_OK) return rc;
    if (num_jobs == 0) return AC_OK;
    if (!workspace || workspace_bytes < l.total)
        return ac::fail(AC_ERR_CAPACITY, "fdn workspace too small: %zu < %zu", workspace_bytes, l.total);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const size_t table_bytes = static_cast<size_t>(num_jobs) * sizeof(ac::FdnJobDev);
    std::vector<unsigned char> local;
    unsigned char *host = static_cast<unsigned char *>(host_staging);
    if (!host) {
        local.assign(table_bytes, 0);
        host = local.data();
    }
    int64_t pool = 0;
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_fdn_job &in = jobs[j];
        ac::FdnJobDev d{};
        std::memcpy(d.absorptive, in.absorptive, sizeof(d.absorptive));
        std::memcpy(d.tone, in.tone, sizeof(d.tone));
        int32_t off = 0;
        for (int i = 0; i < ac::kLines; ++i) {
            d.delays[i] = in.delays[i];
            d.line_start[i] = off;
            off += in.delays[i];
        }
        int32_t ap = 0;
        for (int s = 0; s < AC_FDN_ALLPASS; ++s) {
            d.allpass[s] = in.allpass_delays[s];
            d.allpass_start[s] = ap;
            ap += in.allpass_delays[s];
        }
        d.num_samples = in.num_samples;
        d.preroll = in.preroll;
        d.out = in.out;
        d.pool = pool;
        pool += off;
        std::memcpy(host + j * sizeof(ac::FdnJobDev), &d, sizeof(d));
    }
    AC_CUDA_TRY(cudaMemcpyAsync(ws + l.jobs, host, table_bytes, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));  // pageable source must stay alive
    AC_CUDA_TRY(cudaMemsetAsync(ws + l.pool, 0, static_cast<size_t>(l.pool_doubles) * sizeof(double), stream));
    const int smem = ac::kFixedSmem + l.max_allpass_doubles * static_cast<int>(sizeof(double));
    const int prc = ac::ensure_fdn_smem(smem);
    if (prc != AC_OK) return prc;
    ac::fdn_kernel<<<num_jobs, ac::kFdnThreads, smem, stream>>>(reinterpret_cast<const ac::FdnJobDev *>(ws + l.jobs),
                                                   reinterpret_cast<double *>(ws + l.pool));
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

extern "C" int ac_late_tail_workspace_size(const ac_late_tail_job *jobs, int32_t num_jobs,
                                           const ac_synth_batch_config *config, size_t *bytes) {
    if (!bytes) return ac::fail(AC_ERR_INVALID, "ac_late_tail_workspace_size: null argument");
    ac::LateLayout l;
    const int rc = ac::check_late(jobs, num_jobs, config, false, &l);
    if (rc != AC_OK) return rc;
    *bytes = l.total;
    return AC_OK;
}

extern "C" int ac_late_tail(const ac_late_tail_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                            void *workspace, size_t workspace_bytes, void *host_staging, void *stream_ptr) {
    ac::NvtxRange nvtx_range("ac_late_tail");
    ac::LateLayout l;
    const int rc = ac::check_late(jobs, num_jobs, config, true, &l);
    if (rc != AC_OK) return rc;
    if (num_jobs == 0) return AC_OK;
    if (!workspace || workspace_bytes < l.total)
        return ac::fail(AC_ERR_CAPACITY, "late tail workspace too small: %zu < %zu", workspace_bytes, l.total);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const size_t table_bytes = static_cast<size_t>(num_jobs) * sizeof(ac::LateJobDev);
    std::vector<unsigned char> local;
    unsigned char *host = static_cast<unsigned char *>(host_staging);
    if (!host) {
        local.assign(table_bytes, 0);
        host = local.data();
    }
    float *bands = reinterpret_cast<float *>(ws + l.bands);
    int64_t band_off = 0;
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_late_tail_job &in = jobs[j];
        ac::LateJobDev d{};
        d.traced = in.traced;
        d.fdn = in.fdn;
        d.out = in.out;
        d.component = in.fdn_component;
        d.stats = in.stats;
        d.bands = bands + band_off;
        band_off += static_cast<int64_t>(ac::align256(6 * static_cast<size_t>(in.num_samples) * sizeof(float)) /
                                         sizeof(float));
        for (int b = 0; b < 6; ++b) {
            d.rt60[b] = in.rt60[b];
            d.start[b] = in.start[b];
            d.end[b] = in.end[b];
            d.anchor[b] = in.anchor[b];
        }
        d.changed_from = in.changed_from;
        d.num_samples = in.num_samples;
        d.bin_samples = in.bin_samples;
        d.rate_index = in.rate_index;
        std::memcpy(host + j * sizeof(ac::LateJobDev), &d, sizeof(d));
    }
    AC_CUDA_TRY(cudaMemcpyAsync(ws + l.jobs, host, table_bytes, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));
    const ac::LateJobDev *d_jobs = reinterpret_cast<const ac::LateJobDev *>(ws + l.jobs);
    const int units = 6 * num_jobs;
    ac::late_band_kernel<<<(units + 3) / 4, 32, 0, stream>>>(d_jobs, units, l.longest, *config);
    AC_CUDA_TRY(cudaGetLastError());
    ac::late_mix_kernel<<<units, ac::kMixThreads, 0, stream>>>(d_jobs, *config);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}
