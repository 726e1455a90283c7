// Echogram -> six band impulse responses on the GPU.
//
// Restates acoustic_agent/steam_rt.py:2205-2232 (reconstruct_band_irs) and
// :3070-3083 + :4131-4212 (bandlimit_band_signals, _band_limit, the biquad
// recursion) so that, given the same float32 echogram and noise, every output
// sample is bit-identical to the reference.  This file is compiled with
// -fmad=false: the reference evaluates each multiply and add separately in
// float64, and each biquad section hands its successor a float32-rounded signal.
//
// The raw band signals are materialised first by a fully parallel kernel.  The
// recursion itself is sequential in time, so parallelism comes from elsewhere:
// one warp is a systolic array of 8 four-section low-pass chains.  Lane
// (unit, chain, stage) runs one biquad section and passes its float32 output
// one lane up; section s runs two samples behind section s-1.  A "unit" is one band of one RIR: bands 1-4 need
// two chains (the low-pass at the upper and lower crossover, subtracted),
// bands 0 and 5 one.  Four units per warp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "common.h"
#include "philox.cuh"

namespace ac {
namespace {

constexpr int kSynthBands = 6;
constexpr double kSynthPi = 3.141592653589793;

struct SynthArgs {
    double crossover[100];
    double air_coefficients[6];
    double speed_of_sound;
    int32_t num_rirs;
    int32_t num_bins;
    int32_t spb;
    int32_t sample_rate;
};

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

struct SynthLayout {
    size_t amps, air, wtab, white, raw, total;
};

SynthLayout synth_layout(const ac_synth_params *p) {
    const size_t cells = static_cast<size_t>(p->num_rirs) * kSynthBands * p->num_bins;
    const size_t N = static_cast<size_t>(p->num_bins) * p->samples_per_bin;
    SynthLayout l{};
    size_t off = 0;
    l.amps = off; off = align256(off + cells * sizeof(double));
    l.air = off;  off = align256(off + (p->air ? 0 : cells * sizeof(double)));
    l.wtab = off; off = align256(off + static_cast<size_t>(p->samples_per_bin) * sizeof(double));
    l.white = off; off = align256(off + (p->rng_mode == AC_RNG_PHILOX ? N * sizeof(double) : 0));
    l.raw = off;  off = align256(off + static_cast<size_t>(p->num_rirs) * kSynthBands * N * sizeof(double));
    l.total = off;
    return l;
}

// Envelope amplitudes, air gains, interpolation weights and (Philox mode) noise.
__global__ void synth_prepare_kernel(const float *echo, const double *direct_delays, const __grid_constant__ SynthArgs a,
                                     double *amps, double *air, double *wtab, double *white, uint64_t seed) {
    const size_t cells = static_cast<size_t>(a.num_rirs) * kSynthBands * a.num_bins;
    const size_t N = static_cast<size_t>(a.num_bins) * a.spb;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells; i += stride) {
        // numpy keeps a float32 echogram in float32: clip, divide by float32(4pi), sqrt.
        const float e = echo[i];
        const float cl = e > 0.0f ? e : 0.0f;
        const float amp = sqrtf(cl / static_cast<float>(4.0 * kSynthPi));
        amps[i] = e < static_cast<float>(1e-9) ? 0.0 : static_cast<double>(amp);
        if (air) {
            const int bin = static_cast<int>(i % a.num_bins);
            const int band = static_cast<int>((i / a.num_bins) % kSynthBands);
            const int j = static_cast<int>(i / (static_cast<size_t>(a.num_bins) * kSynthBands));
            // steam_rt.py:2196-2198, path time at the bin centre
            const double t = direct_delays[j] + ((static_cast<double>(bin) + 0.5) * a.spb) / a.sample_rate;
            const double dist = (t > 0.0 ? t : 0.0) * (a.speed_of_sound > 0.0 ? a.speed_of_sound : 0.0);
            const double coeff = a.air_coefficients[band] > 0.0 ? a.air_coefficients[band] : 0.0;
            air[i] = exp(-coeff * dist);
        }
    }
    for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < static_cast<size_t>(a.spb); k += stride)
        wtab[k] = static_cast<double>(k) / static_cast<double>(a.spb);
    if (white) {
        for (size_t n = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; n < N; n += stride) {
            const u32x4 r = noise_draw(seed, static_cast<uint32_t>(n >> 1));
            const double u = (n & 1) ? u01_53(r.z, r.w) : u01_53(r.x, r.y);
            white[n] = -1.0 + 2.0 * u;
        }
    }
}

// Raw band signals (steam_rt.py:2221-2230): the envelope interpolated from the
// previous bin, times the bin's air gain, times the noise -- every sample
// independent, so one thread per sample.
__global__ void synth_raw_kernel(const double *amps, const double *air, const double *wtab, const double *white,
                                 size_t white_stride, const __grid_constant__ SynthArgs a, double *raw) {
    const size_t N = static_cast<size_t>(a.num_bins) * a.spb;
    const size_t total = static_cast<size_t>(a.num_rirs) * kSynthBands * N;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t unit = i / N;            // j * 6 + band
        const size_t n = i - unit * N;
        const size_t j = unit / kSynthBands;
        const int bin = static_cast<int>(n / a.spb);
        const int k = static_cast<int>(n - static_cast<size_t>(bin) * a.spb);
        const size_t row = unit * a.num_bins;
        const double w = wtab[k];
        const double cur = amps[row + bin];
        const double prev = bin == 0 ? cur : amps[row + bin - 1];
        double seg = (1.0 - w) * prev + w * cur;
        seg = seg * air[row + bin];
        raw[i] = seg * white[j * white_stride + n];
    }
}

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

constexpr int kPrefetch = 8;
constexpr int kSkew = 2;  // iterations between consecutive sections
constexpr int kLag = kSkew * 3;  // section 3 runs kLag samples behind section 0

// Lane (unit, chain, stage): section `stage` works on sample it - kSkew*stage.
// The float32 output it produces at iteration it is shuffled one lane up at
// once but consumed there only at it + kSkew, so the shuffle latency never sits
// on the recursion's critical path -- only the section's own y dependency does.
//
// The body is branch-free: before a section's first real sample its input is
// +0.0, and a section whose inputs and state are all +0.0 produces exactly +0.0
// and keeps its state at +0.0 (every product is +0.0 or -0.0 and the sums come
// out +0.0), so the steps while the pipeline fills change nothing.
__global__ void __launch_bounds__(128) synth_filter_kernel(const double *raw, const __grid_constant__ SynthArgs a,
                                                           float *out) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5);
    const int stage = lane & 3;
    const int chain = (lane >> 2) & 1;
    const int unit = warp * 4 + (lane >> 3);
    const int units = a.num_rirs * kSynthBands;
    const bool valid_unit = unit < units;
    const int band = valid_unit ? unit % kSynthBands : 0;
    int cutoff;
    bool active;
    if (band == 0) { cutoff = 0; active = chain == 0; }
    else if (band == kSynthBands - 1) { cutoff = 4; active = chain == 0; }
    else { cutoff = chain == 0 ? band : band - 1; active = true; }
    active = active && valid_unit;
    const double *co = a.crossover + cutoff * 20 + stage * 5;
    Section sec{co[0], co[1], co[2], co[3], co[4], 0.0, 0.0, 0.0, 0.0};
    const bool emits = stage == 3 && chain == 0 && active;
    const bool is_first = stage == 0;
    const int mode = band == 0 ? 0 : (band == kSynthBands - 1 ? 2 : 1);

    const int N = a.num_bins * a.spb;
    const double *x = raw + static_cast<size_t>(valid_unit ? unit : 0) * static_cast<size_t>(N);
    float *out_row = out + static_cast<size_t>(valid_unit ? unit : 0) * static_cast<size_t>(N);

    double ahead[kPrefetch], prev[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
        ahead[u] = (valid_unit && u < N) ? __ldg(x + u) : 0.0;
        prev[u] = 0.0;
    }
    float q1 = 0.0f;  // value the previous section sent last iteration (this section's input next iteration)
    // input part of the first sample (its input is ahead[0] for section 0 and +0.0 otherwise)
    double v = sec.feed(is_first ? ahead[0] : 0.0);
    const int iterations = N + kLag;
    for (int base = 0; base < iterations; base += kPrefetch) {
        double next[kPrefetch];
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            const int m = base + kPrefetch + u;
            next[u] = (valid_unit && m < N) ? __ldg(x + m) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u) {
            const int it = base + u;
            const float y = sec.step(v);
            // input of the next iteration: section 0 reads the prefetched signal,
            // later sections the value their predecessor sent two iterations ago
            const double in_next = is_first ? (u + 1 < kPrefetch ? ahead[u + 1] : next[0]) : static_cast<double>(q1);
            v = sec.feed(in_next);
            const float sent = __shfl_up_sync(full, y, 1);
            const float lower = __shfl_down_sync(full, y, 4);
            q1 = sent;
            // x[it - kLag] is still in registers from the prefetch
            const double x_n = (u >= kLag) ? ahead[u - kLag] : prev[u + kPrefetch - kLag];
            const float band5 = static_cast<float>(x_n - static_cast<double>(y));
            const float o = mode == 0 ? y : (mode == 2 ? band5 : y - lower);
            if (emits && it >= kLag && it < iterations) out_row[it - kLag] = o;
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

extern "C" int ac_synth_workspace_size(const ac_synth_params *p, size_t *bytes) {
    if (!p || !bytes) return ac::fail(AC_ERR_INVALID, "ac_synth_workspace_size: null argument");
    if (p->num_rirs < 0 || p->num_bins < 1 || p->samples_per_bin < 1)
        return ac::fail(AC_ERR_INVALID, "synthesis sizes must be positive");
    *bytes = ac::synth_layout(p).total;
    return AC_OK;
}

extern "C" int ac_synthesize(const float *echograms, const ac_synth_params *p, float *band_irs, void *workspace,
                             size_t workspace_bytes, void *stream_ptr) {
    if (!p || !echograms || !band_irs) return ac::fail(AC_ERR_INVALID, "ac_synthesize: null argument");
    if (p->num_rirs < 0 || p->num_bins < 1 || p->samples_per_bin < 1 || p->sample_rate < 1)
        return ac::fail(AC_ERR_INVALID, "synthesis sizes must be positive");
    const int64_t N = static_cast<int64_t>(p->num_bins) * p->samples_per_bin;
    if (N + 3 > 0x7FFFFFFF) return ac::fail(AC_ERR_CAPACITY, "signal of %lld samples is too long", (long long)N);
    if (p->rng_mode == AC_RNG_REFERENCE && !p->white) return ac::fail(AC_ERR_INVALID, "reference mode needs white noise");
    if (!p->air && !p->direct_delays) return ac::fail(AC_ERR_INVALID, "need an air table or the direct delays");
    if (p->num_rirs == 0) return AC_OK;
    const ac::SynthLayout l = ac::synth_layout(p);
    if (!workspace || workspace_bytes < l.total)
        return ac::fail(AC_ERR_CAPACITY, "synthesis workspace too small: %zu < %zu", workspace_bytes, l.total);
    ac::SynthArgs a;
    std::memcpy(a.crossover, p->crossover, sizeof(a.crossover));
    std::memcpy(a.air_coefficients, p->air_coefficients, sizeof(a.air_coefficients));
    a.speed_of_sound = p->speed_of_sound;
    a.num_rirs = p->num_rirs;
    a.num_bins = p->num_bins;
    a.spb = p->samples_per_bin;
    a.sample_rate = p->sample_rate;
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    double *amps = reinterpret_cast<double *>(ws + l.amps);
    double *air = p->air ? nullptr : reinterpret_cast<double *>(ws + l.air);
    double *wtab = reinterpret_cast<double *>(ws + l.wtab);
    double *white = p->rng_mode == AC_RNG_PHILOX ? reinterpret_cast<double *>(ws + l.white) : nullptr;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t cells = static_cast<size_t>(p->num_rirs) * 6 * p->num_bins;
    const size_t work = std::max<size_t>(cells, static_cast<size_t>(white ? N : p->samples_per_bin));
    const int grid = static_cast<int>(std::min<size_t>((work + 255) / 256, 8192));
    ac::synth_prepare_kernel<<<grid, 256, 0, stream>>>(echograms, p->direct_delays, a, amps, air, wtab, white, p->seed);
    AC_CUDA_TRY(cudaGetLastError());
    const double *air_table = p->air ? p->air : air;
    const double *noise = white ? white : p->white;
    const size_t stride = (white || p->white_shared) ? 0 : static_cast<size_t>(N);
    double *raw = reinterpret_cast<double *>(ws + l.raw);
    const size_t samples = static_cast<size_t>(p->num_rirs) * 6 * static_cast<size_t>(N);
    const int raw_grid = static_cast<int>(std::min<size_t>((samples + 255) / 256, 65536));
    ac::synth_raw_kernel<<<raw_grid, 256, 0, stream>>>(amps, air_table, wtab, noise, stride, a, raw);
    AC_CUDA_TRY(cudaGetLastError());
    const int units = p->num_rirs * 6;
    const int warps = (units + 3) / 4;
    const int threads = 32;  // one warp per block: spread the sequential chains over all SMs
    ac::synth_filter_kernel<<<warps, threads, 0, stream>>>(raw, a, band_irs);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

// ---------------------------------------------------------------------------
// Band synthesis without any device allocation (ac_synthesize_static).
//
// For callers that must not allocate device memory themselves or through us:
// a real-time audio thread, where cudaMalloc can block on the driver for
// milliseconds, or a host engine that owns the whole device-memory budget and
// forbids third-party allocations.  The workspace lives in this file-scope
// array instead; every GPU that loads the library holds it until the process
// exits.  Every call shares it, and it keeps the last call's contents: all
// regions a call reads are written earlier in the same call, so nothing needs
// clearing, but calls that overlap on the GPU (different streams, or threads)
// race on it and must be serialised by the caller.

namespace {

static __device__ __align__(256) unsigned char g_synth_scratch[AC_SYNTH_STATIC_BYTES];

std::mutex g_scratch_mutex;
void *g_scratch_ptr[64] = {nullptr};

// Device address of the static scratch for the current device, looked up once
// per device (the host-side symbol is only a stand-in, never a device address).
int static_scratch(void **out) {
    int device = 0;
    AC_CUDA_TRY(cudaGetDevice(&device));
    if (device < 0 || device >= 64) return ac::fail(AC_ERR_UNSUPPORTED, "device ordinal %d out of range", device);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[device]) {
        void *ptr = nullptr;
        AC_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_synth_scratch));
        g_scratch_ptr[device] = ptr;
    }
    *out = g_scratch_ptr[device];
    return AC_OK;
}

}  // namespace

extern "C" int ac_synthesize_static(const float *echograms, const ac_synth_params *p, float *band_irs,
                                    void *stream_ptr) {
    if (!p || !echograms || !band_irs) return ac::fail(AC_ERR_INVALID, "ac_synthesize_static: null argument");
    if (p->num_rirs < 0 || p->num_bins < 1 || p->samples_per_bin < 1 || p->sample_rate < 1)
        return ac::fail(AC_ERR_INVALID, "synthesis sizes must be positive");
    const int64_t N = static_cast<int64_t>(p->num_bins) * p->samples_per_bin;
    if (N + 3 > 0x7FFFFFFF) return ac::fail(AC_ERR_CAPACITY, "signal of %lld samples is too long", (long long)N);
    if (p->rng_mode == AC_RNG_REFERENCE && !p->white) return ac::fail(AC_ERR_INVALID, "reference mode needs white noise");
    if (!p->air && !p->direct_delays) return ac::fail(AC_ERR_INVALID, "need an air table or the direct delays");
    const ac::SynthLayout l = ac::synth_layout(p);
    if (l.total > static_cast<size_t>(AC_SYNTH_STATIC_BYTES))
        return ac::fail(AC_ERR_CAPACITY,
                        "synthesis of %d RIRs x %lld samples needs %zu bytes of scratch; the static scratch holds %zu: "
                        "split the RIRs over several calls",
                        p->num_rirs, (long long)N, l.total, static_cast<size_t>(AC_SYNTH_STATIC_BYTES));
    if (p->num_rirs == 0) return AC_OK;
    void *scratch = nullptr;
    const int rc = static_scratch(&scratch);
    if (rc != AC_OK) return rc;
    ac::SynthArgs a;
    std::memcpy(a.crossover, p->crossover, sizeof(a.crossover));
    std::memcpy(a.air_coefficients, p->air_coefficients, sizeof(a.air_coefficients));
    a.speed_of_sound = p->speed_of_sound;
    a.num_rirs = p->num_rirs;
    a.num_bins = p->num_bins;
    a.spb = p->samples_per_bin;
    a.sample_rate = p->sample_rate;
    unsigned char *ws = static_cast<unsigned char *>(scratch);
    double *amps = reinterpret_cast<double *>(ws + l.amps);
    double *air = p->air ? nullptr : reinterpret_cast<double *>(ws + l.air);
    double *wtab = reinterpret_cast<double *>(ws + l.wtab);
    double *white = p->rng_mode == AC_RNG_PHILOX ? reinterpret_cast<double *>(ws + l.white) : nullptr;
    double *raw = reinterpret_cast<double *>(ws + l.raw);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t cells = static_cast<size_t>(p->num_rirs) * 6 * p->num_bins;
    const size_t work = std::max<size_t>(cells, static_cast<size_t>(white ? N : p->samples_per_bin));
    const int grid = static_cast<int>(std::min<size_t>((work + 255) / 256, 8192));
    ac::synth_prepare_kernel<<<grid, 256, 0, stream>>>(echograms, p->direct_delays, a, amps, air, wtab, white, p->seed);
    AC_CUDA_TRY(cudaGetLastError());
    const double *air_table = p->air ? p->air : air;
    const double *noise = white ? white : p->white;
    const size_t stride = (white || p->white_shared) ? 0 : static_cast<size_t>(N);
    const size_t samples = static_cast<size_t>(p->num_rirs) * 6 * static_cast<size_t>(N);
    const int raw_grid = static_cast<int>(std::min<size_t>((samples + 255) / 256, 65536));
    ac::synth_raw_kernel<<<raw_grid, 256, 0, stream>>>(amps, air_table, wtab, noise, stride, a, raw);
    AC_CUDA_TRY(cudaGetLastError());
    const int warps = (p->num_rirs * 6 + 3) / 4;
    ac::synth_filter_kernel<<<warps, 32, 0, stream>>>(raw, a, band_irs);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}
