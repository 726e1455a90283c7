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
// recursion itself is sequential in time, so parallelism comes from elsewhere
// (band_filter.cuh): one warp is a systolic array of 8 four-section low-pass chains.  Lane
// (unit, chain, stage) runs one biquad section and passes its float32 output
// one lane up; section s runs kSkew samples behind section s-1.  A "unit" is
// one band of one RIR: bands 1-4 need two chains (the low-pass at the upper
// and lower crossover, subtracted), bands 0 and 5 one.  Four units per warp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "philox.cuh"
#include "band_filter.cuh"

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

__global__ void __launch_bounds__(128) synth_filter_kernel(const double *raw, const __grid_constant__ SynthArgs a,
                                                           float *out) {
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5);
    const int unit = warp * 4 + (lane >> 3);
    const int units = a.num_rirs * kSynthBands;
    const bool valid_unit = unit < units;
    const int band = valid_unit ? unit % kSynthBands : 0;
    const int N = a.num_bins * a.spb;
    const double *x = raw + static_cast<size_t>(valid_unit ? unit : 0) * static_cast<size_t>(N);
    float *out_row = out + static_cast<size_t>(valid_unit ? unit : 0) * static_cast<size_t>(N);
    filter_units(x, out_row, N, valid_unit, band, a.crossover, N + kLag + 2);
}

// ---- ragged batches (ac_synthesize_batch) ----------------------------------

// Device copy of one batch job plus its offsets into the shared arrays.
struct SynthJobDev {
    const float *echogram;
    float *band_irs;
    const double *white;
    const double *air;
    uint64_t seed;
    double direct_delay;
    double speed_of_sound;
    int32_t num_bins;
    int32_t spb;
    int32_t rate_index;
    int32_t rng_mode;
    int64_t cells;    // offset of this job's [6, bins] rows in the amps / air arrays
    int64_t samples;  // offset of this job's [6, N] raw rows, in units of 6 samples
};

// Largest j with prefix[j] <= i (prefix[0] = 0, strictly increasing).
__device__ __forceinline__ int owner(const int64_t *prefix, int num_jobs, int64_t i) {
    int lo = 0, hi = num_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void synth_batch_prepare_kernel(const SynthJobDev *jobs, const int64_t *cell_prefix, int num_jobs,
                                           const __grid_constant__ ac_synth_batch_config cfg, double *amps,
                                           double *air) {
    const int64_t cells = cell_prefix[num_jobs];
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < cells; i += stride) {
        const int j = owner(cell_prefix, num_jobs, i);
        const SynthJobDev &job = jobs[j];
        const int64_t local = i - job.cells;
        const int band = static_cast<int>(local / job.num_bins);
        const int bin = static_cast<int>(local - static_cast<int64_t>(band) * job.num_bins);
        // numpy keeps a float32 echogram in float32: clip, divide by float32(4pi), sqrt.
        const float e = job.echogram[local];
        const float cl = e > 0.0f ? e : 0.0f;
        const float amp = sqrtf(cl / static_cast<float>(4.0 * kSynthPi));
        amps[i] = e < static_cast<float>(1e-9) ? 0.0 : static_cast<double>(amp);
        if (job.air) {
            air[i] = job.air[local];
        } else {
            // steam_rt.py:2196-2198 and :2214-2227: clamped direct delay, path time at the bin centre
            const double delay = job.direct_delay > 0.0 ? job.direct_delay : 0.0;
            const int rate = cfg.sample_rates[job.rate_index];
            const double t = delay + ((static_cast<double>(bin) + 0.5) * job.spb) / rate;
            const double dist = (t > 0.0 ? t : 0.0) * (job.speed_of_sound > 0.0 ? job.speed_of_sound : 0.0);
            const double coeff = cfg.air_coefficients[band] > 0.0 ? cfg.air_coefficients[band] : 0.0;
            air[i] = exp(-coeff * dist);
        }
    }
}

// One thread per (job, sample): the noise value is drawn once and used by all six bands.
__global__ void synth_batch_raw_kernel(const SynthJobDev *jobs, const int64_t *sample_prefix, int num_jobs,
                                       const double *amps, const double *air, double *raw) {
    const int64_t total = sample_prefix[num_jobs];
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < total; i += stride) {
        const int j = owner(sample_prefix, num_jobs, i);
        const SynthJobDev &job = jobs[j];
        const int64_t n = i - sample_prefix[j];
        const int64_t N = static_cast<int64_t>(job.num_bins) * job.spb;
        const int bin = static_cast<int>(n / job.spb);
        const int k = static_cast<int>(n - static_cast<int64_t>(bin) * job.spb);
        const double w = static_cast<double>(k) / static_cast<double>(job.spb);
        double noise;
        if (job.rng_mode == AC_RNG_PHILOX) {
            const u32x4 r = noise_draw(job.seed, static_cast<uint32_t>(n >> 1));
            const double u = (n & 1) ? u01_53(r.z, r.w) : u01_53(r.x, r.y);
            noise = -1.0 + 2.0 * u;
        } else {
            noise = job.white[n];
        }
        double *row = raw + 6 * job.samples + n;
#pragma unroll
        for (int band = 0; band < kSynthBands; ++band) {
            const int64_t c = job.cells + static_cast<int64_t>(band) * job.num_bins + bin;
            const double cur = amps[c];
            const double prev = bin == 0 ? cur : amps[c - 1];
            double seg = (1.0 - w) * prev + w * cur;
            seg = seg * air[c];
            row[band * N] = seg * noise;
        }
    }
}

// Warp w runs units[4w .. 4w+3] (job << 3 | band, or -1); units are ordered
// longest job first, so the four units of a warp have similar lengths.
__global__ void __launch_bounds__(32) synth_batch_filter_kernel(const SynthJobDev *jobs, const int32_t *units,
                                                                int num_units,
                                                                const __grid_constant__ ac_synth_batch_config cfg,
                                                                const double *raw) {
    const int lane = threadIdx.x & 31;
    const int warp = static_cast<int>((blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5);
    const int slot = warp * 4 + (lane >> 3);
    const int code = slot < num_units ? __ldg(units + slot) : -1;
    const bool valid_unit = code >= 0;
    const int j = valid_unit ? code >> 3 : 0;
    const int band = valid_unit ? code & 7 : 0;
    const SynthJobDev &job = jobs[j];
    const int n_len = valid_unit ? job.num_bins * job.spb : 0;
    const int longest = __reduce_max_sync(0xFFFFFFFFu, static_cast<unsigned>(n_len));
    const double *x = raw + 6 * job.samples + static_cast<int64_t>(band) * n_len;
    float *out_row = job.band_irs + static_cast<int64_t>(band) * n_len;
    filter_units(x, out_row, n_len, valid_unit, band, cfg.crossover[valid_unit ? job.rate_index : 0],
                 longest + kLag + 2);
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

namespace ac {
namespace {

// Argument checks shared by ac_synthesize and ac_synthesize_static.
int check_synth(const char *name, const float *echograms, const ac_synth_params *p, const float *band_irs) {
    if (!p || !echograms || !band_irs) return ac::fail(AC_ERR_INVALID, "%s: null argument", name);
    if (p->num_rirs < 0 || p->num_bins < 1 || p->samples_per_bin < 1 || p->sample_rate < 1)
        return ac::fail(AC_ERR_INVALID, "synthesis sizes must be positive");
    const int64_t N = static_cast<int64_t>(p->num_bins) * p->samples_per_bin;
    if (N + 3 > 0x7FFFFFFF) return ac::fail(AC_ERR_CAPACITY, "signal of %lld samples is too long", (long long)N);
    if (p->rng_mode == AC_RNG_REFERENCE && !p->white) return ac::fail(AC_ERR_INVALID, "reference mode needs white noise");
    if (!p->air && !p->direct_delays) return ac::fail(AC_ERR_INVALID, "need an air table or the direct delays");
    return AC_OK;
}

// The three launches of one single-shape synthesis, over a workspace laid out
// by synth_layout(p) (caller-owned or the static scratch; at least l.total bytes).
int enqueue_synthesis(const float *echograms, const ac_synth_params *p, float *band_irs, unsigned char *ws,
                      const SynthLayout &l, cudaStream_t stream) {
    const int64_t N = static_cast<int64_t>(p->num_bins) * p->samples_per_bin;
    SynthArgs a;
    std::memcpy(a.crossover, p->crossover, sizeof(a.crossover));
    std::memcpy(a.air_coefficients, p->air_coefficients, sizeof(a.air_coefficients));
    a.speed_of_sound = p->speed_of_sound;
    a.num_rirs = p->num_rirs;
    a.num_bins = p->num_bins;
    a.spb = p->samples_per_bin;
    a.sample_rate = p->sample_rate;
    double *amps = reinterpret_cast<double *>(ws + l.amps);
    double *air = p->air ? nullptr : reinterpret_cast<double *>(ws + l.air);
    double *wtab = reinterpret_cast<double *>(ws + l.wtab);
    double *white = p->rng_mode == AC_RNG_PHILOX ? reinterpret_cast<double *>(ws + l.white) : nullptr;
    const size_t cells = static_cast<size_t>(p->num_rirs) * 6 * p->num_bins;
    const size_t work = std::max<size_t>(cells, static_cast<size_t>(white ? N : p->samples_per_bin));
    const int grid = static_cast<int>(std::min<size_t>((work + 255) / 256, 8192));
    synth_prepare_kernel<<<grid, 256, 0, stream>>>(echograms, p->direct_delays, a, amps, air, wtab, white, p->seed);
    AC_CUDA_TRY(cudaGetLastError());
    const double *air_table = p->air ? p->air : air;
    const double *noise = white ? white : p->white;
    const size_t stride = (white || p->white_shared) ? 0 : static_cast<size_t>(N);
    double *raw = reinterpret_cast<double *>(ws + l.raw);
    const size_t samples = static_cast<size_t>(p->num_rirs) * 6 * static_cast<size_t>(N);
    const int raw_grid = static_cast<int>(std::min<size_t>((samples + 255) / 256, 65536));
    synth_raw_kernel<<<raw_grid, 256, 0, stream>>>(amps, air_table, wtab, noise, stride, a, raw);
    AC_CUDA_TRY(cudaGetLastError());
    const int units = p->num_rirs * 6;
    const int warps = (units + 3) / 4;
    const int threads = 32;  // one warp per block: spread the sequential chains over all SMs
    synth_filter_kernel<<<warps, threads, 0, stream>>>(raw, a, band_irs);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

}  // namespace
}  // namespace ac

extern "C" int ac_synthesize(const float *echograms, const ac_synth_params *p, float *band_irs, void *workspace,
                             size_t workspace_bytes, void *stream_ptr) {
    ac::NvtxRange nvtx_range("ac_synthesize");
    const int rc = ac::check_synth("ac_synthesize", echograms, p, band_irs);
    if (rc != AC_OK) return rc;
    if (p->num_rirs == 0) return AC_OK;
    const ac::SynthLayout l = ac::synth_layout(p);
    if (!workspace || workspace_bytes < l.total)
        return ac::fail(AC_ERR_CAPACITY, "synthesis workspace too small: %zu < %zu", workspace_bytes, l.total);
    return ac::enqueue_synthesis(echograms, p, band_irs, static_cast<unsigned char *>(workspace), l,
                                 static_cast<cudaStream_t>(stream_ptr));
}

// ---------------------------------------------------------------------------
// Ragged batches: any mix of lengths and sample rates in three launches.

namespace ac {
namespace {

struct SynthBatchLayout {
    size_t jobs, cell_prefix, sample_prefix, units, table_end, amps, air, raw, total;
    int64_t cells, samples;
    int32_t num_units;
};

int check_batch(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *cfg, bool need_buffers,
                SynthBatchLayout *out) {
    if (num_jobs < 0 || (num_jobs > 0 && !jobs) || !cfg)
        return ac::fail(AC_ERR_INVALID, "synthesis batch: null argument");
    if (cfg->num_rates < 1 || cfg->num_rates > AC_SYNTH_MAX_RATES)
        return ac::fail(AC_ERR_INVALID, "synthesis batch: num_rates must be 1..%d", AC_SYNTH_MAX_RATES);
    for (int r = 0; r < cfg->num_rates; ++r)
        if (cfg->sample_rates[r] < 1) return ac::fail(AC_ERR_INVALID, "synthesis batch: sample rate %d < 1", r);
    if (static_cast<int64_t>(num_jobs) > (int64_t{1} << 28))
        return ac::fail(AC_ERR_CAPACITY, "synthesis batch of %d jobs is too large", num_jobs);
    SynthBatchLayout l{};
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_synth_job &job = jobs[j];
        if (job.num_bins < 1 || job.samples_per_bin < 1)
            return ac::fail(AC_ERR_INVALID, "synthesis job %d: sizes must be positive", j);
        const int64_t N = static_cast<int64_t>(job.num_bins) * job.samples_per_bin;
        if (N + 3 > 0x7FFFFFFF) return ac::fail(AC_ERR_CAPACITY, "synthesis job %d: %lld samples is too long", j,
                                                (long long)N);
        if (job.rate_index < 0 || job.rate_index >= cfg->num_rates)
            return ac::fail(AC_ERR_INVALID, "synthesis job %d: rate_index %d out of range", j, job.rate_index);
        if (job.rng_mode != AC_RNG_REFERENCE && job.rng_mode != AC_RNG_PHILOX)
            return ac::fail(AC_ERR_INVALID, "synthesis job %d: unknown rng_mode %d", j, job.rng_mode);
        if (need_buffers) {
            if (!job.echogram || !job.band_irs) return ac::fail(AC_ERR_INVALID, "synthesis job %d: null buffer", j);
            if (job.rng_mode == AC_RNG_REFERENCE && !job.white)
                return ac::fail(AC_ERR_INVALID, "synthesis job %d: reference mode needs white noise", j);
        }
        l.cells += 6 * static_cast<int64_t>(job.num_bins);
        l.samples += N;
    }
    l.num_units = static_cast<int32_t>((6 * static_cast<int64_t>(num_jobs) + 3) / 4 * 4);
    size_t off = 0;
    l.jobs = off;          off = align256(off + static_cast<size_t>(num_jobs) * sizeof(SynthJobDev));
    l.cell_prefix = off;   off = align256(off + (static_cast<size_t>(num_jobs) + 1) * sizeof(int64_t));
    l.sample_prefix = off; off = align256(off + (static_cast<size_t>(num_jobs) + 1) * sizeof(int64_t));
    l.units = off;         off = align256(off + static_cast<size_t>(l.num_units) * sizeof(int32_t));
    l.table_end = off;
    l.amps = off;          off = align256(off + static_cast<size_t>(l.cells) * sizeof(double));
    l.air = off;           off = align256(off + static_cast<size_t>(l.cells) * sizeof(double));
    l.raw = off;           off = align256(off + 6 * static_cast<size_t>(l.samples) * sizeof(double));
    l.total = off;
    *out = l;
    return AC_OK;
}

}  // namespace
}  // namespace ac

extern "C" int ac_synth_batch_workspace_size(const ac_synth_job *jobs, int32_t num_jobs,
                                             const ac_synth_batch_config *config, size_t *bytes) {
    if (!bytes) return ac::fail(AC_ERR_INVALID, "ac_synth_batch_workspace_size: null argument");
    ac::SynthBatchLayout l;
    const int rc = ac::check_batch(jobs, num_jobs, config, false, &l);
    if (rc != AC_OK) return rc;
    *bytes = l.total;
    return AC_OK;
}

namespace {

// Phase 1 (table copy, envelopes and air gains, raw band signals) and phase 2
// (the crossover recursion) of a ragged batch; phase 2 reads only what phase 1
// left in the workspace.
int synth_batch_phase(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                      void *workspace, size_t workspace_bytes, void *host_staging, void *stream_ptr, bool raw_phase,
                      bool filter_phase) {
    ac::SynthBatchLayout l;
    const int rc = ac::check_batch(jobs, num_jobs, config, true, &l);
    if (rc != AC_OK) return rc;
    if (num_jobs == 0) return AC_OK;
    if (!workspace || workspace_bytes < l.total)
        return ac::fail(AC_ERR_CAPACITY, "synthesis batch workspace too small: %zu < %zu", workspace_bytes, l.total);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    const ac::SynthJobDev *d_jobs = reinterpret_cast<const ac::SynthJobDev *>(ws + l.jobs);
    const int32_t *d_units = reinterpret_cast<const int32_t *>(ws + l.units);
    double *raw = reinterpret_cast<double *>(ws + l.raw);
    if (!raw_phase) {
        if (filter_phase) {
            ac::synth_batch_filter_kernel<<<l.num_units / 4, 32, 0, stream>>>(d_jobs, d_units, l.num_units, *config, raw);
            AC_CUDA_TRY(cudaGetLastError());
        }
        return AC_OK;
    }
    std::vector<unsigned char> local;
    unsigned char *host = static_cast<unsigned char *>(host_staging);
    if (!host) {
        local.assign(l.table_end, 0);
        host = local.data();
    }
    ac::SynthJobDev *dev_jobs = reinterpret_cast<ac::SynthJobDev *>(host + l.jobs);
    int64_t *cell_prefix = reinterpret_cast<int64_t *>(host + l.cell_prefix);
    int64_t *sample_prefix = reinterpret_cast<int64_t *>(host + l.sample_prefix);
    int32_t *units = reinterpret_cast<int32_t *>(host + l.units);
    int64_t cells = 0, samples = 0;
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_synth_job &in = jobs[j];
        ac::SynthJobDev d{};
        d.echogram = in.echogram;
        d.band_irs = in.band_irs;
        d.white = in.white;
        d.air = in.air;
        d.seed = in.seed;
        d.direct_delay = in.direct_delay;
        d.speed_of_sound = in.speed_of_sound;
        d.num_bins = in.num_bins;
        d.spb = in.samples_per_bin;
        d.rate_index = in.rate_index;
        d.rng_mode = in.rng_mode;
        d.cells = cells;
        d.samples = samples;
        std::memcpy(dev_jobs + j, &d, sizeof(d));
        cell_prefix[j] = cells;
        sample_prefix[j] = samples;
        cells += 6 * static_cast<int64_t>(in.num_bins);
        samples += static_cast<int64_t>(in.num_bins) * in.samples_per_bin;
    }
    cell_prefix[num_jobs] = cells;
    sample_prefix[num_jobs] = samples;
    // Filter units, longest job first (stable), six per job, padded to whole warps.
    std::vector<int32_t> order(static_cast<size_t>(num_jobs));
    for (int32_t j = 0; j < num_jobs; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return static_cast<int64_t>(jobs[a].num_bins) * jobs[a].samples_per_bin >
               static_cast<int64_t>(jobs[b].num_bins) * jobs[b].samples_per_bin;
    });
    int32_t u = 0;
    for (const int32_t j : order)
        for (int band = 0; band < 6; ++band) units[u++] = (j << 3) | band;
    for (; u < l.num_units; ++u) units[u] = -1;

    AC_CUDA_TRY(cudaMemcpyAsync(ws, host, l.table_end, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));  // pageable source must stay alive
    const int64_t *d_cells = reinterpret_cast<const int64_t *>(ws + l.cell_prefix);
    const int64_t *d_samples = reinterpret_cast<const int64_t *>(ws + l.sample_prefix);
    double *amps = reinterpret_cast<double *>(ws + l.amps);
    double *air = reinterpret_cast<double *>(ws + l.air);
    const int prep_grid = static_cast<int>(std::min<int64_t>((cells + 255) / 256, 8192));
    ac::synth_batch_prepare_kernel<<<prep_grid, 256, 0, stream>>>(d_jobs, d_cells, num_jobs, *config, amps, air);
    AC_CUDA_TRY(cudaGetLastError());
    const int raw_grid = static_cast<int>(std::min<int64_t>((samples + 255) / 256, 65536));
    ac::synth_batch_raw_kernel<<<raw_grid, 256, 0, stream>>>(d_jobs, d_samples, num_jobs, amps, air, raw);
    AC_CUDA_TRY(cudaGetLastError());
    if (filter_phase) {
        ac::synth_batch_filter_kernel<<<l.num_units / 4, 32, 0, stream>>>(d_jobs, d_units, l.num_units, *config, raw);
        AC_CUDA_TRY(cudaGetLastError());
    }
    return AC_OK;
}

}  // namespace

extern "C" int ac_synthesize_batch(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                                   void *workspace, size_t workspace_bytes, void *host_staging, void *stream) {
    ac::NvtxRange nvtx_range("ac_synthesize_batch");
    return synth_batch_phase(jobs, num_jobs, config, workspace, workspace_bytes, host_staging, stream, true, true);
}

extern "C" int ac_synthesize_batch_raw(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                                       void *workspace, size_t workspace_bytes, void *host_staging, void *stream) {
    ac::NvtxRange nvtx_range("ac_synthesize_batch_raw");
    return synth_batch_phase(jobs, num_jobs, config, workspace, workspace_bytes, host_staging, stream, true, false);
}

extern "C" int ac_synthesize_batch_filter(const ac_synth_job *jobs, int32_t num_jobs,
                                          const ac_synth_batch_config *config, void *workspace,
                                          size_t workspace_bytes, void *stream) {
    ac::NvtxRange nvtx_range("ac_synthesize_batch_filter");
    return synth_batch_phase(jobs, num_jobs, config, workspace, workspace_bytes, nullptr, stream, false, true);
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
    ac::NvtxRange nvtx_range("ac_synthesize_static");
    int rc = ac::check_synth("ac_synthesize_static", echograms, p, band_irs);
    if (rc != AC_OK) return rc;
    const int64_t N = static_cast<int64_t>(p->num_bins) * p->samples_per_bin;
    const ac::SynthLayout l = ac::synth_layout(p);
    if (l.total > static_cast<size_t>(AC_SYNTH_STATIC_BYTES))
        return ac::fail(AC_ERR_CAPACITY,
                        "synthesis of %d RIRs x %lld samples needs %zu bytes of scratch; the static scratch holds %zu: "
                        "split the RIRs over several calls",
                        p->num_rirs, (long long)N, l.total, static_cast<size_t>(AC_SYNTH_STATIC_BYTES));
    if (p->num_rirs == 0) return AC_OK;
    void *scratch = nullptr;
    rc = static_scratch(&scratch);
    if (rc != AC_OK) return rc;
    return ac::enqueue_synthesis(echograms, p, band_irs, static_cast<unsigned char *>(scratch), l,
                                 static_cast<cudaStream_t>(stream_ptr));
}
