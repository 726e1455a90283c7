// C ABI entry points: validation, dispatch by precision, device queries.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "scene_internal.h"

namespace ac {

std::string &last_error_slot() {
    static thread_local std::string slot;
    return slot;
}

int device_sm_count(int device) {
    static std::mutex mu;
    static std::vector<int> cache;
    std::lock_guard<std::mutex> lock(mu);
    if (device >= static_cast<int>(cache.size())) cache.resize(device + 1, 0);
    if (cache[device] == 0) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1) sms = 1;
        cache[device] = sms;
    }
    return cache[device];
}

double choose_energy_scale(const ac_scene_s *scene, const ac_trace_params *p) {
    const double R = static_cast<double>(std::max<int64_t>(1, p->num_rays));
    const double B = static_cast<double>(std::max<int32_t>(1, p->num_bounces));
    const double ray_scale = (4.0 * kPi) / R;
    const double imd = std::max(p->irradiance_min_distance, 1e-3);
    const double distance_term = 1.0 / (4.0 * kPi * imd * imd);
    const double w = p->dipole_weight;
    const double gain = std::pow(std::max(1.0, std::fabs(1.0 - 2.0 * w)), std::max(0.0, p->dipole_power));
    const double s_hi = std::max({1.0, std::fabs(scene->max_scattering), std::fabs(scene->min_scattering)});
    const double lobe = s_hi / kPi + (std::max(0.0, p->specular_exponent) + 2.0) / (8.0 * kPi) *
                                         std::max(1.0, std::fabs(1.0 - scene->min_scattering));
    const double growth = std::min(1e300, std::pow(std::max(1.0, scene->max_reflection), B + 1.0));
    const double max_deposit = ray_scale * gain * distance_term * lobe * growth;
    // The accumulators are exact for any number of quanta below 2^32, so only one
    // deposit must fit an int64 quantum: its six-band sum stays below 2^62.
    const double budget = 6.0 * max_deposit;
    int exponent = static_cast<int>(std::floor(std::log2(std::ldexp(1.0, 62) / budget)));
    exponent = std::min(200, std::max(-60, exponent));
    return std::ldexp(1.0, exponent);
}

int validate_trace(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o) {
    if (!scene || !p || !o) return fail(AC_ERR_INVALID, "ac_trace: null argument");
    if (p->num_rays < 1 || p->num_rays > 0x7FFFFFFF) return fail(AC_ERR_INVALID, "num_rays must be in [1, 2^31)");
    if (p->num_bounces < 0 || p->num_bounces > 0xFFFFFE) return fail(AC_ERR_INVALID, "num_bounces must be in [0, 2^24-1)");
    if (p->num_bins < 1) return fail(AC_ERR_INVALID, "num_bins must be positive");
    if (p->num_bins >= (1 << 21))   // (job, bin) fits the 32-bit keys the kernels may match lanes on
        return fail(AC_ERR_CAPACITY, "num_bins %d is too many (at most 2^21 - 1)", p->num_bins);
    if (!(p->bin_duration > 0.0) || !(p->speed_of_sound > 0.0))
        return fail(AC_ERR_INVALID, "bin duration and speed of sound must be positive");
    const double values[] = {p->source[0], p->source[1], p->source[2], p->listener[0], p->listener[1], p->listener[2],
                             p->source_forward[0], p->source_forward[1], p->source_forward[2], p->max_path_length,
                             p->direct_delay, p->listener_radius, p->source_radius, p->irradiance_min_distance,
                             p->specular_exponent, p->dipole_weight, p->dipole_power};
    for (double v : values)
        if (!std::isfinite(v)) return fail(AC_ERR_INVALID, "trace parameters must be finite");
    if (p->precision != AC_PRECISION_FP32 && p->precision != AC_PRECISION_FP64)
        return fail(AC_ERR_INVALID, "precision must be AC_PRECISION_FP32 or AC_PRECISION_FP64");
    if (p->rng_mode != AC_RNG_REFERENCE && p->rng_mode != AC_RNG_PHILOX)
        return fail(AC_ERR_INVALID, "rng_mode must be AC_RNG_REFERENCE or AC_RNG_PHILOX");
    if (p->rng_mode == AC_RNG_REFERENCE && (!p->directions || (p->num_bounces > 0 && (!p->diffuse_random || !p->diffuse_indices))))
        return fail(AC_ERR_INVALID, "reference-stream mode needs directions, diffuse_random and diffuse_indices");
    if (p->num_bounces > 0 && (p->num_bank < 1 || !p->diffuse_bank))
        return fail(AC_ERR_INVALID, "diffuse sample bank is required");
    if (!o->echogram_fx || !o->hit_counts || !o->contrib_counts || !o->surface_energy_fx || !o->counters)
        return fail(AC_ERR_INVALID, "echogram, per-surface and counter outputs are required");
    if (p->render_ambisonics && !o->ambisonic_fx)
        return fail(AC_ERR_INVALID, "render_ambisonics needs the ambisonic accumulator");
    if (p->energy_scale < 0.0 || !std::isfinite(p->energy_scale))
        return fail(AC_ERR_INVALID, "energy_scale must be zero (automatic) or positive");
    if (p->visual_limit < 0 || (p->visual_limit > 0 && p->visual_stride < 1))
        return fail(AC_ERR_INVALID, "visual_limit must be >= 0 and visual_stride >= 1 when candidates are recorded");
    if (p->visual_limit > 0 && (!o->visual_hit_points || !o->visual_surfaces || !o->visual_rays || !o->visual_orders ||
                                !o->visual_distances || !o->visual_gains))
        return fail(AC_ERR_INVALID, "visual_limit > 0 needs every visual-candidate output");
    // Each ray deposits at most once per bounce: fewer than 2^32 quanta per accumulator.
    if (static_cast<double>(p->num_rays) * static_cast<double>(std::max<int32_t>(1, p->num_bounces)) >= 4294967296.0)
        return fail(AC_ERR_CAPACITY, "num_rays * num_bounces must stay below 2^32; split the rays over several jobs");
    return AC_OK;
}

template <typename T>
__global__ void philox_workspace_kernel(uint64_t seed, uint64_t key, int64_t R, int32_t B, int32_t K, T *dirs, T *random,
                                        int32_t *indices) {
    Job<T> job{};
    job.rng_mode = 1;
    job.seed = seed;
    job.stream_key = key;
    job.num_rays = R;
    for (int64_t ri = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; ri < R;
         ri += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        T d[3];
        initial_direction(job, ri, d);
        dirs[3 * ri] = d[0];
        dirs[3 * ri + 1] = d[1];
        dirs[3 * ri + 2] = d[2];
        for (int32_t b = 0; b < B; ++b) {
            const u32x4 r = trace_draw(seed, key, static_cast<uint32_t>(ri), static_cast<uint32_t>(b) + 1u);
            random[static_cast<size_t>(b) * R + ri] = static_cast<T>(u01_53(r.x, r.y));
            indices[static_cast<size_t>(b) * R + ri] = static_cast<int32_t>(below(r.z, static_cast<uint32_t>(K)));
        }
    }
}

std::vector<Partition> partition_jobs(const ac_job *jobs, int32_t count) {
    std::vector<Partition> parts;
    for (int32_t j = 0; j < count; ++j) {
        const bool fp64 = jobs[j].params.precision == AC_PRECISION_FP64;
        const int key = fp64 ? 8 : ((jobs[j].params.rng_mode == AC_RNG_PHILOX ? 2 : 0) |
                                    (jobs[j].params.render_ambisonics ? 1 : 0) |
                                    (jobs[j].params.visual_limit > 0 ? 4 : 0));
        Partition *found = nullptr;
        for (Partition &p : parts)
            if (p.key == key) found = &p;
        if (!found) {
            parts.push_back(Partition{key, fp64, {}});
            found = &parts.back();
        }
        found->indices.push_back(j);
    }
    return parts;
}

size_t partition_bytes(const ac_job *jobs, const Partition &part, const ac_batch_config *cfg) {
    const int32_t n = static_cast<int32_t>(part.indices.size());
    const size_t b = part.fp64 ? batch_workspace_bytes_f64(jobs, part.indices.data(), n, cfg)
                               : batch_workspace_bytes_f32(jobs, part.indices.data(), n, cfg);
    return (b + 255) & ~static_cast<size_t>(255);
}

}  // namespace ac

namespace ac {
namespace {

// Reads n 16-byte words `repeats` times through L2 (ld.global.cg: not cached in L1).
__global__ void read_probe_kernel(const uint4 *buf, size_t n, int repeats, unsigned long long *sink) {
    unsigned acc = 0u;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (int r = 0; r < repeats; ++r)
        for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += stride) {
            const uint4 v = __ldcg(buf + i);
            acc ^= v.x ^ v.y ^ v.z ^ v.w;
        }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);  // a data dependence that keeps every load
}

// Float64 issue-rate probe: eight independent add chains and eight independent
// multiply chains per thread (separate instructions, no fused multiply-add).
__global__ void fp64_probe_kernel(int iterations, double c, double f, unsigned long long *sink) {
    double a[8], m[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        a[j] = threadIdx.x + j;
        m[j] = 1.0 + 1e-9 * (threadIdx.x + j);
    }
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            a[j] = a[j] + c;
            m[j] = m[j] * f;
        }
    }
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc += a[j] + m[j];
    if (acc == -1.0) atomicAdd(sink, 1ull);  // a data dependence that keeps every chain
}

}  // namespace
}  // namespace ac

extern "C" {

const char *ac_last_error(void) { return ac::last_error_slot().c_str(); }

int ac_abi_version(void) { return AC_ABI_VERSION; }

int ac_device_info(int32_t device, char *name, size_t name_len, int32_t *cc_major, int32_t *cc_minor, int32_t *sm_count) {
    cudaDeviceProp prop;
    AC_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (name && name_len) {
        std::strncpy(name, prop.name, name_len - 1);
        name[name_len - 1] = '\0';
    }
    if (cc_major) *cc_major = prop.major;
    if (cc_minor) *cc_minor = prop.minor;
    if (sm_count) *sm_count = prop.multiProcessorCount;
    return AC_OK;
}

int ac_energy_scale(ac_scene_t scene, const ac_trace_params *params, double *scale) {
    if (!scene || !params || !scale) return ac::fail(AC_ERR_INVALID, "ac_energy_scale: null argument");
    *scale = params->energy_scale > 0.0 ? params->energy_scale : ac::choose_energy_scale(scene, params);
    return AC_OK;
}

int ac_trace(ac_scene_t scene, const ac_trace_params *params, const ac_trace_outputs *outputs, void *stream) {
    ac::NvtxRange nvtx_range("ac_trace");
    int rc = ac::validate_trace(scene, params, outputs);
    if (rc != AC_OK) return rc;
    const double scale = params->energy_scale > 0.0 ? params->energy_scale : ac::choose_energy_scale(scene, params);
    if (outputs->scale_out) *outputs->scale_out = scale;
    rc = params->precision == AC_PRECISION_FP64 ? ac::launch_trace_f64(scene, params, outputs, scale, stream)
                                                : ac::launch_trace_f32(scene, params, outputs, scale, stream);
    if (rc != AC_OK) return rc;
    return ac::note_scene_use(scene, stream);
}

int ac_batch_workspace_size(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, size_t *bytes) {
    if (num_jobs < 0 || !bytes || (num_jobs > 0 && !jobs))
        return ac::fail(AC_ERR_INVALID, "ac_batch_workspace_size: bad argument");
    for (int32_t j = 0; j < num_jobs; ++j)
        if (!jobs[j].scene) return ac::fail(AC_ERR_INVALID, "job %d has no scene", j);
    size_t total = 0;
    for (const ac::Partition &part : ac::partition_jobs(jobs, num_jobs)) total += ac::partition_bytes(jobs, part, config);
    *bytes = total;
    return AC_OK;
}

// Jobs run in one launch per (precision, random stream, ambisonics, visual candidates) partition;
// each partition has its own region of the workspace, so the launches are
// simply enqueued one after another on the stream.
int ac_trace_batch(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, void *workspace,
                   size_t workspace_bytes, void *host_staging, void *stream) {
    ac::NvtxRange nvtx_range("ac_trace_batch");
    if (num_jobs < 0 || (num_jobs > 0 && (!jobs || !workspace)))
        return ac::fail(AC_ERR_INVALID, "ac_trace_batch: bad argument");
    for (int32_t j = 0; j < num_jobs; ++j) {
        const int rc = ac::validate_trace(jobs[j].scene, &jobs[j].params, &jobs[j].outputs);
        if (rc != AC_OK) return ac::fail(rc, "job %d: %s", j, ac_last_error());
    }
    size_t offset = 0;
    for (const ac::Partition &part : ac::partition_jobs(jobs, num_jobs)) {
        const size_t bytes = ac::partition_bytes(jobs, part, config);
        if (offset + bytes > workspace_bytes)
            return ac::fail(AC_ERR_CAPACITY, "batch workspace too small: %zu < %zu", workspace_bytes, offset + bytes);
        unsigned char *ws = static_cast<unsigned char *>(workspace) + offset;
        unsigned char *host = host_staging ? static_cast<unsigned char *>(host_staging) + offset : nullptr;
        const int32_t n = static_cast<int32_t>(part.indices.size());
        const int rc = part.fp64 ? ac::launch_batch_f64(jobs, part.indices.data(), n, config, ws, bytes, host, stream)
                                 : ac::launch_batch_f32(jobs, part.indices.data(), n, config, ws, bytes, host, stream);
        if (rc != AC_OK) return rc;
        offset += bytes;
    }
    // jobs of one scene are usually adjacent: note each run of them once
    for (int32_t j = 0; j < num_jobs; ++j) {
        if (j > 0 && jobs[j].scene == jobs[j - 1].scene) continue;
        const int rc = ac::note_scene_use(jobs[j].scene, stream);
        if (rc != AC_OK) return rc;
    }
    return AC_OK;
}

// A submitted batch: the event recorded on the caller's stream after its launches.
struct ac_batch_ticket_s {
    cudaEvent_t done;
};

int ac_batch_submit(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, void *workspace,
                    size_t workspace_bytes, void *host_staging, void *stream, ac_batch_ticket_t *ticket) {
    ac::NvtxRange nvtx_range("ac_batch_submit");
    if (!ticket) return ac::fail(AC_ERR_INVALID, "ac_batch_submit: null ticket");
    *ticket = nullptr;
    const int rc = ac_trace_batch(jobs, num_jobs, config, workspace, workspace_bytes, host_staging, stream);
    if (rc != AC_OK) return rc;
    ac_batch_ticket_s *t = new (std::nothrow) ac_batch_ticket_s();
    if (!t) return ac::fail(AC_ERR_NOMEM, "out of host memory");
    cudaError_t err = cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming);
    if (err == cudaSuccess) {
        err = cudaEventRecord(t->done, static_cast<cudaStream_t>(stream));
        if (err != cudaSuccess) cudaEventDestroy(t->done);
    }
    if (err != cudaSuccess) {
        delete t;
        return ac::fail(AC_ERR_CUDA, "ac_batch_submit: event: %s", cudaGetErrorString(err));
    }
    *ticket = t;
    return AC_OK;
}

int ac_batch_poll(ac_batch_ticket_t ticket, int32_t *done) {
    if (!ticket || !done) return ac::fail(AC_ERR_INVALID, "ac_batch_poll: null argument");
    const cudaError_t err = cudaEventQuery(ticket->done);
    if (err == cudaSuccess) {
        *done = 1;
        return AC_OK;
    }
    if (err == cudaErrorNotReady) {
        cudaGetLastError();   // not-ready is an answer, not a failure: leave no error behind
        *done = 0;
        return AC_OK;
    }
    return ac::fail(AC_ERR_CUDA, "ac_batch_poll: %s", cudaGetErrorString(err));
}

int ac_batch_wait(ac_batch_ticket_t ticket) {
    if (!ticket) return ac::fail(AC_ERR_INVALID, "ac_batch_wait: null ticket");
    AC_CUDA_TRY(cudaEventSynchronize(ticket->done));
    return AC_OK;
}

int ac_batch_release(ac_batch_ticket_t ticket) {
    if (!ticket) return AC_OK;
    const cudaError_t err = cudaEventDestroy(ticket->done);
    delete ticket;
    if (err != cudaSuccess) return ac::fail(AC_ERR_CUDA, "ac_batch_release: %s", cudaGetErrorString(err));
    return AC_OK;
}

int ac_philox_workspace(uint64_t seed, uint64_t stream_key, int64_t num_rays, int32_t num_bounces, int32_t num_bank,
                        int32_t precision, void *directions, void *random, int32_t *indices, void *stream) {
    ac::NvtxRange nvtx_range("ac_philox_workspace");
    if (num_rays < 1 || num_rays > 0x7FFFFFFF || num_bounces < 0 || num_bank < 1 || !directions ||
        (num_bounces > 0 && (!random || !indices)))
        return ac::fail(AC_ERR_INVALID, "ac_philox_workspace: bad argument");
    const int block = 256;
    const int grid = static_cast<int>(std::min<int64_t>((num_rays + block - 1) / block, 4096));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (precision == AC_PRECISION_FP64)
        ac::philox_workspace_kernel<double><<<grid, block, 0, s>>>(seed, stream_key, num_rays, num_bounces, num_bank,
                                                                   static_cast<double *>(directions),
                                                                   static_cast<double *>(random), indices);
    else
        ac::philox_workspace_kernel<float><<<grid, block, 0, s>>>(seed, stream_key, num_rays, num_bounces, num_bank,
                                                                  static_cast<float *>(directions),
                                                                  static_cast<float *>(random), indices);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

int ac_read_bandwidth_probe(const void *buffer, size_t bytes, int32_t repeats, unsigned long long *sink,
                            void *stream) {
    ac::NvtxRange nvtx_range("ac_read_bandwidth_probe");
    if (!buffer || !sink || repeats < 1 || bytes < 16 || (reinterpret_cast<uintptr_t>(buffer) & 15u) != 0)
        return ac::fail(AC_ERR_INVALID, "ac_read_bandwidth_probe: needs a 16-byte aligned buffer and a sink");
    int device = 0;
    AC_CUDA_TRY(cudaGetDevice(&device));
    const int grid = 8 * ac::device_sm_count(device);
    ac::read_probe_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const uint4 *>(buffer),
                                                                                bytes / 16, repeats, sink);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

int ac_fp64_rate_probe(int32_t iterations, unsigned long long *sink, int64_t *ops, void *stream) {
    if (iterations < 1 || !sink || !ops) return ac::fail(AC_ERR_INVALID, "ac_fp64_rate_probe: bad argument");
    int dev = 0, sms = 0;
    AC_CUDA_TRY(cudaGetDevice(&dev));
    AC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = 2 * sms, threads = 256;   // sixteen warps per SM
    ac::fp64_probe_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(iterations, 1e-3, 1.0000000001,
                                                                                    sink);
    AC_CUDA_TRY(cudaGetLastError());
    *ops = static_cast<int64_t>(blocks) * threads * iterations * 16;
    return AC_OK;
}

}  // extern "C"
