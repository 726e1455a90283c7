// Host launchers for the tracer, instantiated once per precision by
// trace_f32.cu and trace_f64.cu.
#pragma once

#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "scene_internal.h"
#include "trace_kernel.cuh"

namespace ac {

constexpr int kDefaultBlock = 256;

// Reference initial values of the visual-candidate arrays (steam_rt.py:4718-4723).
template <typename T>
__device__ __forceinline__ void init_visual(const Job<T> &job, size_t first, size_t step) {
    if (job.visual_limit <= 0) return;
    const size_t L = static_cast<size_t>(job.visual_limit), LB = L * static_cast<size_t>(job.num_bounces);
    for (size_t i = first; i < 3 * LB; i += step) job.visual_hit_points[i] = T(0);
    for (size_t i = first; i < LB; i += step) job.visual_surfaces[i] = -1;
    for (size_t i = first; i < L; i += step) {
        job.visual_rays[i] = -1;
        job.visual_orders[i] = 0;
        job.visual_distances[i] = T(0);
        job.visual_gains[i] = T(0);
    }
}

// Zero every job's accumulators and the work counter (one launch for all jobs).
template <typename T>
__global__ void zero_outputs_kernel(const Job<T> *jobs, int num_jobs, unsigned long long *work_counter) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && work_counter) *work_counter = 0ull;
    for (int j = blockIdx.y; j < num_jobs; j += gridDim.y) {
        const Job<T> &job = jobs[j];
        // word counts: each fixed-point accumulator takes two words
        const size_t nb = 2 * static_cast<size_t>(kBands) * job.num_bins;
        const size_t na = job.ambisonic_fx ? 4 * nb : 0;
        const size_t ns = static_cast<size_t>(job.scene.num_surfaces);
        const size_t total = nb + na + 4 * ns + 8;
        for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
            if (i < nb) job.echogram_fx[i] = 0ull;
            else if (i < nb + na) job.ambisonic_fx[i - nb] = 0ull;
            else if (i < nb + na + ns) job.hit_counts[i - nb - na] = 0ull;
            else if (i < nb + na + 2 * ns) job.contrib_counts[i - nb - na - ns] = 0ull;
            else if (i < nb + na + 4 * ns) job.surface_energy_fx[i - nb - na - 2 * ns] = 0ull;
            else job.counters[i - nb - na - 4 * ns] = 0ull;
        }
        init_visual(job, blockIdx.x * blockDim.x + threadIdx.x, static_cast<size_t>(gridDim.x) * blockDim.x);
    }
}

template <typename T>
__global__ void init_visual_single_kernel(const __grid_constant__ Job<T> job) {
    init_visual(job, blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x,
                static_cast<size_t>(gridDim.x) * blockDim.x);
}

struct FinalizeTargets {
    float *echogram;
    float *ambisonic;
    float *surface_energy;
};

// Fixed point (sum of low halves, sum of high halves) -> double.
__device__ __forceinline__ double fixed_to_double(const unsigned long long *w, double inv_scale) {
    const double v = ldexp(static_cast<double>(static_cast<long long>(w[1])), 32) + static_cast<double>(w[0]);
    return v * inv_scale;
}

// Fixed point -> float32 copies (the reference CUDA backend returns float32).
template <typename T>
__global__ void finalize_kernel(const Job<T> *jobs, const FinalizeTargets *targets, int num_jobs) {
    for (int j = blockIdx.y; j < num_jobs; j += gridDim.y) {
        const Job<T> &job = jobs[j];
        const FinalizeTargets tg = targets[j];
        const double inv = 1.0 / job.energy_scale;
        const size_t nb = static_cast<size_t>(kBands) * job.num_bins;
        const size_t na = (job.ambisonic_fx && tg.ambisonic) ? 4 * nb : 0;
        const size_t ns = tg.surface_energy ? static_cast<size_t>(job.scene.num_surfaces) : 0;
        const size_t ne = tg.echogram ? nb : 0;
        const size_t total = ne + na + ns;
        for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
            if (i < ne) {
                tg.echogram[i] = static_cast<float>(fixed_to_double(job.echogram_fx + 2 * i, inv));
            } else if (i < ne + na) {
                const size_t k = i - ne;
                tg.ambisonic[k] = static_cast<float>(fixed_to_double(job.ambisonic_fx + 2 * k, inv));
            } else {
                const size_t k = i - ne - na;
                tg.surface_energy[k] = static_cast<float>(fixed_to_double(job.surface_energy_fx + 2 * k, inv));
            }
        }
    }
}

template <typename T>
inline void fill_job(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     Job<T> &job) {
    std::memset(&job, 0, sizeof(job));
    job.scene = scene_view<T>(scene);
    for (int a = 0; a < 3; ++a) {
        job.src[a] = static_cast<T>(p->source[a]);
        job.lst[a] = static_cast<T>(p->listener[a]);
        job.fwd[a] = static_cast<T>(p->source_forward[a]);
    }
    job.listener_radius = static_cast<T>(p->listener_radius);
    job.source_radius = static_cast<T>(p->source_radius);
    job.irradiance_min_distance = static_cast<T>(p->irradiance_min_distance);
    job.specular_exponent = static_cast<T>(p->specular_exponent);
    job.dipole_weight = static_cast<T>(p->dipole_weight);
    job.dipole_power = static_cast<T>(p->dipole_power);
    job.ray_scale = static_cast<T>((4.0 * kPi) / static_cast<double>(p->num_rays > 1 ? p->num_rays : 1));
    {
        const T dx = job.lst[0] - job.src[0], dy = job.lst[1] - job.src[1], dz = job.lst[2] - job.src[2];
        job.source_distance = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
    job.speed_of_sound = p->speed_of_sound;
    job.direct_delay = p->direct_delay;
    job.bin_duration = p->bin_duration;
    job.inv_speed_of_sound = 1.0 / p->speed_of_sound;
    job.inv_bin_duration = 1.0 / p->bin_duration;
    job.max_path_length = p->max_path_length;
    job.energy_scale = scale;
    job.num_rays = p->num_rays;
    job.num_bounces = p->num_bounces;
    job.num_bins = p->num_bins;
    job.use_bvh = p->use_bvh ? 1 : 0;
    job.render_ambisonics = p->render_ambisonics ? 1 : 0;
    job.rng_mode = p->rng_mode;
    job.num_bank = p->num_bank;
    job.seed = p->seed;
    job.stream_key = p->stream_key;
    job.directions = static_cast<const T *>(p->directions);
    job.diffuse_random = static_cast<const T *>(p->diffuse_random);
    job.diffuse_indices = p->diffuse_indices;
    job.diffuse_bank = static_cast<const T *>(p->diffuse_bank);
    job.echogram_fx = reinterpret_cast<unsigned long long *>(o->echogram_fx);
    job.ambisonic_fx = p->render_ambisonics ? reinterpret_cast<unsigned long long *>(o->ambisonic_fx) : nullptr;
    job.hit_counts = reinterpret_cast<unsigned long long *>(o->hit_counts);
    job.contrib_counts = reinterpret_cast<unsigned long long *>(o->contrib_counts);
    job.surface_energy_fx = reinterpret_cast<unsigned long long *>(o->surface_energy_fx);
    job.counters = reinterpret_cast<unsigned long long *>(o->counters);
    job.ray_surfaces = o->ray_surfaces;
    if (p->visual_limit > 0) {
        job.visual_limit = p->visual_limit;
        job.visual_stride = p->visual_stride;
        job.visual_hit_points = static_cast<T *>(o->visual_hit_points);
        job.visual_surfaces = o->visual_surfaces;
        job.visual_rays = o->visual_rays;
        job.visual_orders = o->visual_orders;
        job.visual_distances = static_cast<T *>(o->visual_distances);
        job.visual_gains = static_cast<T *>(o->visual_gains);
    }
}

template <typename T, bool kSingle>
inline int persistent_grid(int device, int block, int64_t total_rays, int requested) {
    int per_sm = 0;
    cudaError_t err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<T, kSingle>, block, 0);
    if (err != cudaSuccess || per_sm < 1) per_sm = 1;
    int grid = per_sm * device_sm_count(device);
    if (requested > 0) grid = requested;
    const int64_t needed = (total_rays + block - 1) / block;
    if (needed < grid) grid = static_cast<int>(needed > 0 ? needed : 1);
    return grid;
}

// Single job: the job travels in the kernel's parameter space, so the call
// needs no device allocation and no host->device copy of its own.
template <typename T>
inline int launch_single(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                         void *stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    Job<T> job;
    fill_job<T>(scene, p, o, scale, job);
    AC_CUDA_TRY(cudaSetDevice(scene->device));
    const size_t nb = 2 * static_cast<size_t>(kBands) * p->num_bins;  // two words per accumulator
    AC_CUDA_TRY(cudaMemsetAsync(o->echogram_fx, 0, nb * sizeof(int64_t), stream));
    if (job.ambisonic_fx) AC_CUDA_TRY(cudaMemsetAsync(o->ambisonic_fx, 0, 4 * nb * sizeof(int64_t), stream));
    const size_t ns = static_cast<size_t>(scene->num_surfaces) * sizeof(int64_t);
    AC_CUDA_TRY(cudaMemsetAsync(o->hit_counts, 0, ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->contrib_counts, 0, ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->surface_energy_fx, 0, 2 * ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->counters, 0, 8 * sizeof(int64_t), stream));
    if (job.visual_limit > 0) {
        const size_t cells = 3 * static_cast<size_t>(job.visual_limit) * job.num_bounces;
        init_visual_single_kernel<T><<<static_cast<int>(std::min<size_t>((cells + 255) / 256, 1024)), 256, 0,
                                       stream>>>(job);
        AC_CUDA_TRY(cudaGetLastError());
    }
    const int block = p->block_size > 0 ? p->block_size : kDefaultBlock;
    if (block % 32 != 0 || block > 256) return fail(AC_ERR_INVALID, "block_size must be a multiple of 32 up to 256");
    if (p->num_rays > 0) {
        const int grid = persistent_grid<T, true>(scene->device, block, p->num_rays, p->grid_blocks);
        BatchTable none{};
        trace_kernel<T, true><<<grid, block, 0, stream>>>(job, none);
        AC_CUDA_TRY(cudaGetLastError());
    }
    return AC_OK;
}

template <typename T>
__global__ void finalize_single_kernel(const __grid_constant__ Job<T> job, FinalizeTargets tg) {
    const double inv = 1.0 / job.energy_scale;
    const size_t nb = static_cast<size_t>(kBands) * job.num_bins;
    const size_t na = (job.ambisonic_fx && tg.ambisonic) ? 4 * nb : 0;
    const size_t ns = tg.surface_energy ? static_cast<size_t>(job.scene.num_surfaces) : 0;
    const size_t ne = tg.echogram ? nb : 0;
    const size_t total = ne + na + ns;
    for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i < ne) {
            tg.echogram[i] = static_cast<float>(fixed_to_double(job.echogram_fx + 2 * i, inv));
        } else if (i < ne + na) {
            const size_t k = i - ne;
            tg.ambisonic[k] = static_cast<float>(fixed_to_double(job.ambisonic_fx + 2 * k, inv));
        } else {
            const size_t k = i - ne - na;
            tg.surface_energy[k] = static_cast<float>(fixed_to_double(job.surface_energy_fx + 2 * k, inv));
        }
    }
}

template <typename T>
inline int launch_finalize_single(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o,
                                  double scale, void *stream_ptr) {
    if (!o->echogram && !o->ambisonic && !o->surface_energy) return AC_OK;
    Job<T> job;
    fill_job<T>(scene, p, o, scale, job);
    FinalizeTargets tg{o->echogram, p->render_ambisonics ? o->ambisonic : nullptr, o->surface_energy};
    const size_t total = static_cast<size_t>(kBands) * p->num_bins * 5 + scene->num_surfaces;
    const int grid = static_cast<int>(std::min<size_t>((total + 255) / 256, 1024));
    finalize_single_kernel<T><<<grid, 256, 0, static_cast<cudaStream_t>(stream_ptr)>>>(job, tg);
    AC_CUDA_TRY(cudaGetLastError());
    return AC_OK;
}

// ---------------------------------------------------------------------------
// Batched launch: job table + prefix + finalize targets live in the caller's
// workspace.  Layout (bytes, each part 256-aligned):
//   [0]              work counter (8)
//   [256]            ray prefix int64[count + 1]
//   [..]             Job<T>[count]
//   [..]             FinalizeTargets[count]

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

template <typename T>
inline size_t batch_layout(int32_t count, size_t *off_prefix, size_t *off_jobs, size_t *off_targets) {
    size_t off = 256;
    *off_prefix = off;
    off = align256(off + sizeof(int64_t) * (static_cast<size_t>(count) + 1));
    *off_jobs = off;
    off = align256(off + sizeof(Job<T>) * static_cast<size_t>(count));
    *off_targets = off;
    off = align256(off + sizeof(FinalizeTargets) * static_cast<size_t>(count));
    return off;
}

template <typename T>
inline size_t batch_bytes(int32_t count) {
    size_t a, b, c;
    return batch_layout<T>(count, &a, &b, &c);
}

template <typename T>
inline int launch_batch(const ac_job *jobs_in, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                        void *workspace, size_t workspace_bytes, void *host_staging, void *stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    size_t off_prefix, off_jobs, off_targets;
    const size_t need = batch_layout<T>(count, &off_prefix, &off_jobs, &off_targets);
    if (workspace_bytes < need) return fail(AC_ERR_CAPACITY, "batch workspace too small: %zu < %zu", workspace_bytes, need);
    std::vector<unsigned char> local;
    unsigned char *host = static_cast<unsigned char *>(host_staging);
    if (!host) {
        local.assign(need, 0);
        host = local.data();
    } else {
        std::memset(host, 0, 256);
    }
    int64_t *prefix = reinterpret_cast<int64_t *>(host + off_prefix);
    Job<T> *jobs = reinterpret_cast<Job<T> *>(host + off_jobs);
    FinalizeTargets *targets = reinterpret_cast<FinalizeTargets *>(host + off_targets);
    int device = -1;
    int64_t total = 0;
    for (int32_t k = 0; k < count; ++k) {
        const ac_job &in = jobs_in[indices[k]];
        if (device < 0) device = in.scene->device;
        if (in.scene->device != device) return fail(AC_ERR_INVALID, "batch jobs must share one device");
        double scale = in.params.energy_scale;
        if (!(scale > 0.0)) scale = choose_energy_scale(in.scene, &in.params);
        fill_job<T>(in.scene, &in.params, &in.outputs, scale, jobs[k]);
        if (in.outputs.scale_out) *in.outputs.scale_out = scale;
        prefix[k] = total;
        jobs[k].ray_begin = total;
        total += in.params.num_rays;
        targets[k] = FinalizeTargets{in.outputs.echogram, in.params.render_ambisonics ? in.outputs.ambisonic : nullptr,
                                     in.outputs.surface_energy};
    }
    prefix[count] = total;
    AC_CUDA_TRY(cudaSetDevice(device));
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    AC_CUDA_TRY(cudaMemcpyAsync(ws + off_prefix, host + off_prefix, need - off_prefix, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));  // pageable source must stay alive
    const Job<T> *d_jobs = reinterpret_cast<const Job<T> *>(ws + off_jobs);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    {
        dim3 grid(32, static_cast<unsigned>(std::min<int32_t>(count, 65535)));
        zero_outputs_kernel<T><<<grid, 256, 0, stream>>>(d_jobs, count, counter);
        AC_CUDA_TRY(cudaGetLastError());
    }
    const int block = (cfg && cfg->block_size > 0) ? cfg->block_size : kDefaultBlock;
    if (block % 32 != 0 || block > 256) return fail(AC_ERR_INVALID, "block_size must be a multiple of 32 up to 256");
    if (total > 0) {
        BatchTable table{};
        table.jobs = d_jobs;
        table.ray_begin = reinterpret_cast<const int64_t *>(ws + off_prefix);
        table.num_jobs = count;
        table.total_rays = total;
        table.work_counter = counter;
        const int grid = persistent_grid<T, false>(device, block, total, cfg ? cfg->grid_blocks : 0);
        Job<T> unused;
        std::memset(&unused, 0, sizeof(unused));
        trace_kernel<T, false><<<grid, block, 0, stream>>>(unused, table);
        AC_CUDA_TRY(cudaGetLastError());
    }
    {
        dim3 grid(16, static_cast<unsigned>(std::min<int32_t>(count, 65535)));
        finalize_kernel<T><<<grid, 256, 0, stream>>>(d_jobs, reinterpret_cast<const FinalizeTargets *>(ws + off_targets),
                                                    count);
        AC_CUDA_TRY(cudaGetLastError());
    }
    return AC_OK;
}

}  // namespace ac
