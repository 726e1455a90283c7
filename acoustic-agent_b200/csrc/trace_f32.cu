// Float32 production launches: the warp-uniform scene-scan tracer (trace_fast.cuh).
#include <algorithm>
#include <numeric>
#include <vector>

#include "trace_launch.cuh"

namespace ac {

namespace {

constexpr int kDefaultChunkRays = 32;
// A scene group holds at most this many consecutive jobs, so that (job index mod 1024,
// surface) identifies a (job, surface) pair among the lanes of one warp (hit-count keys).
constexpr int64_t kMaxGroupJobs = 1024;

using FastKernel = void (*)(const Job<float>, const FastScene, const FastTable);

template <bool kSingle, bool kVisual>
FastKernel pick_variant(bool philox, bool amb) {
    if (philox)
        return amb ? trace_fast_kernel<kSingle, true, true, kVisual> : trace_fast_kernel<kSingle, true, false, kVisual>;
    return amb ? trace_fast_kernel<kSingle, false, true, kVisual> : trace_fast_kernel<kSingle, false, false, kVisual>;
}

template <bool kSingle>
FastKernel pick_kernel(bool philox, bool amb, bool visual) {
    return visual ? pick_variant<kSingle, true>(philox, amb) : pick_variant<kSingle, false>(philox, amb);
}

int fast_grid(FastKernel kernel, int device, int block, size_t smem, int64_t total_rays, int requested) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    int grid = requested > 0 ? requested : per_sm * device_sm_count(device);
    const int64_t needed = (total_rays + block - 1) / block;
    if (needed < grid) grid = static_cast<int>(needed > 0 ? needed : 1);
    return grid;
}

// Workspace layout for a float32 batch (each part 256-aligned):
//   [0] chunk counter | group queue counters u64[G] | ray prefix int64[J+1] | Job<float>[J] |
//   FinalizeTargets[J] | FastGroup[G] | FastChunk[NC] | group chunk prefix int64[G+1] | group ray prefix int64[G+1]
// Everything from the ray prefix on is staged on the host and copied in one transfer; the counters are zeroed
// on the device.
struct F32Layout {
    size_t queues, prefix, jobs, targets, groups, chunks, group_chunks, group_rays, total;
};

F32Layout f32_layout(int32_t jobs, int64_t groups, int64_t chunks) {
    F32Layout l{};
    size_t off = 256;
    l.queues = off;       off = align256(off + sizeof(unsigned long long) * static_cast<size_t>(groups));
    l.prefix = off;       off = align256(off + sizeof(int64_t) * (static_cast<size_t>(jobs) + 1));
    l.jobs = off;         off = align256(off + sizeof(Job<float>) * static_cast<size_t>(jobs));
    l.targets = off;      off = align256(off + sizeof(FinalizeTargets) * static_cast<size_t>(jobs));
    l.groups = off;       off = align256(off + sizeof(FastGroup) * static_cast<size_t>(groups));
    l.chunks = off;       off = align256(off + sizeof(FastChunk) * static_cast<size_t>(chunks));
    l.group_chunks = off; off = align256(off + sizeof(int64_t) * (static_cast<size_t>(groups) + 1));
    l.group_rays = off;   off = align256(off + sizeof(int64_t) * (static_cast<size_t>(groups) + 1));
    l.total = off;
    return l;
}

// Jobs sorted by scene so that each scene's rays form one contiguous range.
std::vector<int32_t> scene_order(const ac_job *jobs, const int32_t *indices, int32_t count) {
    std::vector<int32_t> order(indices, indices + count);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return reinterpret_cast<uintptr_t>(jobs[a].scene) < reinterpret_cast<uintptr_t>(jobs[b].scene);
    });
    return order;
}

void count_groups_chunks(const ac_job *jobs, const std::vector<int32_t> &order, int64_t chunk_rays, int64_t *groups,
                         int64_t *chunks) {
    *groups = 0;
    *chunks = 0;
    size_t k = 0;
    while (k < order.size()) {
        const ac_scene_t scene = jobs[order[k]].scene;
        int64_t rays = 0;
        int64_t members = 0;
        while (k < order.size() && jobs[order[k]].scene == scene && members < kMaxGroupJobs) {
            rays += jobs[order[k++]].params.num_rays;
            ++members;
        }
        *groups += 1;
        *chunks += (rays + chunk_rays - 1) / chunk_rays;
    }
}

}  // namespace

int launch_trace_f32(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     void *stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    int entries = 0;
    const int rc = launch_stack_entries(p->stack_entries, scene->fast.num_bvh_nodes > 0 ? scene->bvh_stack_need : 0,
                                        &entries);
    if (rc != AC_OK) return rc;
    Job<float> job;
    fill_job<float>(scene, p, o, scale, job);
    AC_CUDA_TRY(cudaSetDevice(scene->device));
    const size_t nb = 2 * static_cast<size_t>(kBands) * p->num_bins;
    AC_CUDA_TRY(cudaMemsetAsync(o->echogram_fx, 0, nb * sizeof(int64_t), stream));
    if (job.ambisonic_fx) AC_CUDA_TRY(cudaMemsetAsync(o->ambisonic_fx, 0, 4 * nb * sizeof(int64_t), stream));
    const size_t ns = static_cast<size_t>(scene->num_surfaces) * sizeof(int64_t);
    AC_CUDA_TRY(cudaMemsetAsync(o->hit_counts, 0, ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->contrib_counts, 0, ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->surface_energy_fx, 0, 2 * ns, stream));
    AC_CUDA_TRY(cudaMemsetAsync(o->counters, 0, 8 * sizeof(int64_t), stream));
    if (job.visual_limit > 0) {
        const size_t cells = 3 * static_cast<size_t>(job.visual_limit) * job.num_bounces;
        init_visual_single_kernel<float><<<static_cast<int>(std::min<size_t>((cells + 255) / 256, 1024)), 256, 0,
                                           stream>>>(job);
        AC_CUDA_TRY(cudaGetLastError());
    }
    const int block = p->block_size > 0 ? p->block_size : kDefaultBlock;
    if (block % 32 != 0 || block > 256) return fail(AC_ERR_INVALID, "block_size must be a multiple of 32 up to 256");
    FastTable table{};
    table.chunk_rays = kDefaultChunkRays;
    table.chunk_counter = reinterpret_cast<unsigned long long *>(o->counters) + 4;
    const FastKernel kernel = pick_kernel<true>(p->rng_mode == AC_RNG_PHILOX, p->render_ambisonics != 0,
                                                p->visual_limit > 0);
    const size_t smem = stack_smem_bytes(entries);
    const int grid = fast_grid(kernel, scene->device, block, smem, p->num_rays, p->grid_blocks);
    kernel<<<grid, block, smem, stream>>>(job, scene->fast, table);
    AC_CUDA_TRY(cudaGetLastError());
    return launch_finalize_single<float>(scene, p, o, scale, stream_ptr);
}

size_t batch_workspace_bytes_f32(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg) {
    const int64_t chunk_rays = (cfg && cfg->chunk_rays > 0) ? cfg->chunk_rays : kDefaultChunkRays;
    int64_t groups = 0, chunks = 0;
    count_groups_chunks(jobs, scene_order(jobs, indices, count), chunk_rays, &groups, &chunks);
    return f32_layout(count, groups, chunks).total;
}

int launch_batch_f32(const ac_job *jobs_in, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                     void *workspace, size_t workspace_bytes, void *host_staging, void *stream_ptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const int64_t chunk_rays = (cfg && cfg->chunk_rays > 0) ? cfg->chunk_rays : kDefaultChunkRays;
    const std::vector<int32_t> order = scene_order(jobs_in, indices, count);
    int64_t num_groups = 0, num_chunks = 0;
    count_groups_chunks(jobs_in, order, chunk_rays, &num_groups, &num_chunks);
    const F32Layout l = f32_layout(count, num_groups, num_chunks);
    if (workspace_bytes < l.total)
        return fail(AC_ERR_CAPACITY, "batch workspace too small: %zu < %zu", workspace_bytes, l.total);
    std::vector<unsigned char> local;
    unsigned char *host = static_cast<unsigned char *>(host_staging);
    if (!host) {
        local.assign(l.total, 0);
        host = local.data();
    }
    int64_t *prefix = reinterpret_cast<int64_t *>(host + l.prefix);
    Job<float> *jobs = reinterpret_cast<Job<float> *>(host + l.jobs);
    FinalizeTargets *targets = reinterpret_cast<FinalizeTargets *>(host + l.targets);
    FastGroup *groups = reinterpret_cast<FastGroup *>(host + l.groups);
    FastChunk *chunks = reinterpret_cast<FastChunk *>(host + l.chunks);
    int64_t *group_chunks = reinterpret_cast<int64_t *>(host + l.group_chunks);
    int64_t *group_rays = reinterpret_cast<int64_t *>(host + l.group_rays);
    int device = -1, need = 0;
    int64_t total = 0, g = -1, c = 0;
    const ac_scene_s *current = nullptr;
    int64_t group_begin = 0;
    auto close_group = [&](int64_t group_end) {
        group_chunks[g] = c;
        group_rays[g] = group_begin;
        for (int64_t b = group_begin; b < group_end; b += chunk_rays)
            chunks[c++] = FastChunk{b, std::min(b + chunk_rays, group_end), static_cast<int32_t>(g), 0};
    };
    for (int32_t k = 0; k < count; ++k) {
        const ac_job &in = jobs_in[order[k]];
        if (device < 0) device = in.scene->device;
        if (in.scene->device != device) return fail(AC_ERR_INVALID, "batch jobs must share one device");
        if (in.scene->fast.num_bvh_nodes > 0) need = std::max(need, in.scene->bvh_stack_need);
        if (in.scene != current || groups[g].num_jobs >= kMaxGroupJobs) {
            if (g >= 0) close_group(total);
            ++g;
            current = in.scene;
            group_begin = total;
            groups[g] = FastGroup{in.scene->f32, in.scene->fast, k, 0};
        }
        groups[g].num_jobs += 1;
        double scale = in.params.energy_scale;
        if (!(scale > 0.0)) scale = choose_energy_scale(in.scene, &in.params);
        fill_job<float>(in.scene, &in.params, &in.outputs, scale, jobs[k]);
        if (k > 0 && (jobs[k].rng_mode != jobs[0].rng_mode || jobs[k].render_ambisonics != jobs[0].render_ambisonics ||
                      (jobs[k].visual_limit > 0) != (jobs[0].visual_limit > 0)))
            return fail(AC_ERR_INVALID,
                        "one float32 launch needs one random-stream mode, ambisonics and visual-candidate setting");
        if (in.outputs.scale_out) *in.outputs.scale_out = scale;
        prefix[k] = total;
        jobs[k].ray_begin = total;
        total += in.params.num_rays;
        targets[k] = FinalizeTargets{in.outputs.echogram, in.params.render_ambisonics ? in.outputs.ambisonic : nullptr,
                                     in.outputs.surface_energy};
    }
    if (g >= 0) close_group(total);
    int entries = 0;
    const int rc = launch_stack_entries(cfg ? cfg->stack_entries : 0, need, &entries);
    if (rc != AC_OK) return rc;
    prefix[count] = total;
    group_chunks[num_groups] = c;
    group_rays[num_groups] = total;
    AC_CUDA_TRY(cudaSetDevice(device));
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    AC_CUDA_TRY(cudaMemcpyAsync(ws + l.prefix, host + l.prefix, l.total - l.prefix, cudaMemcpyHostToDevice, stream));
    if (!host_staging) AC_CUDA_TRY(cudaStreamSynchronize(stream));
    AC_CUDA_TRY(cudaMemsetAsync(ws + l.queues, 0, sizeof(unsigned long long) * static_cast<size_t>(num_groups), stream));
    const Job<float> *d_jobs = reinterpret_cast<const Job<float> *>(ws + l.jobs);
    unsigned long long *counter = reinterpret_cast<unsigned long long *>(ws);
    {
        dim3 zgrid(32, static_cast<unsigned>(std::min<int32_t>(count, 65535)));
        zero_outputs_kernel<float><<<zgrid, 256, 0, stream>>>(d_jobs, count, counter);
        AC_CUDA_TRY(cudaGetLastError());
    }
    const int block = (cfg && cfg->block_size > 0) ? cfg->block_size : kDefaultBlock;
    if (block % 32 != 0 || block > 256) return fail(AC_ERR_INVALID, "block_size must be a multiple of 32 up to 256");
    if (total > 0) {
        FastTable table{};
        table.jobs = d_jobs;
        table.ray_begin = reinterpret_cast<const int64_t *>(ws + l.prefix);
        table.groups = reinterpret_cast<const FastGroup *>(ws + l.groups);
        table.chunks = reinterpret_cast<const FastChunk *>(ws + l.chunks);
        table.num_chunks = num_chunks;
        table.num_jobs = count;
        table.chunk_rays = static_cast<int32_t>(chunk_rays);
        table.chunk_counter = counter;
        table.group_next = reinterpret_cast<unsigned long long *>(ws + l.queues);
        table.group_chunk_begin = reinterpret_cast<const int64_t *>(ws + l.group_chunks);
        table.group_ray_begin = reinterpret_cast<const int64_t *>(ws + l.group_rays);
        table.num_groups = static_cast<int32_t>(num_groups);
        Job<float> unused;
        std::memset(&unused, 0, sizeof(unused));
        FastScene none{};
        // ac_trace_batch partitions jobs so that one launch has one kernel variant.
        const FastKernel kernel = pick_kernel<false>(jobs[0].rng_mode == AC_RNG_PHILOX, jobs[0].render_ambisonics != 0,
                                                     jobs[0].visual_limit > 0);
        const size_t smem = stack_smem_bytes(entries);
        const int grid = fast_grid(kernel, device, block, smem, total, cfg ? cfg->grid_blocks : 0);
        kernel<<<grid, block, smem, stream>>>(unused, none, table);
        AC_CUDA_TRY(cudaGetLastError());
    }
    {
        dim3 fgrid(16, static_cast<unsigned>(std::min<int32_t>(count, 65535)));
        finalize_kernel<float><<<fgrid, 256, 0, stream>>>(d_jobs, reinterpret_cast<const FinalizeTargets *>(ws + l.targets),
                                                          count);
        AC_CUDA_TRY(cudaGetLastError());
    }
    return AC_OK;
}

}  // namespace ac
