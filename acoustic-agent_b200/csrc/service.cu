// Continuous batching at kernel level (ac_service_*).
//
// The reference traces one job at a time (api.py:583-639 `run_many`, batch.py:139-185, engine.py:64-73).
// A service keeps ONE persistent float32 tracer launch running while the host appends jobs to a ring of job
// slots in device memory: a job submitted while others are being traced is picked up by the warps as they
// run out of work, so requests that arrive during a launch join it instead of waiting for the next one.
//
// Protocol (one service per device; calls on one service are serialised by its lock):
//  * submit: the job descriptors are staged in pinned memory, copied into their slots and the slots' chunk
//    and ray counters and the jobs' outputs zeroed on the service's copy stream, behind the work the caller
//    queued on its own stream before the call (which may still be writing those outputs); once that copy
//    has completed, the count of published jobs in a host-mapped control word is raised.  A launch is
//    started if none is running.
//  * the launch's warps take chunks of rays job by job from the ring (per-job chunk counters); the warp that
//    finishes a job's last ray converts its fixed-point sums into the float32 echogram and writes the job's
//    sequence number into the job's host-mapped done flag.
//  * poll: the host reads the done flags of the jobs in flight.
//  * every wait in the launch is bounded: once every warp of the launch has had nothing to trace for
//    `idle_timeout_ns` the warps leave together and the launch ends; the next submit or poll starts
//    another.  A launch takes jobs below a window of half the ring beyond its first job and then ends, so
//    a slot is rewritten only after every launch that could hold its old contents in L1 has ended.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include <cuda_runtime.h>

#include "common.h"
#include "scene_internal.h"
#include "trace_launch.cuh"

namespace {

constexpr int kMaxLaunches = 2;
constexpr int kLaunchWords = 64;   // three counters and the closing flag, one 128-byte line each

struct Launch {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    unsigned long long *words = nullptr;   // device: the launch's warp counts (FastTable::launch_words)
    bool alive = false;
    int64_t first = 0;          // lowest sequence number it may take
    int64_t window_end = 0;     // it takes jobs below this only
};

}  // namespace

struct ac_service_s {
    int32_t device = 0;
    int64_t capacity = 0;
    int32_t block = 256;
    int32_t grid = 0;
    int32_t chunk_rays = 64;
    int32_t stack_entries = ac::kBvhStack;         // traversal stack entries per lane
    int64_t idle_ns = 20000000;
    ac::ServiceSlot *slots = nullptr;              // device ring
    ac::ServiceSlotState *state = nullptr;         // device
    unsigned long long *words = nullptr;           // device: low-water mark, published copy, refresh time
                                                   // (one 128-byte line each)
    ac::ServiceControl *control = nullptr;         // host, mapped
    ac::ServiceControl *control_dev = nullptr;     // its device address
    ac::ServiceSlot *staging = nullptr;            // pinned, one ring's worth
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copied = nullptr;
    cudaEvent_t caller_ready = nullptr;            // recorded on the submitting caller's stream
    Launch launches[kMaxLaunches];
    int next_launch = 0;
    int64_t next_seq = 0;                          // sequence number of the next submitted job
    int64_t rays_submitted = 0;                    // rays of all jobs submitted so far
    std::vector<int64_t> inflight;                 // submitted, not yet reported done
    int64_t launches_started = 0;
    std::mutex lock;
};

namespace {

int service_fail_cleanup(ac_service_s *s, int code) {
    if (s->slots) cudaFree(s->slots);
    if (s->state) cudaFree(s->state);
    if (s->words) cudaFree(s->words);
    if (s->control) cudaFreeHost(s->control);
    if (s->staging) cudaFreeHost(s->staging);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->copied) cudaEventDestroy(s->copied);
    if (s->caller_ready) cudaEventDestroy(s->caller_ready);
    for (Launch &l : s->launches) {
        if (l.stream) cudaStreamDestroy(l.stream);
        if (l.done) cudaEventDestroy(l.done);
        if (l.words) cudaFree(l.words);
    }
    delete s;
    return code;
}

// Launches that have finished are marked so; returns the lowest first sequence number of those running.
int64_t refresh_launches(ac_service_s *s) {
    int64_t oldest = INT64_MAX;
    for (Launch &l : s->launches) {
        if (!l.alive) continue;
        const cudaError_t q = cudaEventQuery(l.done);
        if (q == cudaSuccess) {
            l.alive = false;
        } else {
            if (q == cudaErrorNotReady) cudaGetLastError();
            oldest = std::min(oldest, l.first);
        }
    }
    return oldest;
}

// Start a launch when jobs are waiting that no running launch's window covers.
int ensure_launch(ac_service_s *s) {
    refresh_launches(s);
    if (s->inflight.empty()) return AC_OK;
    const int64_t newest = s->next_seq - 1;
    int64_t covered = -1;
    for (const Launch &l : s->launches)
        if (l.alive) covered = std::max(covered, l.window_end - 1);
    if (covered >= newest) return AC_OK;
    Launch *slot = nullptr;
    for (Launch &l : s->launches)
        if (!l.alive) slot = &l;
    if (!slot) return AC_OK;   // two launches running; the next poll starts one when a launch ends
    const int64_t first = *std::min_element(s->inflight.begin(), s->inflight.end());
    slot->first = first;
    slot->window_end = first + s->capacity / 2;
    ac::FastTable t{};
    t.slots = s->slots;
    t.slot_state = s->state;
    t.control = s->control_dev;
    t.low_water = s->words;
    t.published_copy = s->words + 16;
    t.refresh_at = s->words + 32;
    t.window_first = slot->first;
    t.window_end = slot->window_end;
    t.idle_ns = s->idle_ns;
    t.mask = s->capacity - 1;
    t.launch_words = slot->words;
    AC_CUDA_TRY(cudaMemsetAsync(slot->words, 0, kLaunchWords * sizeof(unsigned long long), slot->stream));
    ac::Job<float> unused;
    std::memset(&unused, 0, sizeof(unused));
    ac::FastScene none{};
    ac::trace_fast_kernel<false, true, false, false, true>
        <<<s->grid, s->block, ac::stack_smem_bytes(s->stack_entries), slot->stream>>>(unused, none, t);
    AC_CUDA_TRY(cudaGetLastError());
    AC_CUDA_TRY(cudaEventRecord(slot->done, slot->stream));
    slot->alive = true;
    s->launches_started += 1;
    return AC_OK;
}

__global__ void zero_slots_kernel(const ac::ServiceSlot *slots, ac::ServiceSlotState *state, int64_t first,
                                  int32_t count, int64_t mask) {
    for (int j = blockIdx.y; j < count; j += gridDim.y) {
        const int64_t slot = (first + j) & mask;
        const ac::Job<float> &job = slots[slot].job;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            state[slot].chunks_taken = 0ull;
            state[slot].rays_finished = 0ull;
        }
        const size_t nb = 2 * static_cast<size_t>(ac::kBands) * job.num_bins;
        const size_t ns = static_cast<size_t>(job.scene.num_surfaces);
        const size_t total = nb + 4 * ns + 8;
        for (size_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
            if (i < nb) job.echogram_fx[i] = 0ull;
            else if (i < nb + ns) job.hit_counts[i - nb] = 0ull;
            else if (i < nb + 2 * ns) job.contrib_counts[i - nb - ns] = 0ull;
            else if (i < nb + 4 * ns) job.surface_energy_fx[i - nb - 2 * ns] = 0ull;
            else job.counters[i - nb - 4 * ns] = 0ull;
        }
    }
}

}  // namespace

extern "C" int ac_service_create(const ac_service_config *cfg, ac_service_t *out) {
    ac::NvtxRange nvtx_range("ac_service_create");
    if (!cfg || !out) return ac::fail(AC_ERR_INVALID, "ac_service_create: null argument");
    *out = nullptr;
    const int64_t capacity = cfg->capacity > 0 ? cfg->capacity : 4096;
    if (capacity < 64 || capacity > (1 << 20) || (capacity & (capacity - 1)))
        return ac::fail(AC_ERR_INVALID, "ac_service_create: capacity must be a power of two in 64..2^20");
    const int block = cfg->block_size > 0 ? cfg->block_size : 256;
    if (block % 32 != 0 || block > 256) return ac::fail(AC_ERR_INVALID, "block_size must be a multiple of 32 up to 256");
    if (cfg->chunk_rays < 0 || cfg->blocks_per_sm < 0 || cfg->blocks_per_sm > 8 || cfg->idle_timeout_ns < 0 ||
        cfg->reserve_blocks < 0 ||
        cfg->stack_entries < 0 || cfg->stack_entries > ac::kBvhStack)
        return ac::fail(AC_ERR_INVALID,
                        "ac_service_create: bad chunk_rays, blocks_per_sm, stack_entries, reserve_blocks or "
                        "idle_timeout_ns");
    ac_service_s *s = new (std::nothrow) ac_service_s();
    if (!s) return ac::fail(AC_ERR_NOMEM, "out of host memory");
    s->device = cfg->device;
    s->capacity = capacity;
    s->block = block;
    s->chunk_rays = cfg->chunk_rays > 0 ? cfg->chunk_rays : 64;
    s->stack_entries = cfg->stack_entries > 0 ? cfg->stack_entries : ac::kBvhStack;
    s->idle_ns = cfg->idle_timeout_ns > 0 ? cfg->idle_timeout_ns : 20000000;
    cudaError_t err = cudaSetDevice(s->device);
    if (err != cudaSuccess) {
        ac::fail(AC_ERR_CUDA, "ac_service_create: cudaSetDevice: %s", cudaGetErrorString(err));
        return service_fail_cleanup(s, AC_ERR_CUDA);
    }
    const int per_sm = cfg->blocks_per_sm > 0 ? cfg->blocks_per_sm : 2;
    s->grid = per_sm * ac::device_sm_count(s->device) - cfg->reserve_blocks;
    if (s->grid < 1) {
        ac::fail(AC_ERR_INVALID, "ac_service_create: reserve_blocks leaves no blocks");
        return service_fail_cleanup(s, AC_ERR_INVALID);
    }
    const size_t control_bytes = sizeof(ac::ServiceControl) + sizeof(long long) * static_cast<size_t>(capacity);
    if (cudaMalloc(&s->slots, sizeof(ac::ServiceSlot) * capacity) != cudaSuccess ||
        cudaMalloc(&s->state, sizeof(ac::ServiceSlotState) * capacity) != cudaSuccess ||
        cudaMalloc(&s->words, 48 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&s->control), control_bytes, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void **>(&s->staging), sizeof(ac::ServiceSlot) * capacity,
                      cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        ac::fail(AC_ERR_NOMEM, "ac_service_create: could not allocate the job ring (%lld slots)", (long long)capacity);
        return service_fail_cleanup(s, AC_ERR_NOMEM);
    }
    std::memset(s->control, 0xFF, control_bytes);   // done flags: -1 (no job)
    s->control->published = 0;
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->control_dev), s->control, 0) != cudaSuccess ||
        cudaMemset(s->words, 0, 48 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->caller_ready, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        ac::fail(AC_ERR_CUDA, "ac_service_create: set-up failed");
        return service_fail_cleanup(s, AC_ERR_CUDA);
    }
    for (Launch &l : s->launches) {
        if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc(&l.words, kLaunchWords * sizeof(unsigned long long)) != cudaSuccess) {
            cudaGetLastError();
            ac::fail(AC_ERR_CUDA, "ac_service_create: stream set-up failed");
            return service_fail_cleanup(s, AC_ERR_CUDA);
        }
    }
    *out = s;
    return AC_OK;
}

extern "C" int ac_service_submit(ac_service_t s, const ac_job *jobs, int32_t num_jobs, int64_t *first_seq,
                                 void *stream) {
    ac::NvtxRange nvtx_range("ac_service_submit");
    if (!s || num_jobs < 0 || (num_jobs > 0 && !jobs) || !first_seq)
        return ac::fail(AC_ERR_INVALID, "ac_service_submit: bad argument");
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_job &in = jobs[j];
        const int rc = ac::validate_trace(in.scene, &in.params, &in.outputs);
        if (rc != AC_OK) return ac::fail(rc, "job %d: %s", j, ac_last_error());
        if (in.scene->device != s->device) return ac::fail(AC_ERR_INVALID, "job %d: scene on another device", j);
        if (in.params.precision != AC_PRECISION_FP32 || in.params.rng_mode != AC_RNG_PHILOX ||
            in.params.render_ambisonics || in.params.visual_limit > 0 || in.outputs.ray_surfaces)
            return ac::fail(AC_ERR_INVALID, "job %d: the service traces float32 Philox jobs without ambisonics, "
                            "visual candidates or recorded rays", j);
        if (in.params.num_bounces < 1) return ac::fail(AC_ERR_INVALID, "job %d: needs at least one bounce", j);
        if (in.scene->fast.num_bvh_nodes > 0 && in.scene->bvh_stack_need > s->stack_entries)
            return ac::fail(AC_ERR_INVALID, "job %d: its scene needs %d traversal stack entries, the service has %d",
                            j, in.scene->bvh_stack_need, s->stack_entries);
    }
    std::lock_guard<std::mutex> guard(s->lock);
    *first_seq = s->next_seq;
    if (num_jobs == 0) return AC_OK;
    AC_CUDA_TRY(cudaSetDevice(s->device));
    // a slot is rewritten only when its previous job is done and reported, and no running launch's window
    // reaches back to that job (it could hold the old descriptor in L1)
    const int64_t oldest_launch = refresh_launches(s);
    const int64_t oldest_inflight =
        s->inflight.empty() ? s->next_seq : *std::min_element(s->inflight.begin(), s->inflight.end());
    const int64_t last = s->next_seq + num_jobs - 1;
    if (last - oldest_inflight >= s->capacity / 2 || (oldest_launch != INT64_MAX && last >= oldest_launch + s->capacity))
        return ac::fail(AC_ERR_CAPACITY, "ac_service_submit: the job ring is full (%lld jobs in flight); poll and "
                        "retry", (long long)s->inflight.size());
    for (int32_t j = 0; j < num_jobs; ++j) {
        const ac_job &in = jobs[j];
        const int64_t seq = s->next_seq + j;
        ac::ServiceSlot &sl = s->staging[seq & (s->capacity - 1)];
        std::memset(&sl, 0, sizeof(sl));
        double scale = in.params.energy_scale;
        if (!(scale > 0.0)) scale = ac::choose_energy_scale(in.scene, &in.params);
        if (in.outputs.scale_out) *in.outputs.scale_out = scale;
        ac::fill_job<float>(in.scene, &in.params, &in.outputs, scale, sl.job);
        sl.fast = in.scene->fast;
        sl.echogram = in.outputs.echogram;
        sl.surface_energy = in.outputs.surface_energy;
        sl.seq = seq;
        sl.chunk_rays = s->chunk_rays;
        sl.num_chunks = (in.params.num_rays + s->chunk_rays - 1) / s->chunk_rays;
        sl.scene_id = reinterpret_cast<uint64_t>(in.scene);
        sl.ray_offset = s->rays_submitted;
        s->rays_submitted += in.params.num_rays;
        s->control->done[seq & (s->capacity - 1)] = -1;
    }
    // copy the slots (one or two runs of the ring), zero the jobs' sums and counters -- after what the caller
    // queued on its stream so far (e.g. its own initialisation of the outputs), which could otherwise land
    // on top of the first rays' sums
    AC_CUDA_TRY(cudaEventRecord(s->caller_ready, static_cast<cudaStream_t>(stream)));
    AC_CUDA_TRY(cudaStreamWaitEvent(s->copy_stream, s->caller_ready, 0));
    const int64_t mask = s->capacity - 1;
    int64_t seq = s->next_seq;
    int32_t left = num_jobs;
    while (left > 0) {
        const int64_t at = seq & mask;
        const int32_t run = static_cast<int32_t>(std::min<int64_t>(left, s->capacity - at));
        AC_CUDA_TRY(cudaMemcpyAsync(s->slots + at, s->staging + at, sizeof(ac::ServiceSlot) * run,
                                    cudaMemcpyHostToDevice, s->copy_stream));
        seq += run;
        left -= run;
    }
    dim3 zgrid(16, static_cast<unsigned>(std::min<int32_t>(num_jobs, 65535)));
    zero_slots_kernel<<<zgrid, 256, 0, s->copy_stream>>>(s->slots, s->state, s->next_seq, num_jobs, mask);
    AC_CUDA_TRY(cudaGetLastError());
    AC_CUDA_TRY(cudaEventRecord(s->copied, s->copy_stream));
    AC_CUDA_TRY(cudaEventSynchronize(s->copied));
    for (int32_t j = 0; j < num_jobs; ++j) s->inflight.push_back(s->next_seq + j);
    s->next_seq += num_jobs;
    __atomic_store_n(&s->control->published, static_cast<long long>(s->next_seq), __ATOMIC_RELEASE);
    return ensure_launch(s);
}

extern "C" int ac_service_poll(ac_service_t s, int64_t *done_seqs, int32_t max_done, int32_t *num_done) {
    if (!s || !num_done || max_done < 0 || (max_done > 0 && !done_seqs))
        return ac::fail(AC_ERR_INVALID, "ac_service_poll: bad argument");
    std::lock_guard<std::mutex> guard(s->lock);
    AC_CUDA_TRY(cudaSetDevice(s->device));
    int32_t n = 0;
    const int64_t mask = s->capacity - 1;
    for (size_t k = 0; k < s->inflight.size() && n < max_done;) {
        const int64_t seq = s->inflight[k];
        if (__atomic_load_n(&s->control->done[seq & mask], __ATOMIC_ACQUIRE) == seq) {
            done_seqs[n++] = seq;
            s->inflight[k] = s->inflight.back();
            s->inflight.pop_back();
        } else {
            ++k;
        }
    }
    *num_done = n;
    // a launch that ended (idle, or its window used up) while jobs still wait is replaced
    for (Launch &l : s->launches) {
        if (!l.alive) continue;
        const cudaError_t q = cudaEventQuery(l.done);
        if (q != cudaSuccess && q != cudaErrorNotReady)
            return ac::fail(AC_ERR_CUDA, "ac_service_poll: launch failed: %s", cudaGetErrorString(q));
        if (q == cudaErrorNotReady) cudaGetLastError();
    }
    return ensure_launch(s);
}

extern "C" int ac_service_info(ac_service_t s, ac_service_stats *stats) {
    if (!s || !stats) return ac::fail(AC_ERR_INVALID, "ac_service_info: null argument");
    std::lock_guard<std::mutex> guard(s->lock);
    refresh_launches(s);
    stats->submitted = s->next_seq;
    stats->in_flight = static_cast<int64_t>(s->inflight.size());
    stats->launches = s->launches_started;
    int32_t alive = 0;
    stats->warps_alive = 0;
    stats->warps_waiting = 0;
    for (const Launch &l : s->launches) {
        if (!l.alive) continue;
        alive += 1;
        unsigned long long words[kLaunchWords];
        AC_CUDA_TRY(cudaMemcpyAsync(words, l.words, sizeof(words), cudaMemcpyDeviceToHost, s->copy_stream));
        AC_CUDA_TRY(cudaStreamSynchronize(s->copy_stream));
        stats->warps_alive += static_cast<int64_t>(words[0]);
        stats->warps_waiting += static_cast<int64_t>(words[16]);
    }
    stats->running_launches = alive;
    stats->capacity = s->capacity;
    stats->grid_blocks = s->grid;
    return AC_OK;
}

extern "C" int ac_service_inspect(ac_service_t s, int64_t seq, ac_service_job_state *out) {
    if (!s || !out) return ac::fail(AC_ERR_INVALID, "ac_service_inspect: null argument");
    std::lock_guard<std::mutex> guard(s->lock);
    if (seq < 0 || seq >= s->next_seq || seq < s->next_seq - s->capacity)
        return ac::fail(AC_ERR_INVALID, "ac_service_inspect: %lld is not one of the last %lld jobs submitted",
                        (long long)seq, (long long)s->capacity);
    AC_CUDA_TRY(cudaSetDevice(s->device));
    const int64_t slot = seq & (s->capacity - 1);
    ac::ServiceSlotState st{};
    unsigned long long low = 0;
    AC_CUDA_TRY(cudaMemcpyAsync(&st, s->state + slot, sizeof(st), cudaMemcpyDeviceToHost, s->copy_stream));
    AC_CUDA_TRY(cudaMemcpyAsync(&low, s->words, sizeof(low), cudaMemcpyDeviceToHost, s->copy_stream));
    AC_CUDA_TRY(cudaStreamSynchronize(s->copy_stream));
    const ac::ServiceSlot &sl = s->staging[slot];   // the descriptor as submitted
    std::memset(out, 0, sizeof(*out));
    out->seq = seq;
    out->chunks = sl.num_chunks;
    out->chunks_taken = static_cast<int64_t>(st.chunks_taken);
    out->rays = sl.job.num_rays;
    out->rays_finished = static_cast<int64_t>(st.rays_finished);
    out->done_seq = __atomic_load_n(&s->control->done[slot], __ATOMIC_ACQUIRE);
    out->low_water = static_cast<int64_t>(low);
    out->in_flight = std::find(s->inflight.begin(), s->inflight.end(), seq) != s->inflight.end() ? 1 : 0;
    return AC_OK;
}

extern "C" int ac_service_destroy(ac_service_t s) {
    ac::NvtxRange nvtx_range("ac_service_destroy");
    if (!s) return AC_OK;
    cudaSetDevice(s->device);
    // every launch ends on its own once no work is left (bounded idle wait): wait for them
    for (Launch &l : s->launches)
        if (l.alive) cudaEventSynchronize(l.done);
    cudaStreamSynchronize(s->copy_stream);
    return service_fail_cleanup(s, AC_OK);
}
