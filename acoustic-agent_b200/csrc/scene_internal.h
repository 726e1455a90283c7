// Device-resident scene: the surface SoA packed into 16-byte aligned quads,
// one copy per precision, plus the host-side facts the launchers need.
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "acoustic_rt.h"
#include "trace_fast.cuh"

struct ac_scene_s {
    int32_t device = 0;
    int64_t num_surfaces = 0;
    int64_t num_corners = 0;
    int64_t node_count = 0;
    int64_t leaf_count = 0;
    int32_t max_leaf = 0;
    void *storage_f32 = nullptr;
    void *storage_f64 = nullptr;
    size_t bytes_f32 = 0;
    size_t bytes_f64 = 0;
    ac::SceneDev<float> f32{};
    ac::SceneDev<double> f64{};
    ac::FastScene fast{};          // float32 cluster scan data (inside storage_f32)
    int32_t cluster_size = 8;
    int64_t num_clusters = 0;
    int32_t traversal = AC_TRAVERSAL_SCAN;  // what the float32 kernel uses for this scene
    int32_t bvh_depth = 0;
    int64_t bvh_nodes = 0;
    int32_t bvh_width = 0;
    int32_t bvh_stack_need = 0;
    double max_reflection = 0.0;   // bound used when choosing the fixed-point scale
    double max_scattering = 0.0;
    double min_scattering = 0.0;
    // Last use of the scene on each stream that launched work reading it: an
    // event recorded after that work.  ac_scene_destroy orders the frees after
    // all of them, so a scene may be destroyed while kernels that read it are
    // still queued on streams that do not synchronise with the legacy stream.
    std::mutex use_lock;
    std::vector<std::pair<cudaStream_t, cudaEvent_t>> uses;
};

namespace ac {

template <typename T>
inline const SceneDev<T> &scene_view(const ac_scene_s *s);
template <>
inline const SceneDev<float> &scene_view<float>(const ac_scene_s *s) { return s->f32; }
template <>
inline const SceneDev<double> &scene_view<double>(const ac_scene_s *s) { return s->f64; }

// Power-of-two fixed-point scale: the largest deposit the scene and parameters
// allow, summed over the six bands, maps to at most 2^62.
double choose_energy_scale(const ac_scene_s *scene, const ac_trace_params *p);

// Validates trace parameters against a scene (host-side, before any launch).
int validate_trace(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o);

int device_sm_count(int device);

// Records, after the work just enqueued on `stream`, that `scene` is in use
// there (see ac_scene_s::uses).  Work enqueued while the stream is being
// captured into a CUDA graph is not recorded: the graph's owner keeps the
// scene alive while the graph can still run.
int note_scene_use(ac_scene_s *scene, void *stream);

// Per-precision launchers (trace_f32.cu / trace_f64.cu).
int launch_trace_f32(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     void *stream);
int launch_trace_f64(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     void *stream);
int launch_batch_f32(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                     void *workspace, size_t bytes, void *host_staging, void *stream);
int launch_batch_f64(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                     void *workspace, size_t bytes, void *host_staging, void *stream);
size_t batch_workspace_bytes_f32(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg);
size_t batch_workspace_bytes_f64(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg);

// Jobs of one batch launch: same precision, random-stream mode and ambisonics setting.
struct Partition {
    int key;
    bool fp64;
    std::vector<int32_t> indices;
};
std::vector<Partition> partition_jobs(const ac_job *jobs, int32_t count);
size_t partition_bytes(const ac_job *jobs, const Partition &part, const ac_batch_config *cfg);

}  // namespace ac
