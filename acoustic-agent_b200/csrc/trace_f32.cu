// FP32 production instantiation of the tracer (FMA contraction allowed).
#include "trace_launch.cuh"

namespace ac {

int launch_trace_f32(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     void *stream) {
    int rc = launch_single<float>(scene, p, o, scale, stream);
    if (rc != AC_OK) return rc;
    return launch_finalize_single<float>(scene, p, o, scale, stream);
}

int launch_batch_f32(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                     void *workspace, size_t bytes, void *host_staging, void *stream) {
    return launch_batch<float>(jobs, indices, count, cfg, workspace, bytes, host_staging, stream);
}

size_t batch_workspace_bytes_f32(int32_t count) { return batch_bytes<float>(count); }

}  // namespace ac
