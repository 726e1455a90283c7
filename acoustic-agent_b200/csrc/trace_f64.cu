// FP64 parity instantiation of the tracer.  Built with -fmad=false: every
// multiply and add rounds on its own, as in the Numba float64 reference.
#include "trace_launch.cuh"

namespace ac {

int launch_trace_f64(const ac_scene_s *scene, const ac_trace_params *p, const ac_trace_outputs *o, double scale,
                     void *stream) {
    int rc = launch_single<double>(scene, p, o, scale, stream);
    if (rc != AC_OK) return rc;
    return launch_finalize_single<double>(scene, p, o, scale, stream);
}

int launch_batch_f64(const ac_job *jobs, const int32_t *indices, int32_t count, const ac_batch_config *cfg,
                     void *workspace, size_t bytes, void *host_staging, void *stream) {
    return launch_batch<double>(jobs, indices, count, cfg, workspace, bytes, host_staging, stream);
}

size_t batch_workspace_bytes_f64(const ac_job *, const int32_t *, int32_t count, const ac_batch_config *) {
    return batch_bytes<double>(count);
}

}  // namespace ac
