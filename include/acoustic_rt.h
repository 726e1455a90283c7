/*
 * acoustic_rt.h -- C ABI of the B200 reflection-tracing backend for
 * Acoustic Agent.
 *
 * One shared library (libacoustic_rt.so) holds the sm_100a kernels and this
 * ABI.  Every entry point returns an int status (AC_OK or a negative AC_ERR_*
 * code); nothing throws across the ABI and nothing calls exit/abort.  A
 * human-readable message for the last failure on the calling thread is
 * available from ac_last_error().
 *
 * Threading: scene handles are immutable after ac_scene_create and may be
 * shared between threads; each caller thread should use its own CUDA stream.
 * All device work is asynchronous on the stream passed in (a cudaStream_t,
 * passed as void*; NULL = the legacy default stream).
 *
 * Reference interfaces replaced (paths inside the Acoustic Agent project):
 *   ac_bvh_build        acoustic_agent/bvh.py:8-77                   build_bvh
 *   ac_bvh_build_device the same, on the GPU (steam_rt.py:881 calls build_bvh)
 *   ac_scene_create     acoustic_agent/steam_rt.py:834-924           _scene_kernel_arrays
 *                       + acoustic_agent/steam_rt_cuda.py:76-115     device upload / cache
 *   ac_trace            acoustic_agent/steam_rt.py:1757-1804         trace_energy_field
 *                       (kernels: steam_rt.py:4708-4850, steam_rt_cuda.py:491-710)
 *   ac_trace_batch      acoustic_agent/api.py:477-639, batch.py:139-185, engine.py:64-73
 *                       (the per-job loops, run as one persistent launch;
 *                       ac_batch_submit / _poll / _wait / _release queue it)
 *   ac_synthesize       acoustic_agent/steam_rt.py:2205-2232         reconstruct_band_irs
 *                       + steam_rt.py:3070-3083                      bandlimit_band_signals
 *   ac_synthesize_batch the same per RIR, over the per-job loops of engine.py:64-73 and
 *                       batch.py:139-185 (one ragged batch instead of one call per RIR)
 */
#ifndef ACOUSTIC_RT_H
#define ACOUSTIC_RT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AC_ABI_VERSION 2

#define AC_OK 0
#define AC_ERR_INVALID (-1)     /* bad argument, shape or value (reference: ValueError) */
#define AC_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define AC_ERR_NOMEM (-3)       /* device or host allocation failed */
#define AC_ERR_UNSUPPORTED (-4) /* no usable sm_100 device, or option not built */
#define AC_ERR_CAPACITY (-5)    /* a size exceeds a fixed capacity */

enum { AC_KIND_WALL = 0, AC_KIND_HORIZONTAL = 1, AC_KIND_BOX = 2 };
enum { AC_PRECISION_FP32 = 0, AC_PRECISION_FP64 = 1 };
enum { AC_RNG_REFERENCE = 0, AC_RNG_PHILOX = 1 };
/* How the float32 kernel finds the closest surface (results are the same):
 * SCAN walks kind-separated clusters of surfaces in warp lockstep (best for a
 * room with tens of surfaces); BVH lets every lane descend its own path of a
 * surface-area-heuristic BVH over walls and boxes with a short stack (best
 * for multi-room scenes with hundreds of surfaces); HYBRID scans the walls in
 * lockstep and descends a BVH over the boxes only; AUTO picks by size (scan
 * up to 16 walls and boxes, hybrid with up to 16 walls, BVH beyond). */
enum { AC_TRAVERSAL_AUTO = 0, AC_TRAVERSAL_SCAN = 1, AC_TRAVERSAL_BVH = 2, AC_TRAVERSAL_HYBRID = 3 };

typedef struct ac_scene_s *ac_scene_t;

/* Output of ac_bvh_build.  The caller allocates every array with room for
 * 2*num_surfaces-1 nodes and num_surfaces primitives. */
typedef struct ac_bvh {
    double *bounds_min;   /* [nodes,3] */
    double *bounds_max;   /* [nodes,3] */
    int64_t *start;       /* [nodes] first primitive slot of a leaf, -1 for inner nodes */
    int64_t *count;       /* [nodes] primitives in a leaf, 0 for inner nodes */
    int64_t *escape;      /* [nodes] preorder index of the node after this subtree */
    int64_t *primitives;  /* [num_surfaces] surface index per primitive slot */
    int64_t node_count;
    int64_t leaf_count;
    int64_t max_depth;
} ac_bvh;

/* Scene surfaces in the reference's SoA layout (all float64, row-major).
 * If bvh_node_count == 0 the library builds the BVH itself from the padded
 * per-surface AABBs in surface_bounds_min/max (ac_bvh_build, leaf size 4). */
typedef struct ac_scene_desc {
    int64_t num_surfaces;
    const int64_t *kinds;        /* [S] AC_KIND_* */
    const double *wall_a;        /* [S,2] */
    const double *wall_delta;    /* [S,2] */
    const double *wall_z;        /* [S,2] */
    const double *z_values;      /* [S] */
    const double *box_center;    /* [S,2] */
    const double *box_axis_u;    /* [S,2] */
    const double *box_axis_v;    /* [S,2] */
    const double *box_half;      /* [S,2] */
    const double *box_z;         /* [S,2] */
    const double *normals;       /* [S,3] */
    const double *reflection;    /* [S,6] energy reflection = 1 - absorption */
    const double *scattering;    /* [S] band-mean scattering */
    int64_t num_corners;
    const double *corners;       /* [C,2] room polygon for horizontal surfaces */
    const double *surface_bounds_min; /* [S,3] padded AABBs (used when the BVH is built here) */
    const double *surface_bounds_max; /* [S,3] */
    int64_t bvh_node_count;      /* 0: build here with leaf size 4 */
    const double *bvh_bounds_min;
    const double *bvh_bounds_max;
    const int64_t *bvh_start;
    const int64_t *bvh_count;
    const int64_t *bvh_escape;
    const int64_t *bvh_primitives;
    int32_t device;              /* CUDA device ordinal that will own the scene */
    int32_t cluster_size;        /* surfaces per cluster of the float32 scan (0: 32) */
    int32_t traversal;           /* float32 kernel: AC_TRAVERSAL_AUTO / _SCAN / _BVH / _HYBRID */
    int32_t bvh_leaf;            /* float32 BVH: surfaces per leaf, 1..8 (0: 1) */
    int32_t bvh_width;           /* float32 BVH: children per inner node, 2 or 4 (0: the library's default) */
    int32_t reserved;
} ac_scene_desc;

typedef struct ac_scene_info {
    int64_t num_surfaces;
    int64_t num_corners;
    int64_t node_count;
    int64_t leaf_count;
    int64_t device_bytes;        /* device memory held by the scene */
    int32_t device;
    int32_t max_leaf;
    int64_t num_clusters;        /* clusters of the float32 scan */
    int32_t traversal;           /* what the float32 kernel uses: AC_TRAVERSAL_SCAN, _BVH or _HYBRID */
    int32_t bvh_depth;           /* float32 BVH: inner-node levels (0 in scan mode) */
    int64_t bvh_nodes;           /* float32 BVH: inner nodes (0 in scan mode) */
    int32_t bvh_width;           /* float32 BVH: children per inner node (0 in scan mode) */
    int32_t bvh_stack_need;      /* float32 BVH: traversal stack entries a ray can need, the sentinel
                                    included (the least `stack_entries` a launch over it may use) */
} ac_scene_info;

/* One trace: rays from the listener, next-event estimation to the source.
 * Field meanings follow steam_rt.py:1822-1890 (the kernel arguments). */
typedef struct ac_trace_params {
    double source[3];
    double listener[3];
    double source_forward[3];
    int64_t num_rays;
    int32_t num_bounces;
    int32_t num_bins;
    double bin_duration;
    double speed_of_sound;
    double max_path_length;      /* duration * c */
    double direct_delay;         /* |source - listener| / c */
    double listener_radius;
    double source_radius;
    double irradiance_min_distance;
    double specular_exponent;
    double dipole_weight;
    double dipole_power;
    int32_t use_bvh;             /* 0: linear scan over all surfaces, 1: BVH */
    int32_t render_ambisonics;   /* 1: also fill the first-order ambisonic echogram */
    int32_t precision;           /* AC_PRECISION_FP32 (production) or AC_PRECISION_FP64 (parity) */
    int32_t rng_mode;            /* AC_RNG_REFERENCE: arrays below; AC_RNG_PHILOX: on-device stream */
    uint64_t seed;               /* Philox key part 1 */
    uint64_t stream_key;         /* Philox key part 2 (scene identity) */
    /* reference-stream arrays, DEVICE pointers, element type double for FP64
     * and float for FP32 (diffuse_indices is int32 in both):
     * directions [R,3], diffuse_random [B,R], diffuse_indices [B,R]. */
    const void *directions;
    const void *diffuse_random;
    const int32_t *diffuse_indices;
    const void *diffuse_bank;    /* [K,3] device, element type as above; both RNG modes */
    int32_t num_bank;
    int32_t block_size;          /* 0: library default */
    double energy_scale;         /* fixed-point scale (a power of two); 0: library picks (ac_energy_scale) */
    int32_t grid_blocks;         /* 0: library default (persistent, SM-count based) */
    /* Visual-path candidates (steam_rt.py:1853-1860, kernel :4718-4731, :4765-4769,
     * :4821-4824): rays with ray % visual_stride == 0 and ray / visual_stride <
     * visual_limit record their hit points and their strongest contribution.
     * visual_limit = 0: none. */
    int32_t visual_limit;
    int32_t visual_stride;
    /* Float32 BVH scenes: entries of each lane's traversal stack (shared
     * memory, 1 KiB per entry per 256-thread block).  0: the library maximum
     * (32); otherwise bvh_stack_need of the scene .. 32, else AC_ERR_INVALID.
     * A schedule knob: results do not depend on it. */
    int32_t stack_entries;
} ac_trace_params;

/* Outputs.  All pointers are DEVICE memory owned by the caller.  Energies
 * are accumulated as exact fixed point: each deposit is rounded to an integer
 * quantum q = round(energy * scale) (|q| <= 2^62), and each accumulator is a
 * pair of int64 words holding the sum of the quanta's low 32 bits (unsigned)
 * and the sum of their high parts q >> 32 (signed):
 *     value = (word[1] * 2^32 + word[0]) / scale.
 * The sums are exact and independent of order while fewer than 2^32 quanta
 * reach one accumulator, which num_rays * num_bounces < 2^32 guarantees (the
 * call rejects larger jobs with AC_ERR_CAPACITY).  The accumulators are zeroed
 * by the call itself; NULL optional outputs are skipped. */
typedef struct ac_trace_outputs {
    int64_t *echogram_fx;        /* [6,bins,2] required */
    int64_t *ambisonic_fx;       /* [6,4,bins,2] when render_ambisonics */
    int64_t *hit_counts;         /* [S] required */
    int64_t *contrib_counts;     /* [S] required */
    int64_t *surface_energy_fx;  /* [S,2] required */
    int64_t *counters;           /* [8] required: actual_bounces, active_rays, ray_bounces, shadow_rays,
                                    work counter (scratch), 3 reserved */
    float *echogram;             /* [6,bins] optional dequantized copy */
    float *ambisonic;            /* [6,4,bins] optional */
    float *surface_energy;       /* [S] optional */
    int32_t *ray_surfaces;       /* [R,B] optional per-ray hit surface per bounce, -1 after termination */
    double *scale_out;           /* optional host pointer: receives the fixed-point scale used */
    /* Visual-path candidates, required when visual_limit > 0 (L = visual_limit,
     * B = num_bounces; element type float for FP32, double for FP64); the call
     * initialises them like the reference (0, and -1 for the index arrays). */
    void *visual_hit_points;     /* [L,B,3] offset hit point of each bounce */
    int32_t *visual_surfaces;    /* [L,B] hit surface of each bounce */
    int32_t *visual_rays;        /* [L] ray index of the slot */
    int32_t *visual_orders;      /* [L] bounce + 1 of the strongest contribution */
    void *visual_distances;      /* [L] its path length */
    void *visual_gains;          /* [L] sqrt of its six-band energy */
} ac_trace_outputs;

/* One job of a batched launch: a scene, its trace parameters and outputs. */
typedef struct ac_job {
    ac_scene_t scene;
    ac_trace_params params;
    ac_trace_outputs outputs;
} ac_job;

typedef struct ac_batch_config {
    int32_t block_size;          /* threads per block; 0: library default */
    int32_t chunk_rays;          /* rays per work item a warp takes from the queue; 0: default */
    int32_t grid_blocks;         /* persistent blocks; 0: SM count * occupancy */
    int32_t stack_entries;       /* traversal stack entries per lane (0: 32); at least every BVH scene's
                                    bvh_stack_need, else AC_ERR_INVALID */
} ac_batch_config;

/* Band synthesis of J echograms (steam_rt.py:2205-2232, 3070-3083): per
 * band, the amplitude envelope sqrt(E/4pi) interpolated linearly from the
 * previous bin, times the per-bin air-absorption gain, times white noise,
 * then the six-band crossover (eight-pole low-pass differences). */
typedef struct ac_synth_params {
    int32_t num_rirs;
    int32_t num_bins;
    int32_t samples_per_bin;     /* ceil(bin_duration * fs) */
    int32_t sample_rate;
    int32_t rng_mode;            /* AC_RNG_REFERENCE: noise from `white`; AC_RNG_PHILOX: generated from seed */
    int32_t white_shared;        /* 1: one noise row [N] for all RIRs, 0: [J,N] */
    const double *white;         /* device uniform(-1,1) noise (reference mode) */
    uint64_t seed;               /* noise key in Philox mode */
    const double *air;           /* optional [J,6,bins] device air gains; NULL: computed from the fields below */
    const double *direct_delays; /* [J] device seconds (used when air is NULL) */
    double air_coefficients[6];  /* Np/m per band (acoustics.py:12-22) */
    double speed_of_sound;
    double crossover[100];       /* [5 cutoffs][4 sections][b0,b1,b2,a1,a2] low-pass coefficients */
} ac_synth_params;

const char *ac_last_error(void);
int ac_abi_version(void);

/* Host-only: build the preorder escape-link BVH of bvh.py:8-77. */
int ac_bvh_build(const double *bounds_min, const double *bounds_max, int64_t num_surfaces, int32_t leaf_size,
                 ac_bvh *out);

/* The same tree built on the GPU from device-resident bounds (bvh.py:8-77,
 * build_bvh, for scenes of thousands to millions of surfaces).  The tree's
 * shape depends only on num_surfaces and leaf_size (every split is at n/2),
 * so the host plans it; the device chooses each node's axis and partitions its
 * surfaces about the median of the reference's stable sort order.
 *
 * Host-only sizing: *workspace_bytes of device workspace (256-byte aligned),
 * *staging_bytes of the plan copied to the device each call (pass a pinned
 * buffer of that size as host_staging to keep the call asynchronous; with
 * NULL the call synchronizes `stream` after the copy), *node_count nodes. */
int ac_bvh_device_workspace_size(int64_t num_surfaces, int32_t leaf_size, size_t *workspace_bytes,
                                 size_t *staging_bytes, int64_t *node_count);

/* bounds_min/max: device [S,3] float64.  `out` holds device arrays with room
 * for *node_count nodes and S primitive slots; node_count, leaf_count and
 * max_depth are filled on return.  `status` is one device int32, zeroed by the
 * call and, once the stream reaches the end of the build, OR of
 * AC_BVH_STATUS_*; the arrays are only valid when it reads 0.  S >= 1,
 * S < 2^30, 1 <= leaf_size <= 255. */
enum {
    AC_BVH_STATUS_NONFINITE = 1,   /* reference: "BVH bounds must be finite" */
    AC_BVH_STATUS_ORDER = 2,       /* reference: "BVH maximum bounds must not be below minimum bounds" */
    AC_BVH_STATUS_TIMEOUT = 4,     /* a grid barrier gave up waiting (the build is abandoned) */
    AC_BVH_STATUS_INTERNAL = 8     /* a median search ended without its element (a defect) */
};
int ac_bvh_build_device(const double *bounds_min, const double *bounds_max, int64_t num_surfaces,
                        int32_t leaf_size, ac_bvh *out, int32_t *status, void *workspace, size_t workspace_bytes,
                        void *host_staging, void *stream);

/* Device info for the reference's `cuda` result field. */
int ac_device_info(int32_t device, char *name, size_t name_len, int32_t *cc_major, int32_t *cc_minor,
                   int32_t *sm_count);

/* The scene's device memory comes from the device's stream-ordered pool, so
 * creating or destroying a scene does not wait for work that other streams
 * have in flight; ac_scene_create returns once the upload is complete.
 * ac_trace, ac_trace_batch and ac_direct record an event after the work they
 * enqueue on their stream, and ac_scene_destroy frees the scene's memory only
 * after the last such event of every stream: a scene may be destroyed while
 * that work is still queued.  Work enqueued while a stream is being captured
 * into a CUDA graph is not tracked: destroy the scene only after the graph's
 * last replay has finished.  Destroy each scene once, from one thread, after
 * every call that uses it has returned. */
int ac_scene_create(const ac_scene_desc *desc, ac_scene_t *out);
int ac_scene_destroy(ac_scene_t scene);
int ac_scene_get_info(ac_scene_t scene, ac_scene_info *info);

/* Fixed-point scale the library would pick for these parameters: a power of
 * two that maps the largest possible six-band deposit to at most 2^62. */
int ac_energy_scale(ac_scene_t scene, const ac_trace_params *params, double *scale);

int ac_trace(ac_scene_t scene, const ac_trace_params *params, const ac_trace_outputs *outputs, void *stream);

/* Device (and pinned staging) bytes ac_trace_batch needs for these jobs. */
int ac_batch_workspace_size(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, size_t *bytes);

/* Many jobs (any mix of scenes, ray budgets, bins) in one persistent launch.
 * `workspace` is caller-owned device memory of ac_batch_workspace_size bytes.
 * Host-side it writes the job table into `host_staging` (pinned memory of the
 * same size, or NULL to use a pageable copy). */
int ac_trace_batch(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, void *workspace,
                   size_t workspace_bytes, void *host_staging, void *stream);

/* The persistent queue for hosts without the CUDA runtime: ac_batch_submit is
 * ac_trace_batch plus a completion ticket recorded on `stream` after the
 * launches; ac_batch_poll answers *done = 1 once the batch's outputs are
 * written (0 before, never blocking), ac_batch_wait blocks until then, and
 * ac_batch_release frees the ticket (NULL is accepted).  The workspace and
 * outputs must stay alive until the ticket reports done. */
typedef struct ac_batch_ticket_s *ac_batch_ticket_t;
int ac_batch_submit(const ac_job *jobs, int32_t num_jobs, const ac_batch_config *config, void *workspace,
                    size_t workspace_bytes, void *host_staging, void *stream, ac_batch_ticket_t *ticket);
int ac_batch_poll(ac_batch_ticket_t ticket, int32_t *done);
int ac_batch_wait(ac_batch_ticket_t ticket);
int ac_batch_release(ac_batch_ticket_t ticket);

/* Continuous batching: one persistent float32 trace launch fed while it
 * runs.  Replaces the reference's request loops, which trace one job to
 * completion before the next starts (api.py:583-639 `run_many`,
 * batch.py:139-185, engine.py:64-73), as the batched launch above does, but
 * jobs submitted while others are on the GPU join the running launch: its
 * warps take chunks of rays job by job from a ring of job slots in device
 * memory, so a new job starts as soon as warps run out of older work.
 *
 * ac_service_submit appends jobs (the ac_job of ac_trace_batch; float32,
 * Philox stream, no ambisonics, visual candidates or recorded rays, at least
 * one bounce) and returns their sequence numbers first_seq ..
 * first_seq + num_jobs - 1; it returns once their descriptors are in device
 * memory, and starts a launch if none is running.  It zeroes the jobs'
 * outputs itself, after the work queued on `stream` before the call (the
 * caller's own initialisation of those buffers, say): the jobs are traced
 * only once that work is done.  `stream` NULL: the legacy default stream.
 * When the ring cannot take the jobs yet it fails with
 * AC_ERR_CAPACITY: poll and submit again.  ac_service_poll writes the
 * sequence numbers of jobs whose outputs (fixed-point sums, counters, float32
 * echogram and surface energy) are complete since the last poll; it never
 * blocks.  A job's outputs, and its scene, must stay alive until it is
 * reported done.  Keep polling while jobs are in flight: a launch whose
 * warps find no work for idle_timeout_ns ends on its own (every wait in the
 * kernel is bounded), and a poll or submit starts the next one when needed.
 * Results are the same as ac_trace / ac_trace_batch on the same job: rays are
 * keyed by (seed, stream key, ray) and the sums are exact fixed point.
 * Scenes whose memory is freed and reused for another scene while a launch
 * runs could be read stale from L1: destroy scenes only when
 * ac_service_info reports no running launch.  ac_service_destroy waits for
 * the running launches to end. */
typedef struct ac_service_s *ac_service_t;
typedef struct {
    int32_t device;
    int32_t capacity;            /* job slots in the ring, a power of two (0: 4096); at most half in flight */
    int32_t blocks_per_sm;       /* persistent grid (0: 2, which leaves room for synthesis blocks beside it) */
    int32_t block_size;          /* 0: 256 */
    int32_t chunk_rays;          /* rays a warp takes at a time (0: 64) */
    int32_t stack_entries;       /* traversal stack entries per lane (0: 32); a job whose scene needs more
                                    (bvh_stack_need) is refused at submit */
    int64_t idle_timeout_ns;     /* 0: 20 ms */
    int32_t reserve_blocks;      /* grid = blocks_per_sm * SMs - reserve_blocks: the SMs left one block short
                                    keep room for other kernels (band synthesis) beside the persistent launch */
    int32_t reserved;
} ac_service_config;
typedef struct {
    int64_t submitted;           /* jobs submitted so far (next sequence number) */
    int64_t in_flight;           /* submitted and not yet reported done */
    int64_t launches;            /* persistent launches started so far */
    int32_t running_launches;
    int32_t grid_blocks;
    int64_t capacity;
    int64_t warps_alive;         /* warps of the running launches that may still take work */
    int64_t warps_waiting;       /* of those, the ones waiting for work */
} ac_service_stats;
/* Progress of one submitted job, for monitoring (a job that stops moving is
 * visible here): the counters are read from the device while launches run. */
typedef struct {
    int64_t seq;
    int64_t chunks;              /* chunks of rays the job was split into */
    int64_t chunks_taken;        /* taken by warps so far (may exceed `chunks`: late takers find none) */
    int64_t rays;
    int64_t rays_finished;       /* rays whose sums are complete */
    int64_t done_seq;            /* the slot's done flag: == seq once the job's outputs are final */
    int64_t low_water;           /* jobs below it have no chunks left */
    int32_t in_flight;           /* 1: submitted and not yet reported done by ac_service_poll */
    int32_t reserved;
} ac_service_job_state;
int ac_service_create(const ac_service_config *config, ac_service_t *out);
int ac_service_submit(ac_service_t service, const ac_job *jobs, int32_t num_jobs, int64_t *first_seq,
                      void *stream);
int ac_service_poll(ac_service_t service, int64_t *done_seqs, int32_t max_done, int32_t *num_done);
int ac_service_info(ac_service_t service, ac_service_stats *stats);
/* AC_ERR_INVALID unless `seq` is one of the last `capacity` jobs submitted. */
int ac_service_inspect(ac_service_t service, int64_t seq, ac_service_job_state *state);
int ac_service_destroy(ac_service_t service);

/* Device workspace needed by ac_synthesize. */
int ac_synth_workspace_size(const ac_synth_params *params, size_t *bytes);

/* echograms: [J,6,bins] float32 device.  band_irs: [J,6,bins*spb] float32 device.
 * `workspace` is caller-owned device memory of ac_synth_workspace_size bytes. */
int ac_synthesize(const float *echograms, const ac_synth_params *params, float *band_irs, void *workspace,
                  size_t workspace_bytes, void *stream);

/* ac_synthesize without any device allocation.  No counterpart in the
 * reference (its synthesis runs on the CPU).  For callers that must not
 * allocate device memory: a real-time audio thread, where cudaMalloc can
 * block on the driver for milliseconds, or a host engine that owns the whole
 * device-memory budget and forbids third-party allocations.  The caller passes
 * inputs and outputs as for ac_synthesize; the workspace comes from a static
 * device array of AC_SYNTH_STATIC_BYTES that every GPU loading the library
 * holds until exit.  Calls whose workspace (ac_synth_workspace_size) exceeds
 * it fail with AC_ERR_CAPACITY; split the RIRs over several calls.  The first
 * call on a device looks up the array's device address, so make that first
 * call before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
#define AC_SYNTH_STATIC_BYTES (16u << 20)
int ac_synthesize_static(const float *echograms, const ac_synth_params *params, float *band_irs, void *stream);

/* One RIR of a ragged synthesis batch: reconstruct_band_irs
 * (steam_rt.py:2205-2232) for one echogram, with its own length, sample rate
 * and noise.  Every output sample equals what ac_synthesize gives for the
 * same echogram alone (same noise, same air gains). */
typedef struct ac_synth_job {
    const float *echogram;       /* [6, num_bins] float32 device */
    float *band_irs;             /* [6, num_bins * samples_per_bin] float32 device */
    const double *white;         /* AC_RNG_REFERENCE: [num_bins * samples_per_bin] device uniform(-1, 1) noise */
    const double *air;           /* optional [6, num_bins] device air gains; NULL: computed from direct_delay */
    uint64_t seed;               /* AC_RNG_PHILOX: noise key, the same noise as ac_synthesize with this seed */
    double direct_delay;         /* seconds (steam_rt.py:2214) */
    double speed_of_sound;
    int32_t num_bins;
    int32_t samples_per_bin;     /* ceil(bin_duration * fs) */
    int32_t rate_index;          /* which sample rate / crossover table of the batch config */
    int32_t rng_mode;
} ac_synth_job;

#define AC_SYNTH_MAX_RATES 4
typedef struct ac_synth_batch_config {
    int32_t num_rates;                               /* 1 .. AC_SYNTH_MAX_RATES */
    int32_t sample_rates[AC_SYNTH_MAX_RATES];
    double crossover[AC_SYNTH_MAX_RATES][100];       /* per rate, as ac_synth_params.crossover */
    double air_coefficients[6];                      /* Np/m per band (acoustics.py:12-22) */
} ac_synth_batch_config;

/* Device workspace and pinned staging bytes for ac_synthesize_batch. */
int ac_synth_batch_workspace_size(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                                  size_t *bytes);

/* Any mix of echogram lengths and sample rates in one set of launches (three
 * kernels whatever the batch).  Replaces the per-RIR reconstruct_band_irs
 * calls of engine.py:64-73 / batch.py:139-185.  The job table is written to
 * `host_staging` (pinned, ac_synth_batch_workspace_size bytes, or NULL for a
 * pageable copy) and copied into `workspace` on `stream`; the staging must
 * stay unchanged until the copy has run (for a captured graph: while the
 * graph is replayed). */
int ac_synthesize_batch(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                        void *workspace, size_t workspace_bytes, void *host_staging, void *stream);

/* ac_synthesize_batch in two phases on possibly different streams, for a
 * caller that overlaps the recursion with other work: _raw copies the job
 * table and writes the raw band signals (fully parallel, a fraction of a
 * millisecond); _filter runs the crossover recursion (one warp per four band
 * signals, latency-bound) from what _raw left in `workspace`.  Same jobs,
 * config and workspace for both; _filter must be ordered after _raw. */
int ac_synthesize_batch_raw(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                            void *workspace, size_t workspace_bytes, void *host_staging, void *stream);
int ac_synthesize_batch_filter(const ac_synth_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                               void *workspace, size_t workspace_bytes, void *stream);

/* ---- late reverberation (steam_rt.py:2235-2640) ------------------------
 *
 * One FDN impulse response: _fdn_impulse_kernel(delays, absorptive,
 * preroll + num_samples, allpass_delays, tone)[preroll:]
 * (steam_rt.py:2235-2327, called at :2579-2586).  The delay and filter design
 * (_steam_fdn_delays, _steam_fdn_filter_coefficients, :2330-2470) is host
 * work and arrives here as numbers.  Every output sample is bit-identical to
 * the reference's float64 kernel given the same design. */
#define AC_FDN_LINES 16
#define AC_FDN_ALLPASS 4
#define AC_FDN_MIN_DELAY 128     /* delay lines shorter than this are refused (the reference design keeps them
                                    above 280 samples from 8 kHz up) */
#define AC_FDN_MAX_ALLPASS 4096  /* longest all-pass stage; the shortest must exceed 32 */
typedef struct ac_fdn_job {
    double absorptive[AC_FDN_LINES][6][5];  /* per line and band: b0 b1 b2 a1 a2 */
    double tone[6][5];                      /* output tone-correction sections */
    int32_t delays[AC_FDN_LINES];           /* delay-line lengths in samples */
    int32_t allpass_delays[AC_FDN_ALLPASS]; /* Schroeder all-pass lengths (225, 341, 441, 556 in the reference) */
    int32_t num_samples;                    /* samples written to `out` */
    int32_t preroll;                        /* samples run before the first one written */
    double *out;                            /* device [num_samples] float64 */
} ac_fdn_job;

/* Device workspace (job table + delay lines) and pinned staging bytes for ac_fdn_impulse. */
int ac_fdn_workspace_size(const ac_fdn_job *jobs, int32_t num_jobs, size_t *bytes);

/* Any number of FDN impulse responses in one launch (one 192-thread block per
 * job); the job table is staged as for ac_synthesize_batch. */
int ac_fdn_impulse(const ac_fdn_job *jobs, int32_t num_jobs, void *workspace, size_t workspace_bytes,
                   void *host_staging, void *stream);

/* The hybrid tail of _render_parametric_fdn_late_reverb
 * (steam_rt.py:2588-2640) for one RIR: the FDN impulse is split into six
 * bands by bandlimit_band_signals, each band is scaled so that its energy
 * after `anchor` equals the traced power there decaying at the band's RT60
 * (_late_tail_start_power, :2473-2497), and crossfaded into the traced band
 * signal with the equal-power ramp over [start, end).  Bands with rt60 <= 0
 * keep the unscaled FDN, as in the reference.  Outputs are the float32 casts
 * the reference returns; `stats` receives per band AC_LATE_STATS doubles. */
#define AC_LATE_STATS 8
enum {
    AC_LATE_SCALE = 0,          /* scale_by_band (1 for rt60 <= 0) */
    AC_LATE_POWER = 1,          /* anchor_power_by_band */
    AC_LATE_FDN_ENERGY = 2,     /* fdn_energy_by_band: sum of the scaled FDN band from start */
    AC_LATE_TRACED_TAIL = 3,    /* sum of traced^2 from start */
    AC_LATE_RENDERED_TAIL = 4,  /* sum of out^2 (float64, before the cast) from start */
    AC_LATE_COMPONENT = 5,      /* sum of fdn_component^2 (float64) over the band */
    AC_LATE_CHANGED = 6,        /* 1 if any sample from `changed_from` fails allclose(out, traced, 1e-7, 1e-12) */
};
typedef struct ac_late_tail_job {
    const double *traced;     /* device [6, num_samples] float64 traced band signals */
    const double *fdn;        /* device [num_samples] float64 FDN impulse (ac_fdn_impulse's out) */
    float *out;               /* device [6, num_samples] hybrid band signals */
    float *fdn_component;     /* device [6, num_samples] the crossfaded FDN part of `out` */
    double *stats;            /* device [6, AC_LATE_STATS] */
    double rt60[6];           /* target RT60 per band in seconds */
    int32_t start[6];         /* crossfade start sample per band */
    int32_t end[6];           /* crossfade end sample per band (> start) */
    int32_t anchor[6];        /* sample where the tail power is measured (start, or end at a fitted breakpoint) */
    int32_t changed_from;     /* first sample of the `changed` test (the smallest start) */
    int32_t num_samples;
    int32_t bin_samples;      /* round(bin_duration * fs), at least 1 */
    int32_t rate_index;       /* sample rate / crossover table of the config */
} ac_late_tail_job;

int ac_late_tail_workspace_size(const ac_late_tail_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                                size_t *bytes);
int ac_late_tail(const ac_late_tail_job *jobs, int32_t num_jobs, const ac_synth_batch_config *config,
                 void *workspace, size_t workspace_bytes, void *host_staging, void *stream);

/* ---- direct path (steam_rt.py:1315-1350) ------------------------------
 *
 * The occlusion part of simulate_direct for any number of (source,
 * listener) pairs of one scene, in float64 with the reference's own surface
 * tests (RoomRayScene.closest_hit / any_hit, steam_rt.py:320-352, where a
 * point on the room outline counts as inside): the first surface between
 * listener and source, the volumetric visibility fraction over a sphere of
 * sample points around the source (_volumetric_occlusion, :4215-4240) and,
 * when that is below one, the per-band transmission through the distinct
 * surfaces crossed from both ends (_transmission, :3437-3462).  Distances,
 * gains and delays stay host arithmetic. */
#define AC_DIRECT_MAX_LAYERS 64
typedef struct ac_direct_query {
    double source[3];
    double listener[3];
    double radius;            /* direct_occlusion_radius_m */
    int32_t occlusion;        /* direct_occlusion: 0 leaves occlusion 1 and transmission 1 */
    int32_t volumetric;       /* direct_occlusion_mode == "volumetric"; 0: the blocking surface decides */
    int32_t transmission;     /* direct_transmission: 0 gives zero transmission when occluded */
    int32_t max_layers;       /* max(1, num_transmission_rays), at most AC_DIRECT_MAX_LAYERS */
} ac_direct_query;

typedef struct ac_direct_result {
    double occlusion;         /* visible fraction of the source sphere (or 0 / 1) */
    double transmission[6];
    int32_t occlusion_surface;  /* surface index between listener and source, -1 if none */
    int32_t reserved;
} ac_direct_result;

typedef struct ac_direct_tables {
    const double *unit_samples;   /* device [num_samples, 3]: _sphere_volume_samples(num_samples) */
    int32_t num_samples;          /* direct_occlusion_samples */
    int32_t reserved;
    const double *transmission;   /* device [S, 6] per-surface band transmission */
    const int32_t *surface_group; /* device [S]: surfaces that share a name share a group */
} ac_direct_tables;

/* Device workspace and pinned staging bytes for ac_direct. */
int ac_direct_workspace_size(int32_t num_queries, size_t *bytes);

/* One warp per query on `stream`; results is device memory [num_queries]. */
int ac_direct(ac_scene_t scene, const ac_direct_query *queries, int32_t num_queries, const ac_direct_tables *tables,
              ac_direct_result *results, void *workspace, size_t workspace_bytes, void *host_staging, void *stream);

/* Measurement helper, no counterpart in the reference: reads `bytes` (a
 * multiple of 16 is used) of device memory `repeats` times with 16-byte loads
 * cached in L2 only, on `stream`; time it with events to get the L2 (buffer
 * smaller than L2) or HBM (larger) read bandwidth the tracer's roofline is
 * reported against.  `sink` is one device word the kernel may write. */
int ac_read_bandwidth_probe(const void *buffer, size_t bytes, int32_t repeats, unsigned long long *sink, void *stream);

/* Measurement helper, no counterpart in the reference: launches independent
 * float64 add and multiply chains (separate instructions, as the bit-exact
 * float64 kernels issue them) over every SM on `stream` and returns in *ops
 * the operations launched; time it with events for the float64 issue rate
 * the FDN's roofline is reported against.  `sink` is one device word. */
int ac_fp64_rate_probe(int32_t iterations, unsigned long long *sink, int64_t *ops, void *stream);

/* Test: the device BVH build's grid barrier alone.  `blocks` blocks (1..64)
 * wait for `expected_blocks` arrivals, each giving up after `poll_limit` polls
 * (1..2^26): with expected_blocks > blocks no wait can end, so *status (one
 * device int32, zeroed by the call) reads AC_BVH_STATUS_TIMEOUT once the
 * stream reaches the end, and the kernel has returned.  `workspace`: 8 bytes
 * of device memory, zeroed by the call. */
int ac_bvh_barrier_probe(int32_t blocks, int32_t expected_blocks, int64_t poll_limit, void *workspace,
                         int32_t *status, void *stream);

/* The reference's per-bounce random workspace drawn on the device, bit for
 * bit: replaces the host loop of steam_rt.py:4009-4044
 * (`_diffuse_random_sequence`: for each bounce, `rng.random(R)` then
 * `rng.integers(0, num_bank, R, dtype=int32)` from `rng = default_rng(seed + 1)`)
 * and the upload of its 12 bytes per ray-bounce.  (state, inc) are that
 * generator's 128-bit PCG64 state and increment before its first draw, split
 * into 64-bit halves (numpy's `bit_generator.state`).  Writes `random`
 * [num_bounces, num_rays] (double for AC_PRECISION_FP64, else float, rounded
 * from the double draw) and `indices` [num_bounces, num_rays] int32, device
 * memory, asynchronously on `stream`.  num_bank must be a power of two
 * (AC_ERR_UNSUPPORTED otherwise: numpy's bounded draw can then consume an
 * extra word at an unpredictable place; draw such workspaces on the host);
 * the default bank of 128 qualifies.  The directions of the same workspace
 * (steam_rt.py:3959-3968) use the host's cos/sin and stay on the host. */
int ac_reference_stream(uint64_t state_hi, uint64_t state_lo, uint64_t inc_hi, uint64_t inc_lo, int64_t num_rays,
                        int32_t num_bounces, int32_t num_bank, int32_t precision, void *random, int32_t *indices,
                        void *stream);

/* Debug/test: fill the Philox reference-equivalent workspace the kernels
 * generate internally (directions [R,3], random [B,R], indices [B,R]). */
int ac_philox_workspace(uint64_t seed, uint64_t stream_key, int64_t num_rays, int32_t num_bounces,
                        int32_t num_bank, int32_t precision, void *directions, void *random,
                        int32_t *indices, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ACOUSTIC_RT_H */
