/*
 * turbo_hot.h — C ABI of the B200 (sm_100a) TurboNeRF training hot path.
 *
 * Conventions
 *  - Every entry point returns int: TN_OK (0) or a negative TN_E_* status. No C++
 *    exception crosses this boundary; tn_last_error() gives a message for the calling
 *    thread.
 *  - All buffers are device pointers owned by the caller, in the reference's
 *    structure-of-arrays layout: component c of item i lives at buf[c * stride + i]
 *    (reference: src/workspaces/training-workspace.cuh:87-112). Ray buffers use
 *    `ray_stride`, per-sample buffers `sample_stride`.
 *  - Every compute call takes a cudaStream_t (passed as tn_stream_t, the same type) and
 *    only enqueues work: no host synchronisation, except the functions of the "plain"
 *    family and the *_sync helpers, which reproduce the reference's blocking structure.
 *  - The library owns only the opaque tn_ctx (scratch buffers, device error flags,
 *    tuning table). One context per stream/thread.
 */
#ifndef TURBO_HOT_H
#define TURBO_HOT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* tn_stream_t; /* identical to cudaStream_t */

#define TN_OK 0
#define TN_E_INVALID (-1)     /* an argument is out of range */
#define TN_E_NULL (-2)        /* a required pointer is NULL */
#define TN_E_CAPACITY (-3)    /* a size exceeds a capacity or limit */
#define TN_E_CUDA (-4)        /* a CUDA runtime call failed */
#define TN_E_NO_RAYS (-5)     /* the batch cut found no ray (reference: trainer.cu:162-164) */
#define TN_E_NO_SAMPLES (-6)  /* the batch cut found no sample (reference: trainer.cu:181-183) */
#define TN_E_LEVELS (-7)      /* cascade count outside 1..8 */
#define TN_E_DEVICE (-8)      /* a kernel raised a device-side error flag (see tn_ctx_check) */
#define TN_E_STATE (-9)       /* call not valid in the current state (e.g. during capture) */

/* Device-side error bits reported by tn_ctx_check. */
#define TN_FLAG_GUARD 1u      /* a march loop hit max_iterations */
#define TN_FLAG_CAPACITY 2u   /* an offset + count exceeded the sample capacity */
#define TN_FLAG_NO_RAYS 4u
#define TN_FLAG_NO_SAMPLES 8u
#define TN_FLAG_SPIN 16u      /* a bounded spin-wait gave up */

/* Compositor input activation. */
#define TN_ACT_SIGMA 0        /* input is sigma; d sigma / d input = 1 */
#define TN_ACT_DENSITY 1      /* input is the network density: sigma = exp(min(d,12)-1),
                                 reference density_to_sigma, common-network-kernels.cuh:7-10 */

/* Axis-aligned box; same POD layout as the reference's BoundingBox
 * (src/models/bounding-box.cuh:8-16). contains() is inclusive on both faces. */
typedef struct tn_bbox {
    float min_x, min_y, min_z;
    float max_x, max_y, max_z;
} tn_bbox;

/* Cascaded occupancy grid (reference OccupancyGrid, src/core/occupancy-grid.cuh:22-287).
 * Level k covers the cube [-base*2^k/2, base*2^k/2]^3 with resolution^3 cells; the
 * bitfield holds one byte per Morton-ordered cell, bit k = level k; density holds
 * [n_levels][resolution^3] floats. base_size = 1 reproduces the reference exactly
 * (level extent 2^k, occupancy-grid.cuh:139-141). */
typedef struct tn_grid_desc {
    int32_t n_levels;    /* 1..8 */
    int32_t resolution;  /* power of two, 2..1024 (the reference uses 128) */
    float base_size;     /* extent of level 0 in world units */
    int32_t reserved;
} tn_grid_desc;

/* Step control of the march (reference get_dt, src/utils/raymarching-utils.cuh:7-14,
 * called with dt_max = aabb_size * dt_min at src/core/trainer.cu:102-104). */
typedef struct tn_march_desc {
    float cone_angle;        /* reference NeRFConstants::cone_angle = 1/256 */
    float dt_min;            /* reference min_step_size = sqrt(3)/1024 */
    float dt_max;
    uint32_t max_steps;      /* 0 = unlimited (reference); otherwise samples per ray are capped */
    uint32_t max_iterations; /* loop guard per ray; 0 selects 1<<22. Exceeding it raises TN_FLAG_GUARD */
} tn_march_desc;

/* Per-ray sample ranges of a packed batch. n_rays bounds the launch; when n_rays_dev is
 * non-NULL the kernels read the live ray count from that device word (<= n_rays), so a
 * batch cut computed on the device needs no host round trip. */
typedef struct tn_ray_batch {
    uint32_t n_rays;
    uint32_t ray_stride;
    uint32_t sample_stride;
    uint32_t reserved;
    const uint32_t* counts;      /* [ray] samples per ray */
    const uint32_t* offsets;     /* [ray] first sample of each ray (exclusive scan of counts) */
    const uint32_t* n_rays_dev;  /* optional device count */
} tn_ray_batch;

typedef struct tn_ctx tn_ctx;

/* ---- library / context ------------------------------------------------------------ */
int tn_version(void);
const char* tn_last_error(void);
/* Creates a context on the current CUDA device. */
int tn_ctx_create(tn_ctx** out);
int tn_ctx_destroy(tn_ctx* ctx);
/* Grows the context scratch for batches of up to max_rays rays / max_samples samples
 * (call before stream capture; kernels never allocate). */
int tn_ctx_reserve(tn_ctx* ctx, uint32_t max_rays, uint32_t max_samples);
/* Synchronises `stream`, returns the device error bits raised since the last check in
 * *flags_out and clears them. */
int tn_ctx_check(tn_ctx* ctx, tn_stream_t stream, uint32_t* flags_out);
/* Device pointer of the context's error word (for graph users that read it themselves). */
int tn_ctx_flags_ptr(tn_ctx* ctx, uint32_t** flags_dev);

/* ---- launch shapes and the autotuner ---------------------------------------------------
 * No reference counterpart: the reference fixes its launch shapes (tcnn's linear_kernel,
 * 128 or 512 threads a block). Each field below only changes how the work is split over
 * blocks, warps and lanes. Counts, offsets, samples, per-ray values and gradients are
 * bit-identical for every valid shape; the scalar loss sums of tn_train_losses are the same
 * per-ray terms summed in another order. A context starts with tn_tuning_default. */
typedef struct tn_tuning {
    uint32_t count_rays_per_block;  /* march count, one thread per ray: 32, 64, 128 or 256 (64) */
    uint32_t emit_warps_per_block;  /* march emit: 1, 2, 4, 8 or 16 warps a block (8) */
    uint32_t emit_rays_per_warp;    /* march emit: 1, 2 or 4 rays a warp = 32, 16 or 8 lanes a ray (1) */
    uint32_t loss_rays_per_block;   /* fused losses, one warp per ray: 2, 4 or 8 (4) */
    uint32_t compact_tile;          /* compaction: values a block, 128, 256, 512, 1024 or 2048 (128) */
    uint32_t multi_chunk_rays;      /* multi-scene count: rays per work-stealing chunk, 32..256 (64) */
    uint32_t side_sms;              /* 0 (default) or the SMs kept for work beside the march: every
                                       count block then reserves over half an SM's shared memory,
                                       so that blocks of kernels doing the same (the training
                                       controller's Adam of the previous step) run on other SMs;
                                       below the device's SM count */
} tn_tuning;

void tn_tuning_default(tn_tuning* out);
/* TN_OK when every field holds one of its listed values. */
int tn_tuning_validate(const tn_tuning* t);
/* Sets / reads the shapes later calls on this context use. A tn_march_emit uses the count
 * block size of the tn_march_count before it, whatever the tuning is by then (likewise the
 * multi-scene emit and chunk size). */
int tn_ctx_set_tuning(tn_ctx* ctx, const tn_tuning* t);
int tn_ctx_get_tuning(tn_ctx* ctx, tn_tuning* out);

/* Result of one autotuner call: the candidates tried, the median time of one call with the
 * shape the context had before and with the shape chosen (CUDA events on the caller's stream). */
typedef struct tn_tune_report {
    uint32_t n_candidates;
    float before_ms;
    float best_ms;
} tn_tune_report;

/* ---- ray set-up (a 'next' stage of the reference path) ---------------------------- */
/* Bounding-box clip of initialize_training_rays_and_pixels_kernel
 * (reference src/utils/training-batch-kernels.cuh:122-150): t = max(0, tmin + 1e-5),
 * t_max = min(t_far, tmax), alive = hit && t <= t_max. */
int tn_rays_init_bbox(tn_stream_t stream, uint32_t n_rays, uint32_t ray_stride, const tn_bbox* bbox,
                      float t_far, const float* ori, const float* dir, float* t, float* t_max,
                      uint8_t* alive);

/* ---- fused march + compaction --------------------------------------------------- */
/* Count pass (reference march_and_count_steps_per_ray_kernel,
 * src/utils/training-batch-kernels.cuh:212-298) fused with the batch cut of
 * src/core/trainer.cu:133-183: writes n_steps[ray], clears alive for rays with no step,
 * and writes batch_info[0] = n_rays_cut (rays [0, n_rays_cut) fill the batch),
 * batch_info[1] = n_samples = offsets[n_rays_cut], where offsets is the exclusive scan of
 * n_steps, and batch_info[2] = total samples of all n_rays rays. The offsets themselves are
 * written by tn_march_emit. batch_size is the sample capacity (reference batch_size);
 * batch_size = UINT32_MAX disables the cut (render use: every ray is kept and
 * batch_info = {n_rays, total, total}). */
int tn_march_count(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                   const tn_bbox* bbox, const tn_march_desc* march, uint32_t n_rays, uint32_t ray_stride,
                   const uint32_t* n_rays_dev, const float* ori, const float* dir, const float* ray_t,
                   const float* ray_t_max, uint8_t* alive, uint32_t* n_steps, uint32_t batch_size,
                   uint32_t* batch_info);

/* Emit pass (reference march_and_generate_network_positions_kernel,
 * src/utils/training-batch-kernels.cuh:339-481): for rays [0, batch_info[0]) writes
 * offsets[ray] and, per sample at offsets[ray] + j: t, pos[3] (normalised to [0,1]),
 * dir[3] (0.5*d+0.5), dt (= dt/aabb_size, the compositor's dt), m_norm, dt_norm and
 * img_id (optional, from ray_img_id). offsets holds the exclusive scan of n_steps for all
 * n_rays rays (rays at or beyond the cut emit nothing). Must follow tn_march_count on the
 * same context with the same n_rays: it expands the step positions that pass recorded. */
int tn_march_emit(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                  const tn_bbox* bbox, const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays,
                  uint32_t ray_stride, uint32_t sample_stride, const uint32_t* batch_info,
                  const uint32_t* ray_img_id, const float* ori, const float* dir, const float* ray_t,
                  const uint8_t* alive, const uint32_t* n_steps, uint32_t* offsets,
                  uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                  float* out_m_norm, float* out_dt_norm);
/* Autotuner of the march (tn_tuning count_rays_per_block, then emit_warps_per_block x
 * emit_rays_per_warp): times tn_march_count with every count block size on these rays, keeps
 * the fastest, then tn_march_emit with every emit shape on the counts it produced. The
 * arguments are those of tn_march_count (without n_rays_dev) and tn_march_emit together; on
 * return they hold the outputs of one count + emit call with the chosen shapes. Synchronises
 * the stream; not while it is being captured. Reports may be NULL. */
int tn_autotune_march(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                      const tn_bbox* bbox, const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays,
                      uint32_t ray_stride, const uint32_t* ray_img_id, const float* ori, const float* dir,
                      const float* ray_t, const float* ray_t_max, uint8_t* alive, uint32_t* n_steps,
                      uint32_t batch_size, uint32_t* batch_info, uint32_t sample_stride, uint32_t* offsets,
                      uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                      float* out_m_norm, float* out_dt_norm, tn_tune_report* count_report,
                      tn_tune_report* emit_report);

/* ---- several scenes in one launch (batched multi-scene training) -------------------
 * No single reference call: the reference trains one scene per process. These entry points run
 * the march count and emit of many scenes at once; per scene, counts, offsets and samples equal
 * those of tn_march_count / tn_march_emit without a batch cut (batch_size = UINT32_MAX). */
typedef struct tn_scene {
    tn_grid_desc grid;
    const uint8_t* bitfield;   /* device, R^3 bytes, 16-byte aligned */
    tn_bbox bbox;
    tn_march_desc march;
    float inv_aabb_size;       /* emit: 1 / aabb size of the scene */
    uint32_t ray_begin;        /* first ray of the scene in the shared ray arrays */
    uint32_t n_rays;           /* scenes are given in ray order and do not overlap */
} tn_scene;
#define TN_MAX_SCENES 32

/* Counts the steps of every ray of every scene in one persistent launch: blocks take 64-ray
 * chunks of any scene from a shared counter (work stealing). Writes n_steps and alive for
 * every scene ray, scene_samples[n_scenes] (device, optional: samples per scene) and
 * batch_info[4] (device: total rays, total samples). Samples are packed scene after scene. */
int tn_multi_march_count(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                         uint32_t ray_stride, const float* ori, const float* dir, const float* ray_t,
                         const float* ray_t_max, uint8_t* alive, uint32_t* n_steps, uint32_t* scene_samples,
                         uint32_t* batch_info);
/* Offsets (exclusive scan over all scene rays, in scene order) and the samples of every scene
 * (same outputs as tn_march_emit), after tn_multi_march_count on the same context and scenes. */
int tn_multi_march_emit(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                        uint32_t ray_stride, uint32_t sample_stride, const uint32_t* ray_img_id, const float* ori,
                        const float* dir, const float* ray_t, const uint8_t* alive, const uint32_t* n_steps,
                        uint32_t* offsets, uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir,
                        float* out_dt, float* out_m_norm, float* out_dt_norm);
/* Autotuner of the multi-scene march (multi_chunk_rays, then the emit shape), as
 * tn_autotune_march; the arguments are those of the two multi-scene calls together. */
int tn_autotune_multi(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                      uint32_t ray_stride, const uint32_t* ray_img_id, const float* ori, const float* dir,
                      const float* ray_t, const float* ray_t_max, uint8_t* alive, uint32_t* n_steps,
                      uint32_t* scene_samples, uint32_t* batch_info, uint32_t sample_stride, uint32_t* offsets,
                      uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                      float* out_m_norm, float* out_dt_norm, tn_tune_report* count_report,
                      tn_tune_report* emit_report);

/* Exclusive scan + batch cut of arbitrary counts (reference trainer.cu:146-183 with
 * find_last_lt_presorted, src/utils/parallel-utils.cuh:31-58). batch_info as above. */
int tn_scan_offsets(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                    uint32_t batch_size, uint32_t* batch_info);

/* Allocation-free variant of tn_scan_offsets, with the same outputs (offsets, batch_info),
 * for callers that cannot allocate device memory and hold no tn_ctx: for instance a plugin
 * whose host application owns every device allocation, or a loop that must not pay the
 * device synchronisation of cudaMalloc. No counterpart in the reference (which has no such
 * callers). Its scratch is a fixed array inside the library image (128.25 KiB), held by every
 * device that loads the library until exit.
 *
 * Limit: n <= TN_SCAN_NOALLOC_MAX_COUNTS; larger n returns TN_E_CAPACITY at once.
 *
 * Errors found on the device: with no tn_ctx there is no tn_ctx_check, so the call stores its
 * device-side error bits (TN_FLAG_* above; 0 when the call succeeded) into *error_word, a
 * caller-owned device word written by a plain store at the end of the call (it needs no
 * clearing). They are TN_FLAG_NO_RAYS and TN_FLAG_NO_SAMPLES (the reference's two runtime
 * errors of the batch cut; batch_info then holds n_rays = n_samples = 0) and TN_FLAG_CAPACITY
 * (the total of the counts passed 2^32: offsets past that point are wrong). error_word may be
 * NULL; batch_info[0] == 0 or batch_info[1] == 0 then remain the only signs of an empty cut.
 *
 * The first call on a device (and the first after a cudaDeviceReset) looks up the array's
 * device address, so make that first call before any stream capture. All calls share the
 * array and keep the last call's contents: calls that overlap on the GPU race and must be
 * serialised. */
#define TN_SCAN_NOALLOC_MAX_COUNTS (1u << 21)
int tn_scan_offsets_noalloc(tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                            uint32_t batch_size, uint32_t* batch_info, uint32_t* error_word);

/* Ascending list of the indices i < n with values[i] != 0 (reference
 * generate_nonzero_compaction_indices, src/utils/stream-compaction.cuh:120-139);
 * *count_dev receives the list length. */
int tn_compact_nonzero(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* values, int32_t* out,
                       uint32_t* count_dev);
/* Autotuner of the compaction tile (compact_tile), as tn_autotune_march. */
int tn_autotune_compact(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* values, int32_t* out,
                        uint32_t* count_dev, tn_tune_report* report);

/* ---- compositor (sample tiles over runs of rays, segmented warp scans) ------------ */
/* Forward (reference density_to_ray_rgba_forward, training-kernels-fused.cuh:227-264):
 * rgba[4][ray_stride]; optional per-ray saved state for the backward: depth[ray]
 * (optical depth up to the transmittance cut) and n_used[ray] (samples composited). */
int tn_composite_fwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                     float min_transmittance, const float* density, const float* rgb, const float* dt,
                     float* rgba, float* depth, uint32_t* n_used);

/* Vector-Jacobian product of tn_composite_fwd: given grad_rgba[4][ray_stride], writes
 * dL/d density [sample] and dL/d rgb [3][sample_stride] (zero past each ray's cut).
 * Transmittance is recomputed by a reverse scan from the saved per-ray depth and n_used;
 * no per-sample state from the forward is read. */
int tn_composite_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                     const float* density, const float* rgb, const float* dt, const float* depth,
                     const uint32_t* n_used, const float* grad_rgba, float* dL_ddensity, float* dL_drgb);

/* The store-instead-of-recompute alternative of the pair above (for the memory study of the
 * backward): the forward also writes, for every composited sample, the transmittance after
 * it and its weight (t_saved, w_saved [sample_stride]); the backward reads them instead of
 * recomputing them. Same results within FP32 rounding; 8 more bytes per sample of memory. */
int tn_composite_fwd_store(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                           float min_transmittance, const float* density, const float* rgb, const float* dt,
                           float* rgba, uint32_t* n_used, float* t_saved, float* w_saved);
int tn_composite_bwd_stored(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                            const float* density, const float* rgb, const float* dt, const uint32_t* n_used,
                            const float* t_saved, const float* w_saved, const float* grad_rgba, float* dL_ddensity,
                            float* dL_drgb);

/* Reconstruction loss forward + backward in one pass (reference
 * fused_reconstruction_forward_backward_kernel, training-kernels-fused.cuh:381-498):
 * composite, random-background blend of target and prediction, smooth-L1 loss,
 * dL/dR_c = inv_nrays * huber'(d_c); writes dL/d density and grad_scale * dL/d rgb
 * (zero past the cut). Optional outputs: ray_rgba[4][ray_stride], loss[4][ray_stride],
 * loss_sum[1] (device: inv_nrays * sum over rays of the 4 channel losses). */
int tn_recon_loss_fwd_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                          float min_transmittance, float inv_nrays, float grad_scale, const float* density,
                          const float* rgb, const float* dt, const float* target_rgba, const float* bg_rgb,
                          float* ray_rgba, float* loss, float* loss_sum, float* dL_ddensity, float* dL_drgb);

/* mip-NeRF 360 distortion loss forward (+ backward when dL_ddensity != NULL)
 * (reference mipNeRF360_distortion_loss_forward/backward_kernel,
 * training-kernels-fused.cuh:13-224). ray_loss[ray] = lambda/N * (dt w^2 / 3 + 2 * cross
 * terms); loss_sum[1] = mean over rays; grad_ray (optional) scales each ray's gradient
 * (the reference uses 1). */
int tn_distortion_fwd_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                          float lambda, const float* density, const float* m_norm, const float* dt_norm,
                          const float* grad_ray, float* ray_loss, float* loss_sum, float* dL_ddensity);

/* Gradient merge (reference nerf-network.cu:734-758): grad_out[i] += loss_scale *
 * (dL_rec[i] + dL_dist[i]) then *= t[i]^2 where t[i] < 1 (apply_gradient_distance_scaling,
 * training-kernels-fused.cuh:500-515). dL_dist and t may be NULL. n_samples_dev, when
 * non-NULL, holds the live sample count (<= n_samples). */
int tn_grad_epilogue(tn_stream_t stream, uint32_t n_samples, const uint32_t* n_samples_dev, float loss_scale,
                     const float* dL_rec, const float* dL_dist, const float* t, float* grad_out);

/* Everything between the network forward and backward in one kernel: reconstruction
 * loss fwd/bwd, distortion loss fwd/bwd (lambda > 0) and the gradient merge into
 * grad_density (accumulated, then distance-scaled when t != NULL). dL_drgb receives
 * grad_scale * dL/d rgb. loss_sums[0] = reconstruction loss, loss_sums[1] = distortion. */
int tn_train_losses(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                    float min_transmittance, float inv_nrays, const uint32_t* inv_nrays_from_dev,
                    float grad_scale, float lambda, const float* density, const float* rgb,
                    const float* dt, const float* m_norm, const float* dt_norm, const float* t,
                    const float* target_rgba, const float* bg_rgb, float* ray_rgba, float* grad_density,
                    float* dL_drgb, float* loss_sums);
/* Autotuner of the fused loss kernel's block size (loss_rays_per_block), as
 * tn_autotune_march. grad_density is restored to its values on entry before every call, so
 * on return it holds the result of one call. */
int tn_autotune_losses(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                       float min_transmittance, float inv_nrays, const uint32_t* inv_nrays_from_dev,
                       float grad_scale, float lambda, const float* density, const float* rgb, const float* dt,
                       const float* m_norm, const float* dt_norm, const float* t, const float* target_rgba,
                       const float* bg_rgb, float* ray_rgba, float* grad_density, float* dL_drgb, float* loss_sums,
                       tn_tune_report* report);

/* ---- occupancy grid ------------------------------------------------------------- */
/* Network sample points for (level, cell) pairs (reference
 * generate_grid_cell_network_sample_points_kernel, occupancy-grid-kernels.cu:38-76):
 * out_pos[3][pos_stride] = (cell corner + rand * voxel) * inv_aabb + 0.5. */
int tn_occupancy_sample_points(tn_stream_t stream, const tn_grid_desc* grid, uint32_t n, const int32_t* levels,
                               const uint32_t* cells, const float* rand3, uint32_t rand_stride,
                               float inv_aabb_size, float* out_pos, uint32_t pos_stride);

/* Decay, max-update of the listed (level, cell) pairs and bitfield rebuild in two
 * kernels (reference occupancy-grid-kernels.cu:16-141, trainer.cu:221-311):
 * density *= decay everywhere; for each update u whose selection passes
 * (sample_all, or rand_select[u] < 0.25, or rand_select[u] <= 0.5 and the cell is
 * occupied at its level) density = max(density, act(values[u])); bits = density >
 * threshold; *n_occupied_dev = popcount of the bitfield (optional). */
int tn_occupancy_update(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, float* density,
                        uint8_t* bitfield, uint32_t n_updates, const int32_t* levels, const uint32_t* cells,
                        const float* values, const float* rand_select, int activation, int sample_all,
                        float decay, float threshold, uint32_t* n_occupied_dev);

/* Number of set bits in n_bytes bytes (reference count_1s, src/utils/bit-utils.cuh:52-94). */
int tn_popcount(tn_ctx* ctx, tn_stream_t stream, uint64_t n_bytes, const uint8_t* bytes, uint32_t* out_dev);

/* ---- Adam ---------------------------------------------------------------------- */
/* Reference ngp_adam_step (src/core/adam-optimizer.cuh:48-96), vectorised by 4: params
 * [0, n_grid) are the hash grid (a zero gradient skips the parameter: no moment decay,
 * no step), [n_grid, n_grid+n_mlp) get L2 regularisation. lr is the already-decayed rate
 * (reference 1e-2 / (1 + 3.3e-5 * step), nerf-network.cu:256). weights_copy (optional)
 * receives the updated weights again (the network-precision copy). */
int tn_adam_step(tn_stream_t stream, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale, float lr,
                 float beta1, float beta2, float epsilon, float l2_reg, float* weights, float* weights_copy,
                 const float* gradients, float* first_moments, float* second_moments, uint32_t* param_steps);

/* ---- plain path: one kernel per stage, one thread per ray --------------------------
 * The reference's launch structure, kept as the baseline the fused path is measured
 * against: thrust scans, blocking device->host reads, memsets, dense launches. */
int tn_plain_march_count(tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                         const tn_bbox* bbox, const tn_march_desc* march, uint32_t n_rays, uint32_t ray_stride,
                         const float* ori, const float* dir, const float* ray_t, const float* ray_t_max,
                         uint8_t* alive, uint32_t* n_steps);
/* thrust exclusive_scan + reverse find_if + device->host copy + stream synchronise. */
int tn_plain_scan_cut_sync(tn_stream_t stream, uint32_t n, const uint32_t* n_steps, uint32_t* offsets,
                           uint32_t batch_size, uint32_t* n_rays_out, uint32_t* n_samples_out);
int tn_plain_march_emit(tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                        const tn_bbox* bbox, const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays,
                        uint32_t ray_stride, uint32_t sample_stride, const uint32_t* ray_img_id,
                        const float* ori, const float* dir, const float* ray_t, const uint32_t* offsets,
                        const uint8_t* alive, const uint32_t* n_steps, uint32_t* out_img_id, float* out_t,
                        float* out_pos, float* out_dir, float* out_dt, float* out_m_norm, float* out_dt_norm);
/* memsets + one thread per ray + thrust::reduce with a blocking read of the loss. */
int tn_plain_recon_loss_sync(tn_stream_t stream, const tn_ray_batch* batch, int activation,
                             float min_transmittance, float inv_nrays, float grad_scale, const float* density,
                             const float* rgb, const float* dt, const float* target_rgba, const float* bg_rgb,
                             float* loss, float* dL_ddensity, float* dL_drgb, float* loss_out);
/* memset + forward kernel + backward kernel (per-sample w_cs/wm_cs scratch, caller
 * provided: 2 * sample_stride floats and 5 * ray_stride floats) + thrust::reduce. */
int tn_plain_distortion_sync(tn_stream_t stream, const tn_ray_batch* batch, int activation, float lambda,
                             const float* density, const float* m_norm, const float* dt_norm, float* ray_scratch,
                             float* sample_scratch, float* ray_loss, float* dL_ddensity, float* loss_out);
int tn_plain_grad_epilogue(tn_stream_t stream, uint32_t n_samples, float loss_scale, const float* dL_rec,
                           const float* dL_dist, const float* t, float* grad_out);
int tn_plain_occupancy_update_sync(tn_stream_t stream, const tn_grid_desc* grid, float* density,
                                   uint8_t* bitfield, uint32_t n_updates, const int32_t* levels,
                                   const uint32_t* cells, const float* values, const float* rand_select,
                                   int activation, int sample_all, float decay, float threshold,
                                   uint8_t* count_scratch, uint32_t* n_occupied_out);
int tn_plain_adam_step(tn_stream_t stream, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale,
                       float lr, float beta1, float beta2, float epsilon, float l2_reg, float* weights,
                       float* weights_copy, const float* gradients, float* first_moments, float* second_moments,
                       uint32_t* param_steps);

/* ---- synthetic producer (stand-in for the tiny-cuda-nn network) ------------------ */
/* Gaussian-blob density and sinusoid colour at normalised positions pos[3][pos_stride]
 * (world = (pos - 0.5) * aabb_size). blobs[n_blobs][5] = (cx, cy, cz, std, peak),
 * waves[3][4] = (ax, ay, az, phase) are device arrays. n_dev optional live count. */
int tn_synth_field(tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t pos_stride, const float* pos,
                   float aabb_size, uint32_t n_blobs, const float* blobs, const float* waves, float* sigma,
                   float* rgb, uint32_t out_stride);

/* ---- hash-grid encoding (the tiny-cuda-nn boundary) ---------------------------------
 * The multiresolution hash encoding that the reference builds as tcnn's HashGrid
 * (src/core/nerf-network.cu:27-124: 16 levels of 2 features, 2^19 entries a level, base
 * resolution 16, per-level scale b = exp((ln 2048 aabb - ln 16) / 15), linear interpolation) and
 * runs forward (:431-545) and backward (:668-768). Level l has resolution
 * N_l = floor(base_resolution * per_level_scale^l); a normalised position x in [0,1]^3 takes the
 * trilinear interpolation of the 2 features of its cell's 8 corner vertices; a level whose
 * (N_l + 1)^3 vertices fit in its 2^log2_hashmap_size entries indexes them directly, the others
 * by the spatial hash (x * 1 ^ y * 2654435761 ^ z * 805459861) mod 2^log2_hashmap_size.
 * Parameters [level][2^log2_hashmap_size][2]; features [2 n_levels][stride]. */
typedef struct tn_hashgrid_desc {
    uint32_t n_levels;          /* 1..16 */
    uint32_t log2_hashmap_size; /* entries a level = 2^log2_hashmap_size, 4..24 */
    float base_resolution;      /* N_min >= 1 */
    float per_level_scale;      /* b >= 1 */
} tn_hashgrid_desc;
/* Parameter counts: hash entries (n_levels 2^log2 2 floats) and the linear heads the trainer's
 * hash-grid network adds (density and rgb from the 2 n_levels features: 4 (2 n_levels + 1)). */
int tn_hashgrid_n_params(const tn_hashgrid_desc* desc, uint64_t* n_hash, uint32_t* n_head);
/* Resolution of one level and whether it indexes its vertices directly (dense = 1). */
int tn_hashgrid_level_resolution(const tn_hashgrid_desc* desc, uint32_t level, uint32_t* resolution, int* dense);
/* features[2l + f][i] for the n (n_dev: live count, optional) positions pos[3][stride]. */
int tn_hashgrid_encode(tn_stream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                       uint32_t stride, const float* pos, const float* params, float* features);
/* grads += d features / d params^T dL_dfeatures (atomic adds). With touched_bits (caller-zeroed,
 * n_levels 2^log2 bits), touched_list and touched_count (zero on entry): every entry a live
 * sample touches is listed once as l 2^log2 + index, in no particular order; its bit stays set. */
int tn_hashgrid_backward(tn_stream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                         uint32_t stride, const float* pos, const float* dL_dfeatures, float* grads,
                         uint32_t* touched_bits, uint32_t* touched_list, uint32_t* touched_count);
/* Zeroes the listed entries' gradients (both features) and bitmap words, then the count. */
int tn_hashgrid_clear_touched(tn_stream_t stream, const uint32_t* touched_list, const uint32_t* touched_count,
                              uint32_t max_entries, float* grads, uint32_t* touched_bits);

/* ---- trainer: the controller surface ----------------------------------------------
 * Mirrors the reference's NeRFTrainingController / Trainer (src/controllers/
 * nerf-training-controller.h:23-89, src/core/trainer.cuh:21-70): setup, train_step(),
 * update_occupancy_grid(step), with the TrainingMetrics / OccupancyGridMetrics structs
 * of nerf-training-controller.h:25-51. The network between the march and the losses is
 * pluggable (tn_network); without one the trainer uses its built-in synthetic scene (a
 * Gaussian-blob field for sigma/rgb and fixed sparse hash-grid gradients). */
#define TN_PATH_FUSED 0 /* fused kernels, device batch cut, optional CUDA graph */
#define TN_PATH_PLAIN 1 /* one kernel per stage, thrust, blocking reads (reference structure) */

/* Producer/consumer of per-sample network values (the tiny-cuda-nn boundary). Every
 * callback only enqueues work on `stream`; n is the buffer capacity, n_dev (device) the
 * live count. Positions are normalised to [0,1]^3, [3][stride]. */
typedef struct tn_network {
    void* user;
    int activation; /* TN_ACT_SIGMA or TN_ACT_DENSITY: what `forward` writes into density */
    int (*forward)(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                   const float* pos, const float* dir, float* density, float* rgb);
    /* dL/d density (merged, scaled) and dL/d rgb -> parameter gradients; may be NULL. Both
     * hold the n_dev live samples; entries past them are unspecified. */
    int (*backward)(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                    const float* pos, const float* dir, const float* dL_ddensity, const float* dL_drgb,
                    float* param_grads);
    /* density only, for occupancy updates */
    int (*density)(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                   const float* pos, float* density);
} tn_network;

/* ---- renderer: inference images of one NeRF ---------------------------------------
 * Reference Renderer::submit / perform_task (src/core/renderer.cu:172-646) for one NeRF
 * with an identity transform, through the linear ray batch
 * (src/rendering/ray-batch-coordinators/linear-buffer-ray-batch-coordinator.cu). */

/* Pinhole camera (reference Camera, src/models/camera.cuh:34-137; lens distortion is not
 * part of this surface). transform: camera to world, row-major 3 x 4 [R | t]. */
typedef struct tn_camera {
    int32_t width, height;
    float near, far;                 /* ray origins at `near`, t_max = far - near */
    float focal_x, focal_y;          /* pixels */
    float principal_x, principal_y;  /* pixels */
    float shift_x, shift_y;          /* fractions of the resolution */
    float transform[12];
} tn_camera;

typedef struct tn_render_desc {
    tn_grid_desc grid;
    const uint8_t* bitfield;         /* device, as tn_march_count */
    tn_bbox render_bbox;             /* samples outside it are skipped */
    tn_bbox training_bbox;           /* network positions = (p - min) / (max - min) */
    float dt_min;                    /* reference min_step_size; dt_max = 8 dt_min */
    float cone_angle;                /* reference NeRFConstants::cone_angle */
    float min_transmittance;         /* reference NeRFConstants::min_transmittance = 1e-4 */
    uint32_t batch_size;             /* samples per round; 0 selects 8 per pixel within [2^20, 2^25] */
} tn_render_desc;

typedef struct tn_render_stats {
    uint32_t rays_hit;    /* pixels whose ray meets the render box */
    uint32_t iterations;  /* march/network/composite rounds */
    uint64_t samples;     /* samples sent to the network */
    uint64_t steps;       /* march steps taken (the reference's t += dt steps) */
    uint64_t tests;       /* steps whose sample was tested; the others crossed known-empty cells */
} tn_render_stats;

/* Renders camera->width x camera->height pixels into out_rgba (device, interleaved
 * premultiplied RGBA, pixel i at out_rgba[4 i .. 4 i + 3]; pixels whose ray misses the
 * box are 0). Queries net->forward on packed valid samples. Synchronous: it reads the live
 * ray count back after every round, so not during stream capture. stats may be NULL. */
int tn_render(tn_ctx* ctx, tn_stream_t stream, const tn_render_desc* desc, const tn_camera* camera,
              const tn_network* net, float* out_rgba, tn_render_stats* stats);

/* ---- training rays from posed images ------------------------------------------------
 * Reference initialize_training_rays_and_pixels_kernel + deactivate_rays_with_alpha_threshold_kernel
 * (src/utils/training-batch-kernels.cuh:82-208) as called by Trainer::generate_next_training_batch
 * (src/core/trainer.cu:40-100). Ray i belongs to image (uint32)(i / (n_rays / n_images)), at pixel
 * position p = width * height * random[i] (x = fmod(p, width), y = p / width) of that image's
 * camera (device array of tn_camera, no lens distortion); it is clipped to bbox (t = max(0,
 * t_min + 1e-5), t_max = min(far - near, box exit); alive = 0 when it misses or t_max < t); its
 * target is the RGBA8 texel min(floor(p), w h - 1) of images [n_images][height][width][4] (device)
 * over 255. With alpha_threshold < 1 and alpha_probability < 1, a ray whose target alpha is below
 * the threshold is dropped when random[ray_stride + i] > alpha_probability. Outputs [c][ray_stride];
 * img_id may be NULL. */
int tn_dataset_rays(tn_stream_t stream, uint32_t n_rays, uint32_t ray_stride, uint32_t n_images, int32_t width,
                    int32_t height, const tn_camera* cameras, const uint8_t* images, const tn_bbox* bbox,
                    const float* random, float alpha_threshold, float alpha_probability, float* pix_rgba,
                    uint32_t* img_id, float* ori, float* dir, float* ray_t, float* ray_t_max, uint8_t* alive);

typedef struct tn_trainer_desc {
    tn_grid_desc grid;
    tn_bbox bbox;                       /* training box; aabb size = max_x - min_x */
    uint32_t batch_size;                /* sample capacity per step (reference batch_size) */
    uint32_t n_rays_per_step;           /* rays generated and marched per step */
    float min_step_size;                /* reference NeRFConstants::min_step_size */
    float cone_angle;                   /* reference NeRFConstants::cone_angle */
    uint32_t max_steps_per_ray;         /* 0 = unlimited */
    float min_transmittance;            /* 1e-4 */
    int32_t use_distortion_loss;
    float distortion_lambda;            /* reference 0.01 */
    float loss_scale;                   /* reference LOSS_SCALE (1 with fp32 network values) */
    float occupancy_decay;              /* 0.95 */
    float occupancy_threshold;          /* reference 0.01 * min_step_size */
    uint32_t occupancy_cells_per_step;  /* > 0: re-sample this many random cells in every step */
    uint32_t n_grid_params;             /* parameter layout [hash grid | MLP] */
    uint32_t n_mlp_params;
    float learning_rate;                /* 1e-2, decayed as lr / (1 + decay * step) */
    float learning_rate_decay;          /* 3.3e-5 */
    float beta1, beta2, epsilon, l2_reg;
    int32_t path;                       /* TN_PATH_FUSED or TN_PATH_PLAIN */
    int32_t use_cuda_graph;             /* fused path: capture the step once, replay after */
    uint32_t seed;
    float ray_radius;                   /* synthetic rays: origin sphere radius */
    float ray_jitter;                   /* synthetic rays: direction jitter */
} tn_trainer_desc;

typedef struct tn_training_metrics {
    uint32_t step;
    uint32_t n_rays;
    uint32_t n_samples;
    float loss;
} tn_training_metrics;

typedef struct tn_occupancy_metrics {
    uint32_t n_occupied;
    uint32_t n_total;
} tn_occupancy_metrics;

typedef struct tn_trainer tn_trainer;

/* Fills `out` with the reference defaults. */
int tn_trainer_default_desc(tn_trainer_desc* out);
/* Creates the trainer on the current device: allocates every buffer once (no allocation
 * during steps), initialises the grid like the reference (all bits set, densities 0) and
 * the parameters. `net` may be NULL (built-in synthetic scene). */
int tn_trainer_create(tn_trainer** out, const tn_trainer_desc* desc, const tn_network* net);
int tn_trainer_destroy(tn_trainer* tr);
/* Synthetic scene of the built-in network: n_blobs x (cx, cy, cz, std, peak) and 3 x
 * (ax, ay, az, phase), host arrays. */
int tn_trainer_set_synthetic_field(tn_trainer* tr, uint32_t n_blobs, const float* blobs, const float* waves);
/* Copies a grid state from host memory (density [n_levels][res^3], bitfield [res^3]). */
int tn_trainer_set_grid(tn_trainer* tr, const float* density, const uint8_t* bitfield);
/* Fills the parameter gradient buffer with N(0, std) values on the hash-grid entries that
 * one step's samples touch (and on every MLP weight), zero elsewhere; the built-in
 * network then leaves it unchanged, so every step feeds Adam the same sparse gradients. */
int tn_trainer_init_synthetic_gradients(tn_trainer* tr, float std, uint32_t* n_touched_out);
/* Makes the hash-grid encoding with linear density and colour heads the trainer's network (in
 * place of the synthetic producer): its parameters are the trainer's (hash entries in the grid
 * section, which must hold them exactly; the heads at the start of the MLP section), its
 * backward writes real gradients (the heads' over their parameters, the hash entries' by atomic
 * adds into a cleared gradient section) and lists the hash entries with a nonzero gradient; Adam
 * skips the others as in the reference. Fused path only. */
int tn_trainer_use_hashgrid(tn_trainer* tr, const tn_hashgrid_desc* desc);
/* One training step (reference NeRFTrainingController::train_step,
 * nerf-training-controller.cu:185-212). With metrics == NULL the fused path only enqueues
 * (no host synchronisation); otherwise the call waits and fills the metrics.
 * With tn_tuning side_sms > 0 (the default when at least 16 SMs remain beside a march of
 * 256-ray blocks) the fused path counts ahead: the step's tail (emit, network, losses, Adam,
 * occupancy update) runs beside the next step's rays and march count, which start once the
 * occupancy update has rewritten the grid; results are those of the in-order step, bit for
 * bit. A head counted ahead is dropped when the grid, the ray source or the launch shapes
 * change. */
int tn_trainer_train_step(tn_trainer* tr, tn_training_metrics* metrics);
/* The same step on rays supplied by the caller in host memory (pinned for asynchronous
 * copies): ori/dir [3][n_rays], target_rgba [4][n_rays], bg_rgb [3][n_rays]; n_rays must
 * equal n_rays_per_step. Stands in for the reference's camera/image ray generation
 * (training-batch-kernels.cuh:82-187); the box clip runs on the device. */
int tn_trainer_train_step_rays(tn_trainer* tr, uint32_t n_rays, const float* ori, const float* dir,
                               const float* target_rgba, const float* bg_rgb, tn_training_metrics* metrics);
/* The same step as tn_trainer_train_step_rays, pipelined for a training loop that feeds rays
 * from the host: the call copies this step's rays in and enqueues the tail of the previous
 * pipelined step beside this step's rays and march count (its head), then returns the
 * previous step's metrics in *previous, waiting for that step's tail only, so the GPU always
 * has work queued. previous->step = 0 on the first pipelined call (after a synchronous read:
 * tn_trainer_sync_metrics runs the last step's tail and returns its metrics). A previous step's
 * device error is reported by this call's status. The host arrays of a step must stay
 * unchanged until the call after it returns. Fused path only. */
int tn_trainer_train_step_rays_pipelined(tn_trainer* tr, uint32_t n_rays, const float* ori, const float* dir,
                                         const float* target_rgba, const float* bg_rgb,
                                         tn_training_metrics* previous);
/* Runs one fused step eagerly with events between its stages and writes the stage times
 * (ms): rays, march count, march emit, network forward, losses, network backward,
 * Adam, occupancy query (cell sampling and the density network), occupancy update. */
int tn_trainer_profile_step(tn_trainer* tr, float* stage_ms, uint32_t max_stages, uint32_t* n_stages);
/* Tunes the trainer's launch shapes on its own batch (the rays of the last step, or freshly
 * generated synthetic rays before the first one): the march (count and emit) and the fused
 * losses. Leaves weights, optimizer state and the occupancy grid untouched; the next step
 * captures its graph again with the chosen shapes. reports[3] (may be NULL): count, emit,
 * losses. Synchronous. */
int tn_trainer_autotune(tn_trainer* tr, tn_tune_report* reports);
/* Runs the tail of a pipelined caller-ray step still pending (tn_trainer_train_step_rays_pipelined
 * leaves it to the next call) and waits for the trainer's stream. tn_trainer_buffer, the
 * snapshot, render and metric calls do the same first. */
int tn_trainer_flush(tn_trainer* tr);
/* Clears the training data (reference NeRFTrainingController::reset_training,
 * src/controllers/nerf-training-controller.cu:108-120, bound at
 * src/api/python_bindings.cu:453-457): parameters re-drawn from the seed, Adam moments and
 * per-parameter step counts zero, every occupancy bit set and densities zero
 * (occupancy-grid.cuh:81-85), step counter and metrics zero.
 * Buffers, launch shapes, the dataset and the network are kept. Synchronous. */
int tn_trainer_reset(tn_trainer* tr);
/* Launch shapes of the trainer's context; setting them (validated) makes the next step
 * capture its graph again. */
int tn_trainer_get_tuning(tn_trainer* tr, tn_tuning* out);
int tn_trainer_set_tuning(tn_trainer* tr, const tn_tuning* t);
/* Renders the trainer's scene (its grid, training box, cone angle, transmittance cut and
 * network) with tn_render (reference NeRFRenderingController::submit,
 * src/controllers/nerf-rendering-controller.cu:50). render_bbox NULL selects the training
 * box; min_step_size <= 0 the trainer's; batch_size 0 the tn_render default.
 * A pending caller-ray step completes first. */
int tn_trainer_render(tn_trainer* tr, const tn_camera* camera, const tn_bbox* render_bbox, float min_step_size,
                      uint32_t batch_size, float* out_rgba, tn_render_stats* stats);
/* Trains on rays from posed images instead of the built-in synthetic rays (the reference trains
 * on its Dataset, src/core/trainer.cu:40-100): n_images cameras and RGBA8 images
 * [n_images][height][width][4], host arrays, copied to the device. Every step draws its pixel
 * positions, alpha-selection draws and background colours from the trainer's seed and step
 * (tn_dataset_rays). The next step captures its graph again. */
int tn_trainer_set_dataset(tn_trainer* tr, uint32_t n_images, int32_t width, int32_t height, const tn_camera* cameras,
                           const uint8_t* images);
/* The training controller's alpha selection (reference NeRFTrainingController::
 * alpha_selection_threshold / alpha_selection_probability, nerf-training-controller.h:75-76):
 * while both are below 1, dataset rays whose target alpha is below the threshold are kept with
 * the given probability. Defaults 1, 1 (off). */
int tn_trainer_set_alpha_selection(tn_trainer* tr, float threshold, float probability);
/* .turbo snapshots (reference FileManager::save / load, src/services/file-manager.cuh:18-198):
 * the reference's 300-byte header, the fp32 parameters ([hash grid | MLP]: n_density_params
 * carries the hash-grid count, n_color_params the MLP count) and the occupancy bitfield, which
 * the reference's loader reads; then a resume block of this library (Adam moments and step
 * counts, grid densities, the trainer's step counters) that the reference's loader ignores.
 * Save completes a pending caller-ray step first and synchronises. Load restores into a trainer
 * created with the same parameter counts, grid and box: everything the file holds, so a file
 * with the resume block continues training exactly; a reference file (no resume block) sets
 * the parameters and the bitfield and leaves the rest. */
typedef struct tn_turbo_info {
    uint64_t n_params;
    uint64_t file_bytes;
    uint32_t n_occ_grid_bits;
    uint32_t aabb_scale;
    uint32_t has_resume;
    uint32_t step_count;
    uint32_t n_levels, resolution;
    char dataset_path[256];
} tn_turbo_info;
int tn_trainer_save(tn_trainer* tr, const char* path, const char* dataset_path);
int tn_trainer_load(tn_trainer* tr, const char* path);
/* Reads a .turbo file's header and resume block (no GPU work). */
int tn_turbo_file_info(const char* path, tn_turbo_info* out);
/* 0/1: kernel nodes in the captured step graph (synthetic / caller rays), 2: graph nodes,
 * 3: samples processed so far, 4: rays used so far, 5: steps (3-5 synchronise). */
int tn_trainer_stat(tn_trainer* tr, int which, uint64_t* out);
/* Reference NeRFTrainingController::update_occupancy_grid (nerf-training-controller.cu:
 * 214-226, trainer.cu:221-311): decay, every cell of every level re-sampled through the
 * network (all selected while training_step < 256), bits, popcount. Synchronous. */
int tn_trainer_update_occupancy_grid(tn_trainer* tr, uint32_t training_step, tn_occupancy_metrics* metrics);
/* Waits for the trainer's stream and reads the last step's metrics. */
int tn_trainer_sync_metrics(tn_trainer* tr, tn_training_metrics* metrics);
int tn_trainer_stream(tn_trainer* tr, tn_stream_t* out);
/* Device pointers of the trainer's state, for inspection and tests:
 * 0 weights, 1 gradients, 2 first moments, 3 second moments, 4 param steps, 5 grid
 * density, 6 bitfield, 7 sample t, 8 sample pos, 9 sample dt, 10 ray offsets,
 * 11 ray n_steps, 12 batch_info[4], 13 network density, 14 network rgb,
 * 15 grad density, 16 dL/drgb, 17 ray origins, 18 ray directions, 19 ray t,
 * 20 ray t_max, 21 ray alive, 22 target rgba, 23 background rgb, 24 m_norm, 25 dt_norm,
 * 26 the dataset rays' draws [2][n_rays] (pixel, alpha selection; NULL without a dataset),
 * the last step's occupancy update inputs (occupancy_cells_per_step entries each): 27 levels,
 * 28 Morton cells, 29 network density values, 30 selection draws; with the hash-grid network:
 * 31 the hash entries with a nonzero gradient after the last step (l 2^log2 + index, in no
 * particular order; the entries Adam updates), 32 their count (uint32). */
int tn_trainer_buffer(tn_trainer* tr, int which, void** ptr, uint64_t* bytes);

#ifdef __cplusplus
}
#endif

#endif /* TURBO_HOT_H */
