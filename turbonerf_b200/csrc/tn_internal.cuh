// Host-side internals shared by the library's translation units: the context, error
// reporting and argument checks.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "tn_common.cuh"

struct tn_ctx {
    int device = 0;
    uint32_t* flags = nullptr;          // device error word (TN_FLAG_*)
    uint32_t* tickets = nullptr;        // [16] last-block counters, always left at zero
    uint32_t* block_u32 = nullptr;      // per-block u32 aggregates / prefixes
    size_t block_u32_cap = 0;
    float* block_f32 = nullptr;         // per-block float partials
    size_t block_f32_cap = 0;
    uint8_t* mip = nullptr;             // coarse occupancy mip built by tn_march_count
    size_t mip_cap = 0;
    float* slots = nullptr;             // per-ray step positions recorded by tn_march_count
    size_t slots_cap = 0;
    uint32_t slot_cap = 0;              // slots per ray of the last tn_march_count
    uint32_t slot_rays = 0;             // n_rays of the last tn_march_count
    tn_tuning tune{64, 8, 1, 4, 128, 64, 0};  // launch shapes (tn_tuning_default)
    uint32_t count_group_used = 0;      // rays per block of the last tn_march_count (its emit's grouping)
    uint32_t multi_chunk_used = 0;      // rays per chunk of the last tn_multi_march_count
    uint8_t* render_ws = nullptr;       // ray and sample buffers of tn_render
    size_t render_ws_cap = 0;
};

namespace tn {

enum Ticket : int {
    TICKET_MARCH = 0,
    TICKET_SCAN = 1,
    TICKET_RECON = 2,
    TICKET_DIST = 3,
    TICKET_TRAIN = 4,
    TICKET_POPCOUNT = 5,
    TICKET_COMPACT = 6,
    TICKET_MULTI = 7,        // multi-scene count: chunks finished
    TICKET_MULTI_WORK = 8,   // multi-scene count: next chunk to take
    TICKET_COUNT = 16,
};

void set_error(const char* fmt, ...);
int fail(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
int check_launch(const char* what);
int ensure_block_u32(tn_ctx* ctx, size_t n);
int ensure_block_f32(tn_ctx* ctx, size_t n);
int ensure_mip(tn_ctx* ctx, size_t bytes);
int ensure_slots(tn_ctx* ctx, size_t n);
int ensure_render_ws(tn_ctx* ctx, size_t bytes);
bool stream_capturing(cudaStream_t s);
int num_sms();

// Host-side IEEE single arithmetic, identical to the device expressions they replace
// (volatile keeps the compiler from folding or contracting them).
inline GridView make_grid_view(const tn_grid_desc& d, const uint8_t* bits) {
    GridView g{};
    g.n_levels = d.n_levels;
    g.res = d.resolution;
    g.res_f = (float)d.resolution;
    volatile float one = 1.0f, halfc = 0.5f;
    g.inv_res = one / g.res_f;
    g.base = d.base_size;
    g.bits = bits;
    for (int k = 0; k < MAX_LEVELS; ++k) {
        volatile float ls = g.base * (float)(1 << k);
        g.ls[k] = ls;
        g.inv_ls[k] = one / ls;
        g.half[k] = halfc * ls;
        g.cell[k] = ls * g.inv_res;
    }
    return g;
}

int validate_grid(const tn_grid_desc* grid);

// Shared memory that a block reserves so that no second block reserving as much fits on its
// SM: just over half of the SM's shared memory (blocks of the march count and of the kernels
// that run beside it on other SMs).
size_t exclusive_smem();
// Lets kernel `func` take the device's opt-in shared memory (less its static shared memory) as
// dynamic shared memory.
int allow_optin_smem(const void* func);

// Where the fused Adam runs: by default one 256-thread block per 1024 parameters over the whole
// GPU; with max_blocks, at most that many 1024-thread blocks (a grid-stride loop), each
// reserving reserve_smem bytes of shared memory. enable: a device flag; the update runs only
// when it is non-zero.
struct AdamPlacement {
    uint32_t max_blocks = 0;
    size_t reserve_smem = 0;
    const uint32_t* enable = nullptr;
};

// Internal launchers (device-side parameters for graph replays).
int launch_adam(cudaStream_t stream, bool plain, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale,
                float lr, const float* lr_dev, float beta1, float beta2, float epsilon, float l2_reg, float* weights,
                float* weights_copy, const float* gradients, float* first_moments, float* second_moments,
                uint32_t* param_steps, const AdamPlacement& place = AdamPlacement{});
// The hash-grid network (hashgrid.cu) over params [hash entries | heads], for batches of up to
// cap samples and density queries of up to qcap; *handle owns its buffers.
int hashnet_create(const tn_hashgrid_desc* desc, const float* params, uint32_t cap, uint32_t qcap, tn_network* out,
                   void** handle);
void hashnet_destroy(void* handle);
// Device count (and *list) of the entries the network's last backward touched.
const uint32_t* hashnet_touched(void* handle, const uint32_t** list);
// tn_train_losses; accumulate false writes the merged density gradient over grad_density.
int train_losses(tn_ctx* ctx, cudaStream_t stream, const tn_ray_batch* batch, int activation, float min_transmittance,
                 float inv_nrays, const uint32_t* inv_nrays_from_dev, float grad_scale, float lambda,
                 const float* density, const float* rgb, const float* dt, const float* m_norm, const float* dt_norm,
                 const float* t, const float* target_rgba, const float* bg_rgb, float* ray_rgba, float* grad_density,
                 float* dL_drgb, float* loss_sums, bool accumulate);
int launch_occupancy_update(tn_ctx* ctx, cudaStream_t stream, const tn_grid_desc* grid, float* density,
                            uint8_t* bitfield, uint32_t n_updates, const int32_t* levels, const uint32_t* cells,
                            const float* values, const float* rand_select, int activation, int sample_all,
                            const uint32_t* sample_all_dev, const uint32_t* n_dev, float decay, float threshold,
                            uint32_t* n_occupied_dev, uint8_t* bitfield_out = nullptr,
                            cudaEvent_t bits_done = nullptr, bool bits_ready = false);
// The bitfield launch_occupancy_update will write into bitfield_out, computed before it from
// settled densities without changing them (the selection rule reads `bitfield`, the policy
// *sample_all_dev); equal to the update's bits bit for bit.
int launch_occupancy_bits_ahead(cudaStream_t stream, const tn_grid_desc* grid, const float* density,
                                const uint8_t* bitfield, uint8_t* bitfield_out, uint32_t n_updates,
                                const int32_t* levels, const uint32_t* cells, const float* values,
                                const float* rand_select, int activation, const uint32_t* sample_all_dev, float decay,
                                float threshold);
int launch_occupancy_scatter(cudaStream_t stream, const tn_grid_desc* grid, float* density, const uint8_t* bitfield,
                             uint32_t n_updates, const int32_t* levels, const uint32_t* cells, const float* values,
                             const float* rand_select, int activation, int sample_all, float decay);
int launch_occupancy_sweep(cudaStream_t stream, const tn_grid_desc* grid, float* density, uint8_t* bitfield,
                           float decay, float threshold, uint32_t* n_occupied_dev);
int launch_plain_occ_decay(cudaStream_t stream, const tn_grid_desc* grid, float* density, float decay);
int launch_plain_occ_update(cudaStream_t stream, const tn_grid_desc* grid, float* density, const uint8_t* bitfield,
                            uint32_t n_updates, const int32_t* levels, const uint32_t* cells, const float* values,
                            const float* rand_select, int activation, int sample_all);
int launch_plain_occ_bits_sync(cudaStream_t stream, const tn_grid_desc* grid, const float* density, uint8_t* bitfield,
                               float threshold, uint8_t* count_scratch, uint32_t* n_occupied_out);
int launch_synth_rays(cudaStream_t stream, uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* step_dev,
                      float radius, float jitter, const tn_bbox& b, float t_far, float* ori, float* dir, float* target,
                      float* bg, float* ray_t, float* ray_t_max, uint8_t* alive);
int launch_synth_cells(cudaStream_t stream, uint32_t n, uint32_t seed, const uint32_t* step_dev, int n_levels,
                       uint32_t volume, int32_t* levels, uint32_t* cells, float* rand3, uint32_t rand_stride,
                       float* rand_sel);
int launch_synth_level_cells(cudaStream_t stream, uint32_t n, uint32_t start, int level, uint32_t seed, uint32_t salt,
                             int32_t* levels, uint32_t* cells, float* rand3, uint32_t rand_stride, float* rand_sel);
int launch_synth_hash_grads(cudaStream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t ps, const float* pos,
                            int n_levels, uint32_t log2_table, int n_features, float base_res, float per_level_scale,
                            uint32_t seed, float std, float* grads);
int launch_synth_params(cudaStream_t stream, uint32_t n, uint32_t n_grid, uint32_t seed, float* w);
int check_dataset(uint32_t n_images, int32_t width, int32_t height);

// .turbo snapshot (snapshot.cu): the reference's header and sections (FileManager::save,
// src/services/file-manager.cuh:18-120), then this library's resume block.
struct TurboHeader {
    char project_name[16];  // "TurboNeRF"
    char dataset_path[256];
    uint32_t version;       // 0
    uint32_t n_color_params;
    uint32_t n_density_params;
    uint32_t n_appearance_embedding_params;
    uint32_t n_occ_grid_bits;
    uint32_t aabb_scale;
    uint32_t n_appearances;
};
static_assert(sizeof(TurboHeader) == 300, "the reference's NeRFFileData layout");

struct TurboResume {
    char magic[8];  // "TNRESUME"
    uint32_t version;
    uint32_t n_levels, resolution;
    uint32_t n_grid_params, n_mlp_params;
    uint32_t step_count;
    uint64_t samples_total, rays_total;
};

int read_turbo_file(const char* path, TurboHeader* header, TurboResume* resume, bool* has_resume, uint64_t* size);
int launch_dataset_rays(cudaStream_t stream, uint32_t n_rays, uint32_t rs, uint32_t n_images, int32_t width,
                        int32_t height, const tn_camera* cameras, const uint8_t* images, const tn_bbox& bbox,
                        const float* random, float alpha_threshold, float alpha_probability, float* pix_rgba,
                        uint32_t* img_id, float* ori, float* dir, float* ray_t, float* ray_tmax, uint8_t* alive);
int launch_dataset_draws(cudaStream_t stream, uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* step_dev,
                         float* random, float* bg);

}  // namespace tn

#define TN_REQUIRE(cond, code, ...) \
    do { if (!(cond)) return tn::fail((code), __VA_ARGS__); } while (0)
#define TN_NONNULL(p) TN_REQUIRE((p) != nullptr, TN_E_NULL, "%s: %s is NULL", __func__, #p)
