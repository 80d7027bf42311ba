// Runs the reference's own hot-path kernels on the CPU (test infrastructure only).
//
// This file compiles TurboNeRF's kernel sources unchanged, straight from the reference tree
// (the include paths below resolve under <reference>/src), against the host stand-ins in
// oracle/refstub/ for CUDA and for the un-vendored tiny-cuda-nn, json, stb and thrust headers.
// A __global__ kernel is then a plain function; the launchers below call it once per CUDA
// thread, setting the thread-local threadIdx / blockIdx / blockDim first, with OpenMP over
// blocks of 128 threads (every kernel here is one independent thread per ray, sample, cell or
// parameter, with no shared memory and no synchronisation). The library built from it,
// oracle/_ref/libturbonerf_ref.so, pins the oracle restatement (oracle/oracle.cpp) and the
// fixtures under tests/golden/ to the reference's arithmetic.
//
// Arithmetic: IEEE fp32 in the order the reference's source writes it, with no contraction of
// a*b+c (-ffp-contract=off). Integer outputs (march counts, emitted samples, bits, popcounts,
// Adam step counts) are therefore the reference source's own. Outputs that go through the
// reference's fast intrinsics (__expf in density_to_sigma / sigma_to_alpha) use the C
// library's expf here, so they agree with a GPU build of the same source to a few ulp.
//
// Not run: update_occupancy_with_density_kernel (utils/occupancy-grid-kernels.cu:79-116). It
// calls OccupancyGrid::update_sigma_at (core/occupancy-grid.cuh:217-224), which is declared
// float and never returns; a host compiler may treat the end of that function as unreachable
// and delete the kernel's store (g++ 13 does, at every optimisation level). The oracle's
// restatement of that kernel stays pinned by its own closed-form tests.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "utils/training-batch-kernels.cuh"
#include "utils/training-kernels-fused.cuh"
#include "utils/occupancy-grid-kernels.cu"
#include "utils/bit-utils.cu"
#include "core/adam-optimizer.cuh"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

namespace {

constexpr uint32_t kBlock = 128;

// Calls body() once for every thread of a 1-D launch of n threads in blocks of kBlock.
template <typename F>
void launch_linear(uint64_t n, F body) {
    const int64_t n_blocks = (int64_t)((n + kBlock - 1) / kBlock);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t b = 0; b < n_blocks; ++b) {
        blockDim = dim3(kBlock);
        gridDim = dim3((unsigned)n_blocks);
        blockIdx = uint3{(unsigned)b, 0u, 0u};
        for (uint32_t t = 0; t < kBlock; ++t) {
            threadIdx = uint3{t, 0u, 0u};
            body();
        }
    }
}

// The reference's grid object over host memory: n_levels cascades of res^3 cells, the given
// bitfield (res^3 bytes) and densities (n_levels * res^3 floats, may be null = zero).
struct HostGrid {
    turbo::OccupancyGrid grid;
    HostGrid(int n_levels, int res, const uint8_t* bits, const float* density) : grid(0, res) {
        grid.n_levels = n_levels;
        grid.initialize_if_needed(nullptr, true);
        std::memcpy(grid.get_bitfield(), bits, (size_t)res * res * res);
        if (density) std::memcpy(grid.get_density(), density, sizeof(float) * (size_t)n_levels * res * res * res);
    }
    ~HostGrid() { grid.free_device_memory(); }
};

turbo::BoundingBox make_bbox(const float* b) {
    turbo::BoundingBox bb;
    bb.min_x = b[0]; bb.min_y = b[1]; bb.min_z = b[2];
    bb.max_x = b[3]; bb.max_y = b[4]; bb.max_z = b[5];
    return bb;
}

}  // namespace

extern "C" {

int ref_num_threads() { return omp_get_max_threads(); }

// march_and_count_steps_per_ray_kernel (utils/training-batch-kernels.cuh:212-298). Ray arrays
// are SoA with stride `stride`; alive (u8) is read and updated, ori / t are read.
void ref_march_count(uint32_t n_rays, uint32_t stride, const float* bbox6, int n_levels, int res,
                     const uint8_t* bitfield, float cone, float dt_min, float dt_max, const float* dir,
                     const float* t_max, uint8_t* alive, float* ori, float* t, uint32_t* n_steps) {
    HostGrid hg(n_levels, res, bitfield, nullptr);
    const turbo::BoundingBox bb = make_bbox(bbox6);
    std::vector<uint8_t> al(alive, alive + n_rays);  // bool storage: 0 or 1
    bool* al_b = reinterpret_cast<bool*>(al.data());
    for (uint32_t i = 0; i < n_rays; ++i) al[i] = alive[i] ? 1 : 0;
    launch_linear(n_rays, [&] {
        turbo::march_and_count_steps_per_ray_kernel(n_rays, stride, &bb, &hg.grid, cone, dt_min, dt_max, dir, t_max,
                                                    al_b, ori, t, n_steps);
    });
    for (uint32_t i = 0; i < n_rays; ++i) alive[i] = al[i];
}

// march_and_generate_network_positions_kernel (utils/training-batch-kernels.cuh:339-481).
void ref_march_emit(uint32_t n_rays, uint32_t stride, const float* bbox6, float inv_aabb, int n_levels, int res,
                    const uint8_t* bitfield, float dt_min, float dt_max, float cone, const uint32_t* img_id,
                    const float* ori, const float* dir, const float* t, const float* t_max,
                    const uint32_t* offsets, const uint8_t* alive, uint32_t* n_steps, uint32_t* out_img_id,
                    float* out_t, float* out_pos, float* out_dir, float* out_dt, float* out_m_norm,
                    float* out_dt_norm) {
    HostGrid hg(n_levels, res, bitfield, nullptr);
    const turbo::BoundingBox bb = make_bbox(bbox6);
    std::vector<uint8_t> al(n_rays);
    for (uint32_t i = 0; i < n_rays; ++i) al[i] = alive[i] ? 1 : 0;
    const bool* al_b = reinterpret_cast<const bool*>(al.data());
    launch_linear(n_rays, [&] {
        turbo::march_and_generate_network_positions_kernel(n_rays, stride, &bb, inv_aabb, &hg.grid, dt_min, dt_max,
                                                           cone, img_id, ori, dir, t, t_max, offsets, al_b, n_steps,
                                                           out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm,
                                                           out_dt_norm);
    });
}

// fused_reconstruction_forward_backward_kernel (utils/training-kernels-fused.cuh:381-498);
// the network's density passes through density_to_sigma, as in the reference.
void ref_fused_reconstruction(uint32_t n_rays, uint32_t stride, float inv_3nrays, float grad_scale,
                              const uint32_t* ray_steps, const uint32_t* ray_offset, const float* random_rgb,
                              const float* target_rgba, const float* density, const float* color, const float* dt,
                              float* loss, float* dl_ddensity, float* dl_dcolor) {
    launch_linear(n_rays, [&] {
        turbo::fused_reconstruction_forward_backward_kernel(n_rays, stride, inv_3nrays, grad_scale, ray_steps,
                                                            ray_offset, random_rgb, target_rgba, density, color, dt,
                                                            loss, dl_ddensity, dl_dcolor);
    });
}

// mipNeRF360_distortion_loss_forward_kernel + _backward_kernel
// (utils/training-kernels-fused.cuh:13-224), with the reference's fixed lambda of 0.01.
// ray5 = [dtw2 | w | wm | wm_w_cs1 | w_wm_cs1] totals per ray (stride n_rays), sample2 =
// [w_cs | wm_cs] per sample (stride sample_stride).
void ref_distortion(uint32_t n_rays, uint32_t sample_stride, const uint32_t* ray_steps, const uint32_t* ray_offset,
                    const float* density, const float* m_norm, const float* dt_norm, float* ray5, float* ray_loss,
                    float* sample2, float* dl_ddensity) {
    float* r = ray5;
    float* w_cs = sample2;
    float* wm_cs = sample2 + sample_stride;
    launch_linear(n_rays, [&] {
        turbo::mipNeRF360_distortion_loss_forward_kernel(n_rays, sample_stride, ray_steps, ray_offset, density, m_norm,
                                                         dt_norm, r, r + n_rays, r + 2 * (size_t)n_rays,
                                                         r + 3 * (size_t)n_rays, r + 4 * (size_t)n_rays, ray_loss,
                                                         w_cs, wm_cs);
    });
    launch_linear(n_rays, [&] {
        turbo::mipNeRF360_distortion_loss_backward_kernel(n_rays, sample_stride, ray_steps, ray_offset, density, r,
                                                          r + n_rays, r + 2 * (size_t)n_rays, r + 3 * (size_t)n_rays,
                                                          r + 4 * (size_t)n_rays, ray_loss, m_norm, dt_norm, w_cs,
                                                          wm_cs, dl_ddensity);
    });
}

// The gradient merge of NerfNetwork::backward (core/nerf-network.cu:734-758): out +=
// scale * in (copy_gradients_kernel<1, true>, utils/common-network-kernels.cuh:41-62), then
// apply_gradient_distance_scaling_kernel (utils/training-kernels-fused.cuh:500-515).
void ref_grad_merge(uint32_t n_samples, float scale, const float* dl_rec, const float* dl_dist, const float* t,
                    float* out) {
    launch_linear(n_samples, [&] { copy_gradients_kernel<1, true>(n_samples, 0, scale, dl_rec, out); });
    if (dl_dist) launch_linear(n_samples, [&] { copy_gradients_kernel<1, true>(n_samples, 0, scale, dl_dist, out); });
    launch_linear(n_samples, [&] { turbo::apply_gradient_distance_scaling_kernel(n_samples, t, out); });
}

// decay_occupancy_grid_values_kernel then update_occupancy_grid_bits_kernel
// (utils/occupancy-grid-kernels.cu:16-34, 118-141) on host copies of the grid.
void ref_occupancy_decay_bits(int n_levels, int res, float decay, float threshold, float* density, uint8_t* bits) {
    HostGrid hg(n_levels, res, bits, density);
    const uint32_t V = (uint32_t)(res * res * res);
    if (decay != 1.0f) launch_linear(V, [&] { turbo::decay_occupancy_grid_values_kernel(&hg.grid, decay); });
    launch_linear(V, [&] { turbo::update_occupancy_grid_bits_kernel(threshold, &hg.grid); });
    std::memcpy(density, hg.grid.get_density(), sizeof(float) * (size_t)n_levels * V);
    std::memcpy(bits, hg.grid.get_bitfield(), V);
}

// The two reference passes of the occupancy update that surround the network query, run in
// place on the caller's arrays: decay_occupancy_grid_values_kernel, and later
// update_occupancy_grid_bits_kernel (the max-update between them is the caller's, see the top of
// this file).
void ref_occupancy_decay(int n_levels, int res, float decay, float* density) {
    std::vector<uint8_t> bits((size_t)res * res * res, 0);
    HostGrid hg(n_levels, res, bits.data(), density);
    const uint32_t V = (uint32_t)(res * res * res);
    launch_linear(V, [&] { turbo::decay_occupancy_grid_values_kernel(&hg.grid, decay); });
    std::memcpy(density, hg.grid.get_density(), sizeof(float) * (size_t)n_levels * V);
}

void ref_occupancy_bits(int n_levels, int res, float threshold, const float* density, uint8_t* bits) {
    HostGrid hg(n_levels, res, bits, density);
    const uint32_t V = (uint32_t)(res * res * res);
    launch_linear(V, [&] { turbo::update_occupancy_grid_bits_kernel(threshold, &hg.grid); });
    std::memcpy(bits, hg.grid.get_bitfield(), V);
}

// generate_grid_cell_network_sample_points_kernel (utils/occupancy-grid-kernels.cu:38-76):
// n_cells cells of one level starting at Morton index start; random [3][stride].
void ref_occupancy_sample_points(int n_levels, int res, uint32_t n_cells, uint32_t stride, uint32_t start, int level,
                                 float inv_aabb, const float* random, float* sample_pos) {
    std::vector<uint8_t> bits((size_t)res * res * res, 0);
    HostGrid hg(n_levels, res, bits.data(), nullptr);
    launch_linear(n_cells, [&] {
        turbo::generate_grid_cell_network_sample_points_kernel(n_cells, stride, start, &hg.grid, level, inv_aabb,
                                                               random, sample_pos);
    });
}

// get_1s_per_uint32 (utils/bit-utils.cu:8-19) over the bitfield's 32-bit words, then the sum
// that count_1s takes with thrust::reduce (utils/bit-utils.cuh:31-72).
uint32_t ref_popcount(const uint8_t* bytes, uint64_t n_bytes) {
    const uint64_t n_words = n_bytes / 4;
    std::vector<uint8_t> counts(n_words);
    std::vector<uint32_t> words(n_words);
    std::memcpy(words.data(), bytes, n_words * 4);
    launch_linear(n_words, [&] { turbo::get_1s_per_uint32(n_words, words.data(), counts.data()); });
    uint32_t total = 0;
    for (uint8_t c : counts) total += c;
    for (uint64_t i = n_words * 4; i < n_bytes; ++i)
        for (int j = 0; j < 8; ++j) total += (bytes[i] >> j) & 1;
    return total;
}

// ngp_adam_step<float> (core/adam-optimizer.cuh:48-96): one step over all n parameters, the
// hash grid first (n_grid) then the network (n_net).
void ref_adam_step(uint32_t n, uint32_t n_grid, uint32_t n_net, float loss_scale, float lr, float beta1, float beta2,
                   float eps, float l2, float* weights_fp, float* weights, const float* grads, float* m, float* v,
                   uint32_t* steps) {
    launch_linear(n, [&] {
        tcnn::ngp_adam_step<float>(n, n_grid, n_grid + n_net, loss_scale, lr, beta1, beta2, eps, l2, weights_fp,
                                   weights, grads, m, v, steps);
    });
}

}  // extern "C"
