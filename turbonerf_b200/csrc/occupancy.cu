// Occupancy grid: density EMA (decay + max-update) and bitfield rebuild.
//
// Fused path (tn_occupancy_update), two kernels:
//  1. scatter: every selected (level, cell) update applies max(density * decay, sigma) at
//     once and marks the cell as already decayed by storing the value negated (densities
//     are non-negative, so the sign bit is free). Duplicate updates of one cell combine
//     through a compare-and-swap loop, which makes the result the maximum of all of them.
//  2. sweep: one pass over all cells, four cells per thread with 16-byte loads per level:
//     decay the unmarked values, unmark the marked ones, threshold every level into the
//     cell's bit byte, write the bitfield and count its set bits.
// This reads and writes the density grid once per update instead of three times
// (reference: decay pass, update pass, bits pass, popcount pass with a host read;
// src/core/trainer.cu:221-311).
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/reduce.h>
#include <thrust/transform_reduce.h>

#include "tn_internal.cuh"

namespace tn {

__device__ __forceinline__ float occ_sigma(int act, float v) { return act == 0 ? v : expf(fminf(v, 12.0f) - 1.0f); }

// generate_grid_cell_network_sample_points_kernel, src/utils/occupancy-grid-kernels.cu:38-76
// with get_voxel_xyz_from_morton_index (src/core/occupancy-grid.cuh:167-182).
__global__ void sample_points_kernel(uint32_t n, int res, float base, const int32_t* __restrict__ levels,
                                     const uint32_t* __restrict__ cells, const float* __restrict__ rand3,
                                     uint32_t rand_stride, float inv_aabb, float* __restrict__ out, uint32_t ps) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = levels[i];
    const uint32_t idx = cells[i];
    const float inv_res = __fdiv_rn(1.0f, (float)res);
    const float ls = __fmul_rn(base, (float)(1 << k));
    const float vs = __fmul_rn(ls, inv_res);
    const int half = res / 2;
    const float vx = __fmul_rn((float)((int)compact1by2(idx) - half), vs);
    const float vy = __fmul_rn((float)((int)compact1by2(idx >> 1) - half), vs);
    const float vz = __fmul_rn((float)((int)compact1by2(idx >> 2) - half), vs);
    const float x = __fadd_rn(vx, __fmul_rn(rand3[i], vs));
    const float y = __fadd_rn(vy, __fmul_rn(rand3[i + rand_stride], vs));
    const float z = __fadd_rn(vz, __fmul_rn(rand3[i + 2 * (size_t)rand_stride], vs));
    out[i] = __fadd_rn(__fmul_rn(x, inv_aabb), 0.5f);
    out[i + ps] = __fadd_rn(__fmul_rn(y, inv_aabb), 0.5f);
    out[i + 2 * (size_t)ps] = __fadd_rn(__fmul_rn(z, inv_aabb), 0.5f);
}

// Selection policy of update_occupancy_with_density_kernel (occupancy-grid-kernels.cu:95-112).
__device__ __forceinline__ bool selected(int sample_all, const float* __restrict__ rand_select, uint32_t u,
                                         const uint8_t* __restrict__ bits, uint32_t idx, int k) {
    if (sample_all) return true;
    const float r = rand_select[u];
    if (r > 0.5f) return false;
    if (r < 0.25f) return true;
    return (bits[idx] & (uint8_t)(1u << k)) != 0;
}

__global__ void occ_scatter_kernel(uint32_t n, uint32_t volume, int n_levels, float* __restrict__ density,
                                   const uint8_t* __restrict__ bits, const int32_t* __restrict__ levels,
                                   const uint32_t* __restrict__ cells, const float* __restrict__ values,
                                   const float* __restrict__ rand_select, int act, int sample_all, float decay,
                                   const uint32_t* __restrict__ sample_all_dev, const uint32_t* __restrict__ n_dev) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= (n_dev ? min(*n_dev, n) : n)) return;
    if (sample_all_dev) sample_all = (int)*sample_all_dev;
    const int k = levels[u];
    const uint32_t idx = cells[u];
    if (k < 0 || k >= n_levels || idx >= volume) return;
    if (!selected(sample_all, rand_select, u, bits, idx, k)) return;
    const float sigma = occ_sigma(act, values[u]);
    uint32_t* p = reinterpret_cast<uint32_t*>(density + (size_t)k * volume + idx);
    uint32_t old = *((volatile uint32_t*)p), assumed;
    do {
        assumed = old;
        const float cur = __uint_as_float(assumed);
        const float v = signbit(cur) ? fmaxf(-cur, sigma) : fmaxf(cur * decay, sigma);
        old = atomicCAS(p, assumed, __float_as_uint(-v));
    } while (old != assumed);
}

__device__ __forceinline__ float settle(float v, float decay) { return signbit(v) ? -v : v * decay; }

// Issues every level's 16-byte load of the thread's four cells before using any of them, so
// each thread keeps n_levels loads in flight. WRITE_DENSITY stores the settled densities;
// WRITE_BITS rebuilds the bitfield; COUNT counts the set bits of the settled densities. The
// one-pass update does all three; the split update runs a bits-only pass first (what the next
// march waits for) and the density write-back after it, beside the march; an update whose bits
// were computed ahead (occ_bits_*_kernel) writes the densities and counts.
template <bool WRITE_DENSITY, bool WRITE_BITS, bool COUNT = WRITE_BITS>
__global__ void __launch_bounds__(256)
occ_sweep_kernel(uint32_t volume4, int n_levels, float* __restrict__ density, uint8_t* __restrict__ bits,
                 float decay, float threshold, uint32_t* __restrict__ n_occupied) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t cnt = 0;
    if (i < volume4) {
        float4* d4 = reinterpret_cast<float4*>(density);
        float4 v[MAX_LEVELS];
#pragma unroll
        for (int k = 0; k < MAX_LEVELS; ++k)
            if (k < n_levels) v[k] = WRITE_DENSITY ? __ldcs(d4 + (size_t)k * volume4 + i) : d4[(size_t)k * volume4 + i];
        uint32_t b0 = 0, b1 = 0, b2 = 0, b3 = 0;
#pragma unroll
        for (int k = 0; k < MAX_LEVELS; ++k) {
            if (k < n_levels) {
                float4 x = v[k];
                x.x = settle(x.x, decay);
                x.y = settle(x.y, decay);
                x.z = settle(x.z, decay);
                x.w = settle(x.w, decay);
                if (WRITE_DENSITY) __stcs(d4 + (size_t)k * volume4 + i, x);
                b0 |= (uint32_t)(x.x > threshold) << k;
                b1 |= (uint32_t)(x.y > threshold) << k;
                b2 |= (uint32_t)(x.z > threshold) << k;
                b3 |= (uint32_t)(x.w > threshold) << k;
            }
        }
        const uint32_t packed = b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
        if (WRITE_BITS) reinterpret_cast<uint32_t*>(bits)[i] = packed;
        cnt = __popc(packed);
    }
    if (COUNT && n_occupied) {
        cnt = warp_sum(cnt);
        __shared__ uint32_t ws[8];
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
            if (t) atomicAdd(n_occupied, t);
        }
    }
}

// The bitfield an occupancy update will write, computed before it without changing the
// densities (which must be settled, as they are between steps): every cell's decayed density
// against the threshold, then the queried cells the update raises or-ed in. A selected query
// (k, cell, sigma) leaves max(decay d, sigma, ...) at the cell, above the threshold exactly when
// one of its max(decay d, sigma) is, so the bits equal the update's bit for bit.
__global__ void __launch_bounds__(256)
occ_bits_decayed_kernel(uint32_t volume4, int n_levels, const float* __restrict__ density,
                        uint8_t* __restrict__ bits, float decay, float threshold) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= volume4) return;
    const float4* d4 = reinterpret_cast<const float4*>(density);
    float4 v[MAX_LEVELS];
#pragma unroll
    for (int k = 0; k < MAX_LEVELS; ++k)
        if (k < n_levels) v[k] = d4[(size_t)k * volume4 + i];
    uint32_t b0 = 0, b1 = 0, b2 = 0, b3 = 0;
#pragma unroll
    for (int k = 0; k < MAX_LEVELS; ++k) {
        if (k < n_levels) {
            b0 |= (uint32_t)(v[k].x * decay > threshold) << k;
            b1 |= (uint32_t)(v[k].y * decay > threshold) << k;
            b2 |= (uint32_t)(v[k].z * decay > threshold) << k;
            b3 |= (uint32_t)(v[k].w * decay > threshold) << k;
        }
    }
    reinterpret_cast<uint32_t*>(bits)[i] = b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
}

__global__ void occ_bits_raise_kernel(uint32_t n, uint32_t volume, int n_levels, const float* __restrict__ density,
                                      const uint8_t* __restrict__ sel_bits, uint8_t* __restrict__ bits,
                                      const int32_t* __restrict__ levels, const uint32_t* __restrict__ cells,
                                      const float* __restrict__ values, const float* __restrict__ rand_select,
                                      int act, const uint32_t* __restrict__ sample_all_dev, float decay,
                                      float threshold) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const int k = levels[u];
    const uint32_t idx = cells[u];
    if (k < 0 || k >= n_levels || idx >= volume) return;
    if (!selected((int)*sample_all_dev, rand_select, u, sel_bits, idx, k)) return;
    const float v = fmaxf(density[(size_t)k * volume + idx] * decay, occ_sigma(act, values[u]));
    if (v > threshold) atomicOr(reinterpret_cast<uint32_t*>(bits) + (idx >> 2), (1u << k) << (8u * (idx & 3u)));
}

__global__ void popcount_kernel(uint64_t n_words, const uint32_t* __restrict__ words, uint64_t n_tail,
                                const uint8_t* __restrict__ tail, uint32_t* __restrict__ out) {
    uint32_t cnt = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_words; i += (uint64_t)gridDim.x * blockDim.x)
        cnt += __popc(words[i]);
    if (blockIdx.x == 0 && threadIdx.x < n_tail) cnt += __popc((uint32_t)tail[threadIdx.x]);
    cnt = warp_sum(cnt);
    __shared__ uint32_t ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        if (t) atomicAdd(out, t);
    }
}

// ---- plain path (reference launch structure) -------------------------------------------
__global__ void plain_decay_kernel(uint32_t volume, int n_levels, float* __restrict__ density, float factor) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= volume) return;
    float* d = density + idx;
    for (int i = 0; i < n_levels; ++i) {
        *d *= factor;
        d += volume;
    }
}

__global__ void plain_update_kernel(uint32_t n, uint32_t volume, int n_levels, float* __restrict__ density,
                                    const uint8_t* __restrict__ bits, const int32_t* __restrict__ levels,
                                    const uint32_t* __restrict__ cells, const float* __restrict__ values,
                                    const float* __restrict__ rand_select, int act, int sample_all) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n) return;
    const int k = levels[u];
    const uint32_t idx = cells[u];
    if (k < 0 || k >= n_levels || idx >= volume) return;
    if (!selected(sample_all, rand_select, u, bits, idx, k)) return;
    const float sigma = act == 0 ? values[u] : __expf(fminf(values[u], 12.0f) - 1.0f);
    // The reference writes fmaxf(value, *ptr) without an atomic (occupancy-grid.cuh:217-224);
    // a CAS loop keeps duplicate (level, cell) updates well defined.
    uint32_t* p = reinterpret_cast<uint32_t*>(density + (size_t)k * volume + idx);
    uint32_t old = *((volatile uint32_t*)p), assumed;
    do {
        assumed = old;
        old = atomicCAS(p, assumed, __float_as_uint(fmaxf(sigma, __uint_as_float(assumed))));
    } while (old != assumed);
}

__global__ void plain_bits_kernel(uint32_t volume, int n_levels, float threshold, const float* __restrict__ density,
                                  uint8_t* __restrict__ bits) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= volume) return;
    uint8_t cell = 0;
    for (int level = 0; level < n_levels; ++level) {
        const uint8_t b = density[(size_t)level * volume + idx] > threshold ? 1 : 0;
        cell |= (uint8_t)(b << level);
    }
    bits[idx] = cell;
}

__global__ void plain_ones_per_u32_kernel(size_t n, const uint32_t* __restrict__ words, uint8_t* __restrict__ counts) {
    const size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (idx >= n) return;
    counts[idx] = (uint8_t)__popc(words[idx]);
}

struct U8ToU32 {
    __host__ __device__ uint32_t operator()(uint8_t v) const { return v; }
};

// Pieces of the update for callers that scatter several batches before one sweep
// (the full-grid update of the reference runs one batch per level and chunk).
int launch_occupancy_scatter(cudaStream_t stream, const tn_grid_desc* grid, float* density, const uint8_t* bitfield,
                             uint32_t n_updates, const int32_t* levels, const uint32_t* cells, const float* values,
                             const float* rand_select, int activation, int sample_all, float decay) {
    if (n_updates == 0) return TN_OK;
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    occ_scatter_kernel<<<(n_updates + 255) / 256, 256, 0, stream>>>(n_updates, volume, grid->n_levels, density,
                                                                    bitfield, levels, cells, values, rand_select,
                                                                    activation, sample_all, decay, nullptr, nullptr);
    return check_launch("occupancy scatter");
}

int launch_occupancy_sweep(cudaStream_t stream, const tn_grid_desc* grid, float* density, uint8_t* bitfield,
                           float decay, float threshold, uint32_t* n_occupied_dev) {
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    if (n_occupied_dev) {
        int st = cuda_status(cudaMemsetAsync(n_occupied_dev, 0, sizeof(uint32_t), stream), "occupancy sweep memset");
        if (st != TN_OK) return st;
    }
    const uint32_t v4 = volume / 4;
    occ_sweep_kernel<true, true><<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density, bitfield, decay,
                                                                       threshold, n_occupied_dev);
    return check_launch("occupancy sweep");
}

int launch_plain_occ_decay(cudaStream_t stream, const tn_grid_desc* grid, float* density, float decay) {
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    plain_decay_kernel<<<(volume + 127) / 128, 128, 0, stream>>>(volume, grid->n_levels, density, decay);
    return check_launch("plain occupancy decay");
}

int launch_plain_occ_update(cudaStream_t stream, const tn_grid_desc* grid, float* density, const uint8_t* bitfield,
                            uint32_t n_updates, const int32_t* levels, const uint32_t* cells, const float* values,
                            const float* rand_select, int activation, int sample_all) {
    if (n_updates == 0) return TN_OK;
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    plain_update_kernel<<<(n_updates + 127) / 128, 128, 0, stream>>>(n_updates, volume, grid->n_levels, density,
                                                                     bitfield, levels, cells, values, rand_select,
                                                                     activation, sample_all);
    return check_launch("plain occupancy update");
}

// Bits + popcount of the reference (update_occupancy_grid_bits_kernel, get_1s_per_uint32 and
// a thrust reduction read back on the host).
int launch_plain_occ_bits_sync(cudaStream_t stream, const tn_grid_desc* grid, const float* density, uint8_t* bitfield,
                               float threshold, uint8_t* count_scratch, uint32_t* n_occupied_out) {
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    plain_bits_kernel<<<(volume + 127) / 128, 128, 0, stream>>>(volume, grid->n_levels, threshold, density, bitfield);
    const size_t words = volume / 4;
    plain_ones_per_u32_kernel<<<(unsigned)((words + 255) / 256), 256, 0, stream>>>(
        words, reinterpret_cast<const uint32_t*>(bitfield), count_scratch);
    int st = check_launch("plain occupancy bits");
    if (st != TN_OK) return st;
    thrust::device_ptr<uint8_t> p(count_scratch);
    *n_occupied_out = thrust::transform_reduce(thrust::cuda::par.on(stream), p, p + words, U8ToU32(), 0u,
                                               thrust::plus<uint32_t>());
    return TN_OK;
}

// Fused occupancy update; sample_all_dev (optional) overrides sample_all from device memory
// and n_dev (optional) bounds the number of live updates, so graph replays can change both.
int launch_occupancy_update(tn_ctx* ctx, cudaStream_t stream, const tn_grid_desc* grid, float* density,
                            uint8_t* bitfield, uint32_t n_updates, const int32_t* levels, const uint32_t* cells,
                            const float* values, const float* rand_select, int activation, int sample_all,
                            const uint32_t* sample_all_dev, const uint32_t* n_dev, float decay, float threshold,
                            uint32_t* n_occupied_dev, uint8_t* bitfield_out, cudaEvent_t bits_done,
                            bool bits_ready) {
    // bits_done: split update; the event is recorded once the bitfield is rebuilt, before the
    // settled densities are written back. bits_ready: bitfield_out already holds the update's
    // bits (launch_occupancy_bits_ahead); the update writes the densities and counts the bits.
    const bool split = bits_done != nullptr;
    TN_NONNULL(ctx);
    int st = validate_grid(grid);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(bitfield);
    if (n_updates) {
        TN_NONNULL(levels); TN_NONNULL(cells); TN_NONNULL(values);
        if (!sample_all || sample_all_dev) TN_NONNULL(rand_select);
    }
    // the selection rule reads `bitfield`; the rebuilt bits go to bitfield_out (default: in place)
    if (!bitfield_out) bitfield_out = bitfield;
    TN_REQUIRE(((uintptr_t)density & 15u) == 0 && ((uintptr_t)bitfield_out & 3u) == 0, TN_E_INVALID,
               "tn_occupancy_update: density must be 16-byte and bitfield 4-byte aligned");
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    if (n_occupied_dev) {
        st = cuda_status(cudaMemsetAsync(n_occupied_dev, 0, sizeof(uint32_t), stream), "tn_occupancy_update memset");
        if (st != TN_OK) return st;
    }
    if (n_updates) {
        occ_scatter_kernel<<<(n_updates + 255) / 256, 256, 0, stream>>>(n_updates, volume, grid->n_levels, density,
                                                                        bitfield, levels, cells, values, rand_select,
                                                                        activation, sample_all, decay, sample_all_dev,
                                                                        n_dev);
        st = check_launch("tn_occupancy_update(scatter)");
        if (st != TN_OK) return st;
    }
    const uint32_t v4 = volume / 4;
    if (bits_ready) {
        occ_sweep_kernel<true, false, true><<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density,
                                                                                 bitfield_out, decay, threshold,
                                                                                 n_occupied_dev);
        return check_launch("tn_occupancy_update(densities, count)");
    }
    if (!split) {
        occ_sweep_kernel<true, true><<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density, bitfield_out,
                                                                           decay, threshold, n_occupied_dev);
        return check_launch("tn_occupancy_update(sweep)");
    }
    occ_sweep_kernel<false, true><<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density, bitfield_out,
                                                                        decay, threshold, n_occupied_dev);
    st = check_launch("tn_occupancy_update(bits)");
    if (st != TN_OK || !bits_done) return st;
    st = cuda_status(cudaEventRecord(bits_done, stream), "occupancy bits done");
    if (st != TN_OK) return st;
    occ_sweep_kernel<true, false><<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density, bitfield_out,
                                                                        decay, threshold, nullptr);
    return check_launch("tn_occupancy_update(densities)");
}

int launch_occupancy_bits_ahead(cudaStream_t stream, const tn_grid_desc* grid, const float* density,
                                const uint8_t* bitfield, uint8_t* bitfield_out, uint32_t n_updates,
                                const int32_t* levels, const uint32_t* cells, const float* values,
                                const float* rand_select, int activation, const uint32_t* sample_all_dev, float decay,
                                float threshold) {
    int st = validate_grid(grid);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(bitfield); TN_NONNULL(bitfield_out); TN_NONNULL(sample_all_dev);
    TN_REQUIRE(((uintptr_t)density & 15u) == 0 && ((uintptr_t)bitfield_out & 3u) == 0, TN_E_INVALID,
               "occupancy bits ahead: density must be 16-byte and bitfield 4-byte aligned");
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    const uint32_t v4 = volume / 4;
    occ_bits_decayed_kernel<<<(v4 + 255) / 256, 256, 0, stream>>>(v4, grid->n_levels, density, bitfield_out, decay,
                                                                   threshold);
    st = check_launch("occupancy bits ahead (decayed)");
    if (st != TN_OK || n_updates == 0) return st;
    occ_bits_raise_kernel<<<(n_updates + 255) / 256, 256, 0, stream>>>(n_updates, volume, grid->n_levels, density,
                                                                       bitfield, bitfield_out, levels, cells, values,
                                                                       rand_select, activation, sample_all_dev, decay,
                                                                       threshold);
    return check_launch("occupancy bits ahead (raised)");
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_occupancy_sample_points(tn_stream_t stream, const tn_grid_desc* grid, uint32_t n, const int32_t* levels,
                               const uint32_t* cells, const float* rand3, uint32_t rand_stride, float inv_aabb_size,
                               float* out_pos, uint32_t pos_stride) {
    int st = validate_grid(grid);
    if (st != TN_OK) return st;
    TN_NONNULL(levels); TN_NONNULL(cells); TN_NONNULL(rand3); TN_NONNULL(out_pos);
    TN_REQUIRE(rand_stride >= n && pos_stride >= n, TN_E_INVALID, "strides must be >= n");
    if (n == 0) return TN_OK;
    sample_points_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, grid->resolution, grid->base_size, levels, cells, rand3,
                                                              rand_stride, inv_aabb_size, out_pos, pos_stride);
    return check_launch("tn_occupancy_sample_points");
}

int tn_occupancy_update(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, float* density, uint8_t* bitfield,
                        uint32_t n_updates, const int32_t* levels, const uint32_t* cells, const float* values,
                        const float* rand_select, int activation, int sample_all, float decay, float threshold,
                        uint32_t* n_occupied_dev) {
    return launch_occupancy_update(ctx, stream, grid, density, bitfield, n_updates, levels, cells, values, rand_select,
                                   activation, sample_all, nullptr, nullptr, decay, threshold, n_occupied_dev);
}

int tn_popcount(tn_ctx* ctx, tn_stream_t stream, uint64_t n_bytes, const uint8_t* bytes, uint32_t* out_dev) {
    TN_NONNULL(ctx); TN_NONNULL(bytes); TN_NONNULL(out_dev);
    int st = cuda_status(cudaMemsetAsync(out_dev, 0, sizeof(uint32_t), stream), "tn_popcount memset");
    if (st != TN_OK) return st;
    TN_REQUIRE(((uintptr_t)bytes & 3u) == 0, TN_E_INVALID, "tn_popcount: bytes must be 4-byte aligned");
    const uint64_t words = n_bytes / 4, tail = n_bytes % 4;
    uint64_t blocks = (words + 255) / 256;
    if (blocks > (uint64_t)num_sms() * 4) blocks = (uint64_t)num_sms() * 4;
    if (blocks == 0) blocks = 1;
    const int grid = (int)blocks;
    popcount_kernel<<<grid, 256, 0, stream>>>(words, reinterpret_cast<const uint32_t*>(bytes), tail, bytes + words * 4,
                                              out_dev);
    return check_launch("tn_popcount");
}

int tn_plain_occupancy_update_sync(tn_stream_t stream, const tn_grid_desc* grid, float* density, uint8_t* bitfield,
                                   uint32_t n_updates, const int32_t* levels, const uint32_t* cells,
                                   const float* values, const float* rand_select, int activation, int sample_all,
                                   float decay, float threshold, uint8_t* count_scratch, uint32_t* n_occupied_out) {
    int st = validate_grid(grid);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(bitfield); TN_NONNULL(count_scratch); TN_NONNULL(n_occupied_out);
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    plain_decay_kernel<<<(volume + 127) / 128, 128, 0, stream>>>(volume, grid->n_levels, density, decay);
    if (n_updates) {
        TN_NONNULL(levels); TN_NONNULL(cells); TN_NONNULL(values);
        plain_update_kernel<<<(n_updates + 127) / 128, 128, 0, stream>>>(n_updates, volume, grid->n_levels, density,
                                                                         bitfield, levels, cells, values, rand_select,
                                                                         activation, sample_all);
    }
    plain_bits_kernel<<<(volume + 127) / 128, 128, 0, stream>>>(volume, grid->n_levels, threshold, density, bitfield);
    const size_t words = volume / 4;
    plain_ones_per_u32_kernel<<<(unsigned)((words + 255) / 256), 256, 0, stream>>>(
        words, reinterpret_cast<const uint32_t*>(bitfield), count_scratch);
    st = check_launch("tn_plain_occupancy_update_sync");
    if (st != TN_OK) return st;
    thrust::device_ptr<uint8_t> p(count_scratch);
    *n_occupied_out = thrust::transform_reduce(thrust::cuda::par.on(stream), p, p + words, U8ToU32(), 0u,
                                               thrust::plus<uint32_t>());
    return TN_OK;
}

}  // extern "C"
