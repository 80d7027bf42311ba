// Shared device helpers for the turbo_hot library (sm_100a).
//
// The march helpers below reproduce the reference's FP32 arithmetic bit for bit, so
// every a*b+c is written with explicit round-to-nearest intrinsics (__fmul_rn,
// __fadd_rn): nvcc would otherwise fuse them into FMAs and the sample positions,
// counts and offsets would no longer match the reference's source semantics.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/turbo_hot.h"

namespace tn {

constexpr int WARP = 32;
constexpr unsigned FULL_MASK = 0xffffffffu;

// Device-side error bits, OR-ed into the context's flag word (read by tn_ctx_check).
enum : uint32_t {
    ERR_GUARD = 1u << 0,       // a march loop hit its iteration limit
    ERR_CAPACITY = 1u << 1,    // an emitted sample or offset exceeded the sample capacity
    ERR_NO_RAYS = 1u << 2,     // the batch cut found no ray
    ERR_NO_SAMPLES = 1u << 3,  // the batch cut found no sample
    ERR_SPIN = 1u << 4,        // a bounded spin-wait gave up
};

__device__ __forceinline__ void raise_flag(uint32_t* flags, uint32_t bit) {
    if (flags) atomicOr(flags, bit);
}

// ------------------------------------------------------------------------------------
// Morton code: 3 x 10-bit interleave, x -> bit 0, y -> bit 1, z -> bit 2 (the layout the
// reference's bitfield uses, src/core/occupancy-grid.cuh:150-182). Published
// "Part1By2"/"Compact1By2" bit-spreading by shifts and masks.
// ------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t part1by2(uint32_t v) {
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__host__ __device__ __forceinline__ uint32_t compact1by2(uint32_t v) {
    v &= 0x09249249u;
    v = (v | (v >> 2)) & 0x030C30C3u;
    v = (v | (v >> 4)) & 0x0300F00Fu;
    v = (v | (v >> 8)) & 0x030000FFu;
    v = (v | (v >> 16)) & 0x000003FFu;
    return v;
}

__host__ __device__ __forceinline__ uint32_t morton3d(uint32_t x, uint32_t y, uint32_t z) {
    return part1by2(x) | (part1by2(y) << 1) | (part1by2(z) << 2);
}

// ------------------------------------------------------------------------------------
// Grid / march arithmetic (exact FP32, no contraction)
// ------------------------------------------------------------------------------------
constexpr int MAX_LEVELS = 8;

// Per-level constants are computed once on the host with the same IEEE operations the
// reference performs inline (level size base * 2^k, its reciprocal 1.0f / size, half size,
// cell size size * (1/R)), so the kernels read them instead of re-deriving them per step.
struct GridView {
    int n_levels;
    int res;
    float res_f;
    float inv_res;     // 1.0f / res_f
    float base;        // level k covers base * 2^k
    const uint8_t* __restrict__ bits;
    float ls[MAX_LEVELS];      // level size
    float inv_ls[MAX_LEVELS];  // 1.0f / level size
    float half[MAX_LEVELS];    // 0.5f * level size
    float cell[MAX_LEVELS];    // level size * inv_res (== inv_res * level size)
};

__device__ __forceinline__ float level_size(const GridView& g, int k) { return g.ls[k]; }

// tcnn::clamp(val, lo, hi) = val < lo ? lo : (hi < val ? hi : val)
__device__ __forceinline__ float clamp_ref(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

// get_dt, src/utils/raymarching-utils.cuh:7-14
__device__ __forceinline__ float get_dt(float t, float cone, float dt_min, float dt_max) {
    return clamp_ref(__fmul_rn(t, cone), dt_min, dt_max);
}

// BoundingBox::contains, src/models/bounding-box.cuh:70-74
__device__ __forceinline__ bool bbox_contains(const tn_bbox& b, float x, float y, float z) {
    return x >= b.min_x && x <= b.max_x && y >= b.min_y && y <= b.max_y && z >= b.min_z && z <= b.max_z;
}

// Quantised coordinate of get_voxel_morton_index (src/core/occupancy-grid.cuh:155-159),
// clamped to the edge cell where the reference would index outside the bitfield.
__device__ __forceinline__ uint32_t cell_coord(float x, float s, float res_f, int res) {
    const float f = __fmul_rn(__fadd_rn(__fmul_rn(x, s), 0.5f), res_f);
    if (!(f >= 0.0f)) return 0u;
    if (f >= res_f) return (uint32_t)(res - 1);
    return (uint32_t)f;
}

__device__ __forceinline__ uint32_t voxel_morton(const GridView& g, int k, float x, float y, float z) {
    const float s = g.inv_ls[k];
    return morton3d(cell_coord(x, s, g.res_f, g.res), cell_coord(y, s, g.res_f, g.res), cell_coord(z, s, g.res_f, g.res));
}

// get_grid_level_at, src/core/occupancy-grid.cuh:232-248
__device__ __forceinline__ int grid_level_at(const GridView& g, float x, float y, float z, float dt) {
    const float m = fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z)));  // all three < half  <=>  max < half
#pragma unroll
    for (int k = 0; k < MAX_LEVELS; ++k) {
        if (k >= g.n_levels) break;
        if (m < g.half[k] && g.cell[k] > dt) return k;
    }
    return g.n_levels - 1;
}

// get_dt_to_next_voxel, src/core/occupancy-grid.cuh:259-282
__device__ __forceinline__ float dt_to_next_voxel(const GridView& g, float px, float py, float pz,
                                                  float dx, float dy, float dz,
                                                  float idx, float idy, float idz,
                                                  float dt_min, int level) {
    const float ils = g.inv_ls[level];
    const float x = __fmul_rn(__fadd_rn(__fmul_rn(px, ils), 0.5f), g.res_f);
    const float y = __fmul_rn(__fadd_rn(__fmul_rn(py, ils), 0.5f), g.res_f);
    const float z = __fmul_rn(__fadd_rn(__fmul_rn(pz, ils), 0.5f), g.res_f);
    const float k = g.cell[level];  // inv_res * level size
    const float tx = __fmul_rn(k, __fmul_rn(__fadd_rn(floorf(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, copysignf(1.0f, dx)), x), 0.5f)), -x), idx));
    const float ty = __fmul_rn(k, __fmul_rn(__fadd_rn(floorf(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, copysignf(1.0f, dy)), y), 0.5f)), -y), idy));
    const float tz = __fmul_rn(k, __fmul_rn(__fadd_rn(floorf(__fadd_rn(__fadd_rn(__fmul_rn(0.5f, copysignf(1.0f, dz)), z), 0.5f)), -z), idz));
    const float t_target = fmaxf(dt_min, fminf(fminf(tx, ty), tz));
    return __fmul_rn(__fdiv_ru(t_target, dt_min), dt_min);
}

// One ray's march state; step() advances it by one loop iteration of
// march_and_count_steps_per_ray_kernel (src/utils/training-batch-kernels.cuh:263-291).
struct RayMarch {
    float ox, oy, oz, dx, dy, dz, idx, idy, idz;
    float t;
};

__device__ __forceinline__ void ray_point(const RayMarch& r, float t, float& x, float& y, float& z) {
    x = __fadd_rn(r.ox, __fmul_rn(t, r.dx));
    y = __fadd_rn(r.oy, __fmul_rn(t, r.dy));
    z = __fadd_rn(r.oz, __fmul_rn(t, r.dz));
}

// Camera::global_ray_at_pixel_xy (src/models/camera.cuh:94-137) without lens distortion: the ray
// through pixel position (x, y) of a pinhole camera (transform: camera to world, row-major 3 x 4),
// origin on the near plane, unit direction, in FP32 with the reference's operation order.
__device__ __forceinline__ void pinhole_ray(const tn_camera& cam, float x, float y, float& ox, float& oy, float& oz,
                                            float& dx, float& dy, float& dz) {
    const float offx = __fadd_rn(__fmul_rn(cam.shift_x, (float)cam.width), -cam.principal_x);
    const float offy = __fadd_rn(__fmul_rn(cam.shift_y, (float)cam.height), -cam.principal_y);
    const float vx = __fdiv_rn(__fadd_rn(__fadd_rn(x, offx), 0.5f), cam.focal_x);
    const float vy = __fdiv_rn(__fadd_rn(__fadd_rn(y, offy), 0.5f), cam.focal_y);
    const float vz = 1.0f;
    const float vlen = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
    const float* m = cam.transform;
    const float gx = __fadd_rn(__fadd_rn(__fmul_rn(m[0], vx), __fmul_rn(m[1], vy)), __fmul_rn(m[2], vz));
    const float gy = __fadd_rn(__fadd_rn(__fmul_rn(m[4], vx), __fmul_rn(m[5], vy)), __fmul_rn(m[6], vz));
    const float gz = __fadd_rn(__fadd_rn(__fmul_rn(m[8], vx), __fmul_rn(m[9], vy)), __fmul_rn(m[10], vz));
    const float gl = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
    dx = __fdiv_rn(gx, gl);
    dy = __fdiv_rn(gy, gl);
    dz = __fdiv_rn(gz, gl);
    ox = __fadd_rn(m[3], __fmul_rn(cam.near, __fmul_rn(vlen, dx)));
    oy = __fadd_rn(m[7], __fmul_rn(cam.near, __fmul_rn(vlen, dy)));
    oz = __fadd_rn(m[11], __fmul_rn(cam.near, __fmul_rn(vlen, dz)));
}

// ------------------------------------------------------------------------------------
// Counter-based random numbers (synthetic inputs and the trainer's own draws)
// ------------------------------------------------------------------------------------
// 32-bit integer hash (PCG output permutation over a mixed counter)
__host__ __device__ __forceinline__ uint32_t hash_u32(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}

__host__ __device__ __forceinline__ uint32_t rng_u32(uint32_t seed, uint32_t stream, uint32_t i, uint32_t k) {
    return hash_u32(hash_u32(hash_u32(seed ^ 0x9E3779B9u) + stream * 0x85EBCA6Bu) ^ (i * 0xC2B2AE35u + k * 0x27D4EB2Fu));
}

// uniform in [0, 1)
__device__ __forceinline__ float rng_uniform(uint32_t seed, uint32_t stream, uint32_t i, uint32_t k) {
    return (float)(rng_u32(seed, stream, i, k) >> 8) * (1.0f / 16777216.0f);
}

// ------------------------------------------------------------------------------------
// Warp scans
// ------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_inclusive_sum(T v, int lane) {
#pragma unroll
    for (int d = 1; d < WARP; d <<= 1) {
        const T u = __shfl_up_sync(FULL_MASK, v, d);
        if (lane >= d) v += u;
    }
    return v;
}

// Inclusive sum from this lane to lane 31 (a reverse scan).
template <typename T>
__device__ __forceinline__ T warp_inclusive_suffix_sum(T v, int lane) {
#pragma unroll
    for (int d = 1; d < WARP; d <<= 1) {
        const T u = __shfl_down_sync(FULL_MASK, v, d);
        if (lane + d < WARP) v += u;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(FULL_MASK, v, d);
    return v;
}

__device__ __forceinline__ uint32_t ld_u32(const uint32_t* p) { return __ldg(p); }

}  // namespace tn
