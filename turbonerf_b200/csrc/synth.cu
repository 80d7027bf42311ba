// Synthetic producer: the stand-in for the tiny-cuda-nn network upstream of the hot path.
// Density = sum of isotropic Gaussian blobs; colour = sigmoid(sin(a . p + phase)) per
// channel. Used by the benchmark and the trainer's built-in scene; not part of the
// reference's algorithm.
#include "tn_internal.cuh"

namespace tn {

__global__ void synth_field_kernel(uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t ps,
                                   const float* __restrict__ pos, float aabb, uint32_t n_blobs,
                                   const float* __restrict__ blobs, const float* __restrict__ waves,
                                   float* __restrict__ sigma, float* __restrict__ rgb, uint32_t os) {
    extern __shared__ float sh[];
    for (uint32_t k = threadIdx.x; k < 5 * n_blobs + 12; k += blockDim.x)
        sh[k] = k < 5 * n_blobs ? blobs[k] : waves[k - 5 * n_blobs];
    __syncthreads();
    const uint32_t n_live = n_dev ? min(*n_dev, n) : n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_live; i += gridDim.x * blockDim.x) {
        const float x = (pos[i] - 0.5f) * aabb;
        const float y = (pos[i + ps] - 0.5f) * aabb;
        const float z = (pos[i + 2 * (size_t)ps] - 0.5f) * aabb;
        float s = 0.0f;
        for (uint32_t b = 0; b < n_blobs; ++b) {
            const float* bl = sh + 5 * b;
            const float dx = x - bl[0], dy = y - bl[1], dz = z - bl[2];
            s += bl[4] * expf(-(dx * dx + dy * dy + dz * dz) / (2.0f * bl[3] * bl[3]));
        }
        if (sigma) sigma[i] = s;
        if (rgb) {
            const float* wv = sh + 5 * n_blobs;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float a = wv[4 * c] * x + wv[4 * c + 1] * y + wv[4 * c + 2] * z + wv[4 * c + 3];
                rgb[i + c * (size_t)os] = 1.0f / (1.0f + expf(-sinf(a)));
            }
        }
    }
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_synth_field(tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t pos_stride, const float* pos,
                   float aabb_size, uint32_t n_blobs, const float* blobs, const float* waves, float* sigma, float* rgb,
                   uint32_t out_stride) {
    TN_NONNULL(pos); TN_NONNULL(blobs); TN_NONNULL(waves);
    TN_REQUIRE(n_blobs >= 1 && n_blobs <= 256, TN_E_INVALID, "n_blobs %u outside 1..256", n_blobs);
    if (n == 0) return TN_OK;
    const int grid = (int)min((n + 255u) / 256u, (uint32_t)num_sms() * 8u);
    const size_t smem = (5 * (size_t)n_blobs + 12) * sizeof(float);
    synth_field_kernel<<<grid, 256, smem, stream>>>(n, n_dev, pos_stride, pos, aabb_size, n_blobs, blobs, waves, sigma,
                                                    rgb, out_stride);
    return check_launch("tn_synth_field");
}

}  // extern "C"

// ---- counter-based random numbers (synthetic inputs only) ---------------------------------
namespace tn {

__device__ __forceinline__ float rng_normal(uint32_t seed, uint32_t stream, uint32_t i, uint32_t k) {
    const float u1 = fmaxf(rng_uniform(seed, stream, i, 2 * k), 1e-7f);
    const float u2 = rng_uniform(seed, stream, i, 2 * k + 1);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Sphere rays (origins uniform on a sphere of `radius`, directions toward the centre plus
// N(0, jitter) per component), random target colours (alpha 1) and backgrounds, and the
// bounding-box clip, for ray i of step *step_dev.
__global__ void synth_rays_kernel(uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* __restrict__ step_dev,
                                  float radius, float jitter, tn_bbox b, float t_far, float* __restrict__ ori,
                                  float* __restrict__ dir, float* __restrict__ target, float* __restrict__ bg,
                                  float* __restrict__ ray_t, float* __restrict__ ray_t_max, uint8_t* __restrict__ alive) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t st = 2u * (step_dev ? *step_dev : 0u);
    float o[3], d[3];
    float on = 0.0f;
    for (int c = 0; c < 3; ++c) { o[c] = rng_normal(seed, st, i, c); on += o[c] * o[c]; }
    on = rsqrtf(fmaxf(on, 1e-20f));
    float dn = 0.0f;
    for (int c = 0; c < 3; ++c) {
        o[c] *= on;
        d[c] = -o[c] + jitter * rng_normal(seed, st + 1u, i, c);
        dn += d[c] * d[c];
        o[c] *= radius;
    }
    dn = rsqrtf(fmaxf(dn, 1e-20f));
    for (int c = 0; c < 3; ++c) {
        d[c] *= dn;
        ori[i + c * (size_t)rs] = o[c];
        dir[i + c * (size_t)rs] = d[c];
        target[i + c * (size_t)rs] = rng_uniform(seed, st, i, 10 + c);
        bg[i + c * (size_t)rs] = rng_uniform(seed, st, i, 20 + c);
    }
    target[i + 3 * (size_t)rs] = 1.0f;
    // bounding-box clip (same arithmetic as rays_init_kernel in march.cu)
    const float ix = __fdiv_rn(1.0f, d[0]), iy = __fdiv_rn(1.0f, d[1]), iz = __fdiv_rn(1.0f, d[2]);
    float t1x = __fmul_rn(__fadd_rn(b.min_x, -o[0]), ix), t2x = __fmul_rn(__fadd_rn(b.max_x, -o[0]), ix);
    float t1y = __fmul_rn(__fadd_rn(b.min_y, -o[1]), iy), t2y = __fmul_rn(__fadd_rn(b.max_y, -o[1]), iy);
    float t1z = __fmul_rn(__fadd_rn(b.min_z, -o[2]), iz), t2z = __fmul_rn(__fadd_rn(b.max_z, -o[2]), iz);
    if (t1x > t2x) { const float s = t1x; t1x = t2x; t2x = s; }
    if (t1y > t2y) { const float s = t1y; t1y = t2y; t2y = s; }
    if (t1z > t2z) { const float s = t1z; t1z = t2z; t2z = s; }
    const float tmin = fmaxf(t1x, fmaxf(t1y, t1z));
    const float tmax = fminf(t2x, fminf(t2y, t2z));
    const float tm = fminf(t_far, tmax);
    const float t = fmaxf(0.0f, __fadd_rn(tmin, 1e-5f));
    const bool ok = (tmax >= tmin) && !(tm < t);
    ray_t[i] = ok ? t : 0.0f;
    ray_t_max[i] = ok ? tm : 0.0f;
    alive[i] = ok ? 1 : 0;
}

// Random (level, cell) pairs with their in-cell offsets and selection draws for the
// occupancy update of step *step_dev. n_dev (optional) receives n.
__global__ void synth_cells_kernel(uint32_t n, uint32_t seed, const uint32_t* __restrict__ step_dev, int n_levels,
                                   uint32_t volume, int32_t* __restrict__ levels, uint32_t* __restrict__ cells,
                                   float* __restrict__ rand3, uint32_t rand_stride, float* __restrict__ rand_sel) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t st = 0x40000000u + (step_dev ? *step_dev : 0u);
    levels[i] = (int32_t)(rng_u32(seed, st, i, 0) % (uint32_t)n_levels);
    cells[i] = rng_u32(seed, st, i, 1) % volume;
    for (int c = 0; c < 3; ++c) rand3[i + c * (size_t)rand_stride] = rng_uniform(seed, st, i, 2 + c);
    rand_sel[i] = rng_uniform(seed, st, i, 5);
}

// All cells of one level in Morton order [start, start + n) with random in-cell offsets.
__global__ void synth_level_cells_kernel(uint32_t n, uint32_t start, int level, uint32_t seed, uint32_t salt,
                                         int32_t* __restrict__ levels, uint32_t* __restrict__ cells,
                                         float* __restrict__ rand3, uint32_t rand_stride, float* __restrict__ rand_sel) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    levels[i] = level;
    cells[i] = start + i;
    for (int c = 0; c < 3; ++c) rand3[i + c * (size_t)rand_stride] = rng_uniform(seed, salt, start + i, 2 + c);
    rand_sel[i] = rng_uniform(seed, salt, start + i, 5);
}

// Hash-grid entries touched by a batch of normalised positions (instant-NGP multiresolution
// hash encoding: level resolution base * scale^l, dense indexing while (res+1)^3 fits the
// table, else the spatial hash with primes 1, 2654435761, 805459861 modulo the table size).
// Every touched entry gets a deterministic N(0, std) gradient for each of its features.
__global__ void synth_hash_grads_kernel(uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t ps,
                                        const float* __restrict__ pos, int n_levels, uint32_t log2_table,
                                        int n_features, float base_res, float per_level_scale, uint32_t seed,
                                        float std, float* __restrict__ grads) {
    const uint32_t live = n_dev ? min(*n_dev, n) : n;
    const uint32_t T = 1u << log2_table;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < live; i += gridDim.x * blockDim.x) {
        const float p[3] = {pos[i], pos[i + ps], pos[i + 2 * (size_t)ps]};
        for (int l = 0; l < n_levels; ++l) {
            const float scale = base_res * exp2f((float)l * log2f(per_level_scale)) - 1.0f;
            const uint32_t res = (uint32_t)ceilf(scale) + 1u;
            const bool dense = (double)(res + 1) * (res + 1) * (res + 1) <= (double)T;
            uint32_t g[3];
            for (int c = 0; c < 3; ++c) g[c] = (uint32_t)floorf(p[c] * scale + 0.5f);
            for (int corner = 0; corner < 8; ++corner) {
                uint32_t q[3];
                for (int c = 0; c < 3; ++c) q[c] = g[c] + ((corner >> c) & 1u);
                uint32_t idx;
                if (dense) idx = (q[0] + q[1] * (res + 1) + q[2] * (res + 1) * (res + 1)) % T;
                else idx = (q[0] * 1u ^ q[1] * 2654435761u ^ q[2] * 805459861u) & (T - 1u);
                for (int f = 0; f < n_features; ++f) {
                    const size_t e = ((size_t)l * T + idx) * n_features + f;
                    grads[e] = std * rng_normal(seed, 0x7777u, (uint32_t)e, 0);
                }
            }
        }
    }
}

__global__ void synth_params_kernel(uint32_t n, uint32_t n_grid, uint32_t seed, float* __restrict__ w) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float u = rng_uniform(seed, 0x5555u, i, 0) * 2.0f - 1.0f;
    w[i] = i < n_grid ? 1e-4f * u : 0.1f * u;
}

}  // namespace tn

namespace tn {

int launch_synth_rays(cudaStream_t stream, uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* step_dev,
                      float radius, float jitter, const tn_bbox& b, float t_far, float* ori, float* dir, float* target,
                      float* bg, float* ray_t, float* ray_t_max, uint8_t* alive) {
    if (n == 0) return TN_OK;
    synth_rays_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, rs, seed, step_dev, radius, jitter, b, t_far, ori, dir,
                                                           target, bg, ray_t, ray_t_max, alive);
    return check_launch("synth_rays");
}

int launch_synth_cells(cudaStream_t stream, uint32_t n, uint32_t seed, const uint32_t* step_dev, int n_levels,
                       uint32_t volume, int32_t* levels, uint32_t* cells, float* rand3, uint32_t rand_stride,
                       float* rand_sel) {
    if (n == 0) return TN_OK;
    synth_cells_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, seed, step_dev, n_levels, volume, levels, cells, rand3,
                                                            rand_stride, rand_sel);
    return check_launch("synth_cells");
}

int launch_synth_level_cells(cudaStream_t stream, uint32_t n, uint32_t start, int level, uint32_t seed, uint32_t salt,
                             int32_t* levels, uint32_t* cells, float* rand3, uint32_t rand_stride, float* rand_sel) {
    if (n == 0) return TN_OK;
    synth_level_cells_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, start, level, seed, salt, levels, cells, rand3,
                                                                  rand_stride, rand_sel);
    return check_launch("synth_level_cells");
}

int launch_synth_hash_grads(cudaStream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t ps, const float* pos,
                            int n_levels, uint32_t log2_table, int n_features, float base_res, float per_level_scale,
                            uint32_t seed, float std, float* grads) {
    if (n == 0) return TN_OK;
    const int grid = (int)min((n + 255u) / 256u, (uint32_t)num_sms() * 8u);
    synth_hash_grads_kernel<<<grid, 256, 0, stream>>>(n, n_dev, ps, pos, n_levels, log2_table, n_features, base_res,
                                                      per_level_scale, seed, std, grads);
    return check_launch("synth_hash_grads");
}

int launch_synth_params(cudaStream_t stream, uint32_t n, uint32_t n_grid, uint32_t seed, float* w) {
    if (n == 0) return TN_OK;
    synth_params_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, n_grid, seed, w);
    return check_launch("synth_params");
}

}  // namespace tn
