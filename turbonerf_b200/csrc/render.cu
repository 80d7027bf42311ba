// Inference rendering of one NeRF: the reference Renderer::perform_task
// (src/core/renderer.cu:172-646) with the kernels of src/utils/rendering-kernels.cu, the linear
// ray batch (src/rendering/ray-batch-coordinators/linear-buffer-ray-batch-coordinator.cu) and the
// pinhole camera (src/models/camera.cuh:94-137), for one NeRF with an identity transform.
//
// Per ray the image value is: from the ray's entry into the render box, cone steps
// t += get_dt(t, cone, dt_min, 8 dt_min); every sample inside the render box whose cell is
// occupied at its level (chosen from the position and the step scaled to the training box) and
// whose unit-cube position lies inside the training box is queried from the network and
// composited front to back, until the transmittance drops below min_transmittance; the ray ends
// once t has passed t_max. The reference marches each live ray a fixed number of steps per
// iteration (the sample budget over the live rays) and only then drops rays past t_max; the
// samples it marches past t_max lie outside the render box (t_max is the box exit whenever the
// camera's far plane lies beyond it) and contribute nothing, so the image does not depend on that
// schedule. Where the reference writes every step of every live ray to strided buffers and
// queries the network on all of them, each iteration here sends only the valid samples:
//   count     -- each live ray walks its steps of this iteration and counts its valid samples;
//   scan      -- offsets of the valid samples (tn_scan_offsets);
//   emit      -- the same walk writes the valid samples' network inputs, packed, and advances t;
//   network forward on the packed samples;
//   composite -- each ray composites its samples in order with its carried transmittance;
//   compaction of the live-ray list (tn_compact_nonzero), whose length sizes the next iteration.
// Output: premultiplied RGBA per pixel, interleaved (pixel i at out[4 i .. 4 i + 3]), the layout
// the reference copies into its render target (copy_packed_rgba_linear_buffer_kernel).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "tn_internal.cuh"

namespace tn {

struct RenderArgs {
    GridView g;
    tn_bbox render_bbox, train_bbox;
    float train_size_x, train_size_y, train_size_z;  // training box extents (pos_to_unit)
    float inv_train_size;                             // 1 / training box size (its x extent)
    float cone, dt_min, dt_max;
    float min_t;
    int act;
    // level choice from float bit patterns (valid when level k's half extent and cell size are
    // level 0's times 2^k exactly, checked on the host): see render_level
    int fast_level;
    int half0_bits, cell0_bits;
};

// get_grid_level_at (occupancy-grid.cuh:232-248): the finest level whose extent holds the point
// (max |coordinate| m < half extent) and whose cell is larger than the step, else the coarsest.
// Both conditions turn true at some level and stay true above it. For positive floats the order
// of values is the order of bit patterns and level j's constants are level 0's patterns plus
// j << 23, so m < half0 2^j <=> j > (bits(m) - bits(half0)) >> 23 (an arithmetic shift is the
// floor), likewise for the step; the level is the larger first level, clamped to the grid.
__device__ __forceinline__ int render_level(const RenderArgs& A, float x, float y, float z, float dt) {
    if (A.fast_level) {
        const float m = fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z)));
        const int jp = (__float_as_int(m) - A.half0_bits) >> 23;
        const int jd = (__float_as_int(dt) - A.cell0_bits) >> 23;
        return min(max(max(jp, jd) + 1, 0), A.g.n_levels - 1);
    }
    return grid_level_at(A.g, x, y, z, dt);
}

// sigma of a network density output (TN_ACT_DENSITY: density_to_sigma,
// common-network-kernels.cuh:7-10) and the opacity 1 - exp(-sigma dt) of one step
__device__ __forceinline__ float render_sigma(int act, float d) {
    return act == TN_ACT_SIGMA ? d : expf(fminf(d, 12.0f) - 1.0f);
}
__device__ __forceinline__ float render_alpha(float x) { return -expm1f(-x); }

// Camera::global_ray_at_pixel_xy (camera.cuh:94-137) without lens distortion, then the box clip of
// prepare_for_linear_raymarching_kernel (rendering-kernels.cu:175-262) for one NeRF: the origin
// moves to the box entry (at least 1e-4 along the ray), t restarts at 0 and t_max becomes
// min(box exit, far - near), both distances from the unmoved origin as in the reference.
// hit[i] = 1 for rays that meet the box.
__global__ void render_rays_kernel(uint32_t n, tn_camera cam, tn_bbox box, float* __restrict__ ori,
                                   float* __restrict__ dir, float* __restrict__ ray_t, float* __restrict__ ray_tmax,
                                   float* __restrict__ trans, uint32_t* __restrict__ hit) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t w = (uint32_t)cam.width;
    const uint32_t py = i / w, px = i - py * w;
    float ox, oy, oz, dx, dy, dz;
    pinhole_ray(cam, (float)px, (float)py, ox, oy, oz, dx, dy, dz);
    // BoundingBox::get_ray_t_intersections, bounding-box.cuh:27-51
    const float ix = __fdiv_rn(1.0f, dx), iy = __fdiv_rn(1.0f, dy), iz = __fdiv_rn(1.0f, dz);
    float t1x = __fmul_rn(__fadd_rn(box.min_x, -ox), ix), t2x = __fmul_rn(__fadd_rn(box.max_x, -ox), ix);
    float t1y = __fmul_rn(__fadd_rn(box.min_y, -oy), iy), t2y = __fmul_rn(__fadd_rn(box.max_y, -oy), iy);
    float t1z = __fmul_rn(__fadd_rn(box.min_z, -oz), iz), t2z = __fmul_rn(__fadd_rn(box.max_z, -oz), iz);
    if (t1x > t2x) { const float s = t1x; t1x = t2x; t2x = s; }
    if (t1y > t2y) { const float s = t1y; t1y = t2y; t2y = s; }
    if (t1z > t2z) { const float s = t1z; t1z = t2z; t2z = s; }
    const float bmin = fmaxf(t1x, fmaxf(t1y, t1z)), bmax = fminf(t2x, fminf(t2y, t2z));
    const bool volume = box.max_x > box.min_x && box.max_y > box.min_y && box.max_z > box.min_z;
    if (!(volume && bmax >= bmin)) {  // misses the NeRF: the pixel stays clear
        hit[i] = 0u;
        return;
    }
    const float t0 = fmaxf(bmin, 1e-4f);
    ox = __fadd_rn(ox, __fmul_rn(t0, dx));
    oy = __fadd_rn(oy, __fmul_rn(t0, dy));
    oz = __fadd_rn(oz, __fmul_rn(t0, dz));
    ori[i] = ox; ori[i + n] = oy; ori[i + 2 * (size_t)n] = oz;
    dir[i] = dx; dir[i + n] = dy; dir[i + 2 * (size_t)n] = dz;
    ray_t[i] = 0.0f;
    ray_tmax[i] = fminf(bmax, __fadd_rn(cam.far, -cam.near));
    trans[i] = 1.0f;
    hit[i] = 1u;
}

// Coarse occupancy: mip[m] is the OR of the 64 bitfield bytes of the 4 x 4 x 4 block of cells
// with Morton index m (cells [64 m, 64 m + 64)), so bit k of mip[idx >> 6] is clear when the
// whole block of cell idx is empty at level k. The same kernel over mip gives the 16 x 16 x 16
// blocks: bit k of mip2[idx >> 12].
__global__ void render_mip_kernel(uint32_t n_blocks, const uint4* __restrict__ bits, uint8_t* __restrict__ mip) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_blocks) return;
    uint32_t v = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint4 u = __ldg(bits + 4 * (size_t)m + q);
        v |= u.x | u.y | u.z | u.w;
    }
    mip[m] = (uint8_t)((v | (v >> 8) | (v >> 16) | (v >> 24)) & 0xFFu);
}

// World coordinate of the cell boundary with index c (scaled coordinate f = c) at level size ls:
// f = (x / ls + 0.5) R  <=>  x = (c / R - 0.5) ls. The skip margin covers its rounding.
__device__ __forceinline__ float cell_boundary(uint32_t c, float inv_res, float ls) {
    return (float)c * inv_res * ls - 0.5f * ls;
}

// The t window in which the sample position o + t d, computed in FP32, lies inside [lo, hi]
// along one axis with a margin on both faces: the faces are pulled in by far more than the
// rounding of the position (o + t d), of these expressions and of the cell coordinate
// (x / ls + 0.5) R, so a step with t in the window gives a cell coordinate strictly inside the
// box. A zero (or below 2^-128) direction leaves the coordinate in place: the window is then
// everything or nothing.
__device__ __forceinline__ void axis_window(float o, float d, float inv_d, float lo, float hi, float ls, float& t_in,
                                            float& t_out) {
    const float e_lo = 4e-6f * (fabsf(lo) + fabsf(o) + ls), e_hi = 4e-6f * (fabsf(hi) + fabsf(o) + ls);
    const float a = lo + e_lo, b = hi - e_hi;
    if (!(fabsf(inv_d) < INFINITY)) {
        // |d| below 2^-128 (or zero): the coordinate moves by less than the margin at any finite t
        const bool inside = o >= a && o <= b;
        t_in = inside ? -INFINITY : INFINITY;
        t_out = inside ? INFINITY : -INFINITY;
    } else if (d > 0.0f) {
        t_in = (a - o) * inv_d;
        t_out = (b - o) * inv_d;
    } else if (d < 0.0f) {
        t_in = (b - o) * inv_d;
        t_out = (a - o) * inv_d;
    } else {
        const bool inside = o >= a && o <= b;
        t_in = inside ? -INFINITY : INFINITY;
        t_out = inside ? INFINITY : -INFINITY;
    }
}

// One round of one ray: from its t, the steps t += get_dt(t) of the reference's march
// (march_rays_and_generate_global_sample_points_kernel, rendering-kernels.cu:264-334), each sample
// tested as filter_and_localize_samples_for_nerf_kernel and assign_normalized_network_inputs_kernel
// do (:336-478, identity transform): inside the render box, occupied at the level that
// get_grid_level_at picks from the position and the step scaled to the training box, and inside
// the training box in unit coordinates. The t of each valid sample goes to slots[c * stride]; the
// round ends after `quota` valid samples or once t has passed t_max (*done).
//
// Empty space: when a sample's cell is empty, the position's cell (or, when the coarse mips say
// so, its whole 4 x 4 x 4 or 16 x 16 x 16 block) at that level k is empty, and the following steps are taken with
// the same FP32 recurrence but without tests while their positions lie inside that box with a
// margin on every face (axis_window). Each of them would read an empty cell at level k, since the
// level choice max(position term, step term) stays k:
//  * inside the box the position lies inside level k's extent, so the position term is <= k;
//  * aligned blocks of 16^3 (R >= 64) and 4^3 (R >= 16) cells and single cells (R >= 4) lie wholly
//    inside or wholly outside the extent of
//    level k - 1; outside it, the position term is >= k (the margin keeps the position clear of
//    the boundary); inside it, the step term must already be >= k at the current step;
//  * the step term only grows along the ray, and is checked to stay <= k at the largest step
//    (dt_max) unless k is the coarsest level.
// The set of valid samples is therefore exactly the step-by-step one.
struct WalkResult {
    uint32_t count;
    bool done;
    uint32_t steps, tests;
};

__device__ WalkResult render_walk(const RenderArgs& A, const RayMarch& r, float dir_len, float& t_io, float tmax,
                                  uint32_t quota, float* __restrict__ slots, uint32_t stride,
                                  const uint8_t* __restrict__ mip, const uint8_t* __restrict__ mip2,
                                  const uint32_t* __restrict__ spread, uint32_t max_iters, uint32_t* flags) {
    const GridView& g = A.g;
    const float dtn_max = __fmul_rn(A.inv_train_size, __fmul_rn(dir_len, A.dt_max));
    const bool cells_ok = g.res >= 4, blocks_ok = g.res >= 16 && mip != nullptr;
    const bool supers_ok = g.res >= 64 && mip2 != nullptr;
    float t = t_io;
    uint32_t c = 0, iters = 0, tests = 0;
    bool done = false;
    while (c < quota) {
        if (t > tmax) {
            done = true;
            break;
        }
        if (++iters > max_iters) {
            raise_flag(flags, ERR_GUARD);
            done = true;
            break;
        }
        const float dt = get_dt(t, A.cone, A.dt_min, A.dt_max);
        float x, y, z;
        ray_point(r, t, x, y, z);
        ++tests;
        if (bbox_contains(A.render_bbox, x, y, z)) {
            const float dt_net = __fmul_rn(A.inv_train_size, __fmul_rn(dir_len, dt));
            const int k = render_level(A, x, y, z, dt_net);
            const float s = g.inv_ls[k];
            const float fx = __fmul_rn(__fadd_rn(__fmul_rn(x, s), 0.5f), g.res_f);
            const float fy = __fmul_rn(__fadd_rn(__fmul_rn(y, s), 0.5f), g.res_f);
            const float fz = __fmul_rn(__fadd_rn(__fmul_rn(z, s), 0.5f), g.res_f);
            // cell coordinates of get_voxel_morton_index, clamped to the grid (cell_coord)
            const uint32_t rm1 = (uint32_t)g.res - 1u;
            const uint32_t cx = min(__float2uint_rz(fx), rm1), cy = min(__float2uint_rz(fy), rm1),
                           cz = min(__float2uint_rz(fz), rm1);
            const uint32_t idx = spread[cx] | spread[g.res + cy] | spread[2 * g.res + cz];
            // the coarse mip first: an empty block needs no read of the bitfield
            const bool block_on = !blocks_ok || ((__ldg(mip + (idx >> 6)) >> k) & 1u);
            if (block_on && ((__ldg(g.bits + idx) >> k) & 1u)) {
                const float ux = __fdiv_rn(__fadd_rn(x, -A.train_bbox.min_x), A.train_size_x);
                const float uy = __fdiv_rn(__fadd_rn(y, -A.train_bbox.min_y), A.train_size_y);
                const float uz = __fdiv_rn(__fadd_rn(z, -A.train_bbox.min_z), A.train_size_z);
                if (ux >= 0.0f && ux <= 1.0f && uy >= 0.0f && uy <= 1.0f && uz >= 0.0f && uz <= 1.0f) {
                    slots[(size_t)c * stride] = t;
                    ++c;
                }
            } else if (cells_ok && fx >= 0.0f && fx < g.res_f && fy >= 0.0f && fy < g.res_f && fz >= 0.0f &&
                       fz < g.res_f && (k == g.n_levels - 1 || dtn_max < g.cell[k])) {
                // the empty box: the 16^3 or 4^3 block when the mips say it is empty, else the cell
                const int sh = block_on ? 0 : ((supers_ok && !((__ldg(mip2 + (idx >> 12)) >> k) & 1u)) ? 4 : 2);
                const uint32_t lx = (cx >> sh) << sh, ly = (cy >> sh) << sh, lz = (cz >> sh) << sh;
                const uint32_t w = 1u << sh, q1 = (uint32_t)g.res >> 2, q3 = 3u * q1;
                const bool inner = lx >= q1 && lx + w <= q3 && ly >= q1 && ly + w <= q3 && lz >= q1 && lz + w <= q3;
                t = __fadd_rn(t, dt);
                if (!inner || k == 0 || !(g.cell[k - 1] > dt_net)) {
                    const float ls = g.ls[k];
                    float ix0, ix1, iy0, iy1, iz0, iz1;
                    axis_window(r.ox, r.dx, r.idx, cell_boundary(lx, g.inv_res, ls),
                                cell_boundary(lx + w, g.inv_res, ls), ls, ix0, ix1);
                    axis_window(r.oy, r.dy, r.idy, cell_boundary(ly, g.inv_res, ls),
                                cell_boundary(ly + w, g.inv_res, ls), ls, iy0, iy1);
                    axis_window(r.oz, r.dz, r.idz, cell_boundary(lz, g.inv_res, ls),
                                cell_boundary(lz + w, g.inv_res, ls), ls, iz0, iz1);
                    const float t_in = fmaxf(ix0, fmaxf(iy0, iz0));
                    const float t_out = fminf(fminf(ix1, fminf(iy1, iz1)), tmax);
                    if (t >= t_in) {
                        // once t cone has reached dt_max every later step is dt_max (t only grows):
                        // four steps per window test; t is monotone, so the fourth decides
                        if (__fmul_rn(t, A.cone) >= A.dt_max) {
                            while (iters + 4u <= max_iters) {
                                const float t4 = __fadd_rn(
                                    __fadd_rn(__fadd_rn(__fadd_rn(t, A.dt_max), A.dt_max), A.dt_max), A.dt_max);
                                if (!(t4 <= t_out)) break;
                                t = t4;
                                iters += 4u;
                            }
                        }
                        while (t <= t_out && iters < max_iters) {
                            t = __fadd_rn(t, get_dt(t, A.cone, A.dt_min, A.dt_max));
                            ++iters;
                        }
                    }
                }
                continue;
            }
        }
        t = __fadd_rn(t, dt);
    }
    t_io = t;
    return {c, done, iters, tests};
}

// One round of every live ray: counts[j] valid samples with their t in slots[c * n_live + j],
// the ray's t advanced; keep[j] = 0 once the ray has passed t_max.
__global__ void render_walk_kernel(RenderArgs A, uint32_t n, uint32_t n_live, uint32_t quota,
                                   const uint32_t* __restrict__ live, const float* __restrict__ ori,
                                   const float* __restrict__ dir, float* __restrict__ ray_t,
                                   const float* __restrict__ ray_tmax, const uint8_t* __restrict__ mip,
                                   const uint8_t* __restrict__ mip2, uint32_t max_iters, uint32_t* __restrict__ counts, float* __restrict__ slots,
                                   uint32_t* __restrict__ keep, unsigned long long* __restrict__ totals,
                                   uint32_t* flags) {
    // Morton spread tables (get_voxel_morton_index), one per axis, pre-shifted: 3 R words
    extern __shared__ uint32_t spread[];
    const uint32_t R = (uint32_t)A.g.res;
    for (uint32_t c = threadIdx.x; c < R; c += blockDim.x) {
        const uint32_t v = part1by2(c);
        spread[c] = v;
        spread[R + c] = v << 1;
        spread[2 * R + c] = v << 2;
    }
    __syncthreads();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t steps = 0, tests = 0;
    if (j < n_live) {
        const uint32_t i = live[j];
        RayMarch r;
        r.ox = ori[i]; r.oy = ori[i + n]; r.oz = ori[i + 2 * (size_t)n];
        r.dx = dir[i]; r.dy = dir[i + n]; r.dz = dir[i + 2 * (size_t)n];
        r.idx = __fdiv_rn(1.0f, r.dx);
        r.idy = __fdiv_rn(1.0f, r.dy);
        r.idz = __fdiv_rn(1.0f, r.dz);
        const float dir_len =
            __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.dx, r.dx), __fmul_rn(r.dy, r.dy)), __fmul_rn(r.dz, r.dz)));
        float t = ray_t[i];
        const WalkResult w =
            render_walk(A, r, dir_len, t, ray_tmax[i], quota, slots + j, n_live, mip, mip2, spread, max_iters, flags);
        ray_t[i] = t;
        counts[j] = w.count;
        keep[j] = w.done ? 0u : 1u;
        steps = w.steps;
        tests = w.tests;
    }
    // steps and tests of the round (statistics)
    const unsigned long long ws = warp_sum((unsigned long long)steps), wt = warp_sum((unsigned long long)tests);
    if ((threadIdx.x & 31u) == 0 && (ws | wt)) {
        atomicAdd(totals, ws);
        atomicAdd(totals + 1, wt);
    }
}

// A warp owns 32 consecutive live rays, whose samples are one contiguous range of the packed
// batch (the offsets are the exclusive scan of the counts in live order): ray_of_sample finds the
// lane whose range holds sample s, the largest r with off[r] <= s, by binary search over the
// warp's offsets in shared memory (lanes past the last live ray hold UINT32_MAX).
constexpr int RW_WARPS = 8;  // warps per block of the expand and composite kernels

__device__ __forceinline__ int ray_of_sample(const uint32_t* off, uint32_t s) {
    int r = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
        if (off[r + step] <= s) r += step;
    return r;
}

// Network inputs of the round's samples, packed at offsets[j]: unit-cube position clamped to
// [0, 1], direction 0.5 d + 0.5, and the step in units of the training box size
// (assign_normalized_network_inputs_kernel, rendering-kernels.cu:404-478). One thread per
// sample of the warp's range, so consecutive lanes write consecutive samples.
__global__ void __launch_bounds__(32 * RW_WARPS)
render_expand_kernel(RenderArgs A, uint32_t n, uint32_t n_live, const uint32_t* __restrict__ live,
                     const float* __restrict__ ori, const float* __restrict__ dir, const uint32_t* __restrict__ counts,
                     const uint32_t* __restrict__ offsets, const float* __restrict__ slots, uint32_t cap,
                     float* __restrict__ s_pos, float* __restrict__ s_dir, float* __restrict__ s_dt, uint32_t* flags) {
    __shared__ uint32_t sh_off[RW_WARPS][32];
    __shared__ float sh_ray[RW_WARPS][7][32];  // o 3 | d 3 | |d|
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t j0 = (blockIdx.x * RW_WARPS + w) * 32u;
    if (j0 >= n_live) return;  // the whole warp leaves
    const uint32_t j = j0 + lane;
    uint32_t off = 0xFFFFFFFFu, end = 0;
    if (j < n_live) {
        const uint32_t i = live[j];
        off = offsets[j];
        end = off + counts[j];
        const float dx = dir[i], dy = dir[i + n], dz = dir[i + 2 * (size_t)n];
        sh_ray[w][0][lane] = ori[i];
        sh_ray[w][1][lane] = ori[i + n];
        sh_ray[w][2][lane] = ori[i + 2 * (size_t)n];
        sh_ray[w][3][lane] = dx;
        sh_ray[w][4][lane] = dy;
        sh_ray[w][5][lane] = dz;
        sh_ray[w][6][lane] = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz)));
    }
    sh_off[w][lane] = off;
    const uint32_t last = min(31u, n_live - 1u - j0);
    const uint32_t base = __shfl_sync(FULL_MASK, off, 0), stop = __shfl_sync(FULL_MASK, end, last);
    __syncwarp();
    if (stop > cap) {
        if (lane == 0) raise_flag(flags, ERR_CAPACITY);
        return;
    }
    for (uint32_t s = base + lane; s < stop; s += 32) {
        const int r = ray_of_sample(sh_off[w], s);
        const float t = slots[(size_t)(s - sh_off[w][r]) * n_live + j0 + r];
        RayMarch ray;
        ray.ox = sh_ray[w][0][r]; ray.oy = sh_ray[w][1][r]; ray.oz = sh_ray[w][2][r];
        ray.dx = sh_ray[w][3][r]; ray.dy = sh_ray[w][4][r]; ray.dz = sh_ray[w][5][r];
        const float dt = get_dt(t, A.cone, A.dt_min, A.dt_max);
        float x, y, z;
        ray_point(ray, t, x, y, z);
        s_pos[s] = clamp_ref(__fdiv_rn(__fadd_rn(x, -A.train_bbox.min_x), A.train_size_x), 0.0f, 1.0f);
        s_pos[s + cap] = clamp_ref(__fdiv_rn(__fadd_rn(y, -A.train_bbox.min_y), A.train_size_y), 0.0f, 1.0f);
        s_pos[s + 2 * (size_t)cap] = clamp_ref(__fdiv_rn(__fadd_rn(z, -A.train_bbox.min_z), A.train_size_z), 0.0f, 1.0f);
        s_dir[s] = __fmaf_rn(0.5f, ray.dx, 0.5f);
        s_dir[s + cap] = __fmaf_rn(0.5f, ray.dy, 0.5f);
        s_dir[s + 2 * (size_t)cap] = __fmaf_rn(0.5f, ray.dz, 0.5f);
        s_dt[s] = __fmul_rn(A.inv_train_size, __fmul_rn(sh_ray[w][6][r], dt));
    }
}

// composite_samples_kernel (rendering-kernels.cu:530-618) after accumulate_nerf_samples_kernel
// (:480-528) for one NeRF: each live ray composites its samples of this round in order. keep[j]
// (set by the walk while t has not passed t_max, kill_terminated_rays_kernel :620-637) is cleared
// when the transmittance falls below min_transmittance.
// The warp walks its sample range in chunks of RC_CHUNK: all lanes load a chunk with coalesced
// reads and compute each sample's opacity, then each lane composites its own ray's samples of the
// chunk in order from shared memory.
constexpr int RC_CHUNK = 128;

__global__ void __launch_bounds__(32 * RW_WARPS)
render_composite_kernel(RenderArgs A, uint32_t n_live, const uint32_t* __restrict__ live,
                        const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets, uint32_t cap,
                        const float* __restrict__ density, const float* __restrict__ rgb,
                        const float* __restrict__ s_dt, float* __restrict__ trans, float* __restrict__ out,
                        uint32_t* __restrict__ keep) {
    __shared__ float sh[RW_WARPS][4][RC_CHUNK];  // alpha | r | g | b
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t j0 = (blockIdx.x * RW_WARPS + w) * 32u;
    if (j0 >= n_live) return;  // the whole warp leaves
    const uint32_t j = j0 + lane;
    const bool has = j < n_live;
    uint32_t i = 0, off = 0, end = 0;
    float T = 1.0f;
    if (has) {
        i = live[j];
        off = offsets[j];
        end = min(off + counts[j], cap);
        T = trans[i];
    }
    const uint32_t last = min(31u, n_live - 1u - j0);
    const uint32_t base = __shfl_sync(FULL_MASK, off, 0), stop = min(__shfl_sync(FULL_MASK, end, last), cap);
    float orr = 0.0f, og = 0.0f, ob = 0.0f, oa = 0.0f;
    bool alive = true;
    for (uint32_t c0 = base; c0 < stop; c0 += RC_CHUNK) {
        const uint32_t cn = min((uint32_t)RC_CHUNK, stop - c0);
        // per sample, in parallel: a = min(alpha, 1) and the colour of one NeRF's sample, the
        // network colour where alpha > 1e-4 and zero below (the reference's (c alpha) / alpha,
        // with the product and quotient, which cancel to within two roundings, left out)
        for (uint32_t q = lane; q < cn; q += 32) {
            const uint32_t s = c0 + q;
            const float alpha = render_alpha(__fmul_rn(render_sigma(A.act, density[s]), s_dt[s]));
            const bool lit = alpha > 0.0001f;
            sh[w][0][q] = fminf(alpha, 1.0f);
            sh[w][1][q] = lit ? rgb[s] : 0.0f;
            sh[w][2][q] = lit ? rgb[s + cap] : 0.0f;
            sh[w][3][q] = lit ? rgb[s + 2 * (size_t)cap] : 0.0f;
        }
        __syncwarp();
        // per ray, in order: the transmittance chain
        const uint32_t lo = max(off, c0), hi = min(end, c0 + cn);
        for (uint32_t s = lo; alive && s < hi; ++s) {
            const uint32_t q = s - c0;
            const float a = sh[w][0][q];
            const float wt = a * T;
            orr = fmaf(wt, sh[w][1][q], orr);
            og = fmaf(wt, sh[w][2][q], og);
            ob = fmaf(wt, sh[w][3][q], ob);
            oa += wt;
            T = T * (1.0f - a);
            if (T < A.min_t) alive = false;
        }
        __syncwarp();
    }
    if (!has) return;
    trans[i] = T;
    float4* px = reinterpret_cast<float4*>(out) + i;
    float4 v = *px;
    v.x += orr; v.y += og; v.z += ob; v.w += oa;
    *px = v;
    if (!alive) keep[j] = 0u;
}

// next live list: the rays whose keep flag is set, in list order
__global__ void render_gather_live_kernel(const uint32_t* __restrict__ n_kept, const int32_t* __restrict__ idx,
                                          const uint32_t* __restrict__ live, uint32_t* __restrict__ next) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < *n_kept) next[k] = live[idx[k]];
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_render(tn_ctx* ctx, tn_stream_t stream, const tn_render_desc* desc, const tn_camera* camera,
              const tn_network* net, float* out_rgba, tn_render_stats* stats) {
    TN_NONNULL(ctx); TN_NONNULL(desc); TN_NONNULL(camera); TN_NONNULL(net);
    TN_REQUIRE(camera->width > 0 && camera->height > 0, TN_E_INVALID, "tn_render: empty image %d x %d", camera->width,
               camera->height);
    TN_REQUIRE(camera->focal_x != 0.0f && camera->focal_y != 0.0f, TN_E_INVALID, "tn_render: zero focal length");
    TN_NONNULL(out_rgba); TN_NONNULL(net->forward); TN_NONNULL(desc->bitfield);
    int st = validate_grid(&desc->grid);
    if (st != TN_OK) return st;
    TN_REQUIRE(desc->dt_min > 0.0f && desc->cone_angle >= 0.0f, TN_E_INVALID, "tn_render: need dt_min > 0, cone >= 0");
    TN_REQUIRE(net->activation == TN_ACT_SIGMA || net->activation == TN_ACT_DENSITY, TN_E_INVALID,
               "tn_render: unknown activation %d", net->activation);
    const tn_bbox& tb = desc->training_bbox;
    TN_REQUIRE(tb.max_x > tb.min_x && tb.max_y > tb.min_y && tb.max_z > tb.min_z, TN_E_INVALID,
               "tn_render: empty training box");
    TN_REQUIRE(((uintptr_t)out_rgba & 15u) == 0, TN_E_INVALID, "tn_render: out_rgba must be 16-byte aligned");
    TN_REQUIRE(!stream_capturing(stream), TN_E_STATE, "tn_render synchronises its stream (not during capture)");
    const uint64_t n64 = (uint64_t)camera->width * (uint64_t)camera->height;
    TN_REQUIRE(n64 <= (1u << 26), TN_E_CAPACITY, "tn_render: %llu pixels exceed 2^26", (unsigned long long)n64);
    const uint32_t n = (uint32_t)n64;
    // 0: a budget from the image size, 8 samples per pixel within [2^20, 2^25] (the reference fixes
    // 1 << 20 and leaves deriving it from the GPU as a to-do, nerf-rendering-controller.cu:20-23)
    const uint32_t batch = desc->batch_size ? desc->batch_size
                                            : (uint32_t)std::min<uint64_t>(std::max<uint64_t>(8 * n64, 1u << 20), 1u << 25);
    TN_REQUIRE(batch <= (1u << 28), TN_E_CAPACITY, "tn_render: batch_size %u exceeds 2^28", batch);
    // live rays x steps never exceeds max(batch, live rays)
    const uint32_t cap = std::max(batch, n);

    RenderArgs A;
    A.g = make_grid_view(desc->grid, desc->bitfield);
    A.render_bbox = desc->render_bbox;
    A.train_bbox = tb;
    {
        volatile float one = 1.0f;
        A.train_size_x = tb.max_x - tb.min_x;
        A.train_size_y = tb.max_y - tb.min_y;
        A.train_size_z = tb.max_z - tb.min_z;
        A.inv_train_size = one / A.train_size_x;
    }
    A.cone = desc->cone_angle;
    A.dt_min = desc->dt_min;
    A.dt_max = 8.0f * desc->dt_min;  // renderer.cu:305
    A.min_t = desc->min_transmittance;
    A.act = net->activation;
    {
        // the bit-pattern level choice needs every level's constants to be level 0's times 2^k
        auto bits_of = [](float f) { int b; memcpy(&b, &f, 4); return b; };
        A.half0_bits = bits_of(A.g.half[0]);
        A.cell0_bits = bits_of(A.g.cell[0]);
        bool ok = std::isnormal(A.g.half[0]) && std::isnormal(A.g.cell[0]) && A.g.half[0] > 0.0f && A.g.cell[0] > 0.0f;
        for (int k = 0; k < A.g.n_levels; ++k)
            ok = ok && bits_of(A.g.half[k]) == A.half0_bits + (k << 23) && bits_of(A.g.cell[k]) == A.cell0_bits + (k << 23);
        A.fast_level = ok ? 1 : 0;
    }
    const size_t spread_bytes = (size_t)3 * desc->grid.resolution * sizeof(uint32_t);  // <= 12 KiB (R <= 1024)

    // workspace: rays [o 3 | d 3 | t | t_max | T] x n floats; pixel lists [live | live2 | counts |
    // offsets | keep | idx] x n u32; counters (16 u32); coarse mips (R^3 / 64 bytes for 4^3 blocks
    // and R^3 / 4096 for 16^3 blocks, each rounded up to 64 bytes); samples [slots | pos 3 | dir 3 |
    // dt | density | rgb 3] x cap floats
    const uint32_t res = (uint32_t)desc->grid.resolution;
    const uint32_t mip_blocks = res >= 16 ? res * res * res / 64 : 0u;
    const uint32_t mip2_blocks = res >= 64 ? mip_blocks / 64 : 0u;
    const size_t ray_words = ((size_t)9 * n + 3) & ~(size_t)3, list_words = ((size_t)6 * n + 3) & ~(size_t)3;
    const size_t mip1_words = ((size_t)mip_blocks + 63) / 64 * 16;
    const size_t mip_words = mip1_words + ((size_t)mip2_blocks + 63) / 64 * 16;
    const size_t smp_words = (size_t)12 * cap;
    st = ensure_render_ws(ctx, (ray_words + list_words + 16 + mip_words + smp_words) * 4);
    if (st != TN_OK) return st;
    float* rays = reinterpret_cast<float*>(ctx->render_ws);
    float *ori = rays, *dir = rays + 3 * (size_t)n, *ray_t = rays + 6 * (size_t)n, *ray_tmax = rays + 7 * (size_t)n,
          *trans = rays + 8 * (size_t)n;
    uint32_t* u32 = reinterpret_cast<uint32_t*>(rays + ray_words);
    uint32_t *live = u32, *live2 = u32 + n, *counts = u32 + 2 * (size_t)n, *offsets = u32 + 3 * (size_t)n,
             *keep = u32 + 4 * (size_t)n;
    int32_t* idx = reinterpret_cast<int32_t*>(u32 + 5 * (size_t)n);
    // [0] live rays, [1..4] batch info, [5] kept rays, [8..11] steps and tests (two u64)
    uint32_t* counters = u32 + list_words;
    unsigned long long* totals = reinterpret_cast<unsigned long long*>(counters + 8);
    uint32_t* info = counters + 1;
    uint8_t* mip = mip_blocks ? reinterpret_cast<uint8_t*>(counters + 16) : nullptr;
    uint8_t* mip2 = mip2_blocks ? reinterpret_cast<uint8_t*>(counters + 16 + mip1_words) : nullptr;
    float* smp = reinterpret_cast<float*>(counters + 16 + mip_words);
    float *slots = smp, *s_pos = smp + (size_t)cap, *s_dir = smp + 4 * (size_t)cap, *s_dt = smp + 7 * (size_t)cap,
          *s_density = smp + 8 * (size_t)cap, *s_rgb = smp + 9 * (size_t)cap;
    TN_REQUIRE(!mip_blocks || ((uintptr_t)desc->bitfield & 15u) == 0, TN_E_INVALID,
               "tn_render: bitfield must be 16-byte aligned");
    const uint32_t max_iters = 1u << 24;  // steps of one ray in one round

    tn_render_stats S{};
    st = cuda_status(cudaMemsetAsync(out_rgba, 0, (size_t)n * 16, stream), "tn_render(clear)");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(counters, 0, 64, stream), "tn_render(counters)");
    if (st == TN_OK && mip_blocks) {
        render_mip_kernel<<<(mip_blocks + 255) / 256, 256, 0, stream>>>(
            mip_blocks, reinterpret_cast<const uint4*>(desc->bitfield), mip);
        st = check_launch("tn_render(mip)");
    }
    if (st == TN_OK && mip2_blocks) {  // the same OR, of the 64 4^3 blocks of each 16^3 block
        render_mip_kernel<<<(mip2_blocks + 255) / 256, 256, 0, stream>>>(
            mip2_blocks, reinterpret_cast<const uint4*>(mip), mip2);
        st = check_launch("tn_render(mip2)");
    }
    if (st == TN_OK) {
        render_rays_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, *camera, desc->render_bbox, ori, dir, ray_t,
                                                                ray_tmax, trans, keep);
        st = check_launch("tn_render(rays)");
    }
    // live list in pixel order
    if (st == TN_OK) st = tn_compact_nonzero(ctx, stream, n, keep, reinterpret_cast<int32_t*>(live), counters);
    uint32_t n_live = 0;
    if (st == TN_OK)
        st = cuda_status(cudaMemcpyAsync(&n_live, counters, 4, cudaMemcpyDeviceToHost, stream), "tn_render(hits)");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_render(sync)");
    S.rays_hit = n_live;
    const uint32_t max_rounds = 1u << 20;
    while (st == TN_OK && n_live > 0 && S.iterations < max_rounds) {
        // each live ray collects up to `quota` valid samples this round (the reference's round is
        // max(batch / live rays, 1) steps, renderer.cu:301)
        const uint32_t quota = std::max(batch / n_live, 1u);
        const int grid = (int)((n_live + 255) / 256);
        render_walk_kernel<<<grid, 256, spread_bytes, stream>>>(A, n, n_live, quota, live, ori, dir, ray_t, ray_tmax,
                                                                mip, mip2, max_iters, counts, slots, keep, totals,
                                                                ctx->flags);
        st = check_launch("tn_render(walk)");
        if (st == TN_OK) st = tn_scan_offsets(ctx, stream, n_live, counts, offsets, 0xffffffffu, info);
        if (st == TN_OK) {
            render_expand_kernel<<<grid, 256, 0, stream>>>(A, n, n_live, live, ori, dir, counts, offsets, slots, cap,
                                                           s_pos, s_dir, s_dt, ctx->flags);
            st = check_launch("tn_render(expand)");
        }
        if (st == TN_OK) st = net->forward(net->user, stream, cap, info + 1, cap, s_pos, s_dir, s_density, s_rgb);
        if (st == TN_OK) {
            render_composite_kernel<<<grid, 256, 0, stream>>>(A, n_live, live, counts, offsets, cap, s_density, s_rgb,
                                                              s_dt, trans, out_rgba, keep);
            st = check_launch("tn_render(composite)");
        }
        if (st == TN_OK) st = tn_compact_nonzero(ctx, stream, n_live, keep, idx, counters + 5);
        if (st == TN_OK) {
            render_gather_live_kernel<<<grid, 256, 0, stream>>>(counters + 5, idx, live, live2);
            st = check_launch("tn_render(live)");
        }
        uint32_t host[5] = {0, 0, 0, 0, 0};  // batch info [0..3], kept rays
        if (st == TN_OK)
            st = cuda_status(cudaMemcpyAsync(host, info, sizeof(host), cudaMemcpyDeviceToHost, stream),
                             "tn_render(live)");
        if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_render(sync)");
        if (st != TN_OK) break;
        S.samples += host[1];
        ++S.iterations;
        n_live = host[4];
        std::swap(live, live2);
    }
    if (st == TN_OK && n_live > 0) st = fail(TN_E_DEVICE, "tn_render: rays still live after %u rounds", max_rounds);
    if (st == TN_OK) {
        unsigned long long tot[2] = {0, 0};
        st = cuda_status(cudaMemcpyAsync(tot, totals, sizeof(tot), cudaMemcpyDeviceToHost, stream), "tn_render(stats)");
        if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_render(sync)");
        S.steps = tot[0];
        S.tests = tot[1];
    }
    uint32_t flags = 0;
    if (st == TN_OK) st = tn_ctx_check(ctx, stream, &flags);
    if (st == TN_OK && (flags & TN_FLAG_CAPACITY)) st = fail(TN_E_CAPACITY, "tn_render: sample capacity exceeded");
    if (st == TN_OK && (flags & TN_FLAG_GUARD)) st = fail(TN_E_DEVICE, "tn_render: a ray took over %u steps in a round", max_iters);
    if (stats) *stats = S;
    return st;
}

}  // extern "C"
