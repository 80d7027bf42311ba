// Occupancy-grid ray marching with sample compaction.
//
// Fused path (tn_march_count + tn_march_emit): no host round trip, one sequential march.
//  * count: one thread per ray runs the reference's DDA loop with its exact arithmetic, written
//    branch-free per step (both successors of t are computed, one is selected) so that a warp's
//    rays never split. Shared memory holds a Morton spread table and a coarse occupancy mip
//    that answers empty 4x4x4 blocks without a global load. A box holding every occupied cell
//    ends each ray's loop where it leaves that box for good (the count cannot change after).
//    The t of every occupied step goes to a per-ray slot. Each 64-ray block reduces its counts;
//    the last block to finish (ticket) scans the block totals and performs the reference's
//    batch cut on the device (batch_info).
//  * emit: one warp per ray rebuilds the ray's offset and expands its recorded steps into the
//    packed sample arrays, one lane per sample (coalesced stores), instead of replaying the march.
// Plain path (tn_plain_*): count kernel, thrust exclusive_scan, reverse find_if, a
// blocking device->host read of the sample count, emit kernel -- the reference's launch
// structure (src/core/trainer.cu:106-216).
#include <thrust/execution_policy.h>
#include <thrust/find.h>
#include <thrust/iterator/reverse_iterator.h>
#include <thrust/scan.h>
#include <thrust/device_ptr.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "tn_internal.cuh"

namespace tn {

constexpr int MARCH_BLOCK = 128;

struct MarchArgs {
    GridView g;
    tn_bbox bbox;
    float cone, dt_min, dt_max;
    float inv_dt_min;  // 1 / dt_min rounded to nearest (host division)
    uint32_t max_steps, max_iters;
};

// Occupancy test (OccupancyGrid::is_occupied_at, src/core/occupancy-grid.cuh:185-207).
__device__ __forceinline__ bool occupied_at(const GridView& g, int k, float x, float y, float z) {
    const uint32_t idx = voxel_morton(g, k, x, y, z);
    return (__ldg(g.bits + idx) & (1u << k)) != 0;
}

__device__ __forceinline__ void load_ray(RayMarch& r, const float* __restrict__ ori, const float* __restrict__ dir,
                                         uint32_t i, uint32_t rs) {
    r.ox = ori[i]; r.oy = ori[i + rs]; r.oz = ori[i + 2 * (size_t)rs];
    r.dx = dir[i]; r.dy = dir[i + rs]; r.dz = dir[i + 2 * (size_t)rs];
    r.idx = __fdiv_rn(1.0f, r.dx);
    r.idy = __fdiv_rn(1.0f, r.dy);
    r.idz = __fdiv_rn(1.0f, r.dz);
}

// march_and_count_steps_per_ray_kernel loop, src/utils/training-batch-kernels.cuh:258-297, in the
// reference's form (plain path).
__device__ uint32_t march_count_ray(const MarchArgs& a, const RayMarch& r, float t_max, uint32_t* flags) {
    uint32_t n = 0, iters = 0;
    float t = r.t;
    while (t < t_max) {
        if (++iters > a.max_iters) { raise_flag(flags, ERR_GUARD); break; }
        float x, y, z;
        ray_point(r, t, x, y, z);
        if (!bbox_contains(a.bbox, x, y, z)) break;
        const float dt = get_dt(t, a.cone, a.dt_min, a.dt_max);
        const int k = grid_level_at(a.g, x, y, z, dt);
        if (occupied_at(a.g, k, x, y, z)) {
            t = __fadd_rn(t, dt);
            ++n;
            if (a.max_steps != 0u && n >= a.max_steps) break;
        } else {
            t = __fadd_rn(t, dt_to_next_voxel(a.g, x, y, z, r.dx, r.dy, r.dz, r.idx, r.idy, r.idz, a.dt_min, k));
        }
    }
    return n;
}

struct SampleOut {
    uint32_t* img_id;
    float* t;
    float* pos;
    float* dir;
    float* dt;
    float* m_norm;
    float* dt_norm;
    uint32_t ss;
};

// assign_normalized_ray_sample, src/utils/training-batch-kernels.cuh:305-331
__device__ __forceinline__ void write_sample(const SampleOut& o, uint32_t s, float x, float y, float z,
                                             const RayMarch& r, float dt, float inv_aabb) {
    const size_t ss = o.ss;
    o.dt[s] = __fmul_rn(inv_aabb, dt);
    o.pos[s] = clamp_ref(__fadd_rn(__fmul_rn(x, inv_aabb), 0.5f), 0.0f, 1.0f);
    o.pos[s + ss] = clamp_ref(__fadd_rn(__fmul_rn(y, inv_aabb), 0.5f), 0.0f, 1.0f);
    o.pos[s + 2 * ss] = clamp_ref(__fadd_rn(__fmul_rn(z, inv_aabb), 0.5f), 0.0f, 1.0f);
    o.dir[s] = __fadd_rn(__fmul_rn(0.5f, r.dx), 0.5f);
    o.dir[s + ss] = __fadd_rn(__fmul_rn(0.5f, r.dy), 0.5f);
    o.dir[s + 2 * ss] = __fadd_rn(__fmul_rn(0.5f, r.dz), 0.5f);
}

// march_and_generate_network_positions_kernel body, src/utils/training-batch-kernels.cuh:405-480
__device__ void march_emit_ray(const MarchArgs& a, RayMarch& r, uint32_t n_steps, uint32_t off, uint32_t img,
                               float inv_aabb, const SampleOut& o) {
    float t = r.t;
    const float t_min = t;
    float t_max = t;
    uint32_t taken = 0, iters = 0;
    while (taken < n_steps) {
        // The count pass already bounded this ray's loop; the guard only protects against
        // inputs that changed between the two passes.
        if (++iters > a.max_iters) break;
        float x, y, z;
        ray_point(r, t, x, y, z);
        const float dt = get_dt(t, a.cone, a.dt_min, a.dt_max);
        const uint32_t s = off + taken;
        if (!bbox_contains(a.bbox, x, y, z)) {
            o.t[s] = t;
            o.m_norm[s] = __fadd_rn(t, __fmul_rn(0.5f, dt));
            o.dt_norm[s] = dt;
            if (o.img_id) o.img_id[s] = img;
            write_sample(o, s, x, y, z, r, dt, inv_aabb);
            ++taken;
            continue;
        }
        const int k = grid_level_at(a.g, x, y, z, dt);
        if (occupied_at(a.g, k, x, y, z)) {
            o.t[s] = t;
            o.m_norm[s] = __fadd_rn(t, __fmul_rn(0.5f, dt));
            o.dt_norm[s] = dt;
            if (o.img_id) o.img_id[s] = img;
            t = __fadd_rn(t, dt);
            t_max = t;
            write_sample(o, s, x, y, z, r, dt, inv_aabb);
            ++taken;
        } else {
            t = __fadd_rn(t, dt_to_next_voxel(a.g, x, y, z, r.dx, r.dy, r.dz, r.idx, r.idy, r.idz, a.dt_min, k));
        }
    }
    const float t_span = fmaxf(__fadd_rn(t_max, -t_min), 1e-6f);
    for (uint32_t j = 0; j < taken; ++j) {
        const uint32_t s = off + j;
        o.m_norm[s] = clamp_ref(__fdiv_rn(__fadd_rn(o.m_norm[s], -t_min), t_span), 0.0f, 1.0f);
        o.dt_norm[s] = __fdiv_rn(o.dt_norm[s], t_span);
    }
}

// Block-wide exclusive scan of one u32 per thread; returns the exclusive prefix and the block
// total in *total. BLOCK bounds the block size; blockDim.x is any multiple of 32 up to it.
template <int BLOCK = MARCH_BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_tot[BLOCK / WARP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t inc = warp_inclusive_sum(v, lane);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    uint32_t before = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < BLOCK / WARP; ++w) {
        if (w >= nw) break;
        const uint32_t x = warp_tot[w];
        if (w < wid) before += x;
        tot += x;
    }
    __syncthreads();
    *total = tot;
    return before + inc - v;
}

// Exclusive scan of the nb per-block totals in block_agg by the one block that runs it, ITEMS
// consecutive totals per thread and one block scan per blockDim.x * ITEMS totals (the totals are
// read with independent loads). visit(b, prefix) receives each block's 64-bit prefix, in order of
// b within a thread; the return value is the 64-bit sum. Within one pass the sums are 32-bit, as
// block_exclusive_scan's are.
template <int BLOCK, int ITEMS, typename Visit>
__device__ __forceinline__ unsigned long long scan_block_totals(uint32_t nb, const uint32_t* block_agg, Visit visit) {
    __shared__ unsigned long long carry_s;
    if (threadIdx.x == 0) carry_s = 0ull;
    __syncthreads();
    const uint32_t per_pass = blockDim.x * ITEMS;
    for (uint32_t base = 0; base < nb; base += per_pass) {
        const uint32_t b0 = base + threadIdx.x * ITEMS;
        uint32_t v[ITEMS];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) v[j] = b0 + j < nb ? *((volatile const uint32_t*)(block_agg + b0 + j)) : 0u;
        uint32_t sum = 0;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const uint32_t t = v[j];
            v[j] = sum;
            sum += t;
        }
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<BLOCK>(sum, &tot);
        const unsigned long long c = carry_s;
#pragma unroll
        for (int j = 0; j < ITEMS; ++j)
            if (b0 + j < nb) visit(b0 + j, c + ex + v[j]);
        __syncthreads();
        if (threadIdx.x == 0) carry_s = c + tot;
        __syncthreads();
    }
    return carry_s;
}

// Last-block epilogue of the count pass: exclusive scan of the block totals into
// block_prefix, then the reference batch cut (src/core/trainer.cu:133-183):
// L = last ray index whose offset < batch_size; n_rays = L; n_samples = offset[L].
// Run by one block of blockDim.x <= BLOCK threads; each entry of block_agg covers blockDim.x rays.
template <int BLOCK = MARCH_BLOCK>
__device__ void scan_blocks_and_cut(uint32_t nb, uint32_t n_live, const uint32_t* __restrict__ counts,
                                    uint32_t* block_agg, uint32_t* block_prefix, uint32_t batch_size,
                                    uint32_t* batch_info, uint32_t* flags) {
    __shared__ int last_block_s;
    __shared__ int last_ray_s;
    if (threadIdx.x == 0) { last_block_s = -1; last_ray_s = -1; }
    const uint32_t bs = blockDim.x;
    const uint32_t nb_live = (n_live + bs - 1) / bs;
    const unsigned long long carry = scan_block_totals<BLOCK, 4>(nb, block_agg, [&](uint32_t b, unsigned long long pre) {
        block_prefix[b] = pre > 0xffffffffull ? 0xffffffffu : (uint32_t)pre;
        if (pre > 0xffffffffull) raise_flag(flags, ERR_CAPACITY);
        if (b < nb_live && pre < batch_size) atomicMax(&last_block_s, (int)b);
    });
    const int lb = last_block_s;
    uint32_t n_rays_cut = 0, n_samples = 0;
    if (batch_size == 0xffffffffu) {
        // no cut (render / inference use): every live ray is kept
        if (threadIdx.x == 0) {
            const unsigned long long total = carry;
            batch_info[0] = n_live;
            batch_info[1] = total > 0xffffffffull ? 0xffffffffu : (uint32_t)total;
            batch_info[2] = batch_info[1];
            if (n_live == 0) raise_flag(flags, ERR_NO_RAYS);
            else if (total == 0) raise_flag(flags, ERR_NO_SAMPLES);
        }
        return;
    }
    if (lb >= 0) {
        const uint32_t i = (uint32_t)lb * bs + threadIdx.x;
        const uint32_t c = i < n_live ? *((volatile const uint32_t*)(counts + i)) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<BLOCK>(c, &tot);
        const uint32_t off = block_prefix[lb] + ex;
        if (i < n_live && off < batch_size) atomicMax(&last_ray_s, (int)i);
        __syncthreads();
        if ((int)i == last_ray_s) {
            n_rays_cut = i;
            n_samples = off;
            batch_info[0] = n_rays_cut;
            batch_info[1] = n_samples;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (last_ray_s < 0) { batch_info[0] = 0; batch_info[1] = 0; }
        const unsigned long long total = carry;
        batch_info[2] = total > 0xffffffffull ? 0xffffffffu : (uint32_t)total;
        const uint32_t nr = last_ray_s < 0 ? 0u : (uint32_t)last_ray_s;
        if (nr == 0) raise_flag(flags, ERR_NO_RAYS);
        else if (*((volatile uint32_t*)(batch_info + 1)) == 0) raise_flag(flags, ERR_NO_SAMPLES);
    }
}

// ---- batch scan of given counts (tn_scan_offsets, tn_scan_offsets_noalloc) ---------------
// Block totals of the counts; returns true in the last block to finish (ticket). BLOCK bounds
// the block size.
template <int BLOCK>
__device__ __forceinline__ bool block_total_and_ticket(uint32_t cnt, uint32_t* block_agg, uint32_t* ticket) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const uint32_t s = warp_sum(cnt);
    __shared__ uint32_t wsum[BLOCK / WARP];
    __shared__ bool is_last;
    if (lane == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < BLOCK / WARP; ++w)
            if (w < nw) tot += wsum[w];
        block_agg[blockIdx.x] = tot;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return is_last;
}

// Pass 1: per-block totals; the last block scans them and applies the batch cut. Every error
// bit of the call is raised by that last block; when flags_out is given, the block also stores
// the final error word there (a plain store, so the caller's word needs no clearing).
__global__ void __launch_bounds__(MARCH_BLOCK)
scan_count_kernel(uint32_t n, const uint32_t* __restrict__ counts, uint32_t batch_size, uint32_t* batch_info,
                  uint32_t* block_agg, uint32_t* block_prefix, uint32_t* ticket, uint32_t* flags,
                  uint32_t* flags_out) {
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    const uint32_t cnt = i < n ? counts[i] : 0u;
    if (!block_total_and_ticket<MARCH_BLOCK>(cnt, block_agg, ticket)) return;
    __threadfence();
    scan_blocks_and_cut<MARCH_BLOCK>(gridDim.x, n, counts, block_agg, block_prefix, batch_size, batch_info, flags);
    __syncthreads();
    if (threadIdx.x == 0) {
        *ticket = 0u;
        if (flags_out) *flags_out = atomicOr(flags, 0u);
    }
}

// Pass 2: offsets = block scan + the block's prefix.
__global__ void __launch_bounds__(MARCH_BLOCK)
scan_offsets_kernel(uint32_t n, const uint32_t* __restrict__ counts, const uint32_t* __restrict__ block_prefix,
                    uint32_t* __restrict__ offsets) {
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    const uint32_t cnt = i < n ? counts[i] : 0u;
    uint32_t tot;
    const uint32_t off = block_exclusive_scan(cnt, &tot) + block_prefix[blockIdx.x];
    if (i < n) offsets[i] = off;
}

// ---- fused march count ----------------------------------------------------------------
// Rays per count block: 64 keeps every SM busy at the 2^14-ray batches of training, where
// each warp is latency-bound on its own rays. block_agg / block_prefix hold one entry per group.
constexpr int COUNT_GROUP_MAX = 256;  // largest count block (tn_tuning::count_rays_per_block)
// The coarse mip (one byte per 4x4x4 block) is staged in shared memory for 16 <= R <= 128.
constexpr int MIP_MIN_RES = 16;
constexpr int MIP_MAX_RES = 128;
constexpr int BOX_INTS = 2 * MAX_LEVELS * 3;  // per level: lo block x,y,z | hi block + 1 x,y,z

__device__ __forceinline__ float pow2i(int e) { return __int_as_float((127 + e) << 23); }

// Level-0 constants of the count loop. Level k's half extent, cell size and reciprocal size are
// level 0's times 2^k (2^-k): scaling by a power of two is exact in IEEE arithmetic, and the
// host checks every level against the per-level table before launching.
struct CountGrid {
    float cell0, inv_ls0, res_f;
    int half0_bits, cell0_bits;  // bit patterns of the level-0 half extent and cell size
    uint32_t res_m1;             // R - 1
    int res_shift;               // log2 R
    uint32_t plane_words;        // R^3 / 32: words per level of the bit-planes
    int n_levels;
    const uint8_t* __restrict__ bits;     // the bitfield, one byte per cell (bit k = level k)
    const uint32_t* __restrict__ planes;  // the same bits as one plane per level, 32 cells per word
};

// get_grid_level_at (occupancy-grid.cuh:232-248): the finest level whose extent holds the point
// (max |coordinate| m < half extent) and whose cell is larger than dt, else the coarsest. Each
// condition turns true at some level and stays true above it, so the answer is the larger of
// the two first levels. For positive floats the order of the values is the order of their bit
// patterns, and level j's constant is level 0's pattern plus j << 23, so
//   m < half0 * 2^j  <=>  j > (bits(m) - bits(half0)) / 2^23,
//   cell0 * 2^j > dt  <=>  j > (bits(dt) - bits(cell0)) / 2^23,
// and the first such j is the quotient (an arithmetic shift) plus one, at least 0.
// NL = 0: the level count is only known at run time (nl_rt).
template <int NL>
__device__ __forceinline__ int count_level(float m, float dt, int half0_bits, int cell0_bits, int nl_rt) {
    const int jp = (__float_as_int(m) - half0_bits) >> 23;
    const int jd = (__float_as_int(dt) - cell0_bits) >> 23;
    return min(max(max(jp, jd) + 1, 0), (NL ? NL : nl_rt) - 1);
}

// a / b rounded toward +infinity for finite a >= b > 0 (the __fdiv_ru of get_dt_to_next_voxel,
// occupancy-grid.cuh:281), from inv_b = 1/b rounded to nearest. q0 = a * inv_b is within two
// ulps of a/b; one Newton correction with the residual a - q0*b (Markstein's division
// refinement) puts q within half an ulp plus a negligible term. RU(a/b) is the smallest float q
// with q*b >= a, so it is q, q's successor or q's predecessor; a fused multiply-add gives the
// residual a - q*b with the sign of the exact residual (no underflow for these operands), which
// decides between them. (An infinite a, which only a direction of three zero components can
// produce, yields NaN instead of infinity; either one ends the march loop the same way.)
__device__ __forceinline__ float div_ru_pos(float a, float b, float inv_b) {
    const float q0 = __fmul_rn(a, inv_b);
    float q = __fmaf_rn(__fmaf_rn(-q0, b, a), inv_b, q0);
    if (__fmaf_rn(-q, b, a) > 0.0f) {
        q = __uint_as_float(__float_as_uint(q) + 1u);
    } else {
        const float d = __uint_as_float(__float_as_uint(q) - 1u);
        if (__fmaf_rn(-d, b, a) <= 0.0f) q = d;
    }
    return q;
}

// One axis of get_dt_to_next_voxel (occupancy-grid.cuh:270-278) from the scaled coordinate
// f = (p / level size + 0.5) * R, which is also the cell coordinate before truncation.
__device__ __forceinline__ float axis_dt(float f, float h, float inv_d, float kcell) {
    return __fmul_rn(kcell, __fmul_rn(__fadd_rn(floorf(__fadd_rn(__fadd_rn(h, f), 0.5f)), -f), inv_d));
}

// Cell coordinate of get_voxel_morton_index, clamped to the grid: the conversion saturates
// (negative and NaN give 0), then the upper edge clamps to R - 1.
__device__ __forceinline__ uint32_t cell_of(float f, uint32_t res_m1) { return min(__float2uint_rz(f), res_m1); }

// The march loop of march_and_count_steps_per_ray_kernel (training-batch-kernels.cuh:258-297),
// branch-free per step so that the 32 rays of a warp never split: both successors of t (the
// occupied step t + dt and the DDA skip) are computed and one is selected. The scaled cell
// coordinates are computed once per step and shared by the Morton lookup and the skip (the
// reference computes the same expression in both, occupancy-grid.cuh:155-159 and :268-272).
//  * t_lim = min(the float below t_max, t_stop) merges `t < t_max` with the tail cut: past
//    t_stop the ray stays outside every occupied cell, so the loop ends with the same count.
//  * the box test (`if (!bbox.contains(p)) break`, training-batch-kernels.cuh:263-265) is made
//    once at the first step and folded into t_lim for the others (box_exit_t below).
//  * LIMIT: max_steps (otherwise unlimited) ends the ray after that many occupied steps.
//  * spread holds three Morton spread tables, pre-shifted for x, y and z.
//  * slots record the t of the first slot_cap occupied steps for the emit pass.
// Order-preserving map of the non-NaN floats to unsigned integers (a < b <=> key(a) < key(b)).
__device__ __forceinline__ uint32_t float_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// The last t >= t0 at which the march's point o + t d (computed fl(o + fl(t d)), as ray_point
// does) still lies on the inner side of the box face the ray leaves through along one axis.
// Both roundings are monotone, so the coordinate is monotone in t and the face test holds on a
// prefix of the floats from t0; the end of the prefix is found by bisection over the float
// order (at most 32 halvings). The caller has checked the test at t0. d == 0: never leaves.
__device__ float axis_exit_t(float o, float d, float lo, float hi, float t0) {
    if (d == 0.0f) return INFINITY;
    uint32_t a = float_key(t0), b = float_key(INFINITY);  // inside at a, outside at b (o + inf d = +-inf)
    while (b - a > 1u) {
        const uint32_t m = a + ((b - a) >> 1);
        const float x = __fadd_rn(o, __fmul_rn(key_float(m), d));
        if (d > 0.0f ? x <= hi : x >= lo) a = m;
        else b = m;
    }
    return key_float(a);
}

// The last t of the loop's steps (from t0 on) whose point the reference's box test accepts,
// given that it accepts the point at t0: along every axis the face test facing the ray's
// origin keeps holding once it holds (the coordinate moves away from that face), so the test
// fails first at the earliest exit over the three axes.
__device__ __forceinline__ float box_exit_t(const tn_bbox& b, const RayMarch& r, float t0) {
    return fminf(axis_exit_t(r.ox, r.dx, b.min_x, b.max_x, t0),
                 fminf(axis_exit_t(r.oy, r.dy, b.min_y, b.max_y, t0), axis_exit_t(r.oz, r.dz, b.min_z, b.max_z, t0)));
}

template <int NL, bool MIP, bool LIMIT>
__device__ uint32_t count_ray_loop(const MarchArgs& a, const CountGrid& cg, const RayMarch& r, float t_lim,
                                   uint32_t max_steps, uint32_t* flags, const uint8_t* __restrict__ mip,
                                   const uint32_t* __restrict__ spread, float* __restrict__ slots,
                                   uint32_t slot_cap) {
    const float hx = __fmul_rn(0.5f, copysignf(1.0f, r.dx));
    const float hy = __fmul_rn(0.5f, copysignf(1.0f, r.dy));
    const float hz = __fmul_rn(0.5f, copysignf(1.0f, r.dz));
    const int cs = cg.res_shift - 2;
    const uint32_t res = 1u << cg.res_shift;
    uint32_t n = 0, iters = 0;
    float t = r.t;
    // Level prediction: the cell lookup and the DDA skip of an iteration run at the level of the
    // previous iteration (kp), while the iteration's own level is found beside them; when the two
    // differ (a ray changes level a handful of times) the iteration is discarded without moving
    // and runs again at the new level. The level choice is then off the chain from t to the next
    // t, and every iteration that counts used the level the reference's loop uses.
    int kp;
    {
        float x, y, z;
        ray_point(r, t, x, y, z);
        const float m = fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z)));
        kp = count_level<NL>(m, get_dt(t, a.cone, a.dt_min, a.dt_max), cg.half0_bits, cg.cell0_bits, cg.n_levels);
    }
    float ils = __fmul_rn(cg.inv_ls0, pow2i(-kp)), kc = __fmul_rn(cg.cell0, pow2i(kp));
    // the iteration guard is part of the loop condition (no branch with a side effect in the
    // body, which stays one straight block); the flag is raised after the loop
    const uint32_t max_iters = a.max_iters;
    while ((t <= t_lim) & (iters < max_iters)) {
        float x, y, z;
        ray_point(r, t, x, y, z);
        const float dt = get_dt(t, a.cone, a.dt_min, a.dt_max);
        const float m = fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z)));
        const int k = count_level<NL>(m, dt, cg.half0_bits, cg.cell0_bits, cg.n_levels);
        const bool same_level = k == kp;
        const float fx = __fmul_rn(__fadd_rn(__fmul_rn(x, ils), 0.5f), cg.res_f);
        const float fy = __fmul_rn(__fadd_rn(__fmul_rn(y, ils), 0.5f), cg.res_f);
        const float fz = __fmul_rn(__fadd_rn(__fmul_rn(z, ils), 0.5f), cg.res_f);
        const uint32_t cx = cell_of(fx, cg.res_m1), cy = cell_of(fy, cg.res_m1), cz = cell_of(fz, cg.res_m1);
        const uint32_t idx = spread[cx] | spread[res + cy] | spread[2 * res + cz];
        bool occ;
        if (MIP) {
            const uint32_t coarse = mip[(((((cz >> 2) << cs) | (cy >> 2)) << cs) | (cx >> 2))];
            const uint32_t word = ((coarse >> kp) & 1u) ? __ldg(cg.planes + kp * cg.plane_words + (idx >> 5)) : 0u;
            occ = (word >> (idx & 31u)) & 1u;
        } else {
            occ = (__ldg(cg.bits + idx) >> kp) & 1u;
        }
        // DDA skip to the next cell boundary: t_target / dt_min rounded up (to a float), times dt_min
        const float tx = axis_dt(fx, hx, r.idx, kc);
        const float ty = axis_dt(fy, hy, r.idy, kc);
        const float tz = axis_dt(fz, hz, r.idz, kc);
        const float t_target = fmaxf(a.dt_min, fminf(fminf(tx, ty), tz));
        const float t_skip = __fadd_rn(t, __fmul_rn(div_ru_pos(t_target, a.dt_min, a.inv_dt_min), a.dt_min));
        // branch-free step: the slot store runs every iteration (a skip's t is overwritten by the
        // next occupied step, and the emit pass reads only the first n slots), so the select of
        // the successor carries no branch
        if (n < slot_cap) slots[n] = t;
        const float t_occ = __fadd_rn(t, dt);
        const float t_next = occ ? t_occ : t_skip;
        t = same_level ? t_next : t;
        n += (same_level & occ) ? 1u : 0u;
        iters += same_level ? 1u : 0u;
        kp = k;
        ils = __fmul_rn(cg.inv_ls0, pow2i(-k));
        kc = __fmul_rn(cg.cell0, pow2i(k));
        if (LIMIT && n >= max_steps) break;
    }
    if (iters >= max_iters && t <= t_lim && !(LIMIT && n >= max_steps)) raise_flag(flags, ERR_GUARD);
    return n;
}

template <int NL, bool MIP>
__device__ uint32_t count_ray(const MarchArgs& a, const CountGrid& cg, const RayMarch& r, float t_lim,
                              uint32_t max_steps, uint32_t* flags, const uint8_t* __restrict__ mip,
                              const uint32_t* __restrict__ spread, float* __restrict__ slots, uint32_t slot_cap) {
    if (!(r.t <= t_lim)) return 0;  // no step (a NaN limit included)
    float x, y, z;
    ray_point(r, r.t, x, y, z);
    if (!bbox_contains(a.bbox, x, y, z)) return 0;  // the first step leaves the box
    t_lim = fminf(t_lim, box_exit_t(a.bbox, r, r.t));
    return max_steps == 0xffffffffu
               ? count_ray_loop<NL, MIP, false>(a, cg, r, t_lim, max_steps, flags, mip, spread, slots, slot_cap)
               : count_ray_loop<NL, MIP, true>(a, cg, r, t_lim, max_steps, flags, mip, spread, slots, slot_cap);
}

// World-space box that holds every occupied cell of every level: per level, the box of its
// occupied 4x4x4 blocks padded by one cell of that level; points beyond the grid clamp to the
// coarsest level's edge cells, so an occupied edge block of that level opens its side to
// infinity. cut = 2 when no cell is occupied.
__device__ void occupied_union(const CountGrid& cg, const int* __restrict__ box, int n_levels, float* u, int* cut) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const int C = 1 << (cg.res_shift - 2);
    bool any = false;
    for (int k = 0; k < n_levels; ++k) {
        if (box[MAX_LEVELS * 3 + k * 3] == 0) continue;  // no occupied block at this level
        any = true;
        const float ls = __int_as_float(cg.half0_bits) * pow2i(k + 1), cw = cg.cell0 * pow2i(k);
        for (int ax = 0; ax < 3; ++ax) {
            const int l = box[k * 3 + ax], h = box[MAX_LEVELS * 3 + k * 3 + ax];
            float wl = (4.0f * (float)l / cg.res_f - 0.5f) * ls - cw;
            float wh = (4.0f * (float)h / cg.res_f - 0.5f) * ls + cw;
            if (k == n_levels - 1) {
                if (l == 0) wl = -INFINITY;
                if (h == C) wh = INFINITY;
            }
            lo[ax] = fminf(lo[ax], wl);
            hi[ax] = fmaxf(hi[ax], wh);
        }
    }
    for (int ax = 0; ax < 3; ++ax) { u[ax] = lo[ax]; u[3 + ax] = hi[ax]; }
    *cut = any ? 1 : 2;
}

// Slab test of the ray against the union box. Returns false when the ray misses it (so it
// meets no occupied cell); otherwise *t_exit is where it leaves the box for good (infinity when
// the test is degenerate). Rounding of o + t d grows with the coordinates: beyond `limit`
// (65536 finest cells) it could exceed the one-cell padding, so such rays keep t_exit = infinity.
__device__ __forceinline__ bool ray_box_exit(const RayMarch& r, const float* u, float t_max, float limit,
                                             float* t_exit) {
    *t_exit = INFINITY;
    const float reach = fmaxf(fabsf(r.ox), fmaxf(fabsf(r.oy), fabsf(r.oz))) +
                        fabsf(t_max) * fmaxf(fabsf(r.dx), fmaxf(fabsf(r.dy), fabsf(r.dz)));
    if (!(reach <= limit)) return true;
    const float o[3] = {r.ox, r.oy, r.oz}, d[3] = {r.dx, r.dy, r.dz}, inv[3] = {r.idx, r.idy, r.idz};
    float te = -INFINITY, tx = INFINITY;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        if (d[ax] == 0.0f) {
            if (!(o[ax] >= u[ax] && o[ax] <= u[3 + ax])) return false;
            continue;
        }
        const float t1 = __fmul_rn(__fadd_rn(u[ax], -o[ax]), inv[ax]);
        const float t2 = __fmul_rn(__fadd_rn(u[3 + ax], -o[ax]), inv[ax]);
        if (t1 != t1 || t2 != t2) return true;
        te = fmaxf(te, fminf(t1, t2));
        tx = fminf(tx, fmaxf(t1, t2));
    }
    if (te > tx) return false;
    *t_exit = tx;
    return true;
}

// One thread per ray, blockDim.x rays per block (a tuning choice, 32..256). Shared memory: the three Morton spread tables
// (3 R words) and, with MIP, the coarse mip (R^3/64 bytes); with MIP the fine test reads the
// per-level bit-planes. The last block to finish scans the group totals and applies the batch
// cut on the device.
template <int NL, bool MIP>
__global__ void __launch_bounds__(COUNT_GROUP_MAX)
march_count_kernel(MarchArgs a, CountGrid cg, uint32_t n_rays, const uint32_t* __restrict__ n_rays_dev, uint32_t rs,
                   const float* __restrict__ ori, const float* __restrict__ dir, const float* __restrict__ ray_t,
                   const float* __restrict__ ray_t_max, uint8_t* __restrict__ alive, uint32_t* counts,
                   uint32_t batch_size, uint32_t* batch_info, uint32_t* block_agg, uint32_t* block_prefix,
                   uint32_t* ticket, uint32_t* flags, const uint8_t* __restrict__ mip_g,
                   const int* __restrict__ box_g, float* __restrict__ slots, uint32_t slot_cap) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* spread = reinterpret_cast<uint32_t*>(smem);
    uint8_t* mip = smem + ((size_t)12 << cg.res_shift);
    __shared__ float ubox_s[6];
    __shared__ int cut_s;
    const uint32_t res = 1u << cg.res_shift;
    for (uint32_t c = threadIdx.x; c < res; c += blockDim.x) {
        const uint32_t v = part1by2(c);
        spread[c] = v;
        spread[res + c] = v << 1;
        spread[2 * res + c] = v << 2;
    }
    if (MIP) {
        const uint32_t n16 = (1u << (3 * (cg.res_shift - 2))) / 16;
        const uint4* src = reinterpret_cast<const uint4*>(mip_g);
        uint4* dst = reinterpret_cast<uint4*>(mip);
#pragma unroll 8
        for (uint32_t k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = __ldg(src + k);
        if (threadIdx.x == 0) occupied_union(cg, box_g, a.g.n_levels, ubox_s, &cut_s);
    }
    __syncthreads();
    const uint32_t n_live = n_rays_dev ? min(*n_rays_dev, n_rays) : n_rays;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t cnt = 0;
    if (i < n_live) {
        if (alive[i]) {
            RayMarch r;
            load_ray(r, ori, dir, i, rs);
            r.t = ray_t[i];
            const float t_max = ray_t_max[i];
            float t_stop = INFINITY;
            bool meets = true;
            if (MIP) {
                if (cut_s == 2) meets = false;
                else meets = ray_box_exit(r, ubox_s, t_max, __fmul_rn(cg.cell0, 65536.0f), &t_stop);
            }
            // t < t_max  <=>  t <= the float just below t_max
            const float below = nextafterf(t_max, -INFINITY);
            const float t_lim = t_stop < below ? t_stop : below;  // a NaN t_max stays NaN
            if (meets)
                cnt = count_ray<NL, MIP>(a, cg, r, t_lim, a.max_steps ? a.max_steps : 0xffffffffu, flags, mip,
                                         spread, slots ? slots + (size_t)i * slot_cap : nullptr,
                                         slots ? slot_cap : 0u);
            if (cnt == 0) alive[i] = 0;
        }
        counts[i] = cnt;
    }
    // make this thread's count visible device-wide before the block reports completion
    __threadfence();
    if (!block_total_and_ticket<COUNT_GROUP_MAX>(cnt, block_agg, ticket)) return;
    __threadfence();
    scan_blocks_and_cut<COUNT_GROUP_MAX>(gridDim.x, n_live, counts, block_agg, block_prefix, batch_size, batch_info,
                                     flags);
    if (threadIdx.x == 0) *ticket = 0u;
}

// Emit pass from the recorded step positions, one warp per ray, so that the rays inside the
// batch (the first ones) spread over every SM. The warp rebuilds its ray's offset from the
// group prefix of the count pass plus the counts of the group's earlier rays, writes it, and
// expands the samples with one lane per sample (coalesced stores of the packed sample arrays).
// Every value is the one the reference's emit loop (training-batch-kernels.cuh:412-480)
// computes from the same t: dt = get_dt(t), the position o + t d, m = t + dt/2, the ray's span
// from its start t to the end of its last step. Rays with more samples than slots fall back to
// replaying their march.
// Writes the n samples of ray r_i at o0.. from its recorded step positions (one lane per sample),
// or, for a ray with more samples than slots, by replaying its march on lane 0.
__device__ __forceinline__ void expand_ray(const MarchArgs& a, float inv_aabb, uint32_t r_i, uint32_t o0, uint32_t n,
                                           uint32_t rs, const uint32_t* __restrict__ img_id,
                                           const float* __restrict__ ori, const float* __restrict__ dir,
                                           const float* __restrict__ ray_t, const SampleOut& o,
                                           const float* __restrict__ slots, uint32_t slot_cap, int lane,
                                           int lanes) {
    RayMarch r;
    load_ray(r, ori, dir, r_i, rs);
    r.t = ray_t[r_i];
    const uint32_t img = img_id ? img_id[r_i] : 0u;
    if (n > slot_cap) {
        if (lane == 0) march_emit_ray(a, r, n, o0, img, inv_aabb, o);
        return;
    }
    const float* sl = slots + (size_t)r_i * slot_cap;
    const float t_last = sl[n - 1];
    const float t_end = __fadd_rn(t_last, get_dt(t_last, a.cone, a.dt_min, a.dt_max));
    const float t_span = fmaxf(__fadd_rn(t_end, -r.t), 1e-6f);
    for (uint32_t j = lane; j < n; j += lanes) {
        const float t = sl[j];
        const float dt = get_dt(t, a.cone, a.dt_min, a.dt_max);
        float x, y, z;
        ray_point(r, t, x, y, z);
        const uint32_t s = o0 + j;
        o.t[s] = t;
        const float m = __fadd_rn(t, __fmul_rn(0.5f, dt));
        o.m_norm[s] = clamp_ref(__fdiv_rn(__fadd_rn(m, -r.t), t_span), 0.0f, 1.0f);
        o.dt_norm[s] = __fdiv_rn(dt, t_span);
        if (o.img_id) o.img_id[s] = img;
        write_sample(o, s, x, y, z, r, dt, inv_aabb);
    }
}

constexpr int EXPAND_THREADS_MAX = 512;  // 16 warps (tn_tuning::emit_warps_per_block)

// Sum over the aligned group of L lanes (all 32 lanes take part).
template <int L>
__device__ __forceinline__ uint32_t group_sum(uint32_t v) {
#pragma unroll
    for (int d = L / 2; d > 0; d >>= 1) v += __shfl_xor_sync(FULL_MASK, v, d);
    return v;
}

// RPW rays per warp (32 / RPW lanes per ray), blockDim.x / 32 warps per block; the count pass
// grouped its rays by 2^group_shift (the block size it ran with).
template <int RPW>
__global__ void __launch_bounds__(EXPAND_THREADS_MAX)
expand_kernel(MarchArgs a, float inv_aabb, uint32_t n_rays, const uint32_t* __restrict__ n_rays_dev, uint32_t rs,
              uint32_t group_shift, const uint32_t* __restrict__ batch_info,
              const uint32_t* __restrict__ block_prefix, const uint32_t* __restrict__ img_id,
              const float* __restrict__ ori, const float* __restrict__ dir, const float* __restrict__ ray_t,
              const uint8_t* __restrict__ alive, const uint32_t* __restrict__ counts,
              uint32_t* __restrict__ offsets, SampleOut o, uint32_t* flags, const float* __restrict__ slots,
              uint32_t slot_cap) {
    constexpr int L = WARP / RPW;
    const uint32_t n_live = n_rays_dev ? min(*n_rays_dev, n_rays) : n_rays;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1);
    const uint32_t r_i = ((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * RPW) + (uint32_t)(lane / L);
    const bool valid = r_i < n_live;
    const uint32_t g0 = (r_i >> group_shift) << group_shift;
    uint32_t part = 0;
    if (valid)
        for (uint32_t j = g0 + sub; j < r_i; j += L) part += counts[j];
    part = group_sum<L>(part);  // every lane of the warp takes part before any leaves
    if (!valid) return;
    const uint32_t o0 = part + block_prefix[r_i >> group_shift];
    const uint32_t n = counts[r_i];
    if (sub == 0) offsets[r_i] = o0;
    if (r_i >= batch_info[0] || n == 0 || !alive[r_i]) return;
    if ((unsigned long long)o0 + n > (unsigned long long)o.ss) {
        if (sub == 0) raise_flag(flags, ERR_CAPACITY);
        return;
    }
    expand_ray(a, inv_aabb, r_i, o0, n, rs, img_id, ori, dir, ray_t, o, slots, slot_cap, sub, L);
}

// Bits k of the four bytes of x (cells 4j .. 4j+3) as four consecutive bits: the mask leaves
// them at bit positions 0, 8, 16, 24, and the multiply by 1 + 2^7 + 2^14 + 2^21 moves them to
// 21..24 without any two partial products meeting.
__device__ __forceinline__ uint32_t gather_level_bits(uint32_t x, int k) {
    return ((((x >> k) & 0x01010101u) * 0x00204081u) >> 21) & 0xFu;
}

// Coarse occupancy mip, x-fastest: byte (cz*C + cy)*C + cx (C = R/4) is the OR of the 64 fine
// bytes of that 4x4x4 block, Morton indices [64m, 64m + 64) with m = morton(cx, cy, cz). Also
//  * writes the per-level bit-planes: bit j of word w of plane k is bit k of cell 32w + j
//    (words 2m and 2m + 1 of every plane come from this block);
//  * reduces, per level, the box of occupied blocks into box[lo x,y,z per level | hi+1 x,y,z
//    per level] (lo starts at a large value, hi at 0), the input of the count pass's tail cut.
__device__ __forceinline__ void build_mip_block(int cshift, int n_levels, const uint4* __restrict__ bits,
                                                uint8_t* __restrict__ mip, int* box, uint32_t* __restrict__ planes,
                                                uint32_t plane_words, uint32_t block) {
    __shared__ int sbox[BOX_INTS];
    if (threadIdx.x < BOX_INTS) sbox[threadIdx.x] = threadIdx.x < BOX_INTS / 2 ? 0x7fffffff : 0;
    __syncthreads();
    const uint32_t C = 1u << cshift;
    const uint32_t c = block * 256 + threadIdx.x;
    uint32_t v = 0, cx = 0, cy = 0, cz = 0;
    if (c < C * C * C) {
        cx = c & (C - 1);
        cy = (c >> cshift) & (C - 1);
        cz = c >> (2 * cshift);
        const uint32_t m = morton3d(cx, cy, cz);
        const uint4* p = bits + (size_t)m * 4;
        uint32_t w[16];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 u = __ldg(p + q);
            w[4 * q] = u.x; w[4 * q + 1] = u.y; w[4 * q + 2] = u.z; w[4 * q + 3] = u.w;
            v |= u.x | u.y | u.z | u.w;
        }
        v = (v | (v >> 8) | (v >> 16) | (v >> 24)) & 0xFFu;
        mip[c] = (uint8_t)v;
        for (int k = 0; k < n_levels; ++k) {
            uint32_t lo = 0, hi = 0;
            if ((v >> k) & 1u) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    lo |= gather_level_bits(w[j], k) << (4 * j);
                    hi |= gather_level_bits(w[8 + j], k) << (4 * j);
                }
            }
            *reinterpret_cast<uint2*>(planes + (size_t)k * plane_words + 2 * (size_t)m) = make_uint2(lo, hi);
        }
    }
    for (int k = 0; k < n_levels; ++k) {
        const bool on = (v >> k) & 1u;
        if (!__any_sync(FULL_MASK, on)) continue;
        const int lx = __reduce_min_sync(FULL_MASK, on ? (int)cx : 0x7fffffff);
        const int ly = __reduce_min_sync(FULL_MASK, on ? (int)cy : 0x7fffffff);
        const int lz = __reduce_min_sync(FULL_MASK, on ? (int)cz : 0x7fffffff);
        const int hx = __reduce_max_sync(FULL_MASK, on ? (int)cx + 1 : 0);
        const int hy = __reduce_max_sync(FULL_MASK, on ? (int)cy + 1 : 0);
        const int hz = __reduce_max_sync(FULL_MASK, on ? (int)cz + 1 : 0);
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&sbox[k * 3 + 0], lx);
            atomicMin(&sbox[k * 3 + 1], ly);
            atomicMin(&sbox[k * 3 + 2], lz);
            atomicMax(&sbox[BOX_INTS / 2 + k * 3 + 0], hx);
            atomicMax(&sbox[BOX_INTS / 2 + k * 3 + 1], hy);
            atomicMax(&sbox[BOX_INTS / 2 + k * 3 + 2], hz);
        }
    }
    __syncthreads();
    if (threadIdx.x < BOX_INTS) {
        const int val = sbox[threadIdx.x];
        if (threadIdx.x < BOX_INTS / 2) {
            if (val != 0x7fffffff) atomicMin(box + threadIdx.x, val);
        } else if (val != 0) {
            atomicMax(box + threadIdx.x, val);
        }
    }
}

__global__ void __launch_bounds__(256)
build_mip_kernel(int cshift, int n_levels, const uint4* __restrict__ bits, uint8_t* __restrict__ mip, int* box,
                 uint32_t* __restrict__ planes, uint32_t plane_words) {
    build_mip_block(cshift, n_levels, bits, mip, box, planes, plane_words, blockIdx.x);
}

// ---- several scenes in one launch ---------------------------------------------------------
// The scenes' rays sit in one set of ray arrays, scene after scene, and their samples are
// packed the same way. Each scene keeps its own grid, bitfield, box and march parameters. The
// count pass is one persistent launch: blocks take chunks of rays (tn_tuning::multi_chunk_rays,
// one thread a ray) of any scene from a shared counter (work stealing) and stage a scene's
// coarse mip when they move to another scene. The block that finishes the last chunk scans all
// chunk totals. The emit pass is one launch over all scenes' rays with the single-scene emit's
// shape. The per-scene results equal those of a tn_march_count / tn_march_emit call per scene
// without a batch cut.
constexpr int MAX_SCENES = 32;

struct SceneParams {
    MarchArgs a;
    CountGrid cg;
    float inv_aabb;
    uint32_t ray_begin, n_rays, chunk_begin;
    int use_mip, cshift;
    uint32_t mip_blocks;  // build_mip blocks of 256 coarse blocks
    uint8_t* mip;
    int* box;
};

struct MultiArgs {
    uint32_t n_scenes, total_chunks, total_rays, spread_res;
    uint32_t chunk_shift;  // rays per work-stealing chunk = 2^chunk_shift = the count block size
    SceneParams sp[MAX_SCENES];
};

__device__ __forceinline__ int scene_of_chunk(const MultiArgs& A, uint32_t chunk) {
    int s = 0;
    for (int k = 1; k < (int)A.n_scenes; ++k)
        if (chunk >= A.sp[k].chunk_begin) s = k;
    return s;
}

__device__ __forceinline__ int scene_of_ray(const MultiArgs& A, uint32_t ray) {
    int s = 0;
    for (int k = 1; k < (int)A.n_scenes; ++k)
        if (ray >= A.sp[k].ray_begin) s = k;
    return s;
}

// Per scene: the occupied-box reduction starts from lo = large, hi = 0.
__global__ void multi_box_init_kernel(const __grid_constant__ MultiArgs A) {
    const uint32_t s = blockIdx.x, i = threadIdx.x;
    if (s < A.n_scenes && A.sp[s].use_mip && i < (uint32_t)BOX_INTS)
        A.sp[s].box[i] = i < (uint32_t)BOX_INTS / 2 ? 0x7fffffff : 0;
}

__global__ void __launch_bounds__(256) multi_build_mip_kernel(const __grid_constant__ MultiArgs A) {
    const SceneParams& sp = A.sp[blockIdx.y];
    if (!sp.use_mip || blockIdx.x >= sp.mip_blocks) return;  // whole blocks leave together
    build_mip_block(sp.cshift, sp.a.g.n_levels, reinterpret_cast<const uint4*>(sp.a.g.bits), sp.mip, sp.box,
                    const_cast<uint32_t*>(sp.cg.planes), sp.cg.plane_words, blockIdx.x);
}

__global__ void __launch_bounds__(COUNT_GROUP_MAX)
multi_count_kernel(const __grid_constant__ MultiArgs A, uint32_t rs, const float* __restrict__ ori,
                   const float* __restrict__ dir, const float* __restrict__ ray_t, const float* __restrict__ ray_t_max,
                   uint8_t* __restrict__ alive, uint32_t* counts, uint32_t* block_agg, uint32_t* block_prefix,
                   uint32_t* work, uint32_t* ticket, uint32_t* flags, float* __restrict__ slots, uint32_t slot_cap,
                   uint32_t* __restrict__ scene_samples, uint32_t* batch_info) {
    extern __shared__ __align__(16) uint8_t smem[];
    uint32_t* spread = reinterpret_cast<uint32_t*>(smem);
    uint8_t* mip = smem + (size_t)12 * A.spread_res;
    __shared__ float ubox_s[6];
    __shared__ int cut_s;
    __shared__ uint32_t chunk_s;
    __shared__ uint32_t wsum[COUNT_GROUP_MAX / WARP];
    __shared__ bool last_s;
    const uint32_t res = A.spread_res;
    for (uint32_t c = threadIdx.x; c < res; c += blockDim.x) {
        const uint32_t v = part1by2(c);
        spread[c] = v;
        spread[res + c] = v << 1;
        spread[2 * res + c] = v << 2;
    }
    int staged = -1;
    for (;;) {
        if (threadIdx.x == 0) chunk_s = atomicAdd(work, 1u);
        __syncthreads();
        const uint32_t chunk = chunk_s;
        if (chunk >= A.total_chunks) break;
        const int s = scene_of_chunk(A, chunk);
        const SceneParams& sp = A.sp[s];
        if (s != staged) {
            if (sp.use_mip) {
                const uint32_t n16 = (1u << (3 * sp.cshift)) / 16;
                const uint4* src = reinterpret_cast<const uint4*>(sp.mip);
                uint4* dst = reinterpret_cast<uint4*>(mip);
#pragma unroll 8
                for (uint32_t k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = __ldg(src + k);
                if (threadIdx.x == 0) occupied_union(sp.cg, sp.box, sp.a.g.n_levels, ubox_s, &cut_s);
            }
            staged = s;
            __syncthreads();
        }
        const uint32_t local = ((chunk - sp.chunk_begin) << A.chunk_shift) + threadIdx.x;
        const uint32_t i = sp.ray_begin + local;
        uint32_t cnt = 0;
        if (local < sp.n_rays) {
            if (alive[i]) {
                RayMarch r;
                load_ray(r, ori, dir, i, rs);
                r.t = ray_t[i];
                const float t_max = ray_t_max[i];
                float t_stop = INFINITY;
                bool meets = true;
                if (sp.use_mip) {
                    if (cut_s == 2) meets = false;
                    else meets = ray_box_exit(r, ubox_s, t_max, __fmul_rn(sp.cg.cell0, 65536.0f), &t_stop);
                }
                const float below = nextafterf(t_max, -INFINITY);
                const float t_lim = t_stop < below ? t_stop : below;
                const uint32_t ms = sp.a.max_steps ? sp.a.max_steps : 0xffffffffu;
                float* sl = slots ? slots + (size_t)i * slot_cap : nullptr;
                const uint32_t sc = slots ? slot_cap : 0u;
                if (meets) {
                    if (sp.use_mip)
                        cnt = count_ray<0, true>(sp.a, sp.cg, r, t_lim, ms, flags, mip, spread, sl, sc);
                    else
                        cnt = count_ray<0, false>(sp.a, sp.cg, r, t_lim, ms, flags, mip, spread, sl, sc);
                }
                if (cnt == 0) alive[i] = 0;
            }
            counts[i] = cnt;
        }
        __threadfence();
        const uint32_t ws = warp_sum(cnt);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = ws;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tot = 0;
            const int nw = blockDim.x >> 5;
#pragma unroll
            for (int w = 0; w < COUNT_GROUP_MAX / WARP; ++w)
                if (w < nw) tot += wsum[w];
            block_agg[chunk] = tot;
            __threadfence();
            last_s = atomicAdd(ticket, 1u) == A.total_chunks - 1;
        }
        __syncthreads();
        if (last_s) {
            __threadfence();
            scan_blocks_and_cut<COUNT_GROUP_MAX>(A.total_chunks, A.total_rays, counts, block_agg, block_prefix,
                                             0xffffffffu, batch_info, flags);
            __syncthreads();
            if (scene_samples && threadIdx.x < A.n_scenes) {
                // a scene's samples start at its first chunk's prefix; scenes without rays at the
                // end of the table start at the batch total
                const uint32_t s0 = threadIdx.x;
                const uint32_t cb = A.sp[s0].chunk_begin;
                const uint32_t ce = s0 + 1 < A.n_scenes ? A.sp[s0 + 1].chunk_begin : A.total_chunks;
                const uint32_t b = cb < A.total_chunks ? block_prefix[cb] : batch_info[2];
                const uint32_t e = ce < A.total_chunks ? block_prefix[ce] : batch_info[2];
                scene_samples[s0] = e - b;
            }
        }
    }
}

template <int RPW>
__global__ void __launch_bounds__(EXPAND_THREADS_MAX)
multi_expand_kernel(const __grid_constant__ MultiArgs A, uint32_t rs, const uint32_t* __restrict__ block_prefix,
                    const uint32_t* __restrict__ img_id, const float* __restrict__ ori, const float* __restrict__ dir,
                    const float* __restrict__ ray_t, const uint8_t* __restrict__ alive,
                    const uint32_t* __restrict__ counts, uint32_t* __restrict__ offsets, SampleOut o, uint32_t* flags,
                    const float* __restrict__ slots, uint32_t slot_cap) {
    constexpr int L = WARP / RPW;
    const int lane = threadIdx.x & 31, sub = lane & (L - 1);
    const uint32_t r_i = ((blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * RPW) + (uint32_t)(lane / L);
    const uint32_t last = A.sp[A.n_scenes - 1].ray_begin + A.sp[A.n_scenes - 1].n_rays;
    const SceneParams& sp = A.sp[scene_of_ray(A, r_i < last ? r_i : 0u)];
    // rays past the end and rays in a gap between scenes do nothing
    const bool valid = r_i < last && r_i - sp.ray_begin < sp.n_rays;
    const uint32_t local = r_i - sp.ray_begin;
    const uint32_t chunk = sp.chunk_begin + (local >> A.chunk_shift);
    const uint32_t g0 = sp.ray_begin + ((local >> A.chunk_shift) << A.chunk_shift);
    uint32_t part = 0;
    if (valid)
        for (uint32_t j = g0 + sub; j < r_i; j += L) part += counts[j];
    part = group_sum<L>(part);  // every lane of the warp takes part before any leaves
    if (!valid) return;
    const uint32_t o0 = part + block_prefix[chunk];
    const uint32_t n = counts[r_i];
    if (sub == 0) offsets[r_i] = o0;
    if (n == 0 || !alive[r_i]) return;
    if ((unsigned long long)o0 + n > (unsigned long long)o.ss) {
        if (sub == 0) raise_flag(flags, ERR_CAPACITY);
        return;
    }
    expand_ray(sp.a, sp.inv_aabb, r_i, o0, n, rs, img_id, ori, dir, ray_t, o, slots, slot_cap, sub, L);
}

// ---- compaction: ascending indices of non-zero values ---------------------------------
// A tile of BLOCK x ITEMS values per block; each thread owns ITEMS consecutive values, so the
// per-thread counts scanned in thread order give ascending output positions.
template <int BLOCK, int ITEMS>
__device__ __forceinline__ uint32_t tile_flags(uint32_t n, const uint32_t* __restrict__ values, uint32_t first,
                                               uint32_t& bits) {
    bits = 0u;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t i = first + (uint32_t)j;
        if (i < n && __ldg(values + i) != 0u) bits |= 1u << j;
    }
    return (uint32_t)__popc(bits);
}

template <int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
compact_count_kernel(uint32_t n, const uint32_t* __restrict__ values, uint32_t* block_agg, uint32_t* block_prefix,
                     uint32_t* count_dev, uint32_t* ticket) {
    const uint32_t first = (blockIdx.x * BLOCK + threadIdx.x) * ITEMS;
    uint32_t bits;
    const uint32_t f = tile_flags<BLOCK, ITEMS>(n, values, first, bits);
    uint32_t s;
    block_exclusive_scan<BLOCK>(f, &s);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        block_agg[blockIdx.x] = s;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const unsigned long long total = scan_block_totals<BLOCK, 4>(
        gridDim.x, block_agg, [&](uint32_t b, unsigned long long pre) { block_prefix[b] = (uint32_t)pre; });
    if (threadIdx.x == 0) {
        *count_dev = (uint32_t)total;
        *ticket = 0u;
    }
}

template <int BLOCK, int ITEMS>
__global__ void __launch_bounds__(BLOCK)
compact_write_kernel(uint32_t n, const uint32_t* __restrict__ values, const uint32_t* __restrict__ block_prefix,
                     int32_t* __restrict__ out) {
    const uint32_t first = (blockIdx.x * BLOCK + threadIdx.x) * ITEMS;
    uint32_t bits;
    const uint32_t f = tile_flags<BLOCK, ITEMS>(n, values, first, bits);
    uint32_t tot;
    uint32_t pos = block_exclusive_scan<BLOCK>(f, &tot) + block_prefix[blockIdx.x];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j)
        if ((bits >> j) & 1u) out[pos++] = (int32_t)(first + (uint32_t)j);
}

// ---- plain path kernels (one thread per ray, reference launch structure) -------------
__global__ void plain_count_kernel(MarchArgs a, uint32_t n_rays, uint32_t rs, const float* __restrict__ ori,
                                   const float* __restrict__ dir, const float* __restrict__ ray_t,
                                   const float* __restrict__ ray_t_max, uint8_t* __restrict__ alive,
                                   uint32_t* __restrict__ n_steps) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays) return;
    if (!alive[i]) { n_steps[i] = 0; return; }
    RayMarch r;
    load_ray(r, ori, dir, i, rs);
    r.t = ray_t[i];
    const uint32_t n = march_count_ray(a, r, ray_t_max[i], nullptr);
    if (n == 0) alive[i] = 0;
    n_steps[i] = n;
}

__global__ void plain_emit_kernel(MarchArgs a, float inv_aabb, uint32_t n_rays, uint32_t rs,
                                  const uint32_t* __restrict__ img_id, const float* __restrict__ ori,
                                  const float* __restrict__ dir, const float* __restrict__ ray_t,
                                  const uint32_t* __restrict__ offsets, const uint8_t* __restrict__ alive,
                                  const uint32_t* __restrict__ n_steps, SampleOut o) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays || !alive[i]) return;
    RayMarch r;
    load_ray(r, ori, dir, i, rs);
    r.t = ray_t[i];
    march_emit_ray(a, r, n_steps[i], offsets[i], img_id ? img_id[i] : 0u, inv_aabb, o);
}

// Bounding-box clip of initialize_training_rays_and_pixels_kernel,
// src/utils/training-batch-kernels.cuh:122-150 and bounding-box.cuh:27-51.
__global__ void rays_init_kernel(uint32_t n, uint32_t rs, tn_bbox b, float t_far, const float* __restrict__ ori,
                                 const float* __restrict__ dir, float* __restrict__ ray_t,
                                 float* __restrict__ ray_t_max, uint8_t* __restrict__ alive) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ox = ori[i], oy = ori[i + rs], oz = ori[i + 2 * (size_t)rs];
    const float dx = dir[i], dy = dir[i + rs], dz = dir[i + 2 * (size_t)rs];
    const float ix = __fdiv_rn(1.0f, dx), iy = __fdiv_rn(1.0f, dy), iz = __fdiv_rn(1.0f, dz);
    float t1x = __fmul_rn(__fadd_rn(b.min_x, -ox), ix), t2x = __fmul_rn(__fadd_rn(b.max_x, -ox), ix);
    float t1y = __fmul_rn(__fadd_rn(b.min_y, -oy), iy), t2y = __fmul_rn(__fadd_rn(b.max_y, -oy), iy);
    float t1z = __fmul_rn(__fadd_rn(b.min_z, -oz), iz), t2z = __fmul_rn(__fadd_rn(b.max_z, -oz), iz);
    if (t1x > t2x) { const float s = t1x; t1x = t2x; t2x = s; }
    if (t1y > t2y) { const float s = t1y; t1y = t2y; t2y = s; }
    if (t1z > t2z) { const float s = t1z; t1z = t2z; t2z = s; }
    const float tmin = fmaxf(t1x, fmaxf(t1y, t1z));
    const float tmax = fminf(t2x, fminf(t2y, t2z));
    if (!(tmax >= tmin)) { alive[i] = 0; ray_t[i] = 0.0f; ray_t_max[i] = 0.0f; return; }
    const float tm = fminf(t_far, tmax);
    const float t = fmaxf(0.0f, __fadd_rn(tmin, 1e-5f));
    if (tm < t) { alive[i] = 0; ray_t[i] = 0.0f; ray_t_max[i] = 0.0f; return; }
    ray_t[i] = t;
    ray_t_max[i] = tm;
    alive[i] = 1;
}

// Budget of the per-ray step-position slots (floats).
constexpr size_t SLOT_BUDGET = 16u << 20;

static uint32_t slot_capacity(uint32_t n_rays, uint32_t max_steps) {
    size_t cap = SLOT_BUDGET / (n_rays ? n_rays : 1);
    if (cap > 1024) cap = 1024;
    if (max_steps && cap > max_steps) cap = max_steps;
    if (cap < 16) cap = 16;
    return (uint32_t)cap;
}

static int make_march_args(const tn_grid_desc* grid, const uint8_t* bitfield, const tn_bbox* bbox,
                           const tn_march_desc* march, MarchArgs& a) {
    int st = validate_grid(grid);
    if (st != TN_OK) return st;
    TN_NONNULL(bitfield);
    TN_NONNULL(bbox);
    TN_NONNULL(march);
    // dt_min >= 1e-30 keeps the residuals of the exact round-up division clear of underflow
    TN_REQUIRE(march->dt_min >= 1e-30f && march->dt_max >= march->dt_min, TN_E_INVALID,
               "march: need 1e-30 <= dt_min <= dt_max (got %g, %g)", march->dt_min, march->dt_max);
    TN_REQUIRE(march->cone_angle >= 0.0f, TN_E_INVALID, "march: cone_angle must be >= 0");
    a.g = make_grid_view(*grid, bitfield);
    a.bbox = *bbox;
    a.cone = march->cone_angle;
    a.dt_min = march->dt_min;
    a.dt_max = march->dt_max;
    volatile float one = 1.0f;
    a.inv_dt_min = one / a.dt_min;
    a.max_steps = march->max_steps;
    a.max_iters = march->max_iterations ? march->max_iterations : (1u << 22);
    return TN_OK;
}

// Level-0 constants of the fused count loop, checked against every level of the per-level table
// (level k must be level 0 scaled by 2^k exactly; base sizes so extreme that this fails are
// rejected).
static int make_count_grid(const MarchArgs& a, CountGrid& cg) {
    const GridView& g = a.g;
    float half0 = g.half[0];
    cg.cell0 = g.cell[0];
    cg.inv_ls0 = g.inv_ls[0];
    cg.res_f = g.res_f;
    cg.res_m1 = (uint32_t)(g.res - 1);
    std::memcpy(&cg.half0_bits, &half0, sizeof(int));
    std::memcpy(&cg.cell0_bits, &cg.cell0, sizeof(int));
    cg.res_shift = 0;
    while ((1 << cg.res_shift) < g.res) ++cg.res_shift;
    cg.plane_words = (uint32_t)(((uint64_t)g.res * g.res * g.res) / 32);
    cg.n_levels = g.n_levels;
    cg.bits = g.bits;
    cg.planes = nullptr;
    for (int k = 0; k < g.n_levels; ++k) {
        const float up = std::ldexp(1.0f, k), dn = std::ldexp(1.0f, -k);
        TN_REQUIRE(g.half[k] == half0 * up && g.cell[k] == cg.cell0 * up && g.inv_ls[k] == cg.inv_ls0 * dn &&
                       std::isnormal(half0 * up) && std::isnormal(cg.cell0 * up) && std::isnormal(cg.inv_ls0 * dn),
                   TN_E_INVALID, "march: base_size %g out of range for %d levels", g.base, g.n_levels);
    }
    return TN_OK;
}

// Per-scene parameters of a multi-scene launch; scratch: per scene [mip | box | planes] in
// ctx->mip, each part 256-byte aligned.
static int make_multi_args(tn_ctx* ctx, uint32_t n_scenes, const tn_scene* scenes, uint32_t ray_stride,
                           uint32_t chunk_rays, MultiArgs& A, bool build_scratch) {
    TN_NONNULL(scenes);
    TN_REQUIRE(n_scenes >= 1 && n_scenes <= (uint32_t)MAX_SCENES, TN_E_INVALID, "n_scenes = %u outside 1..%d", n_scenes,
               MAX_SCENES);
    std::memset(&A, 0, sizeof(A));
    A.n_scenes = n_scenes;
    while ((1u << A.chunk_shift) < chunk_rays) ++A.chunk_shift;
    uint32_t chunk = 0, prev_end = 0, max_res = 0;
    size_t scratch = 0;
    for (uint32_t s = 0; s < n_scenes; ++s) {
        const tn_scene& sc = scenes[s];
        SceneParams& sp = A.sp[s];
        int st = make_march_args(&sc.grid, sc.bitfield, &sc.bbox, &sc.march, sp.a);
        if (st != TN_OK) return st;
        st = make_count_grid(sp.a, sp.cg);
        if (st != TN_OK) return st;
        TN_REQUIRE(sc.ray_begin >= prev_end, TN_E_INVALID, "scene %u: rays must follow the previous scene's", s);
        TN_REQUIRE((uint64_t)sc.ray_begin + sc.n_rays <= ray_stride, TN_E_INVALID, "scene %u: rays beyond ray_stride", s);
        prev_end = sc.ray_begin + sc.n_rays;
        sp.inv_aabb = sc.inv_aabb_size;
        sp.ray_begin = sc.ray_begin;
        sp.n_rays = sc.n_rays;
        sp.chunk_begin = chunk;
        chunk += (sc.n_rays + chunk_rays - 1) >> A.chunk_shift;
        const int res = sc.grid.resolution;
        max_res = std::max<uint32_t>(max_res, (uint32_t)res);
        sp.use_mip = res >= MIP_MIN_RES && res <= MIP_MAX_RES;
        sp.cshift = sp.cg.res_shift - 2;
        if (sp.use_mip) {
            TN_REQUIRE(((uintptr_t)sc.bitfield & 15u) == 0, TN_E_INVALID, "scene %u: bitfield must be 16-byte aligned", s);
            const size_t mip_bytes = (size_t)1 << (3 * sp.cshift);
            sp.mip_blocks = (uint32_t)((mip_bytes + 255) / 256);
            const size_t box_off = (mip_bytes + 255) & ~(size_t)255;
            const size_t planes_off = (box_off + BOX_INTS * sizeof(int) + 255) & ~(size_t)255;
            const size_t end = planes_off + (size_t)sc.grid.n_levels * sp.cg.plane_words * sizeof(uint32_t);
            // pointers are filled once the scratch is allocated
            sp.mip = reinterpret_cast<uint8_t*>(scratch);
            sp.box = reinterpret_cast<int*>(scratch + box_off);
            sp.cg.planes = reinterpret_cast<const uint32_t*>(scratch + planes_off);
            scratch += (end + 255) & ~(size_t)255;
        }
    }
    A.total_chunks = chunk;
    A.total_rays = prev_end;
    A.spread_res = max_res;
    if (build_scratch && scratch) {
        const int st = ensure_mip(ctx, scratch);
        if (st != TN_OK) return st;
    }
    const uintptr_t base = (uintptr_t)ctx->mip;
    for (uint32_t s = 0; s < n_scenes; ++s) {
        SceneParams& sp = A.sp[s];
        if (!sp.use_mip) continue;
        sp.mip = reinterpret_cast<uint8_t*>(base + (uintptr_t)sp.mip);
        sp.box = reinterpret_cast<int*>(base + (uintptr_t)sp.box);
        sp.cg.planes = reinterpret_cast<const uint32_t*>(base + (uintptr_t)sp.cg.planes);
    }
    return TN_OK;
}

// Per-ray step-position slots of a multi-scene launch (a larger budget than one scene's: the
// batch holds many more rays).
constexpr size_t MULTI_SLOT_BUDGET = 64u << 20;

static uint32_t multi_slot_capacity(uint32_t n_rays) {
    size_t cap = MULTI_SLOT_BUDGET / (n_rays ? n_rays : 1);
    cap = std::min<size_t>(std::max<size_t>(cap, 16), 1024);
    return (uint32_t)cap;
}

template <int NL>
static int launch_count_nl(bool mip, uint32_t nb, uint32_t group, size_t smem, cudaStream_t stream, const MarchArgs& a,
                            const CountGrid& cg, uint32_t n_rays, const uint32_t* n_rays_dev, uint32_t rs,
                            const float* ori, const float* dir, const float* ray_t, const float* ray_t_max,
                            uint8_t* alive, uint32_t* counts, uint32_t batch_size, uint32_t* batch_info,
                            uint32_t* block_agg, uint32_t* block_prefix, uint32_t* ticket, uint32_t* flags,
                            const uint8_t* mip_g, const int* box_g, float* slots, uint32_t slot_cap) {
    if (smem > 48 * 1024) {
        // the side_sms reservation: allow the device's opt-in shared memory (set once per kernel)
        static const int optin_status = [] {
            const int st = allow_optin_smem((const void*)march_count_kernel<NL, true>);
            return st == TN_OK ? allow_optin_smem((const void*)march_count_kernel<NL, false>) : st;
        }();
        if (optin_status != TN_OK) return optin_status;
    }
    if (mip)
        march_count_kernel<NL, true><<<nb, group, smem, stream>>>(
            a, cg, n_rays, n_rays_dev, rs, ori, dir, ray_t, ray_t_max, alive, counts, batch_size, batch_info,
            block_agg, block_prefix, ticket, flags, mip_g, box_g, slots, slot_cap);
    else
        march_count_kernel<NL, false><<<nb, group, smem, stream>>>(
            a, cg, n_rays, n_rays_dev, rs, ori, dir, ray_t, ray_t_max, alive, counts, batch_size, batch_info,
            block_agg, block_prefix, ticket, flags, mip_g, box_g, slots, slot_cap);
    return TN_OK;
}

// The two passes of the compaction with a tile of BLOCK x ITEMS values.
template <int BLOCK, int ITEMS>
static void launch_compact(cudaStream_t stream, uint32_t nb, uint32_t n, const uint32_t* values, tn_ctx* ctx,
                           int32_t* out, uint32_t* count_dev) {
    compact_count_kernel<BLOCK, ITEMS><<<nb, BLOCK, 0, stream>>>(n, values, ctx->block_u32, ctx->block_u32 + nb,
                                                                 count_dev, ctx->tickets + TICKET_COMPACT);
    compact_write_kernel<BLOCK, ITEMS><<<nb, BLOCK, 0, stream>>>(n, values, ctx->block_u32 + nb, out);
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_rays_init_bbox(tn_stream_t stream, uint32_t n_rays, uint32_t ray_stride, const tn_bbox* bbox, float t_far,
                      const float* ori, const float* dir, float* t, float* t_max, uint8_t* alive) {
    TN_NONNULL(bbox); TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(t); TN_NONNULL(t_max); TN_NONNULL(alive);
    TN_REQUIRE(ray_stride >= n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", ray_stride, n_rays);
    if (n_rays == 0) return TN_OK;
    rays_init_kernel<<<(n_rays + 255) / 256, 256, 0, stream>>>(n_rays, ray_stride, *bbox, t_far, ori, dir, t, t_max, alive);
    return check_launch("tn_rays_init_bbox");
}

int tn_march_count(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                   const tn_bbox* bbox, const tn_march_desc* march, uint32_t n_rays, uint32_t ray_stride,
                   const uint32_t* n_rays_dev, const float* ori, const float* dir, const float* ray_t,
                   const float* ray_t_max, uint8_t* alive, uint32_t* n_steps, uint32_t batch_size,
                   uint32_t* batch_info) {
    TN_NONNULL(ctx);
    MarchArgs a;
    int st = make_march_args(grid, bitfield, bbox, march, a);
    if (st != TN_OK) return st;
    CountGrid cg;
    st = make_count_grid(a, cg);
    if (st != TN_OK) return st;
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(ray_t_max); TN_NONNULL(alive);
    TN_NONNULL(n_steps); TN_NONNULL(batch_info);
    TN_REQUIRE(n_rays > 0, TN_E_NO_RAYS, "tn_march_count: n_rays = 0");
    TN_REQUIRE(ray_stride >= n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", ray_stride, n_rays);
    const uint32_t group = ctx->tune.count_rays_per_block;
    const uint32_t nb = (n_rays + group - 1) / group;
    st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    // coarse mip of the bitfield, the per-level boxes of occupied blocks and the bit-planes:
    // ctx->mip = [mip (R^3/64 B) | box | planes (n_levels x R^3/8 B, 256-byte aligned)]
    const int res = grid->resolution;
    const bool use_mip = res >= MIP_MIN_RES && res <= MIP_MAX_RES;
    const uint32_t mip_bytes = use_mip ? (uint32_t)(res / 4) * (res / 4) * (res / 4) : 0u;
    const size_t planes_off = ((size_t)mip_bytes + BOX_INTS * sizeof(int) + 255) & ~(size_t)255;
    int* box = nullptr;
    if (use_mip) {
        st = ensure_mip(ctx, planes_off + (size_t)grid->n_levels * cg.plane_words * sizeof(uint32_t));
        if (st != TN_OK) return st;
        TN_REQUIRE(((uintptr_t)bitfield & 15u) == 0, TN_E_INVALID, "bitfield must be 16-byte aligned");
        box = reinterpret_cast<int*>(ctx->mip + mip_bytes);
        cg.planes = reinterpret_cast<const uint32_t*>(ctx->mip + planes_off);
        st = cuda_status(cudaMemsetAsync(box, 0x7f, BOX_INTS / 2 * sizeof(int), stream), "tn_march_count(box)");
        if (st == TN_OK)
            st = cuda_status(cudaMemsetAsync(box + BOX_INTS / 2, 0, BOX_INTS / 2 * sizeof(int), stream),
                             "tn_march_count(box)");
        if (st != TN_OK) return st;
        build_mip_kernel<<<(mip_bytes + 255) / 256, 256, 0, stream>>>(
            cg.res_shift - 2, grid->n_levels, reinterpret_cast<const uint4*>(bitfield), ctx->mip, box,
            reinterpret_cast<uint32_t*>(ctx->mip + planes_off), cg.plane_words);
        st = check_launch("tn_march_count(mip)");
        if (st != TN_OK) return st;
    }
    // per-ray step positions for the emit pass
    const uint32_t slot_cap = slot_capacity(n_rays, march->max_steps);
    st = ensure_slots(ctx, (size_t)n_rays * slot_cap);
    if (st != TN_OK) return st;
    ctx->slot_cap = slot_cap;
    ctx->slot_rays = n_rays;
    size_t smem = (size_t)12 * res + mip_bytes;
    // with SMs kept for other work, each count block holds its SM alone (see exclusive_smem)
    if (ctx->tune.side_sms) smem = std::max(smem, exclusive_smem());
#define TN_COUNT_CASE(NL)                                                                                          \
    case NL:                                                                                                       \
        st = launch_count_nl<NL>(use_mip, nb, group, smem, stream, a, cg, n_rays, n_rays_dev, ray_stride, ori, dir, ray_t,     \
                            ray_t_max, alive, n_steps, batch_size, batch_info, ctx->block_u32, ctx->block_u32 + nb, \
                            ctx->tickets + TICKET_MARCH, ctx->flags, ctx->mip, box, ctx->slots, slot_cap);       \
        break;
    switch (grid->n_levels) {
        TN_COUNT_CASE(1) TN_COUNT_CASE(2) TN_COUNT_CASE(3) TN_COUNT_CASE(4)
        TN_COUNT_CASE(5) TN_COUNT_CASE(6) TN_COUNT_CASE(7) TN_COUNT_CASE(8)
    }
#undef TN_COUNT_CASE
    if (st != TN_OK) return st;
    ctx->count_group_used = group;
    return check_launch("tn_march_count");
}

int tn_march_emit(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                  const tn_bbox* bbox, const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays,
                  uint32_t ray_stride, uint32_t sample_stride, const uint32_t* batch_info,
                  const uint32_t* ray_img_id, const float* ori, const float* dir, const float* ray_t,
                  const uint8_t* alive, const uint32_t* n_steps, uint32_t* offsets,
                  uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                  float* out_m_norm, float* out_dt_norm) {
    TN_NONNULL(ctx);
    MarchArgs a;
    int st = make_march_args(grid, bitfield, bbox, march, a);
    if (st != TN_OK) return st;
    TN_NONNULL(batch_info); TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(alive);
    TN_NONNULL(n_steps); TN_NONNULL(offsets); TN_NONNULL(out_t); TN_NONNULL(out_pos); TN_NONNULL(out_dir);
    TN_NONNULL(out_dt); TN_NONNULL(out_m_norm); TN_NONNULL(out_dt_norm);
    TN_REQUIRE(n_rays > 0, TN_E_NO_RAYS, "tn_march_emit: n_rays = 0");
    TN_REQUIRE(ray_stride >= n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", ray_stride, n_rays);
    const uint32_t group = ctx->count_group_used;
    TN_REQUIRE(group != 0, TN_E_STATE, "tn_march_emit must follow tn_march_count on the same context");
    const uint32_t nb = (n_rays + group - 1) / group;
    TN_REQUIRE(ctx->block_u32_cap >= 2 * (size_t)nb && ctx->slot_rays == n_rays, TN_E_STATE,
               "tn_march_emit must follow tn_march_count on the same context with the same n_rays");
    SampleOut o{out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm, out_dt_norm, sample_stride};
    const uint32_t gshift = (uint32_t)__builtin_ctz(group);
    const uint32_t warps = ctx->tune.emit_warps_per_block, rpw = ctx->tune.emit_rays_per_warp;
    const uint32_t per_block = warps * rpw;
    const uint32_t n_blocks = (n_rays + per_block - 1) / per_block;
#define TN_EXPAND(RPW)                                                                                              \
    expand_kernel<RPW><<<n_blocks, warps * WARP, 0, stream>>>(a, inv_aabb_size, n_rays, nullptr, ray_stride, gshift, \
                                                             batch_info, ctx->block_u32 + nb, ray_img_id, ori, dir,  \
                                                             ray_t, alive, n_steps, offsets, o, ctx->flags,          \
                                                             ctx->slots, ctx->slot_cap)
    if (rpw == 4) TN_EXPAND(4);
    else if (rpw == 2) TN_EXPAND(2);
    else TN_EXPAND(1);
#undef TN_EXPAND
    return check_launch("tn_march_emit");
}

int tn_multi_march_count(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                         uint32_t ray_stride, const float* ori, const float* dir, const float* ray_t,
                         const float* ray_t_max, uint8_t* alive, uint32_t* n_steps, uint32_t* scene_samples,
                         uint32_t* batch_info) {
    TN_NONNULL(ctx);
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(ray_t_max); TN_NONNULL(alive);
    TN_NONNULL(n_steps); TN_NONNULL(batch_info);
    static MultiArgs A;  // large; built under the host lock of the calling thread's launch
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    const uint32_t chunk_rays = ctx->tune.multi_chunk_rays;
    int st = make_multi_args(ctx, n_scenes, scenes, ray_stride, chunk_rays, A, true);
    if (st != TN_OK) return st;
    TN_REQUIRE(A.total_rays > 0, TN_E_NO_RAYS, "tn_multi_march_count: no rays");
    st = ensure_block_u32(ctx, 2 * (size_t)A.total_chunks);
    if (st != TN_OK) return st;
    const uint32_t slot_cap = multi_slot_capacity(A.total_rays);
    st = ensure_slots(ctx, (size_t)A.total_rays * slot_cap);
    if (st != TN_OK) return st;
    ctx->slot_cap = slot_cap;
    ctx->slot_rays = A.total_rays;
    st = cuda_status(cudaMemsetAsync(ctx->tickets + TICKET_MULTI, 0, 2 * sizeof(uint32_t), stream),
                     "tn_multi_march_count(counters)");
    if (st != TN_OK) return st;
    uint32_t max_mip_blocks = 0;
    for (uint32_t s = 0; s < n_scenes; ++s) max_mip_blocks = std::max(max_mip_blocks, A.sp[s].mip_blocks);
    if (max_mip_blocks) {
        multi_box_init_kernel<<<n_scenes, 64, 0, stream>>>(A);
        multi_build_mip_kernel<<<dim3(max_mip_blocks, n_scenes), 256, 0, stream>>>(A);
        st = check_launch("tn_multi_march_count(mip)");
        if (st != TN_OK) return st;
    }
    const size_t smem = (size_t)12 * A.spread_res + (size_t)(MIP_MAX_RES / 4) * (MIP_MAX_RES / 4) * (MIP_MAX_RES / 4);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, multi_count_kernel, (int)chunk_rays, smem);
    const uint32_t grid = std::min<uint32_t>(A.total_chunks, (uint32_t)(num_sms() * std::max(per_sm, 1)));
    ctx->multi_chunk_used = chunk_rays;
    multi_count_kernel<<<grid, chunk_rays, smem, stream>>>(
        A, ray_stride, ori, dir, ray_t, ray_t_max, alive, n_steps, ctx->block_u32, ctx->block_u32 + A.total_chunks,
        ctx->tickets + TICKET_MULTI_WORK, ctx->tickets + TICKET_MULTI, ctx->flags, ctx->slots, slot_cap,
        scene_samples, batch_info);
    return check_launch("tn_multi_march_count");
}

int tn_multi_march_emit(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                        uint32_t ray_stride, uint32_t sample_stride, const uint32_t* ray_img_id, const float* ori,
                        const float* dir, const float* ray_t, const uint8_t* alive, const uint32_t* n_steps,
                        uint32_t* offsets, uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir,
                        float* out_dt, float* out_m_norm, float* out_dt_norm) {
    TN_NONNULL(ctx);
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(alive); TN_NONNULL(n_steps);
    TN_NONNULL(offsets); TN_NONNULL(out_t); TN_NONNULL(out_pos); TN_NONNULL(out_dir); TN_NONNULL(out_dt);
    TN_NONNULL(out_m_norm); TN_NONNULL(out_dt_norm);
    static MultiArgs A;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    TN_REQUIRE(ctx->multi_chunk_used != 0, TN_E_STATE, "tn_multi_march_emit must follow tn_multi_march_count");
    int st = make_multi_args(ctx, n_scenes, scenes, ray_stride, ctx->multi_chunk_used, A, false);
    if (st != TN_OK) return st;
    TN_REQUIRE(ctx->block_u32_cap >= 2 * (size_t)A.total_chunks && ctx->slot_rays == A.total_rays, TN_E_STATE,
               "tn_multi_march_emit must follow tn_multi_march_count on the same context with the same scenes");
    SampleOut o{out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm, out_dt_norm, sample_stride};
    const uint32_t warps = ctx->tune.emit_warps_per_block, rpw = ctx->tune.emit_rays_per_warp;
    const uint32_t per_block = warps * rpw;
    const uint32_t n_blocks = (A.total_rays + per_block - 1) / per_block;
#define TN_MULTI_EXPAND(RPW)                                                                                  \
    multi_expand_kernel<RPW><<<n_blocks, warps * WARP, 0, stream>>>(A, ray_stride, ctx->block_u32 + A.total_chunks, \
                                                                   ray_img_id, ori, dir, ray_t, alive, n_steps,    \
                                                                   offsets, o, ctx->flags, ctx->slots, ctx->slot_cap)
    if (rpw == 4) TN_MULTI_EXPAND(4);
    else if (rpw == 2) TN_MULTI_EXPAND(2);
    else TN_MULTI_EXPAND(1);
#undef TN_MULTI_EXPAND
    return check_launch("tn_multi_march_emit");
}

int tn_scan_offsets(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                    uint32_t batch_size, uint32_t* batch_info) {
    TN_NONNULL(ctx); TN_NONNULL(counts); TN_NONNULL(offsets); TN_NONNULL(batch_info);
    TN_REQUIRE(n > 0, TN_E_NO_RAYS, "tn_scan_offsets: n = 0");
    const uint32_t nb = (n + MARCH_BLOCK - 1) / MARCH_BLOCK;
    int st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    scan_count_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, counts, batch_size, batch_info, ctx->block_u32,
                                                      ctx->block_u32 + nb, ctx->tickets + TICKET_SCAN, ctx->flags,
                                                      nullptr);
    st = check_launch("tn_scan_offsets(count)");
    if (st != TN_OK) return st;
    scan_offsets_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, counts, ctx->block_u32 + nb, offsets);
    return check_launch("tn_scan_offsets(offsets)");
}

// ---- allocation-free scan + batch cut ------------------------------------------------
// Some callers cannot allocate device memory: a plugin whose host application owns the
// whole device heap and forbids extra allocations, or a loop that must not pay cudaMalloc's
// implicit device synchronisation. For them this variant of tn_scan_offsets takes no tn_ctx:
// its scratch (per-block totals and prefixes of the counts, the last-block ticket and an
// error word) is a fixed array in device memory that lives in the library image itself and is
// held by every device that loads the library until the process exits.
//
// Limit: at most TN_SCAN_NOALLOC_MAX_COUNTS counts per call (2 x 16,384 block entries plus 64
// words: 128.25 KiB of scratch). Every call uses the same array, so two calls that overlap on
// the GPU (different streams, or different host threads on one device) race on it; serialise
// them.
constexpr uint32_t NOALLOC_MAX_BLOCKS = TN_SCAN_NOALLOC_MAX_COUNTS / MARCH_BLOCK;
constexpr uint32_t NOALLOC_WORDS = 2 * NOALLOC_MAX_BLOCKS + 64;  // [agg | prefix | ticket, flags, ...]
static __device__ __align__(256) uint32_t g_scan_noalloc_scratch[NOALLOC_WORDS];

// In host code the array's name is a host-side stand-in, not a device address. The device
// address is looked up with cudaGetSymbolAddress once per device, with that device current,
// and cached together with the CUDA context it belongs to: after a cudaDeviceReset the device
// gets a new primary context, the library's module is loaded again, and the address is looked
// up again instead of reusing a stale one. The context is read through the driver entry point
// (the runtime is linked statically and the library does not link libcuda).
typedef int (*CtxGetCurrentFn)(void**);
struct NoallocSlot {
    void* ctx;
    uint32_t* ptr;
};
static NoallocSlot g_scan_noalloc_slot[64] = {};
static std::mutex g_scan_noalloc_mutex;

static int current_context(void** ctx) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        int st = cuda_status(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q),
                             "tn_scan_offsets_noalloc: cudaGetDriverEntryPoint");
        if (st != TN_OK) return st;
        TN_REQUIRE(q == cudaDriverEntryPointSuccess && f != nullptr, TN_E_CUDA,
                   "tn_scan_offsets_noalloc: cuCtxGetCurrent not found");
        fn = reinterpret_cast<CtxGetCurrentFn>(f);
    }
    TN_REQUIRE(fn(ctx) == 0, TN_E_CUDA, "tn_scan_offsets_noalloc: cuCtxGetCurrent failed");
    return TN_OK;
}

static int scan_noalloc_scratch(uint32_t** out) {
    int dev = 0;
    int st = cuda_status(cudaGetDevice(&dev), "tn_scan_offsets_noalloc: cudaGetDevice");
    if (st != TN_OK) return st;
    TN_REQUIRE(dev >= 0 && dev < 64, TN_E_INVALID, "tn_scan_offsets_noalloc: device %d out of range", dev);
    void* ctx = nullptr;
    st = current_context(&ctx);
    if (st != TN_OK) return st;
    std::lock_guard<std::mutex> lock(g_scan_noalloc_mutex);
    NoallocSlot& slot = g_scan_noalloc_slot[dev];
    if (!slot.ptr || !ctx || slot.ctx != ctx) {
        void* p = nullptr;
        // the lookup also makes the runtime's primary context current when none was
        st = cuda_status(cudaGetSymbolAddress(&p, g_scan_noalloc_scratch),
                         "tn_scan_offsets_noalloc: cudaGetSymbolAddress");
        if (st != TN_OK) return st;
        st = current_context(&ctx);
        if (st != TN_OK) return st;
        slot.ptr = static_cast<uint32_t*>(p);
        slot.ctx = ctx;
    }
    *out = slot.ptr;
    return TN_OK;
}

int tn_compact_nonzero(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* values, int32_t* out,
                       uint32_t* count_dev) {
    TN_NONNULL(ctx); TN_NONNULL(values); TN_NONNULL(out); TN_NONNULL(count_dev);
    if (n == 0) return cuda_status(cudaMemsetAsync(count_dev, 0, sizeof(uint32_t), stream), "tn_compact_nonzero");
    const uint32_t tile = ctx->tune.compact_tile;
    const uint32_t nb = (uint32_t)(((uint64_t)n + tile - 1) / tile);
    int st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    switch (tile) {
        case 256: launch_compact<256, 1>(stream, nb, n, values, ctx, out, count_dev); break;
        case 512: launch_compact<256, 2>(stream, nb, n, values, ctx, out, count_dev); break;
        case 1024: launch_compact<256, 4>(stream, nb, n, values, ctx, out, count_dev); break;
        case 2048: launch_compact<256, 8>(stream, nb, n, values, ctx, out, count_dev); break;
        default: launch_compact<128, 1>(stream, nb, n, values, ctx, out, count_dev); break;
    }
    return check_launch("tn_compact_nonzero");
}

int tn_scan_offsets_noalloc(tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                            uint32_t batch_size, uint32_t* batch_info, uint32_t* error_word) {
    TN_NONNULL(counts); TN_NONNULL(offsets); TN_NONNULL(batch_info);
    TN_REQUIRE(n > 0, TN_E_NO_RAYS, "tn_scan_offsets_noalloc: n = 0");
    TN_REQUIRE(n <= TN_SCAN_NOALLOC_MAX_COUNTS, TN_E_CAPACITY,
               "tn_scan_offsets_noalloc: %u counts exceed the fixed scratch limit of %u (use tn_scan_offsets)", n,
               (uint32_t)TN_SCAN_NOALLOC_MAX_COUNTS);
    uint32_t* scratch = nullptr;
    int st = scan_noalloc_scratch(&scratch);
    if (st != TN_OK) return st;
    uint32_t* block_agg = scratch;
    uint32_t* block_prefix = scratch + NOALLOC_MAX_BLOCKS;
    uint32_t* ticket = scratch + 2 * NOALLOC_MAX_BLOCKS;
    uint32_t* flags = ticket + 1;
    // the ticket must start at zero (the last block also leaves it at zero); clear the error word too
    st = cuda_status(cudaMemsetAsync(ticket, 0, 2 * sizeof(uint32_t), stream), "tn_scan_offsets_noalloc: clear");
    if (st != TN_OK) return st;
    const uint32_t nb = (n + MARCH_BLOCK - 1) / MARCH_BLOCK;
    scan_count_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, counts, batch_size, batch_info, block_agg, block_prefix, ticket,
                                                      flags, error_word);
    st = check_launch("tn_scan_offsets_noalloc(count)");
    if (st != TN_OK) return st;
    scan_offsets_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, counts, block_prefix, offsets);
    return check_launch("tn_scan_offsets_noalloc(offsets)");
}

int tn_plain_march_count(tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield, const tn_bbox* bbox,
                         const tn_march_desc* march, uint32_t n_rays, uint32_t ray_stride, const float* ori,
                         const float* dir, const float* ray_t, const float* ray_t_max, uint8_t* alive,
                         uint32_t* n_steps) {
    MarchArgs a;
    int st = make_march_args(grid, bitfield, bbox, march, a);
    if (st != TN_OK) return st;
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(ray_t_max); TN_NONNULL(alive); TN_NONNULL(n_steps);
    if (n_rays == 0) return TN_OK;
    plain_count_kernel<<<(n_rays + 127) / 128, 128, 0, stream>>>(a, n_rays, ray_stride, ori, dir, ray_t, ray_t_max,
                                                                 alive, n_steps);
    return check_launch("tn_plain_march_count");
}

struct LessThan {
    uint32_t v;
    __host__ __device__ bool operator()(uint32_t x) const { return x < v; }
};

int tn_plain_scan_cut_sync(tn_stream_t stream, uint32_t n, const uint32_t* n_steps, uint32_t* offsets,
                           uint32_t batch_size, uint32_t* n_rays_out, uint32_t* n_samples_out) {
    TN_NONNULL(n_steps); TN_NONNULL(offsets); TN_NONNULL(n_rays_out); TN_NONNULL(n_samples_out);
    *n_rays_out = 0;
    *n_samples_out = 0;
    TN_REQUIRE(n > 0, TN_E_NO_RAYS, "tn_plain_scan_cut_sync: n = 0");
    thrust::device_ptr<const uint32_t> in(n_steps);
    thrust::device_ptr<uint32_t> out(offsets);
    thrust::exclusive_scan(thrust::cuda::par.on(stream), in, in + n, out);
    auto rb = thrust::make_reverse_iterator(out + n);
    auto re = thrust::make_reverse_iterator(out);
    auto it = thrust::find_if(thrust::cuda::par.on(stream), rb, re, LessThan{batch_size});
    int last = -1;
    if (it != re) last = (int)thrust::distance(out, it.base() - 1);
    const int max_idx = last - 1;
    TN_REQUIRE(max_idx >= 0, TN_E_NO_RAYS, "No rays were generated for this training batch");
    const uint32_t nr = (uint32_t)(max_idx + 1);
    uint32_t ns = 0;
    int st = cuda_status(cudaMemcpyAsync(&ns, offsets + nr, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream),
                         "tn_plain_scan_cut_sync copy");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_plain_scan_cut_sync sync");
    if (st != TN_OK) return st;
    *n_rays_out = nr;
    *n_samples_out = ns;
    TN_REQUIRE(ns >= 1, TN_E_NO_SAMPLES, "No samples were generated for this training batch");
    return TN_OK;
}

int tn_plain_march_emit(tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield, const tn_bbox* bbox,
                        const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays, uint32_t ray_stride,
                        uint32_t sample_stride, const uint32_t* ray_img_id, const float* ori, const float* dir,
                        const float* ray_t, const uint32_t* offsets, const uint8_t* alive, const uint32_t* n_steps,
                        uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                        float* out_m_norm, float* out_dt_norm) {
    MarchArgs a;
    int st = make_march_args(grid, bitfield, bbox, march, a);
    if (st != TN_OK) return st;
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(offsets); TN_NONNULL(alive); TN_NONNULL(n_steps);
    TN_NONNULL(out_t); TN_NONNULL(out_pos); TN_NONNULL(out_dir); TN_NONNULL(out_dt); TN_NONNULL(out_m_norm);
    TN_NONNULL(out_dt_norm);
    if (n_rays == 0) return TN_OK;
    SampleOut o{out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm, out_dt_norm, sample_stride};
    plain_emit_kernel<<<(n_rays + 127) / 128, 128, 0, stream>>>(a, inv_aabb_size, n_rays, ray_stride, ray_img_id, ori,
                                                                dir, ray_t, offsets, alive, n_steps, o);
    return check_launch("tn_plain_march_emit");
}

}  // extern "C"
