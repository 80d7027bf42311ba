// Occupancy-grid ray marching with sample compaction.
//
// Fused path (tn_march_count + tn_march_emit): no host round trip, one sequential march.
//  * count: one thread per ray runs the reference's DDA loop exactly, with a coarse occupancy
//    mip staged in shared memory to answer empty blocks without a global load, and records
//    the t of every occupied step in a per-ray slot; each 128-ray block reduces its counts;
//    the last block to finish (ticket) scans the block totals and performs the reference's
//    batch cut on the device (batch_info).
//  * emit: the same 128-ray blocks rebuild their rays' offsets with a block scan, then expand
//    the recorded steps into the packed sample arrays, one warp per ray and one lane per
//    sample (coalesced stores), instead of replaying the march.
// Plain path (tn_plain_*): count kernel, thrust exclusive_scan, reverse find_if, a
// blocking device->host read of the sample count, emit kernel -- the reference's launch
// structure (src/core/trainer.cu:106-216).
#include <thrust/execution_policy.h>
#include <thrust/find.h>
#include <thrust/iterator/reverse_iterator.h>
#include <thrust/scan.h>
#include <thrust/device_ptr.h>

#include <mutex>

#include "tn_internal.cuh"

namespace tn {

constexpr int MARCH_BLOCK = 128;

struct MarchArgs {
    GridView g;
    tn_bbox bbox;
    float cone, dt_min, dt_max;
    uint32_t max_steps, max_iters;
};

// Occupancy test (OccupancyGrid::is_occupied_at, src/core/occupancy-grid.cuh:185-207). With a
// coarse mip (one byte per 4x4x4 block of cells = 64 consecutive Morton indices, bit k set when
// any cell of the block is occupied at level k) held in shared memory, an empty block answers
// without touching the fine bitfield; the result is identical by construction.
__device__ __forceinline__ bool occupied_at(const GridView& g, int k, float x, float y, float z,
                                           const uint8_t* __restrict__ mip) {
    const uint32_t idx = voxel_morton(g, k, x, y, z);
    const uint8_t bit = (uint8_t)(1u << k);
    if (mip && !(mip[idx >> 6] & bit)) return false;
    return (__ldg(g.bits + idx) & bit) != 0;
}

__device__ __forceinline__ void load_ray(RayMarch& r, const float* __restrict__ ori, const float* __restrict__ dir,
                                         uint32_t i, uint32_t rs) {
    r.ox = ori[i]; r.oy = ori[i + rs]; r.oz = ori[i + 2 * (size_t)rs];
    r.dx = dir[i]; r.dy = dir[i + rs]; r.dz = dir[i + 2 * (size_t)rs];
    r.idx = __fdiv_rn(1.0f, r.dx);
    r.idy = __fdiv_rn(1.0f, r.dy);
    r.idz = __fdiv_rn(1.0f, r.dz);
}

// march_and_count_steps_per_ray_kernel loop, src/utils/training-batch-kernels.cuh:258-297.
// When `slots` is set, the t of the first `slot_cap` occupied steps is recorded so that the
// emit pass can expand the samples without replaying the march.
__device__ uint32_t march_count_ray(const MarchArgs& a, RayMarch& r, float t_max, uint32_t* flags,
                                    const uint8_t* __restrict__ mip = nullptr, float* __restrict__ slots = nullptr,
                                    uint32_t slot_cap = 0) {
    uint32_t n = 0, iters = 0;
    float t = r.t;
    while (t < t_max) {
        if (++iters > a.max_iters) { raise_flag(flags, ERR_GUARD); break; }
        float x, y, z;
        ray_point(r, t, x, y, z);
        if (!bbox_contains(a.bbox, x, y, z)) break;
        const float dt = get_dt(t, a.cone, a.dt_min, a.dt_max);
        const int k = grid_level_at(a.g, x, y, z, dt);
        if (occupied_at(a.g, k, x, y, z, mip)) {
            if (n < slot_cap) slots[n] = t;
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
        if (occupied_at(a.g, k, x, y, z, nullptr)) {
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

// Block-wide exclusive scan of one u32 per thread (MARCH_BLOCK threads); returns the
// exclusive prefix and the block total in *total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_tot[MARCH_BLOCK / WARP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t inc = warp_inclusive_sum(v, lane);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    uint32_t before = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < MARCH_BLOCK / WARP; ++w) {
        const uint32_t x = warp_tot[w];
        if (w < wid) before += x;
        tot += x;
    }
    __syncthreads();
    *total = tot;
    return before + inc - v;
}

// Last-block epilogue of the count pass: exclusive scan of the block totals into
// block_prefix, then the reference batch cut (src/core/trainer.cu:133-183):
// L = last ray index whose offset < batch_size; n_rays = L; n_samples = offset[L].
__device__ void scan_blocks_and_cut(uint32_t nb, uint32_t n_live, const uint32_t* __restrict__ counts,
                                    uint32_t* block_agg, uint32_t* block_prefix, uint32_t batch_size,
                                    uint32_t* batch_info, uint32_t* flags) {
    __shared__ unsigned long long carry_s;
    __shared__ int last_block_s;
    __shared__ int last_ray_s;
    if (threadIdx.x == 0) { carry_s = 0ull; last_block_s = -1; last_ray_s = -1; }
    __syncthreads();
    const uint32_t nb_live = (n_live + MARCH_BLOCK - 1) / MARCH_BLOCK;
    for (uint32_t base = 0; base < nb; base += MARCH_BLOCK) {
        const uint32_t b = base + threadIdx.x;
        const uint32_t v = b < nb ? *((volatile uint32_t*)(block_agg + b)) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, &tot);
        const unsigned long long pre = carry_s + ex;
        if (b < nb) {
            block_prefix[b] = pre > 0xffffffffull ? 0xffffffffu : (uint32_t)pre;
            if (pre > 0xffffffffull) raise_flag(flags, ERR_CAPACITY);
            if (b < nb_live && pre < batch_size) atomicMax(&last_block_s, (int)b);
        }
        __syncthreads();
        if (threadIdx.x == 0) carry_s += tot;
        __syncthreads();
    }
    const int lb = last_block_s;
    uint32_t n_rays_cut = 0, n_samples = 0;
    if (batch_size == 0xffffffffu) {
        // no cut (render / inference use): every live ray is kept
        if (threadIdx.x == 0) {
            const unsigned long long total = carry_s;
            batch_info[0] = n_live;
            batch_info[1] = total > 0xffffffffull ? 0xffffffffu : (uint32_t)total;
            batch_info[2] = batch_info[1];
            if (n_live == 0) raise_flag(flags, ERR_NO_RAYS);
            else if (total == 0) raise_flag(flags, ERR_NO_SAMPLES);
        }
        return;
    }
    if (lb >= 0) {
        const uint32_t i = (uint32_t)lb * MARCH_BLOCK + threadIdx.x;
        const uint32_t c = i < n_live ? *((volatile const uint32_t*)(counts + i)) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(c, &tot);
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
        const unsigned long long total = carry_s;
        batch_info[2] = total > 0xffffffffull ? 0xffffffffu : (uint32_t)total;
        const uint32_t nr = last_ray_s < 0 ? 0u : (uint32_t)last_ray_s;
        if (nr == 0) raise_flag(flags, ERR_NO_RAYS);
        else if (*((volatile uint32_t*)(batch_info + 1)) == 0) raise_flag(flags, ERR_NO_SAMPLES);
    }
}

// COUNT = true: march each ray; COUNT = false: counts are given (tn_scan_offsets).
template <bool MARCH>
__global__ void __launch_bounds__(MARCH_BLOCK)
count_kernel(MarchArgs a, uint32_t n_rays, const uint32_t* __restrict__ n_rays_dev, uint32_t rs,
             const float* __restrict__ ori, const float* __restrict__ dir, const float* __restrict__ ray_t,
             const float* __restrict__ ray_t_max, uint8_t* __restrict__ alive, uint32_t* counts,
             uint32_t batch_size, uint32_t* batch_info, uint32_t* block_agg, uint32_t* block_prefix,
             uint32_t* ticket, uint32_t* flags, const uint8_t* __restrict__ mip_g, uint32_t mip_bytes,
             float* __restrict__ slots, uint32_t slot_cap) {
    extern __shared__ __align__(16) uint8_t mip_s[];
    if (MARCH && mip_g) {
        // stage the coarse occupancy mip (mip_bytes is a multiple of 16)
        for (uint32_t k = threadIdx.x; k < mip_bytes / 16; k += MARCH_BLOCK)
            reinterpret_cast<uint4*>(mip_s)[k] = __ldg(reinterpret_cast<const uint4*>(mip_g) + k);
        __syncthreads();
    }
    const uint32_t n_live = n_rays_dev ? min(*n_rays_dev, n_rays) : n_rays;
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    uint32_t cnt = 0;
    if (i < n_live) {
        if (MARCH) {
            if (alive[i]) {
                RayMarch r;
                load_ray(r, ori, dir, i, rs);
                r.t = ray_t[i];
                cnt = march_count_ray(a, r, ray_t_max[i], flags, mip_g ? mip_s : nullptr,
                                      slots ? slots + (size_t)i * slot_cap : nullptr, slots ? slot_cap : 0u);
                if (cnt == 0) alive[i] = 0;
            }
            counts[i] = cnt;
        } else {
            cnt = counts[i];
        }
    }
    // make this thread's count visible device-wide before the block reports completion
    __threadfence();
    const int lane = threadIdx.x & 31;
    uint32_t s = warp_sum(cnt);
    __shared__ uint32_t wsum[MARCH_BLOCK / WARP];
    if (lane == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
#pragma unroll
        for (int w = 0; w < MARCH_BLOCK / WARP; ++w) tot += wsum[w];
        block_agg[blockIdx.x] = tot;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    scan_blocks_and_cut(gridDim.x, n_live, counts, block_agg, block_prefix, batch_size, batch_info, flags);
    if (threadIdx.x == 0) *ticket = 0u;
}

template <bool MARCH>
__global__ void __launch_bounds__(MARCH_BLOCK)
emit_kernel(MarchArgs a, float inv_aabb, uint32_t n_rays, const uint32_t* __restrict__ n_rays_dev, uint32_t rs,
            const uint32_t* __restrict__ batch_info, const uint32_t* __restrict__ block_prefix,
            const uint32_t* __restrict__ img_id, const float* __restrict__ ori, const float* __restrict__ dir,
            const float* __restrict__ ray_t, const uint8_t* __restrict__ alive, const uint32_t* __restrict__ counts,
            uint32_t* __restrict__ offsets, SampleOut o, uint32_t* flags) {
    const uint32_t n_live = n_rays_dev ? min(*n_rays_dev, n_rays) : n_rays;
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    const uint32_t cnt = i < n_live ? counts[i] : 0u;
    uint32_t tot;
    const uint32_t off = block_exclusive_scan(cnt, &tot) + block_prefix[blockIdx.x];
    if (i >= n_live) return;
    offsets[i] = off;
    if (!MARCH) return;
    const uint32_t n_cut = batch_info[0];
    if (i >= n_cut || cnt == 0 || !alive[i]) return;
    if ((unsigned long long)off + cnt > (unsigned long long)o.ss) { raise_flag(flags, ERR_CAPACITY); return; }
    RayMarch r;
    load_ray(r, ori, dir, i, rs);
    r.t = ray_t[i];
    march_emit_ray(a, r, cnt, off, img_id ? img_id[i] : 0u, inv_aabb, o);
}

// Emit pass from the recorded step positions: the 128-ray block of the count pass rebuilds its
// offsets, then each warp expands one ray at a time with one lane per sample (coalesced
// stores of the packed sample arrays). Every value is the one the reference's emit loop
// (training-batch-kernels.cuh:412-480) computes from the same t: dt = get_dt(t), the position
// o + t d, m = t + dt/2, the ray's span from its start t to the end of its last step.
// Rays with more samples than slots fall back to replaying their march.
__global__ void __launch_bounds__(MARCH_BLOCK)
expand_kernel(MarchArgs a, float inv_aabb, uint32_t n_rays, const uint32_t* __restrict__ n_rays_dev, uint32_t rs,
              const uint32_t* __restrict__ batch_info, const uint32_t* __restrict__ block_prefix,
              const uint32_t* __restrict__ img_id, const float* __restrict__ ori, const float* __restrict__ dir,
              const float* __restrict__ ray_t, const uint8_t* __restrict__ alive, const uint32_t* __restrict__ counts,
              uint32_t* __restrict__ offsets, SampleOut o, uint32_t* flags, const float* __restrict__ slots,
              uint32_t slot_cap) {
    __shared__ uint32_t off_s[MARCH_BLOCK], cnt_s[MARCH_BLOCK];
    const uint32_t n_live = n_rays_dev ? min(*n_rays_dev, n_rays) : n_rays;
    const uint32_t base = blockIdx.x * MARCH_BLOCK;
    const uint32_t i = base + threadIdx.x;
    const uint32_t c = i < n_live ? counts[i] : 0u;
    uint32_t tot;
    const uint32_t off = block_exclusive_scan(c, &tot) + block_prefix[blockIdx.x];
    const uint32_t n_cut = batch_info[0];
    off_s[threadIdx.x] = off;
    cnt_s[threadIdx.x] = (i < n_live && i < n_cut && c != 0 && alive[i]) ? c : 0u;
    if (i < n_live) offsets[i] = off;
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const size_t ss = o.ss;
    for (int k = 0; k < WARP; ++k) {
        const int local = wid * WARP + k;
        const uint32_t n = cnt_s[local];
        if (n == 0) continue;
        const uint32_t r_i = base + local;
        const uint32_t o0 = off_s[local];
        if ((unsigned long long)o0 + n > (unsigned long long)o.ss) {
            if (lane == 0) raise_flag(flags, ERR_CAPACITY);
            continue;
        }
        RayMarch r;
        load_ray(r, ori, dir, r_i, rs);
        r.t = ray_t[r_i];
        const uint32_t img = img_id ? img_id[r_i] : 0u;
        if (n > slot_cap) {
            if (lane == 0) march_emit_ray(a, r, n, o0, img, inv_aabb, o);
            continue;
        }
        const float* sl = slots + (size_t)r_i * slot_cap;
        const float t_last = sl[n - 1];
        const float t_end = __fadd_rn(t_last, get_dt(t_last, a.cone, a.dt_min, a.dt_max));
        const float t_span = fmaxf(__fadd_rn(t_end, -r.t), 1e-6f);
        for (uint32_t j = lane; j < n; j += WARP) {
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
    (void)ss;
}

// Coarse occupancy mip: byte c = OR of the 64 fine bytes [64c, 64c + 64) (one 4x4x4 block).
__global__ void build_mip_kernel(uint32_t n_coarse, const uint32_t* __restrict__ bits4, uint8_t* __restrict__ mip) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_coarse) return;
    const uint4* p = reinterpret_cast<const uint4*>(bits4) + (size_t)c * 4;
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint4 q = __ldg(p + k);
        v |= q.x | q.y | q.z | q.w;
    }
    mip[c] = (uint8_t)((v | (v >> 8) | (v >> 16) | (v >> 24)) & 0xFFu);
}

// ---- compaction: ascending indices of non-zero values ---------------------------------
__global__ void __launch_bounds__(MARCH_BLOCK)
compact_count_kernel(uint32_t n, const uint32_t* __restrict__ values, uint32_t* block_agg, uint32_t* block_prefix,
                     uint32_t* count_dev, uint32_t* ticket) {
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    const uint32_t f = (i < n && values[i] != 0u) ? 1u : 0u;
    const uint32_t s = __syncthreads_count(f);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
        block_agg[blockIdx.x] = s;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    __shared__ uint32_t carry_s;
    if (threadIdx.x == 0) carry_s = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < gridDim.x; base += MARCH_BLOCK) {
        const uint32_t b = base + threadIdx.x;
        const uint32_t v = b < gridDim.x ? *((volatile uint32_t*)(block_agg + b)) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan(v, &tot);
        if (b < gridDim.x) block_prefix[b] = carry_s + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry_s += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *count_dev = carry_s;
        *ticket = 0u;
    }
}

__global__ void __launch_bounds__(MARCH_BLOCK)
compact_write_kernel(uint32_t n, const uint32_t* __restrict__ values, const uint32_t* __restrict__ block_prefix,
                     int32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * MARCH_BLOCK + threadIdx.x;
    const uint32_t f = (i < n && values[i] != 0u) ? 1u : 0u;
    uint32_t tot;
    const uint32_t pos = block_exclusive_scan(f, &tot) + block_prefix[blockIdx.x];
    if (f) out[pos] = (int32_t)i;
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

// Shared memory available for the coarse mip of the count pass (128^3 cells -> 32 KiB).
constexpr uint32_t MIP_SMEM_MAX = 48u * 1024u;
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
    TN_REQUIRE(march->dt_min > 0.0f && march->dt_max >= march->dt_min, TN_E_INVALID,
               "march: need 0 < dt_min <= dt_max (got %g, %g)", march->dt_min, march->dt_max);
    TN_REQUIRE(march->cone_angle >= 0.0f, TN_E_INVALID, "march: cone_angle must be >= 0");
    a.g = make_grid_view(*grid, bitfield);
    a.bbox = *bbox;
    a.cone = march->cone_angle;
    a.dt_min = march->dt_min;
    a.dt_max = march->dt_max;
    a.max_steps = march->max_steps;
    a.max_iters = march->max_iterations ? march->max_iterations : (1u << 22);
    return TN_OK;
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
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(ray_t_max); TN_NONNULL(alive);
    TN_NONNULL(n_steps); TN_NONNULL(batch_info);
    TN_REQUIRE(n_rays > 0, TN_E_NO_RAYS, "tn_march_count: n_rays = 0");
    TN_REQUIRE(ray_stride >= n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", ray_stride, n_rays);
    const uint32_t nb = (n_rays + MARCH_BLOCK - 1) / MARCH_BLOCK;
    st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    // coarse mip of the bitfield (staged in shared memory by the count pass)
    const uint32_t volume = (uint32_t)grid->resolution * grid->resolution * grid->resolution;
    const uint32_t mip_bytes = volume / 64;
    const bool use_mip = grid->resolution >= 8 && mip_bytes <= MIP_SMEM_MAX;
    if (use_mip) {
        st = ensure_mip(ctx, mip_bytes);
        if (st != TN_OK) return st;
        TN_REQUIRE(((uintptr_t)bitfield & 15u) == 0, TN_E_INVALID, "bitfield must be 16-byte aligned");
        build_mip_kernel<<<(mip_bytes + 255) / 256, 256, 0, stream>>>(mip_bytes, reinterpret_cast<const uint32_t*>(bitfield),
                                                                      ctx->mip);
        st = check_launch("tn_march_count(mip)");
        if (st != TN_OK) return st;
    }
    // per-ray step positions for the emit pass
    const uint32_t slot_cap = slot_capacity(n_rays, march->max_steps);
    st = ensure_slots(ctx, (size_t)n_rays * slot_cap);
    if (st != TN_OK) return st;
    ctx->slot_cap = slot_cap;
    ctx->slot_rays = n_rays;
    const size_t smem = use_mip ? mip_bytes : 0;
    count_kernel<true><<<nb, MARCH_BLOCK, smem, stream>>>(a, n_rays, n_rays_dev, ray_stride, ori, dir, ray_t, ray_t_max,
                                                          alive, n_steps, batch_size, batch_info, ctx->block_u32,
                                                          ctx->block_u32 + nb, ctx->tickets + TICKET_MARCH, ctx->flags,
                                                          use_mip ? ctx->mip : nullptr, use_mip ? mip_bytes : 0u,
                                                          ctx->slots, slot_cap);
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
    const uint32_t nb = (n_rays + MARCH_BLOCK - 1) / MARCH_BLOCK;
    TN_REQUIRE(ctx->block_u32_cap >= 2 * (size_t)nb && ctx->slot_rays == n_rays, TN_E_STATE,
               "tn_march_emit must follow tn_march_count on the same context with the same n_rays");
    SampleOut o{out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm, out_dt_norm, sample_stride};
    expand_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(a, inv_aabb_size, n_rays, nullptr, ray_stride, batch_info,
                                                  ctx->block_u32 + nb, ray_img_id, ori, dir, ray_t, alive, n_steps,
                                                  offsets, o, ctx->flags, ctx->slots, ctx->slot_cap);
    return check_launch("tn_march_emit");
}

int tn_scan_offsets(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                    uint32_t batch_size, uint32_t* batch_info) {
    TN_NONNULL(ctx); TN_NONNULL(counts); TN_NONNULL(offsets); TN_NONNULL(batch_info);
    TN_REQUIRE(n > 0, TN_E_NO_RAYS, "tn_scan_offsets: n = 0");
    const uint32_t nb = (n + MARCH_BLOCK - 1) / MARCH_BLOCK;
    int st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    MarchArgs a{};
    count_kernel<false><<<nb, MARCH_BLOCK, 0, stream>>>(a, n, nullptr, n, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                        const_cast<uint32_t*>(counts), batch_size, batch_info,
                                                        ctx->block_u32, ctx->block_u32 + nb,
                                                        ctx->tickets + TICKET_SCAN, ctx->flags, nullptr, 0u, nullptr,
                                                        0u);
    st = check_launch("tn_scan_offsets(count)");
    if (st != TN_OK) return st;
    SampleOut o{};
    emit_kernel<false><<<nb, MARCH_BLOCK, 0, stream>>>(a, 0.0f, n, nullptr, n, batch_info, ctx->block_u32 + nb,
                                                       nullptr, nullptr, nullptr, nullptr, nullptr, counts, offsets,
                                                       o, ctx->flags);
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
// Limit: at most TN_SCAN_NOALLOC_MAX_COUNTS counts per call (2 x 16,384 block entries =
// 128 KiB of scratch). Every call uses the same array, so two calls that overlap on the GPU
// (different streams, or different host threads on one device) race on it; serialise them.
constexpr uint32_t NOALLOC_MAX_BLOCKS = TN_SCAN_NOALLOC_MAX_COUNTS / MARCH_BLOCK;
constexpr uint32_t NOALLOC_WORDS = 2 * NOALLOC_MAX_BLOCKS + 64;  // [agg | prefix | ticket, flags, ...]
static __device__ __align__(256) uint32_t g_scan_noalloc_scratch[NOALLOC_WORDS];

// The array's name is a host-side stand-in in host code, not a device address: the device
// address is looked up once per device (with that device current) and cached here.
static uint32_t* g_scan_noalloc_ptr[64] = {};
static std::mutex g_scan_noalloc_mutex;

static int scan_noalloc_scratch(uint32_t** out) {
    int dev = 0;
    int st = cuda_status(cudaGetDevice(&dev), "tn_scan_offsets_noalloc: cudaGetDevice");
    if (st != TN_OK) return st;
    TN_REQUIRE(dev >= 0 && dev < 64, TN_E_INVALID, "tn_scan_offsets_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scan_noalloc_mutex);
    if (!g_scan_noalloc_ptr[dev]) {
        void* p = nullptr;
        st = cuda_status(cudaGetSymbolAddress(&p, g_scan_noalloc_scratch),
                         "tn_scan_offsets_noalloc: cudaGetSymbolAddress");
        if (st != TN_OK) return st;
        g_scan_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_scan_noalloc_ptr[dev];
    return TN_OK;
}

int tn_compact_nonzero(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* values, int32_t* out,
                       uint32_t* count_dev) {
    TN_NONNULL(ctx); TN_NONNULL(values); TN_NONNULL(out); TN_NONNULL(count_dev);
    if (n == 0) return cuda_status(cudaMemsetAsync(count_dev, 0, sizeof(uint32_t), stream), "tn_compact_nonzero");
    const uint32_t nb = (n + MARCH_BLOCK - 1) / MARCH_BLOCK;
    int st = ensure_block_u32(ctx, 2 * (size_t)nb);
    if (st != TN_OK) return st;
    compact_count_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, values, ctx->block_u32, ctx->block_u32 + nb, count_dev,
                                                          ctx->tickets + TICKET_COMPACT);
    st = check_launch("tn_compact_nonzero(count)");
    if (st != TN_OK) return st;
    compact_write_kernel<<<nb, MARCH_BLOCK, 0, stream>>>(n, values, ctx->block_u32 + nb, out);
    return check_launch("tn_compact_nonzero(write)");
}

int tn_scan_offsets_noalloc(tn_stream_t stream, uint32_t n, const uint32_t* counts, uint32_t* offsets,
                            uint32_t batch_size, uint32_t* batch_info) {
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
    MarchArgs a{};
    count_kernel<false><<<nb, MARCH_BLOCK, 0, stream>>>(a, n, nullptr, n, nullptr, nullptr, nullptr, nullptr, nullptr,
                                                        const_cast<uint32_t*>(counts), batch_size, batch_info,
                                                        block_agg, block_prefix, ticket, flags, nullptr, 0u, nullptr,
                                                        0u);
    st = check_launch("tn_scan_offsets_noalloc(count)");
    if (st != TN_OK) return st;
    SampleOut o{};
    emit_kernel<false><<<nb, MARCH_BLOCK, 0, stream>>>(a, 0.0f, n, nullptr, n, batch_info, block_prefix, nullptr,
                                                       nullptr, nullptr, nullptr, nullptr, counts, offsets, o, flags);
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
