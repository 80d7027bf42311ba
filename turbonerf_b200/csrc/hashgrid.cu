// Multiresolution hash-grid encoding (sm_100a): the upstream producer of sigma and rgb at the
// tiny-cuda-nn boundary of the reference (src/core/nerf-network.cu:27-124 builds tcnn's HashGrid
// with 16 levels of 2 features, 2^19 entries a level, base resolution 16 and per-level scale
// b = exp((ln 2048 A - ln 16) / 15), linear interpolation; its forward and backward run at
// :431-545 and :668-768). tcnn's source is not part of the reference tree, so this is the
// published algorithm (Mueller et al. 2022, "Instant neural graphics primitives with a
// multiresolution hash encoding", section 3):
//   level l has resolution N_l = floor(N_min b^l); a position x in [0,1]^3 falls in the cell
//   floor(x N_l) with in-cell coordinates f = x N_l - floor(x N_l); the level's feature vector is
//   the trilinear interpolation of the 8 corner vertices' entries; a vertex v indexes its entry
//   directly when the level's (N_l + 1)^3 vertices fit in the table (coarse levels), else by the
//   spatial hash (v_x * 1) xor (v_y * 2654435761) xor (v_z * 805459861) mod T.
// The backward scatters w_c * dL/dfeature into the corner entries' gradients (atomic adds) and
// records, once per entry, every entry a live sample touched: a bitmap and a list, which drive
// the gradient clearing before the next step (and tell which hash entries Adam will see).
//
// Layout: parameters [level][T][2] (one float2 per entry, level l at l T entries); features and
// their gradients [2 L][stride] (feature-major, coalesced per feature). The linear heads that
// stand in for tcnn's density and colour MLPs read the 2 L features of a sample:
//   density = b_s + w_s . f (raw network density; the losses apply the reference's exp
//   activation), rgb_c = sigmoid(b_c + W_c . f).
// Head parameters, after the hash entries: w_s[2L], b_s, then for c = r, g, b: W_c[2L], b_c.
#include <cmath>
#include <vector>

#include "tn_internal.cuh"

namespace tn {

constexpr int HG_F = 2;             // features a level
constexpr int HG_MAX_LEVELS = 16;   // levels
constexpr int HG_MAX_FEAT = HG_F * HG_MAX_LEVELS;

struct HashLevels {
    float scale[HG_MAX_LEVELS];     // N_l
    uint32_t res[HG_MAX_LEVELS];    // N_l
    uint32_t dense[HG_MAX_LEVELS];  // 1: the level's (N_l + 1)^3 vertices index their entries directly
    uint32_t n_levels;
    uint32_t log2_t;
};

// Per-level constants from the descriptor (host, double precision for b^l as the reference's
// host code computes b).
static int hash_levels(const tn_hashgrid_desc* d, HashLevels& H) {
    TN_REQUIRE(d != nullptr, TN_E_NULL, "hash-grid descriptor is NULL");
    TN_REQUIRE(d->n_levels >= 1 && d->n_levels <= (uint32_t)HG_MAX_LEVELS, TN_E_INVALID,
               "n_levels %u not in 1..%d", d->n_levels, HG_MAX_LEVELS);
    TN_REQUIRE(d->log2_hashmap_size >= 4 && d->log2_hashmap_size <= 24, TN_E_INVALID,
               "log2_hashmap_size %u not in 4..24", d->log2_hashmap_size);
    TN_REQUIRE(d->base_resolution >= 1.0f && d->per_level_scale >= 1.0f, TN_E_INVALID,
               "base_resolution and per_level_scale must be at least 1");
    const double T = (double)(1u << d->log2_hashmap_size);
    H.n_levels = d->n_levels;
    H.log2_t = d->log2_hashmap_size;
    for (uint32_t l = 0; l < (uint32_t)HG_MAX_LEVELS; ++l) {
        const double n = l < d->n_levels ? std::floor((double)d->base_resolution *
                                                      std::pow((double)d->per_level_scale, (double)l))
                                         : 1.0;
        TN_REQUIRE(n >= 1.0 && n < 16777216.0, TN_E_INVALID, "level %u resolution %.0f out of range", l, n);
        H.res[l] = (uint32_t)n;
        H.scale[l] = (float)n;
        H.dense[l] = (n + 1.0) * (n + 1.0) * (n + 1.0) <= T ? 1u : 0u;
    }
    return TN_OK;
}

__device__ __forceinline__ uint32_t hg_index(const HashLevels& H, int l, uint32_t x, uint32_t y, uint32_t z) {
    if (H.dense[l]) {
        const uint32_t r = H.res[l] + 1u;
        return x + r * (y + r * z);
    }
    return ((x * 1u) ^ (y * 2654435761u) ^ (z * 805459861u)) & ((1u << H.log2_t) - 1u);
}

// Cell and in-cell coordinate of one coordinate at a level; the cell is clamped to [0, N - 1],
// so that its upper corner is a vertex of the level (a coordinate of exactly 1 has f = 1).
__device__ __forceinline__ void hg_cell(float p, float scale, uint32_t res, uint32_t& i, float& f) {
    const float s = __fmul_rn(p, scale);
    const float fl = fminf(fmaxf(floorf(s), 0.0f), (float)(res - 1u));
    i = (uint32_t)fl;
    f = __fsub_rn(s, fl);
}

// Corner c (bit 0: x + 1, bit 1: y + 1, bit 2: z + 1) of a cell: its entry and trilinear weight
// ((w_x w_y) w_z, each 1 - f or f).
struct HashCorners {
    uint32_t idx[8];
    float w[8];
};

__device__ __forceinline__ void hg_corners(const HashLevels& H, int l, float px, float py, float pz, HashCorners& c) {
    uint32_t ix, iy, iz;
    float fx, fy, fz;
    hg_cell(px, H.scale[l], H.res[l], ix, fx);
    hg_cell(py, H.scale[l], H.res[l], iy, fy);
    hg_cell(pz, H.scale[l], H.res[l], iz, fz);
    const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy), gz = __fsub_rn(1.0f, fz);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
        c.idx[k] = hg_index(H, l, ix + bx, iy + by, iz + bz);
        c.w[k] = __fmul_rn(__fmul_rn(bx ? fx : gx, by ? fy : gy), bz ? fz : gz);
    }
}

__device__ __forceinline__ uint32_t live_count(uint32_t n, const uint32_t* n_dev) {
    return n_dev ? min(*n_dev, n) : n;
}

// One thread per (sample, level): the level's two features, sum over the corners in order of
// w_c * entry (fused multiply-adds).
__global__ void __launch_bounds__(256)
hg_encode_kernel(HashLevels H, uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t pstride, uint32_t stride,
                 const float* __restrict__ pos, const float2* __restrict__ params, float* __restrict__ feat) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (s >= live_count(n, n_dev)) return;
    HashCorners c;
    hg_corners(H, l, pos[s], pos[s + pstride], pos[s + 2 * (size_t)pstride], c);
    const float2* P = params + ((size_t)l << H.log2_t);
    float2 v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = __ldg(P + c.idx[k]);
    float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        a0 = __fmaf_rn(c.w[k], v[k].x, a0);
        a1 = __fmaf_rn(c.w[k], v[k].y, a1);
    }
    feat[(size_t)(HG_F * l) * stride + s] = a0;
    feat[(size_t)(HG_F * l + 1) * stride + s] = a1;
}

// One thread per (sample, level): w_c * dL/dfeature into the corners' entries; each entry a live
// sample touches is listed once (the thread whose atomic or set the entry's bit appends l T + idx).
// Contention is cut three ways: a bit already set is seen with a plain read and skips its atomic;
// the warp's new entries take one counter atomic for the warp; and on levels of resolution up to
// HG_SHARE_RES, where neighbouring samples (consecutive along a ray) share corners, the lanes of a
// warp with the same entry add their contributions in shared memory and one of them makes the
// atomic add.
constexpr int HG_BWD_THREADS = 256;
constexpr uint32_t HG_SHARE_RES = 8192;
__global__ void __launch_bounds__(HG_BWD_THREADS)
hg_backward_kernel(HashLevels H, uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t pstride, uint32_t stride,
                   const float* __restrict__ pos, const float* __restrict__ dfeat, float2* __restrict__ grads,
                   uint32_t* __restrict__ bits, uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
    __shared__ float2 share[HG_BWD_THREADS];
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const bool live = s < live_count(n, n_dev);
    const unsigned active = __ballot_sync(FULL_MASK, live);  // the warp's lanes that continue together
    if (!live) return;
    HashCorners c;
    hg_corners(H, l, pos[s], pos[s + pstride], pos[s + 2 * (size_t)pstride], c);
    const float g0 = dfeat[(size_t)(HG_F * l) * stride + s], g1 = dfeat[(size_t)(HG_F * l + 1) * stride + s];
    const uint32_t base = (uint32_t)l << H.log2_t;
    const bool share_level = H.res[l] <= HG_SHARE_RES;  // the same for the whole block
    // the gradient adds of all 8 corners (reductions without a result: nothing waits for them)
    bool lead[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float2 v = make_float2(__fmul_rn(c.w[k], g0), __fmul_rn(c.w[k], g1));
        lead[k] = true;
        if (share_level) {
            const unsigned peers = __match_any_sync(active, c.idx[k]);
            share[threadIdx.x] = v;
            __syncwarp(active);
            lead[k] = lane == __ffs(peers) - 1;
            if (lead[k]) {
                for (unsigned rest = peers & (peers - 1u); rest; rest &= rest - 1u) {
                    const float2 o = share[(threadIdx.x & ~31u) + (uint32_t)(__ffs(rest) - 1)];
                    v.x += o.x;
                    v.y += o.y;
                }
            }
            __syncwarp(active);
        }
        if (lead[k]) atomicAdd(grads + base + c.idx[k], v);
    }
    if (!bits) return;
    // touched entries: every corner's bitmap word read at once, then the atomic ors of the bits
    // still clear, then one counter atomic for the warp's new entries of all 8 corners
    uint32_t e[8], word[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        e[k] = base + c.idx[k];
        word[k] = lead[k] ? bits[e[k] >> 5] : ~0u;
    }
    bool fresh[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t bit = 1u << (e[k] & 31u);
        fresh[k] = !(word[k] & bit) && !(atomicOr(bits + (e[k] >> 5), bit) & bit);
    }
    unsigned news[8];
    uint32_t total = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        news[k] = __ballot_sync(active, fresh[k]);
        total += (uint32_t)__popc(news[k]);
    }
    if (total == 0) return;
    const int first = __ffs(active) - 1;
    uint32_t at = 0;
    if (lane == first) at = atomicAdd(count, total);
    at = __shfl_sync(active, at, first);
    const unsigned below = (1u << lane) - 1u;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (fresh[k]) list[at + (uint32_t)__popc(news[k] & below)] = e[k];
        at += (uint32_t)__popc(news[k]);
    }
}

// Zeroes the listed entries' gradients and bitmap words (several entries may share a word; all
// write zero).
__global__ void hg_clear_kernel(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count, uint32_t max,
                                float2* __restrict__ grads, uint32_t* __restrict__ bits) {
    const uint32_t nl = min(*count, max);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += gridDim.x * blockDim.x) {
        const uint32_t e = list[k];
        grads[e] = make_float2(0.0f, 0.0f);
        if (bits) bits[e >> 5] = 0u;
    }
}

// Entries with a nonzero gradient (either feature), listed in no particular order: each thread
// takes 8 consecutive entries (four 16-byte loads), a block ranks its nonzero entries with a scan of
// the warps' counts and takes their places with one counter atomic.
constexpr int HG_NZ_THREADS = 256;
__global__ void __launch_bounds__(HG_NZ_THREADS)
hg_nonzero_kernel(uint32_t n_entries, const float4* __restrict__ grads, uint32_t* __restrict__ list,
                  uint32_t* __restrict__ count) {
    __shared__ uint32_t warp_n[HG_NZ_THREADS / WARP];
    __shared__ uint32_t block_at;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t e0 = (blockIdx.x * HG_NZ_THREADS + threadIdx.x) * 8u;
    uint32_t mask = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        if (e0 + 2u * q < n_entries) {  // n_entries is even: the pair's second entry exists too
            const float4 v = grads[e0 / 2u + q];
            if (v.x != 0.0f || v.y != 0.0f) mask |= 1u << (2 * q);
            if (v.z != 0.0f || v.w != 0.0f) mask |= 1u << (2 * q + 1);
        }
    }
    const uint32_t mine = (uint32_t)__popc(mask);
    uint32_t incl = mine;
#pragma unroll
    for (int d = 1; d < WARP; d <<= 1) {
        const uint32_t o = __shfl_up_sync(FULL_MASK, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == WARP - 1) warp_n[wid] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < HG_NZ_THREADS / WARP; ++w) {
            const uint32_t c = warp_n[w];
            warp_n[w] = t;
            t += c;
        }
        block_at = t ? atomicAdd(count, t) : 0u;
    }
    __syncthreads();
    uint32_t at = block_at + warp_n[wid] + incl - mine;
    for (uint32_t m = mask; m; m &= m - 1u) list[at++] = e0 + (uint32_t)(__ffs(m) - 1);
}

// ---- linear heads (the stand-in for tcnn's density and colour MLPs) ------------------------
__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

// One thread per sample: raw density and rgb ([3][ostride]) from the 2 L features ([2L][stride]).
__global__ void __launch_bounds__(256)
hg_heads_forward_kernel(uint32_t nf, uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t stride,
                        const float* __restrict__ feat, const float* __restrict__ head, float* __restrict__ density,
                        float* __restrict__ rgb, uint32_t ostride) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= live_count(n, n_dev)) return;
    float z[4];
#pragma unroll
    for (int o = 0; o < 4; ++o) z[o] = __ldg(head + o * (nf + 1) + nf);
    for (uint32_t j = 0; j < nf; ++j) {
        const float f = feat[(size_t)j * stride + s];
#pragma unroll
        for (int o = 0; o < 4; ++o) z[o] = fmaf(__ldg(head + o * (nf + 1) + j), f, z[o]);
    }
    density[s] = z[0];
    if (rgb) {
#pragma unroll
        for (int c = 0; c < 3; ++c) rgb[(size_t)c * ostride + s] = sigmoid(z[c + 1]);
    }
}

// One thread per sample: dL/dfeature (written) and the heads' parameter gradients, summed over
// the block into partials[block][4][HG_MAX_FEAT + 1] (head o's weights j < nf, then its bias at
// HG_MAX_FEAT; deterministic: fixed lanes, fixed warps).
constexpr int HG_HEAD_THREADS = 256;
constexpr int HG_HEAD_SLOTS = 4 * (HG_MAX_FEAT + 1);
__global__ void __launch_bounds__(HG_HEAD_THREADS)
hg_heads_backward_kernel(uint32_t nf, uint32_t n, const uint32_t* __restrict__ n_dev, uint32_t stride,
                         const float* __restrict__ feat, const float* __restrict__ head,
                         const float* __restrict__ dL_ddensity, const float* __restrict__ dL_drgb,
                         float* __restrict__ dfeat, float* __restrict__ partials) {
    __shared__ float rows[HG_HEAD_THREADS * (HG_MAX_FEAT + 1)];
    __shared__ float runs[HG_HEAD_THREADS];
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool live = s < live_count(n, n_dev);
    float f[HG_MAX_FEAT];
    float dz[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < HG_MAX_FEAT; ++j) f[j] = live && j < (int)nf ? feat[(size_t)j * stride + s] : 0.0f;
    if (live) {
        float z[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            z[c] = __ldg(head + (c + 1) * (nf + 1) + nf);
#pragma unroll
            for (int j = 0; j < HG_MAX_FEAT; ++j)
                if (j < (int)nf) z[c] = fmaf(__ldg(head + (c + 1) * (nf + 1) + j), f[j], z[c]);
        }
        dz[0] = dL_ddensity[s];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float y = sigmoid(z[c]);
            dz[c + 1] = dL_drgb[(size_t)c * stride + s] * y * (1.0f - y);
        }
#pragma unroll
        for (int j = 0; j < HG_MAX_FEAT; ++j) {
            if (j < (int)nf) {
                float g = 0.0f;
#pragma unroll
                for (int o = 0; o < 4; ++o) g = fmaf(dz[o], __ldg(head + o * (nf + 1) + j), g);
                dfeat[(size_t)j * stride + s] = g;
            }
        }
    }
    // the block's sums of dz_o f_j and dz_o, one head at a time: each thread's 33 values to a shared
    // row; 7 groups of threads sum each column over a run of rows; 33 threads add the runs (the
    // order is fixed)
    constexpr int NC = HG_MAX_FEAT + 1;
    constexpr int NG = HG_HEAD_THREADS / NC, RPG = (HG_HEAD_THREADS + NG - 1) / NG;
#pragma unroll
    for (int o = 0; o < 4; ++o) {
#pragma unroll
        for (int j = 0; j < NC; ++j) rows[threadIdx.x * NC + j] = j < HG_MAX_FEAT ? dz[o] * f[j] : dz[o];
        __syncthreads();
        if (threadIdx.x < NG * NC) {
            const int c = threadIdx.x % NC, g = threadIdx.x / NC;
            float v = 0.0f;
            for (int t = g * RPG; t < min((g + 1) * RPG, HG_HEAD_THREADS); ++t) v += rows[t * NC + c];
            runs[g * NC + c] = v;
        }
        __syncthreads();
        if (threadIdx.x < NC) {
            float v = 0.0f;
            for (int g = 0; g < NG; ++g) v += runs[g * NC + threadIdx.x];
            partials[(size_t)blockIdx.x * HG_HEAD_SLOTS + o * NC + threadIdx.x] = v;
        }
        __syncthreads();
    }
    (void)lane;
    (void)wid;
}

// The heads' gradients (head o, weight j < nf at o (nf + 1) + j, bias at o (nf + 1) + nf): one
// block a parameter sums the blocks' partials, each thread a strided run of them, then a fixed tree
// over the threads (deterministic).
constexpr int HG_FINISH_THREADS = 256;
__global__ void __launch_bounds__(HG_FINISH_THREADS)
hg_heads_grad_finish_kernel(uint32_t nf, uint32_t n_blocks, const float* __restrict__ partials,
                            float* __restrict__ grads) {
    __shared__ float warp_s[HG_FINISH_THREADS / WARP];
    const uint32_t k = blockIdx.x;
    const uint32_t o = k / (nf + 1), j = k % (nf + 1);
    const uint32_t slot = o * (HG_MAX_FEAT + 1) + (j < nf ? j : (uint32_t)HG_MAX_FEAT);
    float v = 0.0f;
    for (uint32_t b = threadIdx.x; b < n_blocks; b += HG_FINISH_THREADS) v += partials[(size_t)b * HG_HEAD_SLOTS + slot];
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) warp_s[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < HG_FINISH_THREADS / WARP; ++w) t += warp_s[w];
        grads[k] = t;
    }
}

int hashgrid_encode(cudaStream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                    uint32_t pstride, uint32_t stride, const float* pos, const float* params, float* features) {
    HashLevels H;
    int st = hash_levels(desc, H);
    if (st != TN_OK || n == 0) return st;
    const dim3 grid((n + 255) / 256, H.n_levels);
    hg_encode_kernel<<<grid, 256, 0, stream>>>(H, n, n_dev, pstride, stride, pos,
                                               reinterpret_cast<const float2*>(params), features);
    return check_launch("tn_hashgrid_encode");
}

int hashgrid_backward(cudaStream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                      uint32_t pstride, uint32_t stride, const float* pos, const float* dL_dfeatures, float* grads,
                      uint32_t* touched_bits, uint32_t* touched_list, uint32_t* touched_count) {
    HashLevels H;
    int st = hash_levels(desc, H);
    if (st != TN_OK || n == 0) return st;
    const dim3 grid((n + HG_BWD_THREADS - 1) / HG_BWD_THREADS, H.n_levels);
    hg_backward_kernel<<<grid, HG_BWD_THREADS, 0, stream>>>(H, n, n_dev, pstride, stride, pos, dL_dfeatures,
                                                 reinterpret_cast<float2*>(grads), touched_bits, touched_list,
                                                 touched_count);
    return check_launch("tn_hashgrid_backward");
}

int hashgrid_clear_touched(cudaStream_t stream, const uint32_t* touched_list, const uint32_t* touched_count,
                           uint32_t max_entries, float* grads, uint32_t* touched_bits) {
    hg_clear_kernel<<<num_sms() * 4, 256, 0, stream>>>(touched_list, touched_count, max_entries,
                                                       reinterpret_cast<float2*>(grads), touched_bits);
    int st = check_launch("tn_hashgrid_clear_touched");
    if (st == TN_OK)
        st = cuda_status(cudaMemsetAsync(const_cast<uint32_t*>(touched_count), 0, sizeof(uint32_t), stream),
                         "tn_hashgrid_clear_touched: count");
    return st;
}

// ---- the hash-grid network behind tn_network ------------------------------------------------
struct HashNet {
    tn_hashgrid_desc desc{};
    uint32_t n_features = 0;     // 2 L
    uint64_t n_hash = 0;         // hash parameters (floats): L T 2
    const float* params = nullptr;  // [hash | heads]
    float* feat = nullptr;       // [2L][cap] features of the last forward
    float* dfeat = nullptr;      // [2L][cap]
    float* qfeat = nullptr;      // [2L][qcap] features of density queries
    float* partials = nullptr;   // [blocks][HG_HEAD_SLOTS]
    uint32_t* list = nullptr;    // [L T]
    uint32_t* count = nullptr;   // [1]
    uint32_t cap = 0, qcap = 0;
    ~HashNet() {
        cudaFree(feat); cudaFree(dfeat); cudaFree(qfeat); cudaFree(partials);
        cudaFree(list); cudaFree(count);
    }
};

static const float* head_params(const HashNet* h) { return h->params + h->n_hash; }

static int hashnet_forward(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                           const float* pos, const float* /*dir*/, float* density, float* rgb) {
    auto* h = static_cast<HashNet*>(user);
    cudaStream_t s = (cudaStream_t)stream;
    TN_REQUIRE(n <= h->cap && stride >= n, TN_E_INVALID, "hash-grid network: %u samples past its %u", n, h->cap);
    int st = hashgrid_encode(s, &h->desc, n, n_dev, stride, h->cap, pos, h->params, h->feat);
    if (st != TN_OK || n == 0) return st;
    hg_heads_forward_kernel<<<(n + 255) / 256, 256, 0, s>>>(h->n_features, n, n_dev, h->cap, h->feat,
                                                            head_params(h), density, rgb, stride);
    return check_launch("hash-grid network forward");
}

static int hashnet_density(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                           const float* pos, float* density) {
    auto* h = static_cast<HashNet*>(user);
    cudaStream_t s = (cudaStream_t)stream;
    TN_REQUIRE(n <= h->qcap && stride >= n, TN_E_INVALID, "hash-grid density: %u queries past its %u", n,
               h->qcap);
    int st = hashgrid_encode(s, &h->desc, n, n_dev, stride, h->qcap, pos, h->params, h->qfeat);
    if (st != TN_OK || n == 0) return st;
    hg_heads_forward_kernel<<<(n + 255) / 256, 256, 0, s>>>(h->n_features, n, n_dev, h->qcap, h->qfeat,
                                                            head_params(h), density, nullptr, stride);
    return check_launch("hash-grid network density");
}

static int hashnet_backward(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                            const float* pos, const float* /*dir*/, const float* dL_ddensity, const float* dL_drgb,
                            float* param_grads) {
    auto* h = static_cast<HashNet*>(user);
    cudaStream_t s = (cudaStream_t)stream;
    // the previous step's hash gradients (Adam has read them): a step touches most entries of the
    // fine levels, so one whole-array clear writes less than the entries' scattered sectors would
    const uint64_t entries = h->n_hash / HG_F;
    int st = cuda_status(cudaMemsetAsync(param_grads, 0, h->n_hash * sizeof(float), s), "hash-grid gradients");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(h->count, 0, sizeof(uint32_t), s), "hash-grid count");
    if (st != TN_OK || n == 0) return st;
    const uint32_t blocks = (n + HG_HEAD_THREADS - 1) / HG_HEAD_THREADS;
    hg_heads_backward_kernel<<<blocks, HG_HEAD_THREADS, 0, s>>>(h->n_features, n, n_dev, stride, h->feat,
                                                                head_params(h), dL_ddensity, dL_drgb, h->dfeat,
                                                                h->partials);
    st = check_launch("hash-grid heads backward");
    if (st != TN_OK) return st;
    hg_heads_grad_finish_kernel<<<4 * (h->n_features + 1), HG_FINISH_THREADS, 0, s>>>(h->n_features, blocks,
                                                                                      h->partials,
                                                                                      param_grads + h->n_hash);
    st = check_launch("hash-grid heads gradients");
    if (st != TN_OK) return st;
    st = hashgrid_backward(s, &h->desc, n, n_dev, stride, h->cap, pos, h->dfeat, param_grads, nullptr, nullptr,
                           nullptr);
    if (st != TN_OK) return st;
    // the entries Adam will update: those with a nonzero gradient
    const uint32_t nz_blocks = (uint32_t)((entries + 8ull * HG_NZ_THREADS - 1) / (8ull * HG_NZ_THREADS));
    hg_nonzero_kernel<<<nz_blocks, HG_NZ_THREADS, 0, s>>>((uint32_t)entries, reinterpret_cast<const float4*>(param_grads),
                                                          h->list, h->count);
    return check_launch("hash-grid nonzero entries");
}

// A network over the parameters `params` ([hash entries | heads]) for batches of up to `cap`
// samples (positions with that stride) and density queries of up to `qcap`.
int hashnet_create(const tn_hashgrid_desc* desc, const float* params, uint32_t cap, uint32_t qcap, tn_network* out,
                   void** handle) {
    HashLevels H;
    int st = hash_levels(desc, H);
    if (st != TN_OK) return st;
    auto* h = new HashNet();
    h->desc = *desc;
    h->n_features = HG_F * desc->n_levels;
    h->n_hash = (uint64_t)desc->n_levels << (desc->log2_hashmap_size + 1);
    h->params = params;
    h->cap = cap;
    h->qcap = std::max(qcap, 1u);
    const uint64_t entries = h->n_hash / HG_F;
    const uint32_t blocks = (cap + HG_HEAD_THREADS - 1) / HG_HEAD_THREADS;
    st = cuda_status(cudaMalloc(&h->feat, (size_t)h->n_features * cap * sizeof(float)), "hash-grid features");
    if (st == TN_OK) st = cuda_status(cudaMalloc(&h->dfeat, (size_t)h->n_features * cap * sizeof(float)), "hash-grid dfeat");
    if (st == TN_OK)
        st = cuda_status(cudaMalloc(&h->qfeat, (size_t)h->n_features * h->qcap * sizeof(float)), "hash-grid query features");
    if (st == TN_OK)
        st = cuda_status(cudaMalloc(&h->partials, (size_t)std::max(blocks, 1u) * HG_HEAD_SLOTS * sizeof(float)),
                         "hash-grid partials");
    if (st == TN_OK) st = cuda_status(cudaMalloc(&h->list, (size_t)entries * sizeof(uint32_t)), "hash-grid list");
    if (st == TN_OK) st = cuda_status(cudaMalloc(&h->count, sizeof(uint32_t)), "hash-grid count");
    if (st == TN_OK) st = cuda_status(cudaMemset(h->count, 0, sizeof(uint32_t)), "hash-grid count");
    if (st != TN_OK) {
        delete h;
        return st;
    }
    out->user = h;
    out->activation = TN_ACT_DENSITY;
    out->forward = hashnet_forward;
    out->backward = hashnet_backward;
    out->density = hashnet_density;
    *handle = h;
    return TN_OK;
}

void hashnet_destroy(void* handle) { delete static_cast<HashNet*>(handle); }

// Entries with a nonzero gradient after the last backward (device count, and *list: the
// entries, in no particular order), for inspection and tests.
const uint32_t* hashnet_touched(void* handle, const uint32_t** list) {
    auto* h = static_cast<HashNet*>(handle);
    if (list) *list = h->list;
    return h->count;
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_hashgrid_n_params(const tn_hashgrid_desc* desc, uint64_t* n_hash, uint32_t* n_head) {
    HashLevels H;
    int st = hash_levels(desc, H);
    if (st != TN_OK) return st;
    if (n_hash) *n_hash = (uint64_t)desc->n_levels << (desc->log2_hashmap_size + 1);
    if (n_head) *n_head = 4 * (HG_F * desc->n_levels + 1);
    return TN_OK;
}

int tn_hashgrid_level_resolution(const tn_hashgrid_desc* desc, uint32_t level, uint32_t* resolution,
                                 int* dense) {
    HashLevels H;
    int st = hash_levels(desc, H);
    if (st != TN_OK) return st;
    TN_REQUIRE(level < desc->n_levels, TN_E_INVALID, "level %u past %u", level, desc->n_levels);
    if (resolution) *resolution = H.res[level];
    if (dense) *dense = (int)H.dense[level];
    return TN_OK;
}

int tn_hashgrid_encode(tn_stream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                       uint32_t stride, const float* pos, const float* params, float* features) {
    TN_NONNULL(pos); TN_NONNULL(params); TN_NONNULL(features);
    TN_REQUIRE(stride >= n, TN_E_INVALID, "stride %u < n %u", stride, n);
    return hashgrid_encode((cudaStream_t)stream, desc, n, n_dev, stride, stride, pos, params, features);
}

int tn_hashgrid_backward(tn_stream_t stream, const tn_hashgrid_desc* desc, uint32_t n, const uint32_t* n_dev,
                         uint32_t stride, const float* pos, const float* dL_dfeatures, float* grads,
                         uint32_t* touched_bits, uint32_t* touched_list, uint32_t* touched_count) {
    TN_NONNULL(pos); TN_NONNULL(dL_dfeatures); TN_NONNULL(grads);
    TN_REQUIRE(stride >= n, TN_E_INVALID, "stride %u < n %u", stride, n);
    TN_REQUIRE((touched_bits == nullptr) == (touched_list == nullptr) &&
                   (touched_list == nullptr) == (touched_count == nullptr),
               TN_E_INVALID, "touched_bits, touched_list and touched_count go together");
    return hashgrid_backward((cudaStream_t)stream, desc, n, n_dev, stride, stride, pos, dL_dfeatures, grads,
                             touched_bits, touched_list, touched_count);
}

int tn_hashgrid_clear_touched(tn_stream_t stream, const uint32_t* touched_list, const uint32_t* touched_count,
                              uint32_t max_entries, float* grads, uint32_t* touched_bits) {
    TN_NONNULL(touched_list); TN_NONNULL(touched_count); TN_NONNULL(grads);
    return hashgrid_clear_touched((cudaStream_t)stream, touched_list, touched_count, max_entries, grads,
                                  touched_bits);
}

}  // extern "C"
