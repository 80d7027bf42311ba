// Volume-rendering compositor, reconstruction loss and mip-NeRF 360 distortion loss,
// forward and backward (sm_100a).
//
// Layout: one warp per ray (grid-stride over rays, static assignment so reductions are
// deterministic); the ray's samples are walked in chunks of 32, one sample per lane, with
// coalesced loads of the structure-of-arrays inputs. Running quantities along the ray
// (optical depth, weight sums) are warp-shuffle prefix scans carried across chunks.
//
// Backward passes walk the chunks from the last to the first and obtain every suffix sum
// (sum over later samples) by a reverse scan, instead of subtracting a running prefix from
// the ray total as the reference does (src/utils/training-kernels-fused.cuh:204-208, 310-313).
// Compositor transmittance is recomputed in the backward from the saved per-ray optical
// depth S and the reverse scan of sigma*dt: T_{j+1} = exp(-(S - sum_{i>j} x_i)). No
// per-sample transmittance or weight is stored between forward and backward.
//
// The distortion loss runs without a transmittance cut, so its optical depth can be large;
// its prefix quantities are therefore recomputed in the forward direction from per-chunk
// carries (held in lane registers for the first 64 chunks) rather than by subtraction.
#include <thrust/device_ptr.h>
#include <thrust/execution_policy.h>
#include <thrust/reduce.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>

#include "tn_internal.cuh"

namespace tn {

constexpr int LOSS_WARPS = 8;
constexpr int LOSS_THREADS = LOSS_WARPS * WARP;
constexpr int SAVED_TILES = 64;  // distortion tile carries kept in lane registers (2 per lane)

__device__ __forceinline__ float act_sigma(int act, float d) { return act == 0 ? d : expf(fminf(d, 12.0f) - 1.0f); }
__device__ __forceinline__ float act_dsigma(int act, float sigma) { return act == 0 ? 1.0f : sigma; }

// 1 - exp(-x) for x >= 0 (the opacity of a sample with optical depth x), without a branch: below
// 1/4, x times the first eight terms of (1 - e^-x)/x = sum_k (-x)^k / (k+1)! in Horner form (the
// truncation is below 5e-11 of the result); above, 1 - e^-x from the fast exponential, free of
// cancellation there (its relative error is a few 1e-7). Both are evaluated and one selected.
__device__ __forceinline__ float opacity(float x) {
    float p = fmaf(x, -1.0f / 40320.0f, 1.0f / 5040.0f);
    p = fmaf(p, x, -1.0f / 720.0f);
    p = fmaf(p, x, 1.0f / 120.0f);
    p = fmaf(p, x, -1.0f / 24.0f);
    p = fmaf(p, x, 1.0f / 6.0f);
    p = fmaf(p, x, -0.5f);
    p = fmaf(p, x, 1.0f);
    const float big = 1.0f - __expf(-x);
    return x < 0.25f ? x * p : big;
}

// Exclusive value from an inclusive warp scan: lane 0 gets `carry`.
__device__ __forceinline__ float shift_up(float incl, int lane, float carry) {
    const float v = __shfl_up_sync(FULL_MASK, incl, 1);
    return lane == 0 ? carry : v;
}
// Exclusive value from an inclusive suffix scan: lane 31 gets `carry`.
__device__ __forceinline__ float shift_down(float incl, int lane, float carry) {
    const float v = __shfl_down_sync(FULL_MASK, incl, 1);
    return lane == WARP - 1 ? carry : v;
}

struct Samples {
    const float* __restrict__ density;
    const float* __restrict__ rgb;
    const float* __restrict__ dt;
    const float* __restrict__ m_norm;
    const float* __restrict__ dt_norm;
    const float* __restrict__ t;
    uint32_t ss;
    int act;
};

// Per-ray result of the compositor forward.
struct CompFwd {
    float r, g, b, a;
    float depth;   // optical depth up to and including the last composited sample
    uint32_t used; // samples composited (reference: loop index at the transmittance break + 1)
};

// ---- register-blocked compositor -----------------------------------------------------------
// A ray is processed in blocks of 32 * K samples, lane l owning the K consecutive samples
// [base + K l, base + K l + K). Each running sum along the ray is a prefix (or suffix) inside the
// lane plus one warp scan of the 32 lane totals, so the warp scans once per 32 * K samples, not
// once per 32: a few instructions per sample instead of one full warp scan per sample and sum.
constexpr int CB_K = 4;

// density_to_ray_rgba_forward, src/utils/training-kernels-fused.cuh:227-264, with
// T_j = exp(-sum_{i<j} sigma_i dt_i) and alpha_j = -expm1(-sigma_j dt_j). Sample j is
// composited while T_j >= min_t, i.e. up to and including the first sample after which
// the transmittance drops below min_t.
template <int K>
__device__ CompFwd composite_forward_ray(const Samples& S, uint32_t o, uint32_t n, float min_t, int lane,
                                         float* __restrict__ t_out = nullptr, float* __restrict__ w_out = nullptr) {
    float carry = 0.0f;  // optical depth before the current block
    float ar = 0.0f, ag = 0.0f, ab = 0.0f, aa = 0.0f;
    CompFwd out;
    out.used = n;
    out.depth = 0.0f;
    bool done = false;
    for (uint32_t base = 0; base < n && !done; base += WARP * K) {
        const uint32_t j0 = base + (uint32_t)lane * K;
        float x[K], cr[K], cg[K], cb[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            x[q] = cr[q] = cg[q] = cb[q] = 0.0f;
            if (j0 + q < n) {
                const size_t s = (size_t)o + j0 + q;
                x[q] = act_sigma(S.act, S.density[s]) * S.dt[s];
                cr[q] = S.rgb[s];
                cg[q] = S.rgb[s + S.ss];
                cb[q] = S.rgb[s + 2 * (size_t)S.ss];
            }
        }
        float run = 0.0f, d[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            run += x[q];
            d[q] = run;
        }
        const float lane_incl = warp_inclusive_sum(run, lane);
        const float before = shift_up(lane_incl, lane, 0.0f) + carry;  // depth before the lane's first sample
        float tprev = expf(-before), tn[K], w[K];
        int fq = K;  // the lane's first sample after which T < min_t
#pragma unroll
        for (int q = 0; q < K; ++q) {
            d[q] += before;
            tn[q] = expf(-d[q]);
            w[q] = tprev * -expm1f(-x[q]);
            if (fq == K && j0 + q < n && tn[q] < min_t) fq = q;
            tprev = tn[q];
        }
        const unsigned term = __ballot_sync(FULL_MASK, fq < K);
        const int fl = term ? __ffs(term) - 1 : WARP;
        const int last_q = lane < fl ? K - 1 : (lane == fl ? fq : -1);
        float dsel = 0.0f;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            if (q == fq) dsel = d[q];
            if (q <= last_q && j0 + q < n) {
                ar += w[q] * cr[q];
                ag += w[q] * cg[q];
                ab += w[q] * cb[q];
                aa += w[q];
                if (t_out) {
                    t_out[(size_t)o + j0 + q] = tn[q];  // transmittance after the sample
                    w_out[(size_t)o + j0 + q] = w[q];
                }
            }
        }
        if (term) {
            out.used = base + (uint32_t)fl * K + (uint32_t)__shfl_sync(FULL_MASK, fq, fl) + 1u;
            out.depth = __shfl_sync(FULL_MASK, dsel, fl);
            done = true;
        } else {
            carry += __shfl_sync(FULL_MASK, lane_incl, WARP - 1);
        }
    }
    if (!done) out.depth = carry;
    out.r = warp_sum(ar);
    out.g = warp_sum(ag);
    out.b = warp_sum(ab);
    out.a = warp_sum(aa);
    return out;
}

// Reverse-scan vector-Jacobian product of the compositor for one ray over samples
// [0, used): dL/dsigma_j = dt_j * sum_c g_c (T_{j+1} c_j - sum_{i>j} w_i c_i)
//                        + dt_j * g_a (T_{j+1} - sum_{i>j} w_i);   dL/dc_j = cscale * g_c * w_j,
// with T rebuilt from the forward's optical depth `depth` minus suffix sums of sigma dt.
// The callback `emit(j, valid, dsigma_density, drgb_r, drgb_g, drgb_b)` consumes each sample's
// gradients (dsigma already multiplied by d sigma / d input), blocks from the last one down.
template <int K, typename Emit>
__device__ __forceinline__ void composite_vjp_ray(const Samples& S, uint32_t o, uint32_t used, float depth, float gr,
                                                  float gg, float gb, float ga, float cscale, int lane, Emit&& emit) {
    if (used == 0) return;
    float sx = 0.0f, sr = 0.0f, sg = 0.0f, sb = 0.0f, sa = 0.0f;  // sums over the later blocks
    const uint32_t span = WARP * K;
    for (int64_t base = (int64_t)((used - 1) / span) * span; base >= 0; base -= span) {
        const uint32_t j0 = (uint32_t)base + (uint32_t)lane * K;
        float x[K], cr[K], cg[K], cb[K], dtv[K], sig[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            x[q] = cr[q] = cg[q] = cb[q] = dtv[q] = sig[q] = 0.0f;
            if (j0 + q < used) {
                const size_t s = (size_t)o + j0 + q;
                sig[q] = act_sigma(S.act, S.density[s]);
                dtv[q] = S.dt[s];
                x[q] = sig[q] * dtv[q];
                cr[q] = S.rgb[s];
                cg[q] = S.rgb[s + S.ss];
                cb[q] = S.rgb[s + 2 * (size_t)S.ss];
            }
        }
        // suffix sums of x inside the lane, then over the later lanes and blocks
        float xs[K], run = 0.0f;
#pragma unroll
        for (int q = K - 1; q >= 0; --q) {
            run += x[q];
            xs[q] = run;
        }
        const float lx = warp_inclusive_suffix_sum(run, lane);
        const float ax = shift_down(lx, lane, 0.0f) + sx;  // sum over the samples after the lane's block
        float tn[K], w[K], wr[K], wg[K], wb[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float xi = ax + xs[q];                             // sum_{i>=j} x_i
            const float xe = ax + (q + 1 < K ? xs[q + 1] : 0.0f);    // sum_{i>j} x_i
            const float tj = expf(-fmaxf(depth - xi, 0.0f));
            tn[q] = expf(-fmaxf(depth - xe, 0.0f));
            w[q] = j0 + q < used ? tj * -expm1f(-x[q]) : 0.0f;
            wr[q] = w[q] * cr[q];
            wg[q] = w[q] * cg[q];
            wb[q] = w[q] * cb[q];
        }
        float rs[K], gs[K], bs[K], as[K], rr = 0.0f, rg = 0.0f, rb = 0.0f, ra = 0.0f;
#pragma unroll
        for (int q = K - 1; q >= 0; --q) {
            rr += wr[q]; rs[q] = rr;
            rg += wg[q]; gs[q] = rg;
            rb += wb[q]; bs[q] = rb;
            ra += w[q]; as[q] = ra;
        }
        const float lr = warp_inclusive_suffix_sum(rr, lane), lg = warp_inclusive_suffix_sum(rg, lane);
        const float lb = warp_inclusive_suffix_sum(rb, lane), la = warp_inclusive_suffix_sum(ra, lane);
        const float a_r = shift_down(lr, lane, 0.0f) + sr, a_g = shift_down(lg, lane, 0.0f) + sg;
        const float a_b = shift_down(lb, lane, 0.0f) + sb, a_a = shift_down(la, lane, 0.0f) + sa;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const bool next = q + 1 < K;
            const float r_ex = a_r + (next ? rs[q + 1] : 0.0f), g_ex = a_g + (next ? gs[q + 1] : 0.0f);
            const float b_ex = a_b + (next ? bs[q + 1] : 0.0f), a_ex = a_a + (next ? as[q + 1] : 0.0f);
            const float ds = dtv[q] * (gr * (tn[q] * cr[q] - r_ex) + gg * (tn[q] * cg[q] - g_ex) +
                                       gb * (tn[q] * cb[q] - b_ex) + ga * (tn[q] - a_ex));
            emit(j0 + q, j0 + q < used, ds * act_dsigma(S.act, sig[q]), cscale * gr * w[q], cscale * gg * w[q],
                 cscale * gb * w[q]);
        }
        sx += __shfl_sync(FULL_MASK, lx, 0);
        sr += __shfl_sync(FULL_MASK, lr, 0);
        sg += __shfl_sync(FULL_MASK, lg, 0);
        sb += __shfl_sync(FULL_MASK, lb, 0);
        sa += __shfl_sync(FULL_MASK, la, 0);
    }
}

__device__ __forceinline__ void zero_tail(float* __restrict__ dd, float* __restrict__ drgb, uint32_t ss, uint32_t o,
                                          uint32_t from, uint32_t n, int lane) {
    for (uint32_t j = from + lane; j < n; j += WARP) {
        const size_t s = (size_t)o + j;
        if (dd) dd[s] = 0.0f;
        if (drgb) {
            drgb[s] = 0.0f;
            drgb[s + ss] = 0.0f;
            drgb[s + 2 * (size_t)ss] = 0.0f;
        }
    }
}

// smooth-L1 (beta 1) helpers, src/utils/training-kernels-fused.cuh:344-356
__device__ __forceinline__ float huber(float x) { const float a = fabsf(x); return a < 1.0f ? 0.5f * x * x : a - 0.5f; }
__device__ __forceinline__ float huber_grad(float x) { return fabsf(x) < 1.0f ? x : copysignf(1.0f, x); }

// Reconstruction loss of one ray given its composite (training-kernels-fused.cuh:434-477).
// Returns the sum of the four channel losses; sets the VJP weights g4 of the compositor.
struct ReconGrad { float gr, gg, gb, ga; float l[4]; };

__device__ __forceinline__ ReconGrad recon_grad(const CompFwd& c, float gt_r, float gt_g, float gt_b, float gt_a,
                                               float br, float bgc, float bb, float inv_nrays) {
    const float gt_ac = 1.0f - gt_a;
    const float gtr = gt_r * gt_a + br * gt_ac, gtg = gt_g * gt_a + bgc * gt_ac, gtb = gt_b * gt_a + bb * gt_ac;
    const float ac = 1.0f - c.a;
    const float pr = c.r * c.a + br * ac, pg = c.g * c.a + bgc * ac, pb = c.b * c.a + bb * ac;
    const float dr = pr - gtr, dg = pg - gtg, db = pb - gtb, da = ac - gt_ac;
    ReconGrad g;
    g.l[0] = huber(dr); g.l[1] = huber(dg); g.l[2] = huber(db); g.l[3] = huber(da);
    const float lr = inv_nrays * huber_grad(dr), lg = inv_nrays * huber_grad(dg), lb = inv_nrays * huber_grad(db);
    // pred'_c = R_c A + bg_c (1 - A): d pred'_c = A dR_c + (R_c - bg_c) dA
    // (density_to_ray_rgba_backward, training-kernels-fused.cuh:320-322)
    g.gr = lr * c.a;
    g.gg = lg * c.a;
    g.gb = lb * c.a;
    g.ga = lr * (c.r - br) + lg * (c.g - bgc) + lb * (c.b - bb);
    return g;
}

__device__ __forceinline__ ReconGrad recon_loss_ray(const CompFwd& c, const float* __restrict__ target,
                                                   const float* __restrict__ bg, uint32_t r, uint32_t rs,
                                                   float inv_nrays) {
    return recon_grad(c, target[r], target[r + rs], target[r + 2 * (size_t)rs], target[r + 3 * (size_t)rs], bg[r],
                      bg[r + rs], bg[r + 2 * (size_t)rs], inv_nrays);
}

// ---- distortion -------------------------------------------------------------------------
// Loss of one ray (mipNeRF360_distortion_loss_forward_kernel, training-kernels-fused.cuh:13-120):
//   L = lambda/N * ( (1/3) sum_j dtn_j w_j^2 + sum_{i,j} w_i w_j |m_i - m_j| )
// with w_j = T_j alpha_j from sigma * dt_norm and no transmittance cut. The reference forms the
// cross term as (sum wm_i W_{<i}) - (sum w_i WM_{<i}) and its gradient from suffix sums obtained
// by subtraction (:204-212), which cancels catastrophically in FP32. Here the same quantities
// are accumulated from non-negative terms only:
//   A_j = sum_{l<j} w_l (m_j - m_l) = sum_{i<=j} (m_i - m_{i-1}) W_{<i}     (forward scan)
//   B_j = sum_{l>j} w_l (m_l - m_j) = sum_{i>j}  (m_i - m_{i-1}) W_{>=i}    (reverse scan)
//   cross = 2 sum_j w_j A_j,   dL/dw_j = lambda/N ((2/3) dtn_j w_j + 2 (A_j + B_j))
//   dL/dsigma_j = dtn_j (dL/dw_j T_{j+1} - sum_{l>j} dL/dw_l w_l)
// which is the reference's gradient (:188-223) written without cancelling sums (m is
// non-decreasing along a ray, so every increment m_i - m_{i-1} is >= 0).
struct DistCarry { float x, w, a, m; };

// ---- block-level deterministic sums (per-block partials, last block adds them) ---------
// out[k] = scale[k] * (block-summed v[k]), additionally divided by the live ray count
// *n_dev for the components whose bit is set in dev_mask.
struct FinishScale {
    float s[2];
    const uint32_t* n_dev;
    uint32_t n_host;
    uint32_t dev_mask;
};

template <int NV>
__device__ void block_sum_and_finish(float (&v)[NV], float* partials, uint32_t* ticket, float* out,
                                     const FinishScale fs) {
    __shared__ float red[LOSS_WARPS][NV];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const float s = warp_sum(v[k]);
        if (lane == 0) red[wid][k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            float s = 0.0f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][k];
            partials[(size_t)blockIdx.x * NV + k] = s;
        }
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // every block's partials, four blocks a thread at a time: independent loads from L2 (the
    // other blocks' stores are there; this block never cached them), then the adds
    float acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0f;
    constexpr int U = 4;
    for (uint32_t b0 = threadIdx.x; b0 < gridDim.x; b0 += U * blockDim.x) {
        float x[U][NV];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t b = b0 + (uint32_t)u * blockDim.x;
#pragma unroll
            for (int k = 0; k < NV; ++k) x[u][k] = b < gridDim.x ? __ldcg(partials + (size_t)b * NV + k) : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int k = 0; k < NV; ++k) acc[k] += x[u][k];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const float s = warp_sum(acc[k]);
        if (lane == 0) red[wid][k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t nn = fs.n_dev ? min(*fs.n_dev, fs.n_host) : fs.n_host;
        const float inv_n = nn ? 1.0f / (float)nn : 0.0f;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            float s = 0.0f;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][k];
            s *= fs.s[k];
            if ((fs.dev_mask >> k) & 1u) s *= inv_n;
            if (out) out[k] = s;
        }
        *ticket = 0u;
    }
}

__device__ __forceinline__ uint32_t live_rays(uint32_t n_rays, const uint32_t* n_dev) {
    return n_dev ? min(*n_dev, n_rays) : n_rays;
}

// Two lower bounds at once over ascending offsets: the first i < n with off[i] >= va (lanes
// 0-15) and >= vb (lanes 16-31), n where there is none. Each half probes 16 positions a round and
// keeps the sub-range where the offsets cross its value; every lane of the warp runs every round.
__device__ uint2 warp_lower_bounds(const uint32_t* __restrict__ off, uint32_t n, uint32_t va, uint32_t vb, int lane) {
    const int half = lane >> 4, j = lane & 15;
    const uint32_t v = half ? vb : va;
    uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi]; hi == n or off[hi] >= v
    for (;;) {
        const bool active = hi - lo > 16u;
        if (__ballot_sync(FULL_MASK, active) == 0u) break;
        uint32_t step = 0;
        bool pred = false;
        if (active) {
            step = (hi - lo + 15u) / 16u;
            pred = off[min(lo + (uint32_t)(j + 1) * step, hi) - 1u] >= v;
        }
        const unsigned m = (__ballot_sync(FULL_MASK, pred) >> (16 * half)) & 0xFFFFu;
        if (active) {
            if (m == 0u) {
                lo = hi;
            } else {
                const uint32_t js = (uint32_t)(__ffs(m) - 1);
                const uint32_t nlo = lo + js * step;
                hi = min(lo + (js + 1u) * step, hi) - 1u;
                lo = nlo;
            }
        }
    }
    const bool pred = lo + (uint32_t)j < hi && off[lo + (uint32_t)j] >= v;
    const unsigned m = (__ballot_sync(FULL_MASK, pred) >> (16 * half)) & 0xFFFFu;
    const uint32_t ans = m ? lo + (uint32_t)(__ffs(m) - 1) : hi;
    return make_uint2(__shfl_sync(FULL_MASK, ans, 0), __shfl_sync(FULL_MASK, ans, 16));
}

// The rays of warp w of W under a sample-balanced split: those whose first sample lies in
// [w S / W, (w + 1) S / W), S the batch's samples (offsets ascending); the last warp also takes
// the rays without samples at the end.
__device__ __forceinline__ uint2 balanced_rays(const uint32_t* __restrict__ counts,
                                               const uint32_t* __restrict__ offsets, uint32_t n_live, uint32_t w,
                                               uint32_t W, int lane) {
    const uint32_t total = offsets[n_live - 1] + counts[n_live - 1];
    const uint32_t va = (uint32_t)((uint64_t)total * w / W), vb = (uint32_t)((uint64_t)total * (w + 1) / W);
    uint2 r = warp_lower_bounds(offsets, n_live, va, vb, lane);
    if (w == 0) r.x = 0;
    if (w + 1 == W) r.y = n_live;
    return r;
}

// ---- kernels ----------------------------------------------------------------------------
// ---- sample tiles over several rays (the compositor's launch form) -------------------------
// Each warp owns a run of consecutive rays (`rpw` of them in the distortion tiles; the rays that
// start in its share of the samples in the compositor tiles, balanced_rays), whose samples are one
// contiguous range (offsets are the exclusive scan of the counts), and walks that range in tiles
// of 32 * K samples, lane l owning
// the K consecutive samples [base + K l, base + K l + K). Short rays share a tile and long rays
// span several; every running sum along a ray is a segmented sum: inside a lane, then one
// segmented warp scan of the lane aggregates, then a carry into the next tile. The loads of a
// tile are 32 * K consecutive samples whatever the ray lengths (16-byte vectors when the
// batch's arrays allow: tiles then start at a multiple of 4), and the warp scans once per tile,
// not once per ray or per 32 samples. The warp's ray table sits in shared memory; each lane
// finds the ray of its first sample once per tile and steps to the next ray at ray ends.
constexpr int ST_K = 4;
constexpr int CT_K = 8;  // samples a lane of the compositor forward tiles
constexpr int CV_K = 4;  // samples a lane of the compositor VJP tiles

// Last i < nr with off[i] <= s (rays without samples share their start with the next ray and
// are passed over).
__device__ __forceinline__ int find_ray(const uint32_t* off, int nr, uint32_t s) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const int mid = lo + step;
        if (mid < nr && off[mid] <= s) lo = mid;
    }
    return lo;
}

// Inclusive segmented scans of N values over the lanes, in increasing (SUFFIX = false) or
// decreasing (SUFFIX = true) lane order: a lane with `cut` set starts a new segment there. The
// segment flags travel with the values, so their shuffles overlap.
template <int N, bool SUFFIX>
__device__ __forceinline__ void seg_scan(float (&v)[N], bool cut, int lane) {
    unsigned f = cut ? 1u : 0u;
#pragma unroll
    for (int d = 1; d < WARP; d <<= 1) {
        const unsigned fo = SUFFIX ? __shfl_down_sync(FULL_MASK, f, d) : __shfl_up_sync(FULL_MASK, f, d);
        const bool in = SUFFIX ? lane + d < WARP : lane >= d;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const float vo = SUFFIX ? __shfl_down_sync(FULL_MASK, v[k], d) : __shfl_up_sync(FULL_MASK, v[k], d);
            if (in && !f) v[k] += vo;
        }
        if (in) f |= fo;
    }
}

// The same scans in two parts, for many scans over one set of segments (several of them
// chained, so the flags cannot travel with every one). seg_plan records, per level of the scan (bit l for distance 2^l),
// whether this lane adds the value from the lane that far below (above, SUFFIX): it does when
// that lane exists and no segment start lies in between. seg_scan_plan runs a scan of N values
// from the plan.
template <bool SUFFIX>
__device__ __forceinline__ uint32_t seg_plan(bool cut, int lane) {
    unsigned f = cut ? 1u : 0u;
    uint32_t plan = 0;
#pragma unroll
    for (int l = 0; l < 5; ++l) {
        const int d = 1 << l;
        const unsigned fo = SUFFIX ? __shfl_down_sync(FULL_MASK, f, d) : __shfl_up_sync(FULL_MASK, f, d);
        const bool in = SUFFIX ? lane + d < WARP : lane >= d;
        if (in && !f) plan |= 1u << l;
        if (in) f |= fo;
    }
    return plan;
}

template <int N, bool SUFFIX>
__device__ __forceinline__ void seg_scan_plan(float (&v)[N], uint32_t plan) {
#pragma unroll
    for (int l = 0; l < 5; ++l) {
        const int d = 1 << l;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const float vo = SUFFIX ? __shfl_down_sync(FULL_MASK, v[k], d) : __shfl_up_sync(FULL_MASK, v[k], d);
            if ((plan >> l) & 1u) v[k] += vo;
        }
    }
}

// The K samples of a lane starting at s0: sigma and dt and rgb (16-byte loads when VEC; K is then a
// multiple of 4). Samples outside `in` read as zero.
template <int K, bool VEC, int ACT>
__device__ __forceinline__ void load_tile(const Samples& S, uint32_t s0, const bool (&in)[K], float (&sig)[K],
                                          float (&dtv)[K], float (&cr)[K], float (&cg)[K], float (&cb)[K]) {
    if (VEC) {
        static_assert(!VEC || K % 4 == 0, "vector loads take 4 samples at a time");
#pragma unroll
        for (int v = 0; v < K / 4; ++v) {
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, r = a, g = a, c = a;
            // sv is a multiple of 4; a vector holding an in-range sample (below sample_stride, itself
            // a multiple of 4) ends at or before sample_stride
            const uint32_t sv = s0 + 4u * v;
            bool vin = false;
#pragma unroll
            for (int k = 0; k < 4; ++k) vin = vin || in[4 * v + k];
            if (vin) {
                a = *reinterpret_cast<const float4*>(S.density + sv);
                b = *reinterpret_cast<const float4*>(S.dt + sv);
                r = *reinterpret_cast<const float4*>(S.rgb + sv);
                g = *reinterpret_cast<const float4*>(S.rgb + S.ss + sv);
                c = *reinterpret_cast<const float4*>(S.rgb + 2 * (size_t)S.ss + sv);
            }
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w}, rv[4] = {r.x, r.y, r.z, r.w},
                        gv[4] = {g.x, g.y, g.z, g.w}, cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int q = 4 * v + k;
                sig[q] = in[q] ? act_sigma(ACT, av[k]) : 0.0f;
                dtv[q] = in[q] ? bv[k] : 0.0f;
                cr[q] = in[q] ? rv[k] : 0.0f;
                cg[q] = in[q] ? gv[k] : 0.0f;
                cb[q] = in[q] ? cv[k] : 0.0f;
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            sig[q] = dtv[q] = cr[q] = cg[q] = cb[q] = 0.0f;
            if (in[q]) {
                const size_t s = (size_t)s0 + q;
                sig[q] = act_sigma(ACT, S.density[s]);
                dtv[q] = S.dt[s];
                cr[q] = S.rgb[s];
                cg[q] = S.rgb[s + S.ss];
                cb[q] = S.rgb[s + 2 * (size_t)S.ss];
            }
        }
    }
}

// One lane's K samples of the five sample arrays as loaded (16-byte groups), held in registers
// while the tile before them is computed, so that their load latency hides behind that work.
template <int K>
struct RawTile {
    float4 a[K / 4], b[K / 4], r[K / 4], g[K / 4], c[K / 4];
};

// Loads the 16-byte groups of the lane's K samples from s0 (a multiple of 4) that hold a sample of
// `im` (bit q: sample s0 + q lies in the warp's range); the other groups read as zero.
template <int K>
__device__ __forceinline__ void load_raw(const Samples& S, uint32_t s0, uint32_t im, RawTile<K>& t) {
#pragma unroll
    for (int v = 0; v < K / 4; ++v) {
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        t.a[v] = t.b[v] = t.r[v] = t.g[v] = t.c[v] = z;
        if ((im >> (4 * v)) & 15u) {
            const uint32_t sv = s0 + 4u * v;
            t.a[v] = *reinterpret_cast<const float4*>(S.density + sv);
            t.b[v] = *reinterpret_cast<const float4*>(S.dt + sv);
            t.r[v] = *reinterpret_cast<const float4*>(S.rgb + sv);
            t.g[v] = *reinterpret_cast<const float4*>(S.rgb + S.ss + sv);
            t.c[v] = *reinterpret_cast<const float4*>(S.rgb + 2 * (size_t)S.ss + sv);
        }
    }
}

// load_tile's outputs from a raw tile: samples outside `in` read as zero.
template <int K, int ACT>
__device__ __forceinline__ void unpack_tile(const RawTile<K>& t, const bool (&in)[K], float (&sig)[K],
                                            float (&dtv)[K], float (&cr)[K], float (&cg)[K], float (&cb)[K]) {
#pragma unroll
    for (int v = 0; v < K / 4; ++v) {
        const float av[4] = {t.a[v].x, t.a[v].y, t.a[v].z, t.a[v].w}, bv[4] = {t.b[v].x, t.b[v].y, t.b[v].z, t.b[v].w},
                    rv[4] = {t.r[v].x, t.r[v].y, t.r[v].z, t.r[v].w}, gv[4] = {t.g[v].x, t.g[v].y, t.g[v].z, t.g[v].w},
                    cv[4] = {t.c[v].x, t.c[v].y, t.c[v].z, t.c[v].w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int q = 4 * v + k;
            sig[q] = in[q] ? act_sigma(ACT, av[k]) : 0.0f;
            dtv[q] = in[q] ? bv[k] : 0.0f;
            cr[q] = in[q] ? rv[k] : 0.0f;
            cg[q] = in[q] ? gv[k] : 0.0f;
            cb[q] = in[q] ? cv[k] : 0.0f;
        }
    }
}

// Bits of the lane's K samples from s0 that lie in [s_begin, s_end).
template <int K>
__device__ __forceinline__ uint32_t tile_range_mask(uint32_t s0, uint32_t s_begin, uint32_t s_end) {
    const uint32_t lo = s_begin > s0 ? min(s_begin - s0, (uint32_t)K) : 0u;
    const uint32_t hi = s_end > s0 ? min(s_end - s0, (uint32_t)K) : 0u;
    return ((1u << hi) - 1u) & ~((1u << lo) - 1u);
}

// L2 prefetch of one tile of samples [s, s + 32 K) of the five sample arrays (density, dt and the
// three rgb planes), one 128-byte line per lane for the first 5 * 32 K / 32 lanes: the next tile's
// loads then find their lines in L2 instead of DRAM. Lines past the arrays' end are not touched.
template <int K>
__device__ __forceinline__ void prefetch_tile(const Samples& S, uint32_t s, int lane) {
    constexpr int LINES = WARP * K / 32;  // 128-byte lines of one array per tile
#pragma unroll
    for (int i = lane; i < 5 * LINES; i += WARP) {
        const int arr = i / LINES, line = i % LINES;
        const uint32_t at = s + (uint32_t)line * 32u;
        if (at < S.ss) {
            const float* base = arr == 0 ? S.density : arr == 1 ? S.dt : S.rgb + (size_t)(arr - 2) * S.ss;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(base + at));
        }
    }
}

// Head bits of one tile of 32 K samples [base, base + 32 K] (one word more for the sample after
// the tile): bit d is set when a non-empty ray of the warp starts at base + d, or when the warp's
// samples end there. `off` is the lane's ray start (lanes at or past `nne` hold none). Returns, for
// lane l, the K + 1 bits from sample base + K l.
template <int K>
__device__ __forceinline__ uint32_t tile_head_bits(uint32_t* words, uint32_t base, uint32_t off, int nne,
                                                   uint32_t s_end, int lane) {
    if (lane <= K) words[lane] = 0u;
    __syncwarp();
    const uint32_t d = off - base;  // wraps for rays that started before the tile
    if (lane < nne && d <= (uint32_t)(WARP * K)) atomicOr(&words[d >> 5], 1u << (d & 31));
    const uint32_t e = s_end - base;
    if (lane == 0 && e <= (uint32_t)(WARP * K)) atomicOr(&words[e >> 5], 1u << (e & 31));
    __syncwarp();
    const uint32_t p0 = (uint32_t)lane * K;
    return __funnelshift_r(words[p0 >> 5], words[(p0 >> 5) + 1], p0 & 31);
}

// Ordinal (among the warp's non-empty rays, starts `off` ascending) of the ray holding sample s:
// the last k < nne with off[k] <= s, or -1 before the first start (the part of a warp's first
// 16-byte group that precedes its rays).
__device__ __forceinline__ int ray_ordinal(const uint32_t* off, int nne, uint32_t s) {
    if (off[0] > s) return -1;
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const int mid = lo + step;
        if (mid < nne && off[mid] <= s) lo = mid;
    }
    return lo;
}

// Compositor forward over the rays of each warp (density_to_ray_rgba_forward,
// src/utils/training-kernels-fused.cuh:227-264). Termination is decided on the optical depth
// d = sum sigma dt: sample j is composited while the depth before it is at most
// depth_max = -ln(min_t) (transmittance >= min_t), and the first sample whose depth after it
// exceeds depth_max is the last one composited. The weights use the transmittance as a product
// of (1 - alpha) inside each lane from exp(-depth) at the lane's first sample.
// Ray boundaries come from the tile's head bits (one word per 32 samples, built once per tile):
// a lane tests bits instead of searching the ray table per sample, and one segment plan serves
// the optical-depth scan and the colour scan. The alpha of a ray is 1 - exp(-d) at its
// terminating sample (the sum of its weights, without rounding accumulated over the samples;
// `opacity`, a few 1e-7 relative), stored with the depth and the sample count there; its colour sums are stored at its last sample
// (the ray open at the lane's start, after the colour scan).
// One group of the forward tiles: rays [r0, r0 + nr) (consecutive samples), walked in tiles of
// 32 K samples. t_off, t_rid and t_head are the warp's tables.
template <int K, bool VEC, int ACT, bool STORE>
__device__ __forceinline__ void composite_fwd_group(const Samples& S, uint32_t r0, int nr, uint32_t rs,
                                                    const uint32_t* __restrict__ counts,
                                                    const uint32_t* __restrict__ offsets, float depth_max,
                                                    float* __restrict__ rgba, float* __restrict__ depth,
                                                    uint32_t* __restrict__ n_used, float* __restrict__ t_out,
                                                    float* __restrict__ w_out, uint32_t* t_off, uint32_t* t_rid,
                                                    uint32_t* t_head, int lane) {
    uint32_t o = 0, c = 0;
    if (lane < nr) {
        o = offsets[r0 + lane];
        c = counts[r0 + lane];
        if (c == 0) {  // a ray without samples
            const uint32_t r = r0 + lane;
            rgba[r] = 0.0f; rgba[r + rs] = 0.0f; rgba[r + 2 * (size_t)rs] = 0.0f; rgba[r + 3 * (size_t)rs] = 0.0f;
            if (depth) depth[r] = 0.0f;
            if (n_used) n_used[r] = 0u;
        }
    }
    const unsigned ne = __ballot_sync(FULL_MASK, c > 0u);
    if (ne == 0u) return;
    if (c > 0u) {
        const int k = __popc(ne & ((1u << lane) - 1u));
        t_off[k] = o;
        t_rid[k] = r0 + (uint32_t)lane;
    }
    const int nne = __popc(ne);
    const uint32_t s_begin = __shfl_sync(FULL_MASK, o, __ffs(ne) - 1);
    const uint32_t s_end = __shfl_sync(FULL_MASK, o + c, 31 - __clz(ne));
    __syncwarp();
    const uint32_t my_off = lane < nne ? t_off[lane] : 0u;
    float cx = 0.0f, c3[3] = {0.0f, 0.0f, 0.0f};  // depth and colour sums of the ray open at the tile start
    constexpr uint32_t SPAN = WARP * K;
    const uint32_t b_first = VEC ? (s_begin & ~3u) : s_begin;
    // with 16-byte loads the next tile's samples are loaded before this tile is computed (cur, nxt)
    // and the third tile from here prefetched into L2 (the distance measured best)
    RawTile<K> cur, nxt;
    if (VEC) {
        const uint32_t s0f = b_first + (uint32_t)lane * K;
        load_raw<K>(S, s0f, tile_range_mask<K>(s0f, s_begin, s_end), cur);
    }
    for (uint32_t base = b_first; base < s_end; base += SPAN) {
        if (VEC) {
            const uint32_t s0n = base + SPAN + (uint32_t)lane * K;
            if (base + SPAN < s_end) load_raw<K>(S, s0n, tile_range_mask<K>(s0n, s_begin, s_end), nxt);
            if (base + 3 * SPAN < s_end) prefetch_tile<K>(S, base + 3 * SPAN, lane);
        } else if (base + SPAN < s_end) {
            prefetch_tile<K>(S, base + SPAN, lane);
        }
        const uint32_t win = tile_head_bits<K>(t_head, base, my_off, nne, s_end, lane);
        constexpr uint32_t LANE_BITS = (1u << K) - 1u;
        const uint32_t hm = win & LANE_BITS, lm = (win >> 1) & LANE_BITS;  // ray starts; ray ends
        const uint32_t s0 = base + (uint32_t)lane * K;
        const uint32_t im = tile_range_mask<K>(s0, s_begin, s_end);  // samples inside [s_begin, s_end)
        bool in[K];
#pragma unroll
        for (int q = 0; q < K; ++q) in[q] = (im >> q) & 1u;
        float x[K], dtv[K], cr[K], cg[K], cb[K];
        if (VEC) {
            unpack_tile<K, ACT>(cur, in, x, dtv, cr, cg, cb);
            cur = nxt;
        } else {
            load_tile<K, false, ACT>(S, s0, in, x, dtv, cr, cg, cb);
        }
#pragma unroll
        for (int q = 0; q < K; ++q) x[q] *= dtv[q];
        // optical depth: the lane's aggregate from its last ray start, one segmented scan
        const bool cut = hm != 0u;
        const uint32_t plan = seg_plan<false>(cut, lane);
        float agg[1];
        {
            float a = 0.0f;
#pragma unroll
            for (int q = 0; q < K; ++q) a = ((hm >> q) & 1u) ? x[q] : a + x[q];
            agg[0] = (lane == 0 && !cut) ? a + cx : a;
        }
        seg_scan_plan<1, false>(agg, plan);
        float run = __shfl_up_sync(FULL_MASK, agg[0], 1);
        if (lane == 0) run = cx;
        const int k0 = ray_ordinal(t_off, nne, s0);  // the ray open at the lane's first sample
        float tb = __expf(-run);  // transmittance before the lane's first sample
        float a3[3] = {0.0f, 0.0f, 0.0f};
        float f3[3] = {0.0f, 0.0f, 0.0f};
        bool first_end = false;  // the ray open at the lane's start ends in the lane
        uint32_t term_bits = 0u;  // the lane's terminating samples
        float run_q[K];           // the optical depth after each sample
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const bool h = (hm >> q) & 1u;
            const float excl = h ? 0.0f : run;
            tb = h ? 1.0f : tb;
#pragma unroll
            for (int k = 0; k < 3; ++k) a3[k] = h ? 0.0f : a3[k];
            run = excl + x[q];
            const bool comp = in[q] && excl <= depth_max;
            const float al = opacity(x[q]);
            const float w = comp ? tb * al : 0.0f;
            const float tn = fmaf(-tb, al, tb);  // transmittance after the sample
            if (STORE && comp) {
                t_out[s0 + q] = tn;
                w_out[s0 + q] = w;
            }
            a3[0] = fmaf(w, cr[q], a3[0]);
            a3[1] = fmaf(w, cg[q], a3[1]);
            a3[2] = fmaf(w, cb[q], a3[2]);
            const bool last = in[q] && ((lm >> q) & 1u);
            // the ray's terminating sample: its depth, samples used and alpha are stored after the
            // loop (term_bits, run_q), so that the loop carries no branch for them
            const bool term = comp && (run > depth_max || last);
            term_bits |= (uint32_t)term << q;
            run_q[q] = run;
            if (last) {  // an in-range sample: at or after the warp's first ray start
                if ((hm & ((2u << q) - 1u)) == 0u) {
                    first_end = true;  // the ray began in an earlier lane: completed after the colour scan
#pragma unroll
                    for (int c = 0; c < 3; ++c) f3[c] = a3[c];
                } else {
                    const uint32_t r = t_rid[k0 + __popc(hm & ((2u << q) - 2u))];
                    rgba[r] = a3[0]; rgba[r + rs] = a3[1]; rgba[r + 2 * (size_t)rs] = a3[2];
                }
            }
            tb = tn;
        }
        while (term_bits) {
            const int q = __ffs(term_bits) - 1;
            term_bits &= term_bits - 1u;
            float d = run_q[0];
#pragma unroll
            for (int j = 1; j < K; ++j) d = q == j ? run_q[j] : d;
            const int k = k0 + __popc(hm & ((2u << q) - 2u));
            const uint32_t r = t_rid[k];
            if (depth) depth[r] = d;
            if (n_used) n_used[r] = s0 + q - t_off[k] + 1u;
            rgba[r + 3 * (size_t)rs] = opacity(d);
        }
        // colour sums of the ray open at each lane's end, over the lanes
        if (lane == 0 && !cut) {
#pragma unroll
            for (int k = 0; k < 3; ++k) a3[k] += c3[k];
        }
        seg_scan_plan<3, false>(a3, plan);
        float e3[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            e3[k] = __shfl_up_sync(FULL_MASK, a3[k], 1);
            if (lane == 0) e3[k] = c3[k];
        }
        if (first_end) {
            const uint32_t r = t_rid[k0];
            rgba[r] = e3[0] + f3[0]; rgba[r + rs] = e3[1] + f3[1]; rgba[r + 2 * (size_t)rs] = e3[2] + f3[2];
        }
        // carries of the ray open at the end of the tile (lane 31 holds the tile's last samples)
        cx = __shfl_sync(FULL_MASK, agg[0], WARP - 1);
#pragma unroll
        for (int k = 0; k < 3; ++k) c3[k] = __shfl_sync(FULL_MASK, a3[k], WARP - 1);
        __syncwarp();  // every lane has read the tile's head words
    }
}

// The tile kernels launch one wave of resident warps; each warp takes the rays whose first sample
// lies in its equal share of the batch's samples (balanced_rays), in groups of up to 32 rays.
template <int K, bool VEC, int ACT, bool STORE>
__global__ void __launch_bounds__(LOSS_THREADS, 2)
composite_fwd_tiles_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rs,
                           const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets, float depth_max,
                           float* __restrict__ rgba, float* __restrict__ depth, uint32_t* __restrict__ n_used,
                           float* __restrict__ t_out, float* __restrict__ w_out) {
    static_assert(K % 4 == 0 && K <= 16, "16-byte groups, at most 16 samples a lane");
    __shared__ uint32_t t_off[LOSS_WARPS][WARP], t_rid[LOSS_WARPS][WARP], t_head[LOSS_WARPS][K + 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    if (n_live == 0) return;
    const uint2 rr = balanced_rays(counts, offsets, n_live, blockIdx.x * LOSS_WARPS + wid, gridDim.x * LOSS_WARPS, lane);
    for (uint32_t r0 = rr.x; r0 < rr.y; r0 += WARP) {
        composite_fwd_group<K, VEC, ACT, STORE>(S, r0, (int)min((uint32_t)WARP, rr.y - r0), rs, counts, offsets,
                                                depth_max, rgba, depth, n_used, t_out, w_out, t_off[wid], t_rid[wid],
                                                t_head[wid], lane);
        __syncwarp();  // the warp's tables are reused by the next group
    }
}

// Compositor VJP over the rays of each warp (semantics of composite_vjp_ray): tiles from the end
// of the warp's samples down. With the ray's upstream gradient g = (gr, gg, gb, ga) and
// u_j = gr r_j + gg g_j + gb b_j + ga, dL/dsigma_j = dt_j (T_{j+1} u_j - sum_{i>j} w_i u_i) over the
// composited samples: one segmented suffix sum of w u. The transmittance at each lane's first
// sample comes from the ray's forward depth minus the segmented suffix sum of x = sigma dt (one
// exponential a lane); inside the lane it is the product of (1 - alpha), restarted at ray starts.
// Samples of a ray at or past its `used` get zero gradients.
// One group of the VJP tiles: rays [r0, r0 + nr), tiles from the last. t_off, t_lim, t_dep, t_g
// and t_head are the warp's tables.
template <int K, bool VEC, int ACT>
__device__ __forceinline__ void composite_bwd_group(const Samples& S, uint32_t r0, int nr, uint32_t rs,
                                                    const uint32_t* __restrict__ counts,
                                                    const uint32_t* __restrict__ offsets,
                                                    const float* __restrict__ depth,
                                                    const uint32_t* __restrict__ n_used,
                                                    const float* __restrict__ grad_rgba, float* __restrict__ dd,
                                                    float* __restrict__ drgb, uint32_t* t_off, uint32_t* t_lim,
                                                    float* t_dep, float4* t_g, uint32_t* t_head, int lane) {
    uint32_t o = 0, c = 0;
    if (lane < nr) {
        o = offsets[r0 + lane];
        c = counts[r0 + lane];
    }
    const unsigned ne = __ballot_sync(FULL_MASK, c > 0u);
    if (ne == 0u) return;
    if (c > 0u) {
        const uint32_t r = r0 + (uint32_t)lane;
        const int k = __popc(ne & ((1u << lane) - 1u));
        t_off[k] = o;
        t_lim[k] = o + min(n_used[r], c);  // end of the composited samples
        t_dep[k] = depth[r];
        t_g[k] = make_float4(grad_rgba[r], grad_rgba[r + rs], grad_rgba[r + 2 * (size_t)rs],
                                  grad_rgba[r + 3 * (size_t)rs]);
    }
    const int nne = __popc(ne);
    const uint32_t s_begin = __shfl_sync(FULL_MASK, o, __ffs(ne) - 1);
    const uint32_t s_end = __shfl_sync(FULL_MASK, o + c, 31 - __clz(ne));
    __syncwarp();
    const uint32_t my_off = lane < nne ? t_off[lane] : 0u;
    const uint32_t b0 = VEC ? (s_begin & ~3u) : s_begin;
    const uint32_t span = WARP * K;
    const uint32_t n_tiles = (s_end - b0 + span - 1) / span;
    float cx = 0.0f, cu = 0.0f;  // suffix sums of x and w u of the ray open at the tile end
    // with 16-byte loads the next tile's samples (the one below) are loaded before this tile is
    // computed (cur, nxt); an L2 prefetch further ahead measured slower here (its instructions
    // cost more than it saves)
    RawTile<K> cur, nxt;
    if (VEC) {
        const uint32_t s0l = b0 + (n_tiles - 1) * span + (uint32_t)lane * K;
        load_raw<K>(S, s0l, tile_range_mask<K>(s0l, s_begin, s_end), cur);
    }
    for (int t = (int)n_tiles - 1; t >= 0; --t) {
        const uint32_t base = b0 + (uint32_t)t * span;
        if (VEC) {
            if (t > 0) {
                const uint32_t s0n = base - span + (uint32_t)lane * K;
                load_raw<K>(S, s0n, tile_range_mask<K>(s0n, s_begin, s_end), nxt);
            }
        } else if (t > 0) {
            prefetch_tile<K>(S, base - span, lane);
        }
        const uint32_t win = tile_head_bits<K>(t_head, base, my_off, nne, s_end, lane);
        constexpr uint32_t LANE_BITS = (1u << K) - 1u;
        const uint32_t hm = win & LANE_BITS, lm = (win >> 1) & LANE_BITS;  // ray starts; ray ends
        const uint32_t s0 = base + (uint32_t)lane * K;
        const uint32_t im = tile_range_mask<K>(s0, s_begin, s_end);
        const int k0 = ray_ordinal(t_off, nne, s0);
        bool in[K], valid[K];
        float4 g[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            in[q] = (im >> q) & 1u;
            // -1 only for samples before the warp's first start, which are outside the range
            const int k = max(k0 + __popc(hm & ((2u << q) - 2u)), 0);
            valid[q] = in[q] && s0 + q < t_lim[k];
            g[q] = t_g[k];
        }
        float x[K], dtv[K], cr[K], cg[K], cb[K];
        if (VEC) {
            unpack_tile<K, ACT>(cur, valid, x, dtv, cr, cg, cb);
            cur = nxt;
        } else {
            load_tile<K, false, ACT>(S, s0, valid, x, dtv, cr, cg, cb);
        }
        float sig[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            sig[q] = x[q];
            x[q] *= dtv[q];
        }
        // suffix sums of x: the lane's aggregate is its samples up to its first ray end
        const bool cut = lm != 0u;
        const uint32_t plan = seg_plan<true>(cut, lane);
        float vx[1];
        {
            float a = 0.0f;
#pragma unroll
            for (int q = K - 1; q >= 0; --q) a = ((lm >> q) & 1u) ? x[q] : a + x[q];
            vx[0] = (lane == WARP - 1 && !cut) ? a + cx : a;
        }
        seg_scan_plan<1, true>(vx, plan);
        // transmittance before and after each sample, weights, u and w u
        float tn[K], w[K], u[K], wu[K];
        {
            float T = __expf(-fmaxf(t_dep[max(k0, 0)] - vx[0], 0.0f));
#pragma unroll
            for (int q = 0; q < K; ++q) {
                T = ((hm >> q) & 1u) ? 1.0f : T;
                const float al = opacity(x[q]);
                w[q] = valid[q] ? T * al : 0.0f;
                tn[q] = fmaf(-T, al, T);
                u[q] = fmaf(g[q].x, cr[q], fmaf(g[q].y, cg[q], fmaf(g[q].z, cb[q], g[q].w)));
                wu[q] = w[q] * u[q];
                T = tn[q];
            }
        }
        float vu[1];
        {
            float a = 0.0f;
#pragma unroll
            for (int q = K - 1; q >= 0; --q) a = ((lm >> q) & 1u) ? wu[q] : a + wu[q];
            vu[0] = (lane == WARP - 1 && !cut) ? a + cu : a;
        }
        seg_scan_plan<1, true>(vu, plan);
        float e = __shfl_down_sync(FULL_MASK, vu[0], 1);  // sum of w u after the lane, ray open at its end
        if (lane == WARP - 1) e = cu;
        float o_d[K], o_r[K], o_g[K], o_b[K];
#pragma unroll
        for (int q = K - 1; q >= 0; --q) {
            e = ((lm >> q) & 1u) ? 0.0f : e;  // sums over i > j within the ray
            const float ds = dtv[q] * (tn[q] * u[q] - e);
            o_d[q] = valid[q] ? ds * act_dsigma(ACT, sig[q]) : 0.0f;
            o_r[q] = g[q].x * w[q];
            o_g[q] = g[q].y * w[q];
            o_b[q] = g[q].z * w[q];
            e += wu[q];
        }
#pragma unroll
        for (int v = 0; v < K / 4; ++v) {
            const bool all_in = ((im >> (4 * v)) & 15u) == 15u;
            const uint32_t sv = s0 + 4u * v;
            if (VEC && all_in) {
                *reinterpret_cast<float4*>(dd + sv) = make_float4(o_d[4 * v], o_d[4 * v + 1], o_d[4 * v + 2], o_d[4 * v + 3]);
                *reinterpret_cast<float4*>(drgb + sv) = make_float4(o_r[4 * v], o_r[4 * v + 1], o_r[4 * v + 2], o_r[4 * v + 3]);
                *reinterpret_cast<float4*>(drgb + S.ss + sv) =
                    make_float4(o_g[4 * v], o_g[4 * v + 1], o_g[4 * v + 2], o_g[4 * v + 3]);
                *reinterpret_cast<float4*>(drgb + 2 * (size_t)S.ss + sv) =
                    make_float4(o_b[4 * v], o_b[4 * v + 1], o_b[4 * v + 2], o_b[4 * v + 3]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int q = 4 * v + k;
                    if (!in[q]) continue;
                    const size_t s = (size_t)s0 + q;
                    dd[s] = o_d[q];
                    drgb[s] = o_r[q];
                    drgb[s + S.ss] = o_g[q];
                    drgb[s + 2 * (size_t)S.ss] = o_b[q];
                }
            }
        }
        cx = __shfl_sync(FULL_MASK, vx[0], 0);
        cu = __shfl_sync(FULL_MASK, vu[0], 0);
        __syncwarp();  // every lane has read the tile's head words
    }
}

template <int K, bool VEC, int ACT>
__global__ void __launch_bounds__(LOSS_THREADS, 3)
composite_bwd_tiles_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rs,
                           const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                           const float* __restrict__ depth, const uint32_t* __restrict__ n_used,
                           const float* __restrict__ grad_rgba, float* __restrict__ dd, float* __restrict__ drgb) {
    static_assert(K % 4 == 0 && K <= 16, "16-byte groups, at most 16 samples a lane");
    __shared__ uint32_t t_off[LOSS_WARPS][WARP], t_lim[LOSS_WARPS][WARP], t_head[LOSS_WARPS][K + 1];
    __shared__ float t_dep[LOSS_WARPS][WARP];
    __shared__ float4 t_g[LOSS_WARPS][WARP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    if (n_live == 0) return;
    const uint2 rr = balanced_rays(counts, offsets, n_live, blockIdx.x * LOSS_WARPS + wid, gridDim.x * LOSS_WARPS, lane);
    for (uint32_t r0 = rr.x; r0 < rr.y; r0 += WARP) {
        composite_bwd_group<K, VEC, ACT>(S, r0, (int)min((uint32_t)WARP, rr.y - r0), rs, counts, offsets, depth, n_used,
                                         grad_rgba, dd, drgb, t_off[wid], t_lim[wid], t_dep[wid], t_g[wid],
                                         t_head[wid], lane);
        __syncwarp();
    }
}

// ---- distortion loss over sample tiles ------------------------------------------------------
// The distortion loss forward and backward (mipNeRF360_distortion_loss_forward_kernel /
// _backward_kernel, training-kernels-fused.cuh:13-224, with the sums A, B above) in the tile
// form of the compositor: a warp owns `rpw` consecutive rays and walks their samples in tiles of
// 32 * K, lane l owning K consecutive samples. Forward, tiles in increasing order: per sample the
// optical depth before it, the weight w = T (1 - e^-x), the weight sum before it W_<, the
// increment dm of m and A = sum dm W_<, each a segmented scan of the lane aggregates with a
// carry into the next tile; the per-ray loss k (sum dtn w^2 / 3 + 2 sum w A), k = lambda / n,
// is a segmented sum closed at the ray's last sample. The carry at each tile's start (x, w, a, m
// of the ray open there) is kept, two tiles per lane, for the backward. Backward, tiles in
// decreasing order: the tile's forward quantities rebuilt from its carry, then the segmented
// suffix sums W_>=, F = sum dm W_>= (B = F of the next sample) and sum g w over later samples,
// with g = k ((2/3) dtn w + 2 (A + B)) and dL/dsigma = dtn (g T_{j+1} - sum_{l>j} g_l w_l).
// Tiles past the kept ones replay the forward from the last kept carry.

struct DistTile {
    float sig[ST_K], dtn[ST_K], w[ST_K], tn[ST_K], dm[ST_K], a[ST_K];
};

// Forward quantities of one tile from the carry `c` of the ray open at its start; `next` is the
// carry at its end.
template <bool VEC, int ACT>
__device__ __forceinline__ void dist_tile_forward(const Samples& S, uint32_t s0, const bool (&in)[ST_K],
                                                  const bool (&head)[ST_K], bool any_head, uint32_t plan, int lane,
                                                  const DistCarry& c, DistCarry& next, DistTile& d) {
    constexpr int K = ST_K;
    float m[K];
    if (VEC) {
        bool vin = false;
#pragma unroll
        for (int q = 0; q < K; ++q) vin = vin || in[q];
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, e = a;
        if (vin) {  // s0 is a multiple of 4 and the vector ends at or before the sample stride
            a = *reinterpret_cast<const float4*>(S.density + s0);
            b = *reinterpret_cast<const float4*>(S.dt_norm + s0);
            e = *reinterpret_cast<const float4*>(S.m_norm + s0);
        }
        const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w}, ev[4] = {e.x, e.y, e.z, e.w};
#pragma unroll
        for (int q = 0; q < K; ++q) {
            d.sig[q] = in[q] ? act_sigma(ACT, av[q]) : 0.0f;
            d.dtn[q] = in[q] ? bv[q] : 0.0f;
            m[q] = in[q] ? ev[q] : 0.0f;
        }
    } else {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            d.sig[q] = d.dtn[q] = m[q] = 0.0f;
            if (in[q]) {
                d.sig[q] = act_sigma(ACT, S.density[s0 + q]);
                d.dtn[q] = S.dt_norm[s0 + q];
                m[q] = S.m_norm[s0 + q];
            }
        }
    }
    // optical depth before each sample, weights, transmittance after each sample
    float x[K];
    float agg[1] = {0.0f};
#pragma unroll
    for (int q = 0; q < K; ++q) {
        x[q] = d.sig[q] * d.dtn[q];
        if (head[q]) agg[0] = 0.0f;
        agg[0] += x[q];
    }
    if (lane == 0 && !any_head) agg[0] += c.x;
    seg_scan_plan<1, false>(agg, plan);
    float run = shift_up(agg[0], lane, c.x);
    // T before the lane's first sample; inside a ray the transmittance before a sample is the one
    // after the previous sample, the same exp of the same depth. After a sample it is exp(-depth),
    // not T (1 - alpha), which cancels once e^-x is small.
    float tj = expf(-run);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        if (head[q]) { run = 0.0f; tj = 1.0f; }
        run += x[q];
        d.w[q] = in[q] ? tj * opacity(x[q]) : 0.0f;
        d.tn[q] = expf(-run);
        tj = d.tn[q];
    }
    next.x = __shfl_sync(FULL_MASK, agg[0], WARP - 1);
    // weight sums before each sample
    float wex[K];
    agg[0] = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        if (head[q]) agg[0] = 0.0f;
        agg[0] += d.w[q];
    }
    if (lane == 0 && !any_head) agg[0] += c.w;
    seg_scan_plan<1, false>(agg, plan);
    run = shift_up(agg[0], lane, c.w);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        wex[q] = head[q] ? 0.0f : run;
        run = wex[q] + d.w[q];
    }
    next.w = __shfl_sync(FULL_MASK, agg[0], WARP - 1);
    // increments of m (the first sample of a ray has none) and A = sum dm W_<
    const float m_before = shift_up(m[K - 1], lane, c.m);
    agg[0] = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const float mp = head[q] ? m[q] : (q ? m[q - 1] : m_before);
        d.dm[q] = in[q] ? fmaxf(m[q] - mp, 0.0f) : 0.0f;
        if (head[q]) agg[0] = 0.0f;
        agg[0] += d.dm[q] * wex[q];
    }
    if (lane == 0 && !any_head) agg[0] += c.a;
    seg_scan_plan<1, false>(agg, plan);
    run = shift_up(agg[0], lane, c.a);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        run = (head[q] ? 0.0f : run) + d.dm[q] * wex[q];
        d.a[q] = run;
    }
    next.a = __shfl_sync(FULL_MASK, agg[0], WARP - 1);
    next.m = __shfl_sync(FULL_MASK, m[K - 1], WARP - 1);
}

// Sample flags of a tile: in range, first / last sample of its ray, and the ray's index in the
// warp's table.
__device__ __forceinline__ void tile_flags(const uint32_t* t_off, const uint32_t* t_end, int nr, uint32_t s_begin,
                                           uint32_t s_end, uint32_t s0, bool (&in)[ST_K], bool (&head)[ST_K],
                                           bool (&last)[ST_K], int (&ri)[ST_K]) {
    int cur = find_ray(t_off, nr, s0 > s_begin ? s0 : s_begin);
    uint32_t coff = t_off[cur], cend = t_end[cur];
#pragma unroll
    for (int q = 0; q < ST_K; ++q) {
        const uint32_t s = s0 + q;
        in[q] = s >= s_begin && s < s_end;
        while (in[q] && s >= cend) {  // the next ray with samples
            ++cur;
            coff = t_off[cur];
            cend = t_end[cur];
        }
        ri[q] = cur;
        head[q] = in[q] && s == coff;
        last[q] = in[q] && s + 1 == cend;
    }
}

template <bool VEC, int ACT>
__global__ void __launch_bounds__(LOSS_THREADS)
distortion_tiles_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rpw,
                        const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets, float lambda,
                        const float* __restrict__ grad_ray, float* __restrict__ ray_loss, float* loss_sum,
                        float* __restrict__ dd, float* partials, uint32_t* ticket) {
    constexpr int K = ST_K;
    __shared__ uint32_t t_off[LOSS_WARPS][WARP], t_end[LOSS_WARPS][WARP];
    __shared__ float t_k[LOSS_WARPS][WARP], t_gs[LOSS_WARPS][WARP];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    const uint32_t r0 = (blockIdx.x * LOSS_WARPS + wid) * rpw;
    float acc[1] = {0.0f};
    if (r0 < n_live) {  // whole warps; every thread reaches the block sum below
        const int nr = (int)min(rpw, n_live - r0);
        if (lane < nr) {
            const uint32_t r = r0 + lane, o = offsets[r], n = counts[r];
            t_off[wid][lane] = o;
            t_end[wid][lane] = o + n;
            t_k[wid][lane] = n ? lambda / (float)n : 0.0f;
            t_gs[wid][lane] = grad_ray ? grad_ray[r] : 1.0f;
            if (n == 0 && ray_loss) ray_loss[r] = 0.0f;
        }
        __syncwarp();
        const uint32_t s_begin = t_off[wid][0], s_end = t_end[wid][nr - 1];
        const uint32_t b0 = VEC ? (s_begin & ~3u) : s_begin;
        const uint32_t span = WARP * K;
        const uint32_t n_tiles = s_end > b0 ? (s_end - b0 + span - 1) / span : 0u;
        // forward: carries kept for the backward (tile t in lane t % 32, slot t / 32)
        DistCarry keep0{0.0f, 0.0f, 0.0f, 0.0f}, keep1 = keep0;
        DistCarry c{0.0f, 0.0f, 0.0f, 0.0f};
        float cl[2] = {0.0f, 0.0f};  // running loss sums (sum dtn w^2, sum w A) of the open ray
        for (uint32_t t = 0; t < n_tiles; ++t) {
            if ((uint32_t)lane == (t & 31u)) {
                if (t < 32u) keep0 = c; else if (t < 64u) keep1 = c;
            }
            const uint32_t s0 = b0 + t * span + (uint32_t)lane * K;
            bool in[K], head[K], last[K];
            int ri[K];
            tile_flags(t_off[wid], t_end[wid], nr, s_begin, s_end, s0, in, head, last, ri);
            bool any_head = false;
#pragma unroll
            for (int q = 0; q < K; ++q) any_head = any_head || head[q];
            const uint32_t plan = seg_plan<false>(any_head, lane);
            DistTile d;
            DistCarry nx;
            dist_tile_forward<VEC, ACT>(S, s0, in, head, any_head, plan, lane, c, nx, d);
            float l2[2] = {0.0f, 0.0f};
#pragma unroll
            for (int q = 0; q < K; ++q) {
                if (head[q]) l2[0] = l2[1] = 0.0f;
                l2[0] += d.dtn[q] * d.w[q] * d.w[q];
                l2[1] += d.w[q] * d.a[q];
            }
            if (lane == 0 && !any_head) { l2[0] += cl[0]; l2[1] += cl[1]; }
            seg_scan_plan<2, false>(l2, plan);
            float e2[2] = {shift_up(l2[0], lane, cl[0]), shift_up(l2[1], lane, cl[1])};
#pragma unroll
            for (int q = 0; q < K; ++q) {
                if (head[q]) e2[0] = e2[1] = 0.0f;
                e2[0] += d.dtn[q] * d.w[q] * d.w[q];
                e2[1] += d.w[q] * d.a[q];
                if (last[q]) {
                    const float loss = t_k[wid][ri[q]] * ((1.0f / 3.0f) * e2[0] + 2.0f * e2[1]);
                    if (ray_loss) ray_loss[r0 + (uint32_t)ri[q]] = loss;
                    acc[0] += loss;
                }
            }
            cl[0] = __shfl_sync(FULL_MASK, l2[0], WARP - 1);
            cl[1] = __shfl_sync(FULL_MASK, l2[1], WARP - 1);
            c = nx;
        }
        if (dd) {
            // backward: tiles from the last; suffix carries of the ray open at each tile's end
            float sw = 0.0f, sf = 0.0f, sg = 0.0f;
            for (int t = (int)n_tiles - 1; t >= 0; --t) {
                DistCarry ct;
                if (t < SAVED_TILES) {
                    const DistCarry& kc = t < 32 ? keep0 : keep1;
                    const int src = t & 31;
                    ct.x = __shfl_sync(FULL_MASK, kc.x, src);
                    ct.w = __shfl_sync(FULL_MASK, kc.w, src);
                    ct.a = __shfl_sync(FULL_MASK, kc.a, src);
                    ct.m = __shfl_sync(FULL_MASK, kc.m, src);
                } else {  // replay the forward from the last kept carry
                    const int src = (SAVED_TILES - 1) & 31;
                    ct.x = __shfl_sync(FULL_MASK, keep1.x, src);
                    ct.w = __shfl_sync(FULL_MASK, keep1.w, src);
                    ct.a = __shfl_sync(FULL_MASK, keep1.a, src);
                    ct.m = __shfl_sync(FULL_MASK, keep1.m, src);
                    for (int u = SAVED_TILES - 1; u < t; ++u) {
                        const uint32_t su = b0 + (uint32_t)u * span + (uint32_t)lane * K;
                        bool in[K], head[K], last[K];
                        int ri[K];
                        tile_flags(t_off[wid], t_end[wid], nr, s_begin, s_end, su, in, head, last, ri);
                        bool any_head = false;
#pragma unroll
                        for (int q = 0; q < K; ++q) any_head = any_head || head[q];
                        DistTile du;
                        DistCarry nx;
                        dist_tile_forward<VEC, ACT>(S, su, in, head, any_head, seg_plan<false>(any_head, lane), lane,
                                                    ct, nx, du);
                        ct = nx;
                    }
                }
                const uint32_t s0 = b0 + (uint32_t)t * span + (uint32_t)lane * K;
                bool in[K], head[K], last[K];
                int ri[K];
                tile_flags(t_off[wid], t_end[wid], nr, s_begin, s_end, s0, in, head, last, ri);
                bool any_head = false, any_tail = false;
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    any_head = any_head || head[q];
                    any_tail = any_tail || last[q];
                }
                DistTile d;
                DistCarry nx;
                dist_tile_forward<VEC, ACT>(S, s0, in, head, any_head, seg_plan<false>(any_head, lane), lane, ct, nx,
                                            d);
                const uint32_t splan = seg_plan<true>(any_tail, lane);
                // W_>= (inclusive suffix of w)
                float agg[1] = {0.0f};
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    if (last[q]) agg[0] = 0.0f;
                    agg[0] += d.w[q];
                }
                if (lane == WARP - 1 && !any_tail) agg[0] += sw;
                seg_scan_plan<1, true>(agg, splan);
                float run = shift_down(agg[0], lane, sw);
                float wge[K];
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    wge[q] = (last[q] ? 0.0f : run) + d.w[q];
                    run = wge[q];
                }
                sw = __shfl_sync(FULL_MASK, agg[0], 0);
                // B = sum over later samples of dm W_>=
                agg[0] = 0.0f;
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    if (last[q]) agg[0] = 0.0f;
                    agg[0] += d.dm[q] * wge[q];
                }
                if (lane == WARP - 1 && !any_tail) agg[0] += sf;
                seg_scan_plan<1, true>(agg, splan);
                run = shift_down(agg[0], lane, sf);
                float g[K];
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    const float b = last[q] ? 0.0f : run;
                    g[q] = t_k[wid][ri[q]] * ((2.0f / 3.0f) * d.dtn[q] * d.w[q] + 2.0f * (d.a[q] + b));
                    run = b + d.dm[q] * wge[q];
                }
                sf = __shfl_sync(FULL_MASK, agg[0], 0);
                // sum over later samples of g w, and the gradient
                agg[0] = 0.0f;
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    if (last[q]) agg[0] = 0.0f;
                    agg[0] += g[q] * d.w[q];
                }
                if (lane == WARP - 1 && !any_tail) agg[0] += sg;
                seg_scan_plan<1, true>(agg, splan);
                run = shift_down(agg[0], lane, sg);
                float o[K];
#pragma unroll
                for (int q = K - 1; q >= 0; --q) {
                    const float later = last[q] ? 0.0f : run;
                    o[q] = in[q] ? t_gs[wid][ri[q]] * d.dtn[q] * (g[q] * d.tn[q] - later) * act_dsigma(ACT, d.sig[q])
                                 : 0.0f;
                    run = later + g[q] * d.w[q];
                }
                sg = __shfl_sync(FULL_MASK, agg[0], 0);
                bool all_in = true;
#pragma unroll
                for (int q = 0; q < K; ++q) all_in = all_in && in[q];
                if (VEC && all_in) {
                    *reinterpret_cast<float4*>(dd + s0) = make_float4(o[0], o[1], o[2], o[3]);
                } else {
#pragma unroll
                    for (int q = 0; q < K; ++q)
                        if (in[q]) dd[s0 + q] = o[q];
                }
            }
        }
    }
    if (loss_sum) block_sum_and_finish<1>(acc, partials, ticket, loss_sum, FinishScale{{1.0f, 0.0f}, n_dev, n_rays, 1u});
}

// VJP of the compositor from the forward's stored per-sample transmittance (after the sample)
// and weights, the alternative to recomputing them (composite_bwd_tiles_kernel): the same suffix
// sums, read instead of rebuilt.
__global__ void __launch_bounds__(LOSS_THREADS)
composite_bwd_stored_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rs,
                            const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                            const uint32_t* __restrict__ n_used, const float* __restrict__ t_saved,
                            const float* __restrict__ w_saved, const float* __restrict__ grad_rgba,
                            float* __restrict__ dd, float* __restrict__ drgb) {
    const int lane = threadIdx.x & 31;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    const uint32_t nw = gridDim.x * LOSS_WARPS;
    for (uint32_t r = blockIdx.x * LOSS_WARPS + (threadIdx.x >> 5); r < n_live; r += nw) {
        const uint32_t o = offsets[r], n = counts[r];
        const uint32_t used = min(n_used[r], n);
        const float gr = grad_rgba[r], gg = grad_rgba[r + rs], gb = grad_rgba[r + 2 * (size_t)rs],
                    ga = grad_rgba[r + 3 * (size_t)rs];
        zero_tail(dd, drgb, S.ss, o, used, n, lane);
        float su = 0.0f;  // sum over later chunks of w u, u = gr r + gg g + gb b + ga
        if (used == 0) continue;
        for (int base = (int)(((used - 1) / WARP) * WARP); base >= 0; base -= WARP) {
            const uint32_t j = (uint32_t)base + lane;
            const bool valid = j < used;
            float u = 0.0f, w = 0.0f, tn = 0.0f, dtv = 0.0f, sigma = 0.0f;
            float cr = 0.0f, cg = 0.0f, cb = 0.0f;
            if (valid) {
                const size_t s = (size_t)o + j;
                sigma = act_sigma(S.act, S.density[s]);
                dtv = S.dt[s];
                cr = S.rgb[s]; cg = S.rgb[s + S.ss]; cb = S.rgb[s + 2 * (size_t)S.ss];
                tn = t_saved[s];
                w = w_saved[s];
                u = gr * cr + gg * cg + gb * cb + ga;
            }
            const float incl = warp_inclusive_suffix_sum(w * u, lane) + su;
            const float u_ex = shift_down(incl, lane, su);
            if (valid) {
                const size_t s = (size_t)o + j;
                dd[s] = dtv * (tn * u - u_ex) * act_dsigma(S.act, sigma);
                drgb[s] = gr * w;
                drgb[s + S.ss] = gg * w;
                drgb[s + 2 * (size_t)S.ss] = gb * w;
            }
            su = __shfl_sync(FULL_MASK, incl, 0);
        }
    }
}

__global__ void __launch_bounds__(LOSS_THREADS)
recon_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rs, const uint32_t* __restrict__ counts,
             const uint32_t* __restrict__ offsets, float min_t, float inv_nrays, float grad_scale,
             const float* __restrict__ target, const float* __restrict__ bg, float* __restrict__ ray_rgba,
             float* __restrict__ loss, float* loss_sum, float* __restrict__ dd, float* __restrict__ drgb,
             float* partials, uint32_t* ticket) {
    const int lane = threadIdx.x & 31;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    const uint32_t nw = gridDim.x * LOSS_WARPS;
    float acc[1] = {0.0f};
    for (uint32_t r = blockIdx.x * LOSS_WARPS + (threadIdx.x >> 5); r < n_live; r += nw) {
        const uint32_t o = offsets[r], n = counts[r];
        const CompFwd c = composite_forward_ray<CB_K>(S, o, n, min_t, lane);
        const ReconGrad g = recon_loss_ray(c, target, bg, r, rs, inv_nrays);
        if (lane == 0) {
            if (ray_rgba) {
                ray_rgba[r] = c.r; ray_rgba[r + rs] = c.g; ray_rgba[r + 2 * (size_t)rs] = c.b;
                ray_rgba[r + 3 * (size_t)rs] = c.a;
            }
            if (loss) {
                loss[r] = g.l[0]; loss[r + rs] = g.l[1]; loss[r + 2 * (size_t)rs] = g.l[2]; loss[r + 3 * (size_t)rs] = g.l[3];
            }
            acc[0] += g.l[0] + g.l[1] + g.l[2] + g.l[3];
        }
        zero_tail(dd, drgb, S.ss, o, c.used, n, lane);
        composite_vjp_ray<CB_K>(S, o, c.used, c.depth, g.gr, g.gg, g.gb, g.ga, grad_scale, lane,
                                [&](uint32_t j, bool valid, float ds, float xr, float xg, float xb) {
                                    if (!valid) return;
                                    const size_t s = (size_t)o + j;
                                    dd[s] = ds;
                                    drgb[s] = xr;
                                    drgb[s + S.ss] = xg;
                                    drgb[s + 2 * (size_t)S.ss] = xb;
                                });
    }
    if (loss_sum) block_sum_and_finish<1>(acc, partials, ticket, loss_sum, FinishScale{{inv_nrays, 0.0f}, nullptr, 0u, 0u});
}

// ---- register-blocked rays -----------------------------------------------------------------
// A ray of at most RB_MAX samples is held in registers, lane l owning the consecutive samples
// [RB_SPL*l, RB_SPL*l + RB_SPL). Its inputs are read once, and each running sum along the ray is
// a prefix inside the lane plus one warp scan of the lane totals (instead of one warp scan per
// 32-sample chunk). Longer rays take the chunked path.
constexpr int RB_SPL = 8;
constexpr uint32_t RB_MAX = RB_SPL * WARP;

// In place inclusive prefix along the ray plus `carry` (the sum before this block of samples);
// returns the sum before the lane's first sample, so that the exclusive prefix of sample q is
// (q ? v[q-1] : returned value).
template <int K>
__device__ __forceinline__ float blk_prefix(float (&v)[K], int lane, float carry = 0.0f) {
#pragma unroll
    for (int q = 1; q < K; ++q) v[q] += v[q - 1];
    const float before = shift_up(warp_inclusive_sum(v[K - 1], lane), lane, 0.0f) + carry;
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] += before;
    return before;
}

// In place inclusive suffix along the ray plus `carry` (the sum after this block of samples);
// returns the sum after the lane's last sample, so that the exclusive suffix of sample q is
// (q < K-1 ? v[q+1] : returned value).
template <int K>
__device__ __forceinline__ float blk_suffix(float (&v)[K], int lane, float carry = 0.0f) {
#pragma unroll
    for (int q = K - 2; q >= 0; --q) v[q] += v[q + 1];
    const float after = shift_down(warp_inclusive_suffix_sum(v[0], lane), lane, 0.0f) + carry;
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] += after;
    return after;
}

// ---- shared-memory staging of one ray's samples ----------------------------------------
// Each input array of the ray is copied with cp.async into a per-warp buffer, all of them before
// a single wait, so the ray pays one memory latency; results go back through the same buffers
// with coalesced stores. A buffer array holds RB_PITCH floats. Rays of at most RB_MAX samples use
// the slot layout: slot i at i + 4 (i / 32), so that every 16-byte group of slots (4c .. 4c + 3)
// stays whole and aligned, and lane l reads its slots 8l .. 8l + 7 as two 16-byte loads without
// bank conflicts (8 consecutive lanes cover the 32 banks). With 16-byte staging the ray's first
// sample sits in slot o mod 4 (o its first sample in the batch), so that the copies are whole
// aligned groups. The chunks of longer rays use the layout j + j / 32 (one sample per lane
// per copy).
constexpr int RB_PITCH = RB_MAX + RB_MAX / WARP * 4;
enum StageArray : int { SA_SIG = 0, SA_DT, SA_R, SA_G, SA_B, SA_DTN, SA_M, SA_T, SA_GD, SA_N };
constexpr size_t TL_STAGE_BYTES = (size_t)SA_N * RB_PITCH * sizeof(float);  // one warp's staging buffer

__device__ __forceinline__ uint32_t skew(uint32_t j) { return j + (j >> 5); }
__device__ __forceinline__ uint32_t slot4(uint32_t i) { return i + ((i >> 5) << 2); }

__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async16(float* dst, const float* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void stage_segment(float* buf, const float* __restrict__ src, size_t o, uint32_t n,
                                              int lane) {
    for (uint32_t j = (uint32_t)lane; j < n; j += WARP) cp_async4(buf + skew(j), src + o + j);
}

__device__ __forceinline__ void store_segment(float* __restrict__ dst, const float* buf, size_t o, uint32_t n,
                                              int lane) {
    for (uint32_t j = (uint32_t)lane; j < n; j += WARP) dst[o + j] = buf[skew(j)];
}

// Samples [o, o + n) of src into the slots from e: with VEC the whole 16-byte groups of
// [o - e, o + n) (e = o mod 4; src 16-byte aligned), else one sample per copy (e = 0).
template <bool VEC>
__device__ __forceinline__ void stage_slots(float* buf, const float* __restrict__ src, uint32_t o, uint32_t e,
                                            uint32_t n, int lane) {
    if (VEC) {
        const uint32_t groups = (e + n + 3u) >> 2;
        const float* base = src + (o - e);
        for (uint32_t c = (uint32_t)lane; c < groups; c += WARP) cp_async16(buf + slot4(4u * c), base + 4u * c);
    } else {
        for (uint32_t j = (uint32_t)lane; j < n; j += WARP) cp_async4(buf + slot4(j), src + o + j);
    }
}

// Slots [e, e + n) back to dst[o, o + n): whole 16-byte groups in one store, the ray's partial
// first and last groups sample by sample (their other samples belong to neighbouring rays).
template <bool VEC>
__device__ __forceinline__ void store_slots(float* __restrict__ dst, const float* buf, uint32_t o, uint32_t e,
                                            uint32_t n, int lane) {
    if (VEC) {
        const uint32_t groups = (e + n + 3u) >> 2, end = e + n;
        float* base = dst + (o - e);
        for (uint32_t c = (uint32_t)lane; c < groups; c += WARP) {
            const uint32_t i = 4u * c;
            const float4 v = *reinterpret_cast<const float4*>(buf + slot4(i));
            if (i >= e && i + 4u <= end) {
                *reinterpret_cast<float4*>(base + i) = v;
            } else {
                if (i >= e && i < end) base[i] = v.x;
                if (i + 1u >= e && i + 1u < end) base[i + 1u] = v.y;
                if (i + 2u >= e && i + 2u < end) base[i + 2u] = v.z;
                if (i + 3u >= e && i + 3u < end) base[i + 3u] = v.w;
            }
        }
    } else {
        for (uint32_t j = (uint32_t)lane; j < n; j += WARP) dst[o + j] = buf[slot4(j)];
    }
}

// The lane's K slots K lane .. K lane + K - 1 (K a multiple of 4).
template <int K>
__device__ __forceinline__ void read_slots(const float* buf, int lane, float (&v)[K]) {
    const float4* p = reinterpret_cast<const float4*>(buf + slot4((uint32_t)(K * lane)));
#pragma unroll
    for (int c = 0; c < K / 4; ++c) {
        const float4 a = p[c];
        v[4 * c] = a.x; v[4 * c + 1] = a.y; v[4 * c + 2] = a.z; v[4 * c + 3] = a.w;
    }
}
template <int K>
__device__ __forceinline__ void write_slots(float* buf, int lane, const float (&v)[K]) {
    float4* p = reinterpret_cast<float4*>(buf + slot4((uint32_t)(K * lane)));
#pragma unroll
    for (int c = 0; c < K / 4; ++c) p[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
}

// e^-x for the transmittances and opacities of the fused loss kernel: the fast intrinsic, whose
// relative error at the optical depths that matter here (x below about 20) is a few 1e-6.
__device__ __forceinline__ float exp_neg(float x) { return __expf(-x); }


// One ray of at most 32 K samples (32 K - o mod 4 with VEC) of the fused training losses, in
// the slot layout, with the compositor's transmittance and weights kept from its forward:
// compositor forward (training-kernels-fused.cuh:227-264), reconstruction loss (:434-477),
// compositor VJP (:269-341), distortion forward/backward in the non-cancelling form above, and
// the gradient merge with the distance scaling (nerf-network.cu:734-758). `sm` is the warp's
// staging buffer, SA_N arrays of RB_PITCH floats. Lane l owns the slots K l .. K l + K - 1,
// sample j = slot - e; slots outside the ray read as zero (their staged values belong to other
// rays). `accumulate`: the merged gradient is added to grad_density (else written over it).
template <bool VEC, int K>
__device__ __forceinline__ void train_losses_ray_blocked(const Samples& S, uint32_t r, uint32_t o, uint32_t n,
                                                         int lane, float min_t, float inv_nrays, float grad_scale,
                                                         float lambda, const float* __restrict__ target,
                                                         const float* __restrict__ bg, uint32_t rs,
                                                         float* __restrict__ ray_rgba,
                                                         float* __restrict__ grad_density, float* __restrict__ drgb,
                                                         float& acc_rec, float& acc_dist, float* sm, bool accumulate) {
    static_assert(K % 4 == 0 && K <= RB_SPL, "slots are read in 16-byte groups");
    const uint32_t e = VEC ? (o & 3u) : 0u;
    const uint32_t j0 = (uint32_t)lane * K - e;  // sample of the lane's first slot (wraps below the ray)
    const size_t ss = S.ss;
    float* const b_sig = sm + SA_SIG * RB_PITCH;
    float* const b_dt = sm + SA_DT * RB_PITCH;
    float* const b_r = sm + SA_R * RB_PITCH;
    float* const b_g = sm + SA_G * RB_PITCH;
    float* const b_b = sm + SA_B * RB_PITCH;
    float* const b_dtn = sm + SA_DTN * RB_PITCH;
    float* const b_m = sm + SA_M * RB_PITCH;
    float* const b_t = sm + SA_T * RB_PITCH;
    float* const b_gd = sm + SA_GD * RB_PITCH;
    // every input of the ray in flight at once; the per-ray inputs of the loss meanwhile
    __syncwarp();  // the previous ray's write-back reads of the buffers are done
    stage_slots<VEC>(b_sig, S.density, o, e, n, lane);
    stage_slots<VEC>(b_dt, S.dt, o, e, n, lane);
    stage_slots<VEC>(b_r, S.rgb, o, e, n, lane);
    stage_slots<VEC>(b_g, S.rgb + ss, o, e, n, lane);
    stage_slots<VEC>(b_b, S.rgb + 2 * ss, o, e, n, lane);
    if (lambda > 0.0f) {
        stage_slots<VEC>(b_dtn, S.dt_norm, o, e, n, lane);
        stage_slots<VEC>(b_m, S.m_norm, o, e, n, lane);
    }
    if (S.t) stage_slots<VEC>(b_t, S.t, o, e, n, lane);
    if (accumulate) stage_slots<VEC>(b_gd, grad_density, o, e, n, lane);
    const float gt_r = target[r], gt_g = target[r + rs], gt_b = target[r + 2 * (size_t)rs];
    const float gt_a = target[r + 3 * (size_t)rs];
    const float bg_r = bg[r], bg_g = bg[r + rs], bg_b = bg[r + 2 * (size_t)rs];
    cp_async_wait_all();
    __syncwarp();
    bool valid[K];
#pragma unroll
    for (int q = 0; q < K; ++q) valid[q] = j0 + q < n;
    float sig[K], dt[K], cr[K], cg[K], cb[K];
    read_slots(b_sig, lane, sig);
    read_slots(b_dt, lane, dt);
    read_slots(b_r, lane, cr);
    read_slots(b_g, lane, cg);
    read_slots(b_b, lane, cb);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        sig[q] = valid[q] ? act_sigma(S.act, sig[q]) : 0.0f;
        dt[q] = valid[q] ? dt[q] : 0.0f;
        cr[q] = valid[q] ? cr[q] : 0.0f;
        cg[q] = valid[q] ? cg[q] : 0.0f;
        cb[q] = valid[q] ? cb[q] : 0.0f;
    }
    // ---- compositor forward: T after each sample, weights, the transmittance cut
    float T[K], w[K];
    uint32_t used = n;
    float depth;
    {
        float p[K];
#pragma unroll
        for (int q = 0; q < K; ++q) p[q] = sig[q] * dt[q];
        blk_prefix(p, lane);
#pragma unroll
        for (int q = 0; q < K; ++q) T[q] = exp_neg(p[q]);
        const float t_in = shift_up(T[K - 1], lane, 1.0f);
        int first_q = K;
        float cut_depth = 0.0f;
#pragma unroll
        for (int q = K - 1; q >= 0; --q) {
            w[q] = (q ? T[q - 1] : t_in) * opacity(sig[q] * dt[q]);
            if (valid[q] && T[q] < min_t) { first_q = q; cut_depth = p[q]; }
        }
        const unsigned term = __ballot_sync(FULL_MASK, first_q < K);
        if (term) {
            const int fl = __ffs(term) - 1;
            used = (uint32_t)fl * K + (uint32_t)__shfl_sync(FULL_MASK, first_q, fl) + 1u - e;
            depth = __shfl_sync(FULL_MASK, cut_depth, fl);
        } else {
            depth = __shfl_sync(FULL_MASK, p[K - 1], WARP - 1);
        }
    }
    float ar = 0.0f, ag = 0.0f, ab = 0.0f, aa = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        w[q] = j0 + q < used ? w[q] : 0.0f;
        ar += w[q] * cr[q];
        ag += w[q] * cg[q];
        ab += w[q] * cb[q];
        aa += w[q];
    }
    CompFwd c;
    c.r = warp_sum(ar); c.g = warp_sum(ag); c.b = warp_sum(ab); c.a = warp_sum(aa);
    c.depth = depth;
    c.used = used;
    const ReconGrad g = recon_grad(c, gt_r, gt_g, gt_b, gt_a, bg_r, bg_g, bg_b, inv_nrays);
    if (lane == 0) {
        if (ray_rgba) {
            ray_rgba[r] = c.r; ray_rgba[r + rs] = c.g; ray_rgba[r + 2 * (size_t)rs] = c.b;
            ray_rgba[r + 3 * (size_t)rs] = c.a;
        }
        acc_rec += g.l[0] + g.l[1] + g.l[2] + g.l[3];
    }
    // ---- compositor VJP. The upstream weights gr, gg, gb, ga are the same for the whole ray, so
    // the four suffix sums of w c and w enter only through sum_{i>j} w_i u_i with
    // u = gr cr + gg cg + gb cb + ga: one suffix scan.
    float ds[K];
    {
        float su[K], cu[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            cu[q] = g.gr * cr[q] + g.gg * cg[q] + g.gb * cb[q] + g.ga;
            su[q] = w[q] * cu[q];
        }
        const float su_after = blk_suffix(su, lane);
        float dr[K], dg[K], db[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float u_ex = q < K - 1 ? su[q + 1] : su_after;
            const float d = dt[q] * (T[q] * cu[q] - u_ex);
            ds[q] = j0 + q < used ? grad_scale * d * act_dsigma(S.act, sig[q]) : 0.0f;
            dr[q] = grad_scale * g.gr * w[q];
            dg[q] = grad_scale * g.gg * w[q];
            db[q] = grad_scale * g.gb * w[q];
        }
        write_slots(b_r, lane, dr);
        write_slots(b_g, lane, dg);
        write_slots(b_b, lane, db);
    }
    // ---- distortion forward and backward (all n samples, no transmittance cut)
    if (lambda > 0.0f) {
        float dtn[K], mm[K];
        read_slots(b_dtn, lane, dtn);
        read_slots(b_m, lane, mm);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            dtn[q] = valid[q] ? dtn[q] : 0.0f;
            mm[q] = valid[q] ? mm[q] : 0.0f;
        }
        float wd[K], tnext[K], dm[K], A[K];
        {
            float p[K];
#pragma unroll
            for (int q = 0; q < K; ++q) p[q] = sig[q] * dtn[q];
            blk_prefix(p, lane);
#pragma unroll
            for (int q = 0; q < K; ++q) tnext[q] = exp_neg(p[q]);  // T_{j+1}
            const float t_in = shift_up(tnext[K - 1], lane, 1.0f);
#pragma unroll
            for (int q = 0; q < K; ++q)
                wd[q] = valid[q] ? (q ? tnext[q - 1] : t_in) * opacity(sig[q] * dtn[q]) : 0.0f;
        }
        {
            float W[K];
#pragma unroll
            for (int q = 0; q < K; ++q) W[q] = wd[q];
            const float w_before = blk_prefix(W, lane);
            // m of the previous sample; the first sample has no increment
            const float m_in = __shfl_up_sync(FULL_MASK, mm[K - 1], 1);
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float m_prev = q ? mm[q - 1] : m_in;
                dm[q] = valid[q] && j0 + q != 0u ? fmaxf(mm[q] - m_prev, 0.0f) : 0.0f;
                A[q] = dm[q] * (q ? W[q - 1] : w_before);
            }
            blk_prefix(A, lane);
        }
        float uni = 0.0f, cross = 0.0f;
#pragma unroll
        for (int q = 0; q < K; ++q) { uni += dtn[q] * wd[q] * wd[q]; cross += wd[q] * A[q]; }
        uni = warp_sum(uni);
        cross = warp_sum(cross);
        const float k = n ? lambda / (float)n : 0.0f;
        if (lane == 0) acc_dist += k * ((1.0f / 3.0f) * uni + 2.0f * cross);
        float Wge[K];
#pragma unroll
        for (int q = 0; q < K; ++q) Wge[q] = wd[q];
        blk_suffix(Wge, lane);
        float f[K];
#pragma unroll
        for (int q = 0; q < K; ++q) f[q] = dm[q] * Wge[q];
        const float f_after = blk_suffix(f, lane);
        float gw[K], gq[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float b = q < K - 1 ? f[q + 1] : f_after;  // B_j
            gq[q] = k * ((2.0f / 3.0f) * dtn[q] * wd[q] + 2.0f * (A[q] + b));
            gw[q] = gq[q] * wd[q];
        }
        const float gw_after = blk_suffix(gw, lane);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const float gw_ex = q < K - 1 ? gw[q + 1] : gw_after;
            const float dd = grad_scale * dtn[q] * (gq[q] * tnext[q] - gw_ex) * act_dsigma(S.act, sig[q]);
            ds[q] += valid[q] ? dd : 0.0f;
        }
    }
    // ---- gradient merge: copy_gradients_kernel<1,true> twice + apply_gradient_distance_scaling_kernel
    {
        float gd[K], tt[K];
        if (accumulate) {
            read_slots(b_gd, lane, gd);
        } else {
#pragma unroll
            for (int q = 0; q < K; ++q) gd[q] = 0.0f;
        }
        if (S.t) read_slots(b_t, lane, tt);
#pragma unroll
        for (int q = 0; q < K; ++q) {
            float v = gd[q] + ds[q];
            if (S.t) v = tt[q] < 1.0f ? v * (tt[q] * tt[q]) : v;
            gd[q] = v;
        }
        write_slots(b_gd, lane, gd);
    }
    __syncwarp();
    store_slots<VEC>(grad_density, b_gd, o, e, n, lane);
    store_slots<VEC>(drgb, b_r, o, e, n, lane);
    store_slots<VEC>(drgb + ss, b_g, o, e, n, lane);
    store_slots<VEC>(drgb + 2 * ss, b_b, o, e, n, lane);
}

// Rays longer than RB_MAX: the same computation over super-chunks of RB_MAX samples in the
// blocked layout. The compositor forward carries its running sums from chunk to chunk; its VJP
// walks the chunks from the last and rebuilds the transmittance from the ray's optical depth
// and the suffix sums of sigma * dt, as the chunked path does. The distortion forward keeps each
// chunk's starting carry (lane c holds chunk c for c < 32; later chunks replay from chunk 31),
// and its backward recomputes each chunk's forward quantities from that carry.
struct ScCarry { float x, w, a, m; };

struct ScStore {
    ScCarry s;
    __device__ __forceinline__ void put(uint32_t c, int lane, const ScCarry& v) {
        if (c < 32u && (uint32_t)lane == c) s = v;
    }
    __device__ __forceinline__ ScCarry get(uint32_t c) const {
        const int src = (int)min(c, 31u);
        ScCarry v;
        v.x = __shfl_sync(FULL_MASK, s.x, src);
        v.w = __shfl_sync(FULL_MASK, s.w, src);
        v.a = __shfl_sync(FULL_MASK, s.a, src);
        v.m = __shfl_sync(FULL_MASK, s.m, src);
        return v;
    }
};

// Distortion forward of one super-chunk from its carry: weights w_j, T_{j+1}, the increments of
// m and A_j, and the next chunk's carry; adds the chunk's uni and cross terms (per lane).
template <int K>
__device__ __forceinline__ void sc_dist_forward(const float (&sig)[K], const float (&dtn)[K], const float (&mm)[K],
                                                uint32_t j0, uint32_t n, int lane, const ScCarry& c, float (&wd)[K],
                                                float (&tnext)[K], float (&dm)[K], float (&A)[K], ScCarry& next,
                                                float& uni, float& cross) {
    float p[K];
#pragma unroll
    for (int q = 0; q < K; ++q) p[q] = sig[q] * dtn[q];
    const float before = blk_prefix(p, lane, c.x);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const float em = expm1f(-sig[q] * dtn[q]);
        const float tj = expf(-(q ? p[q - 1] : before));
        wd[q] = j0 + q < n ? tj * -em : 0.0f;
        tnext[q] = expf(-p[q]);  // T_{j+1}; T_j (1 + em) cancels once e^-x is small
    }
    float W[K];
#pragma unroll
    for (int q = 0; q < K; ++q) W[q] = wd[q];
    const float w_before = blk_prefix(W, lane, c.w);
    const float m_in = __shfl_up_sync(FULL_MASK, mm[K - 1], 1);
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const float m_prev = q ? mm[q - 1] : (lane ? m_in : c.m);
        dm[q] = j0 + q < n ? fmaxf(mm[q] - m_prev, 0.0f) : 0.0f;
        A[q] = dm[q] * (q ? W[q - 1] : w_before);
    }
    blk_prefix(A, lane, c.a);
#pragma unroll
    for (int q = 0; q < K; ++q) { uni += dtn[q] * wd[q] * wd[q]; cross += wd[q] * A[q]; }
    // only a chunk that is followed by another one passes its carry on, and such a chunk is full
    next.x = __shfl_sync(FULL_MASK, p[K - 1], WARP - 1);
    next.w = __shfl_sync(FULL_MASK, W[K - 1], WARP - 1);
    next.a = __shfl_sync(FULL_MASK, A[K - 1], WARP - 1);
    next.m = __shfl_sync(FULL_MASK, mm[K - 1], WARP - 1);
}

template <int K>
__device__ __forceinline__ void sc_load_dist(const Samples& S, uint32_t o, uint32_t j0, uint32_t n, float (&sig)[K],
                                             float (&dtn)[K], float (&mm)[K]) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const bool valid = j0 + q < n;
        const size_t s = (size_t)o + j0 + q;
        sig[q] = valid ? act_sigma(S.act, S.density[s]) : 0.0f;
        dtn[q] = valid ? S.dt_norm[s] : 0.0f;
        mm[q] = valid ? S.m_norm[s] : 0.0f;
    }
}

// A ray of more than RB_MAX samples: the same three passes as the blocked path (compositor
// forward to the cut, distortion forward, reversed backward with the merge), each over chunks
// of RB_MAX samples that are staged through the warp's buffer `sm` with cp.async, with the
// chunk's outputs written back through the buffer in coalesced rows.
__device__ __noinline__ void train_losses_ray_long(const Samples& S, uint32_t r, uint32_t o, uint32_t n, int lane,
                                                   float min_t, float inv_nrays, float grad_scale, float lambda,
                                                   const float* __restrict__ target, const float* __restrict__ bg,
                                                   uint32_t rs, float* __restrict__ ray_rgba,
                                                   float* __restrict__ grad_density, float* __restrict__ drgb,
                                                   float& acc_rec, float& acc_dist, float* sm,
                                                   bool accumulate) {
    constexpr int K = RB_SPL;
    const size_t ss = S.ss;
    const uint32_t nch = (n + RB_MAX - 1) / RB_MAX;
    const uint32_t l0 = (uint32_t)lane * K;  // the lane's first sample inside a chunk
    float* const b_sig = sm + SA_SIG * RB_PITCH;
    float* const b_dt = sm + SA_DT * RB_PITCH;
    float* const b_r = sm + SA_R * RB_PITCH;
    float* const b_g = sm + SA_G * RB_PITCH;
    float* const b_b = sm + SA_B * RB_PITCH;
    float* const b_dtn = sm + SA_DTN * RB_PITCH;
    float* const b_m = sm + SA_M * RB_PITCH;
    float* const b_t = sm + SA_T * RB_PITCH;
    float* const b_gd = sm + SA_GD * RB_PITCH;
    // Each pass stages a chunk's inputs into the warp's buffer (one round trip to memory) and
    // reads them from there; the chunk's samples are [c0, c0 + len).
    auto chunk_len = [&](uint32_t c) { return min(RB_MAX, n - c * RB_MAX); };
    auto stage_done = [&]() { cp_async_wait_all(); __syncwarp(); };
    // ---- compositor forward over the chunks up to the transmittance cut
    float cx = 0.0f, tin = 1.0f;
    float ar = 0.0f, ag = 0.0f, ab = 0.0f, aa = 0.0f;
    uint32_t used = n;
    float depth = 0.0f;
    for (uint32_t c = 0; c < nch; ++c) {
        const size_t c0 = (size_t)o + (size_t)c * RB_MAX;
        const uint32_t len = chunk_len(c);
        __syncwarp();  // the previous chunk's reads of the buffer are done
        stage_segment(b_sig, S.density, c0, len, lane);
        stage_segment(b_dt, S.dt, c0, len, lane);
        stage_segment(b_r, S.rgb, c0, len, lane);
        stage_segment(b_g, S.rgb + ss, c0, len, lane);
        stage_segment(b_b, S.rgb + 2 * ss, c0, len, lane);
        stage_done();
        const uint32_t j0 = c * RB_MAX + l0;
        float x[K], p[K], T[K];
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const bool valid = l0 + q < len;
            const uint32_t k = skew(l0 + q);
            x[q] = valid ? act_sigma(S.act, b_sig[k]) * b_dt[k] : 0.0f;
            p[q] = x[q];
        }
        blk_prefix(p, lane, cx);
#pragma unroll
        for (int q = 0; q < K; ++q) T[q] = expf(-p[q]);
        const float t_lane = shift_up(T[K - 1], lane, tin);
        int first_q = K;
        float cut_depth = 0.0f;
#pragma unroll
        for (int q = K - 1; q >= 0; --q)
            if (j0 + q < n && T[q] < min_t) { first_q = q; cut_depth = p[q]; }
        const unsigned term = __ballot_sync(FULL_MASK, first_q < K);
        uint32_t cut = n;
        if (term) {
            const int fl = __ffs(term) - 1;
            cut = c * RB_MAX + (uint32_t)fl * K + (uint32_t)__shfl_sync(FULL_MASK, first_q, fl) + 1u;
            depth = __shfl_sync(FULL_MASK, cut_depth, fl);
        }
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const uint32_t j = j0 + q;
            if (j < cut) {
                const uint32_t k = skew(l0 + q);
                const float w = (q ? T[q - 1] : t_lane) * -expm1f(-x[q]);
                ar += w * b_r[k]; ag += w * b_g[k]; ab += w * b_b[k]; aa += w;
            }
        }
        if (term) { used = cut; break; }
        cx = __shfl_sync(FULL_MASK, p[K - 1], WARP - 1);
        tin = __shfl_sync(FULL_MASK, T[K - 1], WARP - 1);
        depth = cx;
    }
    CompFwd cf;
    cf.r = warp_sum(ar); cf.g = warp_sum(ag); cf.b = warp_sum(ab); cf.a = warp_sum(aa);
    cf.depth = depth;
    cf.used = used;
    const ReconGrad g = recon_loss_ray(cf, target, bg, r, rs, inv_nrays);
    if (lane == 0) {
        if (ray_rgba) {
            ray_rgba[r] = cf.r; ray_rgba[r + rs] = cf.g; ray_rgba[r + 2 * (size_t)rs] = cf.b;
            ray_rgba[r + 3 * (size_t)rs] = cf.a;
        }
        acc_rec += g.l[0] + g.l[1] + g.l[2] + g.l[3];
    }
    // distortion inputs of chunk c from the buffer (staged by the caller of this lambda)
    auto dist_from_buffer = [&](uint32_t len, float (&sig)[K], float (&dtn)[K], float (&mm)[K]) {
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const bool valid = l0 + q < len;
            const uint32_t k = skew(l0 + q);
            sig[q] = valid ? act_sigma(S.act, b_sig[k]) : 0.0f;
            dtn[q] = valid ? b_dtn[k] : 0.0f;
            mm[q] = valid ? b_m[k] : 0.0f;
        }
    };
    auto stage_dist = [&](uint32_t c) {
        const size_t c0 = (size_t)o + (size_t)c * RB_MAX;
        const uint32_t len = chunk_len(c);
        __syncwarp();
        stage_segment(b_sig, S.density, c0, len, lane);
        stage_segment(b_dtn, S.dt_norm, c0, len, lane);
        stage_segment(b_m, S.m_norm, c0, len, lane);
        stage_done();
        return len;
    };
    // ---- distortion forward over all chunks, keeping each chunk's starting carry
    ScStore store;
    store.s = ScCarry{0.0f, 0.0f, 0.0f, 0.0f};
    const float kd = lambda > 0.0f ? lambda / (float)n : 0.0f;
    if (lambda > 0.0f) {
        ScCarry c{0.0f, 0.0f, 0.0f, S.m_norm[o]};  // m_{-1} := m_0 (zero first increment)
        float uni = 0.0f, cross = 0.0f;
        for (uint32_t ci = 0; ci < nch; ++ci) {
            store.put(ci, lane, c);
            const uint32_t j0 = ci * RB_MAX + l0;
            float sig[K], dtn[K], mm[K], wd[K], tnext[K], dm[K], A[K];
            dist_from_buffer(stage_dist(ci), sig, dtn, mm);
            ScCarry nx;
            sc_dist_forward(sig, dtn, mm, j0, n, lane, c, wd, tnext, dm, A, nx, uni, cross);
            c = nx;
        }
        uni = warp_sum(uni);
        cross = warp_sum(cross);
        if (lane == 0) acc_dist += kd * ((1.0f / 3.0f) * uni + 2.0f * cross);
    }
    // ---- backward over the chunks from the last
    float sx = 0.0f;                                   // compositor: sum of x after the chunk
    float sr = 0.0f, sg = 0.0f, sb = 0.0f, sa = 0.0f;  // compositor: sums of w c, w after the chunk
    float sw = 0.0f, sf = 0.0f, sgw = 0.0f;           // distortion suffix sums after the chunk
    for (int ci = (int)nch - 1; ci >= 0; --ci) {
        const uint32_t j0 = (uint32_t)ci * RB_MAX + l0;
        const size_t c0 = (size_t)o + (size_t)ci * RB_MAX;
        const uint32_t len = chunk_len((uint32_t)ci);
        // chunks beyond 31 replay the distortion forward from chunk 31 (reads straight from memory)
        ScCarry dc = store.get((uint32_t)ci);
        if (lambda > 0.0f) {
            for (uint32_t k = 31u; k < (uint32_t)ci; ++k) {
                float sig[K], dtn[K], mm[K], wd[K], tnext[K], dm[K], A[K];
                const uint32_t jk = k * RB_MAX + l0;
                sc_load_dist(S, o, jk, n, sig, dtn, mm);
                ScCarry nx;
                float u0 = 0.0f, c0_ = 0.0f;
                sc_dist_forward(sig, dtn, mm, jk, n, lane, dc, wd, tnext, dm, A, nx, u0, c0_);
                dc = nx;
            }
        }
        __syncwarp();
        stage_segment(b_sig, S.density, c0, len, lane);
        stage_segment(b_dt, S.dt, c0, len, lane);
        stage_segment(b_r, S.rgb, c0, len, lane);
        stage_segment(b_g, S.rgb + ss, c0, len, lane);
        stage_segment(b_b, S.rgb + 2 * ss, c0, len, lane);
        if (lambda > 0.0f) {
            stage_segment(b_dtn, S.dt_norm, c0, len, lane);
            stage_segment(b_m, S.m_norm, c0, len, lane);
        }
        if (S.t) stage_segment(b_t, S.t, c0, len, lane);
        if (accumulate) stage_segment(b_gd, grad_density, c0, len, lane);
        stage_done();
        float ds[K];
#pragma unroll
        for (int q = 0; q < K; ++q) ds[q] = 0.0f;
        float w[K];
#pragma unroll
        for (int q = 0; q < K; ++q) w[q] = 0.0f;
        if ((uint32_t)ci * RB_MAX < used) {
            float sig[K], dt[K], cr[K], cg[K], cb[K];
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const bool valid = j0 + q < used;
                const uint32_t k = skew(l0 + q);
                sig[q] = valid ? act_sigma(S.act, b_sig[k]) : 0.0f;
                dt[q] = valid ? b_dt[k] : 0.0f;
                cr[q] = valid ? b_r[k] : 0.0f;
                cg[q] = valid ? b_g[k] : 0.0f;
                cb[q] = valid ? b_b[k] : 0.0f;
            }
            // T before / after sample j from the optical depth and the suffix sums of x
            float xs[K];
#pragma unroll
            for (int q = 0; q < K; ++q) xs[q] = sig[q] * dt[q];
            const float xs_after = blk_suffix(xs, lane, sx);
            float ta[K], vr[K], vg[K], vb[K], va[K];
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float xs_ex = q < K - 1 ? xs[q + 1] : xs_after;
                const float tj = expf(-fmaxf(depth - xs[q], 0.0f));
                ta[q] = expf(-fmaxf(depth - xs_ex, 0.0f));
                w[q] = j0 + q < used ? tj * -expm1f(-sig[q] * dt[q]) : 0.0f;
                vr[q] = w[q] * cr[q]; vg[q] = w[q] * cg[q]; vb[q] = w[q] * cb[q]; va[q] = w[q];
            }
            const float ar_ = blk_suffix(vr, lane, sr), ag_ = blk_suffix(vg, lane, sg);
            const float ab_ = blk_suffix(vb, lane, sb), aa_ = blk_suffix(va, lane, sa);
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float r_ex = q < K - 1 ? vr[q + 1] : ar_, g_ex = q < K - 1 ? vg[q + 1] : ag_;
                const float b_ex = q < K - 1 ? vb[q + 1] : ab_, a_ex = q < K - 1 ? va[q + 1] : aa_;
                const float tn = ta[q];
                const float d = dt[q] * (g.gr * (tn * cr[q] - r_ex) + g.gg * (tn * cg[q] - g_ex) +
                                         g.gb * (tn * cb[q] - b_ex) + g.ga * (tn - a_ex));
                if (j0 + q < used) ds[q] = grad_scale * d * act_dsigma(S.act, sig[q]);
            }
            sx = __shfl_sync(FULL_MASK, xs[0], 0);
            sr = __shfl_sync(FULL_MASK, vr[0], 0); sg = __shfl_sync(FULL_MASK, vg[0], 0);
            sb = __shfl_sync(FULL_MASK, vb[0], 0); sa = __shfl_sync(FULL_MASK, va[0], 0);
        }
        if (lambda > 0.0f) {
            float sig[K], dtn[K], mm[K], wd[K], tnext[K], dm[K], A[K];
            dist_from_buffer(len, sig, dtn, mm);
            ScCarry nx;
            float u0 = 0.0f, c0_ = 0.0f;
            sc_dist_forward(sig, dtn, mm, j0, n, lane, dc, wd, tnext, dm, A, nx, u0, c0_);
            float Wge[K];
#pragma unroll
            for (int q = 0; q < K; ++q) Wge[q] = wd[q];
            blk_suffix(Wge, lane, sw);
            float f[K];
#pragma unroll
            for (int q = 0; q < K; ++q) f[q] = dm[q] * Wge[q];
            const float f_after = blk_suffix(f, lane, sf);
            float gw[K], gq[K];
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float b = q < K - 1 ? f[q + 1] : f_after;
                gq[q] = kd * ((2.0f / 3.0f) * dtn[q] * wd[q] + 2.0f * (A[q] + b));
                gw[q] = gq[q] * wd[q];
            }
            const float gw_after = blk_suffix(gw, lane, sgw);
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const float gw_ex = q < K - 1 ? gw[q + 1] : gw_after;
                if (j0 + q < n) ds[q] += grad_scale * dtn[q] * (gq[q] * tnext[q] - gw_ex) * act_dsigma(S.act, sig[q]);
            }
            sw = __shfl_sync(FULL_MASK, Wge[0], 0);
            sf = __shfl_sync(FULL_MASK, f[0], 0);
            sgw = __shfl_sync(FULL_MASK, gw[0], 0);
        }
        // outputs through the buffer: dL/drgb (zero past the cut) and the merged density gradient
        __syncwarp();  // every lane has read the chunk's inputs
#pragma unroll
        for (int q = 0; q < K; ++q) {
            if (l0 + q < len) {
                const uint32_t k = skew(l0 + q);
                b_r[k] = grad_scale * g.gr * w[q];
                b_g[k] = grad_scale * g.gg * w[q];
                b_b[k] = grad_scale * g.gb * w[q];
                float gd = (accumulate ? b_gd[k] : 0.0f) + ds[q];
                if (S.t) { const float tt = b_t[k]; if (tt < 1.0f) gd *= tt * tt; }
                b_gd[k] = gd;
            }
        }
        __syncwarp();
        store_segment(grad_density, b_gd, c0, len, lane);
        store_segment(drgb, b_r, c0, len, lane);
        store_segment(drgb + ss, b_g, c0, len, lane);
        store_segment(drgb + 2 * ss, b_b, c0, len, lane);
    }
}

// Reconstruction + distortion forward/backward + gradient merge, one warp per ray with its own
// staging buffer (dynamic shared memory, 10.1 KB a warp); W warps a block (tn_tuning
// loss_rays_per_block: 2, 4 or 8) and 16 / W blocks an SM (128 registers a thread) keep 16 rays
// in flight per SM. VEC: 16-byte staging (every sample array 16-byte aligned, stride a multiple
// of 4). The grid is every resident warp (or fewer), each taking rays in turn: a batch of many
// waves (the rays of several scenes) is one persistent launch.
template <int W, bool VEC>
__global__ void __launch_bounds__(W * WARP, 16 / W)
train_losses_kernel(Samples S, uint32_t n_rays, const uint32_t* n_dev, uint32_t rs, const uint32_t* __restrict__ counts,
                    const uint32_t* __restrict__ offsets, float min_t, float inv_nrays_host,
                    const uint32_t* __restrict__ inv_from, float grad_scale, float lambda,
                    const float* __restrict__ target, const float* __restrict__ bg, float* __restrict__ ray_rgba,
                    float* __restrict__ grad_density, float* __restrict__ drgb, float* loss_sums, float* partials,
                    uint32_t* ticket, bool accumulate) {
    extern __shared__ __align__(16) float stage[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t n_live = live_rays(n_rays, n_dev);
    float inv_nrays = inv_nrays_host;
    if (inv_from) { const uint32_t nn = *inv_from; inv_nrays = nn ? 1.0f / (float)nn : 0.0f; }
    const float lam = lambda > 0.0f ? lambda : 0.0f;
    float acc[2] = {0.0f, 0.0f};
    float* const sm = stage + (size_t)wid * SA_N * RB_PITCH;
    auto one_ray = [&](uint32_t r) {
        const uint32_t o = offsets[r], n = counts[r];
        const uint32_t span = n + (VEC ? (o & 3u) : 0u);  // slots the ray takes
        if (span <= RB_MAX)
            train_losses_ray_blocked<VEC, RB_SPL>(S, r, o, n, lane, min_t, inv_nrays, grad_scale, lam, target, bg, rs,
                                                  ray_rgba, grad_density, drgb, acc[0], acc[1], sm, accumulate);
        else
            train_losses_ray_long(S, r, o, n, lane, min_t, inv_nrays, grad_scale, lam, target, bg, rs, ray_rgba,
                                  grad_density, drgb, acc[0], acc[1], sm, accumulate);
    };
    for (uint32_t r = blockIdx.x * W + wid; r < n_live; r += gridDim.x * W) one_ray(r);
    if (loss_sums) {
        acc[0] *= inv_nrays;
        block_sum_and_finish<2>(acc, partials, ticket, loss_sums, FinishScale{{1.0f, 1.0f}, n_dev, n_rays, 2u});
    }
}

__global__ void grad_epilogue_kernel(uint32_t n, const uint32_t* __restrict__ n_dev, float scale,
                                     const float* __restrict__ rec, const float* __restrict__ dist,
                                     const float* __restrict__ t, float* __restrict__ out) {
    const uint32_t n_live = n_dev ? min(*n_dev, n) : n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_live; i += gridDim.x * blockDim.x) {
        float g = out[i] + scale * rec[i];
        if (dist) g += scale * dist[i];
        if (t) { const float tt = t[i]; if (tt < 1.0f) g *= tt * tt; }
        out[i] = g;
    }
}

// ---- plain path: one thread per ray, reference structure --------------------------------
__device__ __forceinline__ float plain_sigma(int act, float d) { return act == 0 ? d : __expf(fminf(d, 12.0f) - 1.0f); }

__global__ void plain_recon_kernel(uint32_t n_rays, uint32_t rs, uint32_t ss, int act, float min_t, float inv_nrays,
                                   float grad_scale, const uint32_t* __restrict__ counts,
                                   const uint32_t* __restrict__ offsets, const float* __restrict__ bg,
                                   const float* __restrict__ target, const float* __restrict__ density,
                                   const float* __restrict__ rgb, const float* __restrict__ dtb,
                                   float* __restrict__ loss, float* __restrict__ dd, float* __restrict__ drgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays) return;
    const uint32_t o = offsets[i], n = counts[i];
    const float* sr = rgb + o;
    const float* sg = rgb + o + ss;
    const float* sb = rgb + o + 2 * (size_t)ss;
    const float* sd = density + o;
    const float* sdt = dtb + o;
    float r = 0, g = 0, b = 0, a = 0, trans = 1.0f;
    for (uint32_t k = 0; k < n; ++k) {
        const float alpha = 1.0f - __expf(-plain_sigma(act, sd[k]) * sdt[k]);
        const float w = trans * alpha;
        r += w * sr[k]; g += w * sg[k]; b += w * sb[k]; a += w;
        trans *= (1.0f - alpha);
        if (trans < min_t) break;
    }
    const float gt_r = target[i], gt_g = target[i + rs], gt_b = target[i + 2 * (size_t)rs], gt_a = target[i + 3 * (size_t)rs];
    const float br = bg[i], bgc = bg[i + rs], bb = bg[i + 2 * (size_t)rs];
    const float gac = 1.0f - gt_a;
    const float gtr = gt_r * gt_a + br * gac, gtg = gt_g * gt_a + bgc * gac, gtb = gt_b * gt_a + bb * gac;
    const float ac = 1.0f - a;
    const float pr = r * a + br * ac, pg = g * a + bgc * ac, pb = b * a + bb * ac;
    const float dr = pr - gtr, dg = pg - gtg, db = pb - gtb, da = ac - gac;
    loss[i] = huber(dr); loss[i + rs] = huber(dg); loss[i + 2 * (size_t)rs] = huber(db); loss[i + 3 * (size_t)rs] = huber(da);
    const float lr = inv_nrays * huber_grad(dr), lg = inv_nrays * huber_grad(dg), lb = inv_nrays * huber_grad(db);
    const float cdr = r - br, cdg = g - bgc, cdb = b - bb;
    float cr = r, cg = g, cb = b, ca = a;
    trans = 1.0f;
    for (uint32_t k = 0; k < n; ++k) {
        const float sig = plain_sigma(act, sd[k]);
        const float alpha = 1.0f - __expf(-sig * sdt[k]);
        const float w = trans * alpha;
        const float kk = trans - w;
        cr -= w * sr[k]; cg -= w * sg[k]; cb -= w * sb[k]; ca -= w;
        float dRr = sdt[k] * (kk * sr[k] - cr), dRg = sdt[k] * (kk * sg[k] - cg), dRb = sdt[k] * (kk * sb[k] - cb);
        const float dRa = sdt[k] * (kk - ca);
        dRr = dRr * a + cdr * dRa;
        dRg = dRg * a + cdg * dRa;
        dRb = dRb * a + cdb * dRa;
        dd[o + k] = (lr * dRr + lg * dRg + lb * dRb) * (act == 0 ? 1.0f : sig);
        const float dRc = w * a;
        drgb[o + k] = grad_scale * lr * dRc;
        drgb[o + k + ss] = grad_scale * lg * dRc;
        drgb[o + k + 2 * (size_t)ss] = grad_scale * lb * dRc;
        trans *= 1.0f - alpha;
        if (trans < min_t) break;
    }
}

__global__ void plain_dist_fwd_kernel(uint32_t n_rays, uint32_t rs, int act, float lambda,
                                      const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                                      const float* __restrict__ density, const float* __restrict__ mb,
                                      const float* __restrict__ dtb, float* __restrict__ ray5,
                                      float* __restrict__ ray_loss, float* __restrict__ w_cs_b,
                                      float* __restrict__ wm_cs_b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays) return;
    const uint32_t n = counts[i];
    if (n == 0) {
        ray_loss[i] = 0.0f;
        for (int k = 0; k < 5; ++k) ray5[i + k * (size_t)rs] = 0.0f;
        return;
    }
    const uint32_t o = offsets[i];
    float cw = 0, cwm = 0, cdtw2 = 0, cwmw = 0, cwwm = 0, trans = 1.0f, pw = 0, pwm = 0, b0 = 0, b1 = 0, uni = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const float dt = dtb[o + k];
        const float alpha = 1.0f - __expf(-plain_sigma(act, density[o + k]) * dt);
        const float w = alpha * trans;
        const float m = mb[o + k];
        const float wm = w * m;
        const float a0 = wm * pw, a1 = w * pwm, a2 = dt * w * w;
        cw += w; cwm += wm; cdtw2 += a2; cwmw += a0; cwwm += a1;
        w_cs_b[o + k] = cw;
        wm_cs_b[o + k] = cwm;
        b0 += a0; b1 += a1; uni += a2;
        pw = cw; pwm = cwm;
        trans *= (1.0f - alpha);
    }
    const float kk = lambda / (float)n;
    ray_loss[i] = kk * ((1.0f / 3.0f) * uni + 2.0f * (b0 - b1));
    ray5[i] = cdtw2; ray5[i + rs] = cw; ray5[i + 2 * (size_t)rs] = cwm; ray5[i + 3 * (size_t)rs] = cwmw;
    ray5[i + 4 * (size_t)rs] = cwwm;
}

__global__ void plain_dist_bwd_kernel(uint32_t n_rays, uint32_t rs, int act, float lambda,
                                      const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                                      const float* __restrict__ density, const float* __restrict__ ray5,
                                      const float* __restrict__ mb, const float* __restrict__ dtb,
                                      const float* __restrict__ w_cs_b, const float* __restrict__ wm_cs_b,
                                      float* __restrict__ dd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays) return;
    const uint32_t n = counts[i];
    if (n == 0) return;
    const uint32_t o = offsets[i];
    float cdtw2 = ray5[i], cw = ray5[i + rs], cwm = ray5[i + 2 * (size_t)rs], cwmw = ray5[i + 3 * (size_t)rs],
          cwwm = ray5[i + 4 * (size_t)rs];
    float trans = 1.0f, pw = 0.0f, pwm = 0.0f;
    const float kk = lambda / (float)n;
    for (uint32_t k = 0; k < n; ++k) {
        const float dt = dtb[o + k];
        const float sig = plain_sigma(act, density[o + k]);
        const float alpha = 1.0f - __expf(-sig * dt);
        const float T = trans;
        const float w = alpha * T;
        const float m = mb[o + k];
        const float wm = w * m;
        const float wcs = w_cs_b[o + k], wmcs = wm_cs_b[o + k];
        const float dw = T * (dt * (1.0f - alpha));
        const float dwm = m * dw;
        const float tw = T - w;
        cw -= w; cwm -= wm; cdtw2 -= dt * w * w; cwmw -= wm * pw; cwwm -= w * pwm;
        const float db0 = dwm * pw + dt * (cwm * (wcs + tw) - 2.0f * cwmw);
        const float db1 = dw * pwm + dt * (cw * (m * tw + wmcs) - 2.0f * cwwm);
        const float du = 2.0f * dt * (dt * w * tw - cdtw2);
        dd[o + k] = kk * (2.0f * (db0 - db1) + (1.0f / 3.0f) * du) * (act == 0 ? 1.0f : sig);
        pw = wcs; pwm = wmcs;
        trans *= (1.0f - alpha);
    }
}

__global__ void plain_copy_gradients_kernel(uint32_t n, float scale, const float* __restrict__ in, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = scale * in[i] + out[i];
}

__global__ void plain_distance_scaling_kernel(uint32_t n, const float* __restrict__ t, float* __restrict__ g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float tt = t[i];
    if (tt >= 1.0f) return;
    g[i] *= tt * tt;
}

// Resident blocks per SM of each loss kernel, queried once per kernel.
static int blocks_per_sm(const void* kernel, int threads, size_t dyn_smem = 0) {
    static std::mutex mu;
    static std::vector<std::pair<const void*, int>> known;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto& kv : known)
        if (kv.first == kernel) return kv.second;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem);
    if (per_sm <= 0) per_sm = 1;
    known.emplace_back(kernel, per_sm);
    return per_sm;
}

static int loss_grid(const void* kernel, uint32_t n_rays, int threads = LOSS_THREADS, size_t dyn_smem = 0) {
    const int per_sm = blocks_per_sm(kernel, threads, dyn_smem);
    const uint32_t want = (n_rays + threads / WARP - 1) / (threads / WARP);
    const uint32_t cap = (uint32_t)(num_sms() * per_sm);
    return (int)max(1u, min(want, cap));
}

template <int W, bool VEC>
static int launch_train_losses_v(tn_ctx* ctx, cudaStream_t stream, const tn_ray_batch* batch, const Samples& S,
                                 float min_t, float inv_nrays, const uint32_t* inv_from, float grad_scale,
                                 float lambda, const float* target, const float* bg, float* ray_rgba,
                                 float* grad_density, float* drgb, float* loss_sums, bool accumulate) {
    const size_t smem = W * TL_STAGE_BYTES;
    static std::once_flag once;
    std::call_once(once, [&] {
        cudaFuncSetAttribute(train_losses_kernel<W, VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    });
    const int grid = loss_grid((const void*)train_losses_kernel<W, VEC>, batch->n_rays, W * WARP, smem);
    int st = ensure_block_f32(ctx, (size_t)grid * 2);
    if (st != TN_OK) return st;
    train_losses_kernel<W, VEC><<<grid, W * WARP, smem, stream>>>(
        S, batch->n_rays, batch->n_rays_dev, batch->ray_stride, batch->counts, batch->offsets, min_t, inv_nrays,
        inv_from, grad_scale, lambda, target, bg, ray_rgba, grad_density, drgb, loss_sums, ctx->block_f32,
        ctx->tickets + TICKET_TRAIN, accumulate);
    return check_launch("tn_train_losses");
}

// 16-byte staging when every per-sample array the kernel reads or writes is 16-byte aligned and
// the sample stride is a multiple of 4 (then no 16-byte group of a ray reaches past the arrays).
template <int W>
static int launch_train_losses(tn_ctx* ctx, cudaStream_t stream, const tn_ray_batch* batch, const Samples& S,
                               float min_t, float inv_nrays, const uint32_t* inv_from, float grad_scale, float lambda,
                               const float* target, const float* bg, float* ray_rgba, float* grad_density,
                               float* drgb, float* loss_sums, bool accumulate) {
    const uintptr_t m = (uintptr_t)S.density | (uintptr_t)S.rgb | (uintptr_t)S.dt | (uintptr_t)S.m_norm |
                        (uintptr_t)S.dt_norm | (uintptr_t)S.t | (uintptr_t)grad_density | (uintptr_t)drgb;
    if ((m & 15u) == 0 && (S.ss & 3u) == 0)
        return launch_train_losses_v<W, true>(ctx, stream, batch, S, min_t, inv_nrays, inv_from, grad_scale, lambda,
                                              target, bg, ray_rgba, grad_density, drgb, loss_sums, accumulate);
    return launch_train_losses_v<W, false>(ctx, stream, batch, S, min_t, inv_nrays, inv_from, grad_scale, lambda,
                                           target, bg, ray_rgba, grad_density, drgb, loss_sums, accumulate);
}

// Rays per warp of the sample-tile kernels, from the batch's mean samples per ray
// (sample_stride / n_rays, an upper bound): up to 4 tiles (32 * ST_K samples each) of samples per
// warp while that leaves at least 32 warps per SM (the setup of a warp's range and its partly
// filled first and last tiles are then paid once per 4 tiles), else 1 tile per warp; more when
// the grid would otherwise take more than one wave of resident warps.
static uint32_t tile_rays_per_warp(const tn_ray_batch* b, const void* kernel, uint32_t max_tiles = 0,
                                   int k = ST_K) {
    const double mean = b->n_rays ? std::max(1.0, (double)b->sample_stride / (double)b->n_rays) : 1.0;
    const double per_tile = (double)(WARP * k);
    const double fill = (double)b->sample_stride / (per_tile * num_sms() * 32.0);
    const double tiles = std::min(4.0, std::max(1.0, std::floor(fill)));
    uint32_t rpw = (uint32_t)std::min(32.0, std::max(1.0, std::floor(tiles * per_tile / mean)));
    // when the grid would take more than one wave of resident warps, enough rays per warp (at most
    // 32) that it takes one: no partly filled last wave
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, LOSS_THREADS, 0) == cudaSuccess && per_sm > 0) {
        const uint64_t resident = (uint64_t)num_sms() * (uint64_t)per_sm * LOSS_WARPS;
        const uint64_t warps = (b->n_rays + rpw - 1) / rpw;
        if (warps > resident) rpw = (uint32_t)std::min<uint64_t>(32, (b->n_rays + resident - 1) / resident);
    }
    // a kernel that keeps per-tile state for max_tiles tiles: rays of about that many tiles a warp
    if (max_tiles) rpw = std::min(rpw, (uint32_t)std::max(1.0, std::floor(max_tiles * per_tile / mean)));
    return rpw;
}

// 16-byte sample vectors: every per-sample array 16-byte aligned and the stride a multiple of 4.
static bool tile_vec(const Samples& S, const void* a, const void* b) {
    const uintptr_t m = (uintptr_t)S.density | (uintptr_t)S.rgb | (uintptr_t)S.dt | (uintptr_t)a | (uintptr_t)b;
    return (m & 15u) == 0 && (S.ss & 3u) == 0;
}

// One wave of resident warps for a sample-balanced launch, at least eight rays a warp on average.
static int balanced_grid(uint32_t n_rays, const void* kernel) {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, LOSS_THREADS, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const uint32_t wave = (uint32_t)num_sms() * (uint32_t)per_sm;
    const uint32_t want = (std::max(1u, n_rays / 8u) + LOSS_WARPS - 1) / LOSS_WARPS;
    return (int)std::max(1u, std::min(wave, want));
}

static int tile_grid(uint32_t n_rays, uint32_t rpw) {
    const uint32_t warps = (n_rays + rpw - 1) / rpw;
    return (int)((warps + LOSS_WARPS - 1) / LOSS_WARPS);
}

// Launch of the compositor forward tiles, specialised on the vector loads, the activation and
// whether per-sample transmittance and weights are stored. depth_max = -ln(min_transmittance).
static void launch_composite_fwd_tiles(cudaStream_t stream, const tn_ray_batch* b, const Samples& S,
                                       float min_t, float* rgba, float* depth, uint32_t* n_used, float* t_out,
                                       float* w_out) {
    const float depth_max = min_t > 0.0f ? -logf(min_t) : INFINITY;
    const bool vec = tile_vec(S, t_out, w_out), store = t_out != nullptr;
    const int grid = balanced_grid(b->n_rays, vec ? (const void*)composite_fwd_tiles_kernel<CT_K, true, 0, false>
                                                  : (const void*)composite_fwd_tiles_kernel<CT_K, false, 0, false>);
#define TN_FWD_TILES(V, A, ST)                                                                                  \
    composite_fwd_tiles_kernel<CT_K, V, A, ST><<<grid, LOSS_THREADS, 0, stream>>>(                              \
        S, b->n_rays, b->n_rays_dev, b->ray_stride, b->counts, b->offsets, depth_max, rgba, depth, n_used,       \
        t_out, w_out)
    const int key = (vec ? 4 : 0) | (S.act ? 2 : 0) | (store ? 1 : 0);
    switch (key) {
        case 0: TN_FWD_TILES(false, 0, false); break;
        case 1: TN_FWD_TILES(false, 0, true); break;
        case 2: TN_FWD_TILES(false, 1, false); break;
        case 3: TN_FWD_TILES(false, 1, true); break;
        case 4: TN_FWD_TILES(true, 0, false); break;
        case 5: TN_FWD_TILES(true, 0, true); break;
        case 6: TN_FWD_TILES(true, 1, false); break;
        default: TN_FWD_TILES(true, 1, true); break;
    }
#undef TN_FWD_TILES
}

static void launch_composite_bwd_tiles(cudaStream_t stream, const tn_ray_batch* b, const Samples& S,
                                       const float* depth, const uint32_t* n_used, const float* grad_rgba, float* dd,
                                       float* drgb) {
    const bool vec = tile_vec(S, dd, drgb);
    const int grid = balanced_grid(b->n_rays, vec ? (const void*)composite_bwd_tiles_kernel<CV_K, true, 0>
                                                  : (const void*)composite_bwd_tiles_kernel<CV_K, false, 0>);
#define TN_BWD_TILES(V, A)                                                                                      \
    composite_bwd_tiles_kernel<CV_K, V, A><<<grid, LOSS_THREADS, 0, stream>>>(                                  \
        S, b->n_rays, b->n_rays_dev, b->ray_stride, b->counts, b->offsets, depth, n_used, grad_rgba, dd,         \
        drgb)
    const int key = (vec ? 2 : 0) | (S.act ? 1 : 0);
    switch (key) {
        case 0: TN_BWD_TILES(false, 0); break;
        case 1: TN_BWD_TILES(false, 1); break;
        case 2: TN_BWD_TILES(true, 0); break;
        default: TN_BWD_TILES(true, 1); break;
    }
#undef TN_BWD_TILES
}

static int check_batch(const tn_ray_batch* b) {
    TN_REQUIRE(b != nullptr, TN_E_NULL, "ray batch is NULL");
    TN_NONNULL(b->counts);
    TN_NONNULL(b->offsets);
    TN_REQUIRE(b->ray_stride >= b->n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", b->ray_stride, b->n_rays);
    return TN_OK;
}

// tn_train_losses, and the trainer's form that writes the merged gradient over grad_density
// instead of adding to it (accumulate false: no zeroing pass before it).
int train_losses(tn_ctx* ctx, cudaStream_t stream, const tn_ray_batch* batch, int activation, float min_transmittance,
                 float inv_nrays, const uint32_t* inv_nrays_from_dev, float grad_scale, float lambda,
                 const float* density, const float* rgb, const float* dt, const float* m_norm, const float* dt_norm,
                 const float* t, const float* target_rgba, const float* bg_rgb, float* ray_rgba, float* grad_density,
                 float* dL_drgb, float* loss_sums, bool accumulate) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(target_rgba); TN_NONNULL(bg_rgb);
    TN_NONNULL(grad_density); TN_NONNULL(dL_drgb);
    if (lambda > 0.0f) { TN_NONNULL(m_norm); TN_NONNULL(dt_norm); }
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, m_norm, dt_norm, t, batch->sample_stride, activation};
    switch (ctx->tune.loss_rays_per_block) {
        case 2: return launch_train_losses<2>(ctx, stream, batch, S, min_transmittance, inv_nrays, inv_nrays_from_dev,
                                              grad_scale, lambda, target_rgba, bg_rgb, ray_rgba, grad_density,
                                              dL_drgb, loss_sums, accumulate);
        case 8: return launch_train_losses<8>(ctx, stream, batch, S, min_transmittance, inv_nrays, inv_nrays_from_dev,
                                              grad_scale, lambda, target_rgba, bg_rgb, ray_rgba, grad_density,
                                              dL_drgb, loss_sums, accumulate);
        default: return launch_train_losses<4>(ctx, stream, batch, S, min_transmittance, inv_nrays,
                                               inv_nrays_from_dev, grad_scale, lambda, target_rgba, bg_rgb, ray_rgba,
                                               grad_density, dL_drgb, loss_sums, accumulate);
    }
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_composite_fwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                     float min_transmittance, const float* density, const float* rgb, const float* dt,
                     float* rgba, float* depth, uint32_t* n_used) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(rgba);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, nullptr, nullptr, nullptr, batch->sample_stride, activation};
    launch_composite_fwd_tiles(stream, batch, S, min_transmittance, rgba, depth, n_used, nullptr, nullptr);
    return check_launch("tn_composite_fwd");
}

int tn_composite_fwd_store(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                           float min_transmittance, const float* density, const float* rgb, const float* dt,
                           float* rgba, uint32_t* n_used, float* t_saved, float* w_saved) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(rgba); TN_NONNULL(n_used);
    TN_NONNULL(t_saved); TN_NONNULL(w_saved);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, nullptr, nullptr, nullptr, batch->sample_stride, activation};
    launch_composite_fwd_tiles(stream, batch, S, min_transmittance, rgba, nullptr, n_used, t_saved, w_saved);
    return check_launch("tn_composite_fwd_store");
}

int tn_composite_bwd_stored(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                            const float* density, const float* rgb, const float* dt, const uint32_t* n_used,
                            const float* t_saved, const float* w_saved, const float* grad_rgba, float* dL_ddensity,
                            float* dL_drgb) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(n_used); TN_NONNULL(t_saved);
    TN_NONNULL(w_saved); TN_NONNULL(grad_rgba); TN_NONNULL(dL_ddensity); TN_NONNULL(dL_drgb);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, nullptr, nullptr, nullptr, batch->sample_stride, activation};
    const int grid = loss_grid((const void*)composite_bwd_stored_kernel, batch->n_rays);
    composite_bwd_stored_kernel<<<grid, LOSS_THREADS, 0, stream>>>(
        S, batch->n_rays, batch->n_rays_dev, batch->ray_stride, batch->counts, batch->offsets, n_used, t_saved,
        w_saved, grad_rgba, dL_ddensity, dL_drgb);
    return check_launch("tn_composite_bwd_stored");
}

int tn_composite_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                     const float* density, const float* rgb, const float* dt, const float* depth,
                     const uint32_t* n_used, const float* grad_rgba, float* dL_ddensity, float* dL_drgb) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(depth); TN_NONNULL(n_used);
    TN_NONNULL(grad_rgba); TN_NONNULL(dL_ddensity); TN_NONNULL(dL_drgb);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, nullptr, nullptr, nullptr, batch->sample_stride, activation};
    launch_composite_bwd_tiles(stream, batch, S, depth, n_used, grad_rgba, dL_ddensity, dL_drgb);
    return check_launch("tn_composite_bwd");
}

int tn_recon_loss_fwd_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                          float min_transmittance, float inv_nrays, float grad_scale, const float* density,
                          const float* rgb, const float* dt, const float* target_rgba, const float* bg_rgb,
                          float* ray_rgba, float* loss, float* loss_sum, float* dL_ddensity, float* dL_drgb) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(target_rgba); TN_NONNULL(bg_rgb);
    TN_NONNULL(dL_ddensity); TN_NONNULL(dL_drgb);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, rgb, dt, nullptr, nullptr, nullptr, batch->sample_stride, activation};
    const int grid = loss_grid((const void*)recon_kernel, batch->n_rays);
    st = ensure_block_f32(ctx, (size_t)grid * 2);
    if (st != TN_OK) return st;
    recon_kernel<<<grid, LOSS_THREADS, 0, stream>>>(S, batch->n_rays, batch->n_rays_dev, batch->ray_stride, batch->counts,
                                                    batch->offsets, min_transmittance, inv_nrays, grad_scale,
                                                    target_rgba, bg_rgb, ray_rgba, loss, loss_sum, dL_ddensity,
                                                    dL_drgb, ctx->block_f32, ctx->tickets + TICKET_RECON);
    return check_launch("tn_recon_loss_fwd_bwd");
}

int tn_distortion_fwd_bwd(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation, float lambda,
                          const float* density, const float* m_norm, const float* dt_norm, const float* grad_ray,
                          float* ray_loss, float* loss_sum, float* dL_ddensity) {
    TN_NONNULL(ctx);
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(m_norm); TN_NONNULL(dt_norm);
    TN_REQUIRE(activation == TN_ACT_SIGMA || activation == TN_ACT_DENSITY, TN_E_INVALID, "unknown activation %d", activation);
    if (batch->n_rays == 0) return TN_OK;
    Samples S{density, nullptr, nullptr, m_norm, dt_norm, nullptr, batch->sample_stride, activation};
    const uintptr_t al = (uintptr_t)density | (uintptr_t)m_norm | (uintptr_t)dt_norm | (uintptr_t)dL_ddensity;
    const bool vec = (al & 15u) == 0 && (batch->sample_stride & 3u) == 0;
    const uint32_t rpw = tile_rays_per_warp(
        batch, vec ? (const void*)distortion_tiles_kernel<true, 0> : (const void*)distortion_tiles_kernel<false, 0>,
        SAVED_TILES / 2);
    const int grid = tile_grid(batch->n_rays, rpw);
    st = ensure_block_f32(ctx, (size_t)grid * 2);
    if (st != TN_OK) return st;
#define TN_DIST_TILES(V, A)                                                                                     \
    distortion_tiles_kernel<V, A><<<grid, LOSS_THREADS, 0, stream>>>(                                           \
        S, batch->n_rays, batch->n_rays_dev, rpw, batch->counts, batch->offsets, lambda, grad_ray, ray_loss,     \
        loss_sum, dL_ddensity, ctx->block_f32, ctx->tickets + TICKET_DIST)
    switch ((vec ? 2 : 0) | (activation ? 1 : 0)) {
        case 0: TN_DIST_TILES(false, 0); break;
        case 1: TN_DIST_TILES(false, 1); break;
        case 2: TN_DIST_TILES(true, 0); break;
        default: TN_DIST_TILES(true, 1); break;
    }
#undef TN_DIST_TILES
    return check_launch("tn_distortion_fwd_bwd");
}

int tn_grad_epilogue(tn_stream_t stream, uint32_t n_samples, const uint32_t* n_samples_dev, float loss_scale,
                     const float* dL_rec, const float* dL_dist, const float* t, float* grad_out) {
    TN_NONNULL(dL_rec); TN_NONNULL(grad_out);
    if (n_samples == 0) return TN_OK;
    const int grid = (int)min((n_samples + 255u) / 256u, (uint32_t)num_sms() * 8u);
    grad_epilogue_kernel<<<grid, 256, 0, stream>>>(n_samples, n_samples_dev, loss_scale, dL_rec, dL_dist, t, grad_out);
    return check_launch("tn_grad_epilogue");
}

int tn_train_losses(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                    float min_transmittance, float inv_nrays, const uint32_t* inv_nrays_from_dev, float grad_scale,
                    float lambda, const float* density, const float* rgb, const float* dt, const float* m_norm,
                    const float* dt_norm, const float* t, const float* target_rgba, const float* bg_rgb,
                    float* ray_rgba, float* grad_density, float* dL_drgb, float* loss_sums) {
    return tn::train_losses(ctx, stream, batch, activation, min_transmittance, inv_nrays, inv_nrays_from_dev,
                            grad_scale, lambda, density, rgb, dt, m_norm, dt_norm, t, target_rgba, bg_rgb, ray_rgba,
                            grad_density, dL_drgb, loss_sums, true);
}

// fused_reconstruction_loss_forward_backward launch structure (src/core/nerf-network.cu:547-602):
// two memsets, one thread per ray, thrust::reduce of the 4 x n_rays losses, blocking read.
int tn_plain_recon_loss_sync(tn_stream_t stream, const tn_ray_batch* batch, int activation, float min_transmittance,
                             float inv_nrays, float grad_scale, const float* density, const float* rgb, const float* dt,
                             const float* target_rgba, const float* bg_rgb, float* loss, float* dL_ddensity,
                             float* dL_drgb, float* loss_out) {
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(rgb); TN_NONNULL(dt); TN_NONNULL(target_rgba); TN_NONNULL(bg_rgb);
    TN_NONNULL(loss); TN_NONNULL(dL_ddensity); TN_NONNULL(dL_drgb); TN_NONNULL(loss_out);
    TN_REQUIRE(batch->n_rays_dev == nullptr, TN_E_INVALID, "plain path takes a host ray count");
    const uint32_t n = batch->n_rays, rs = batch->ray_stride, ss = batch->sample_stride;
    st = cuda_status(cudaMemsetAsync(dL_ddensity, 0, (size_t)ss * sizeof(float), stream), "plain recon memset");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(dL_drgb, 0, 3 * (size_t)ss * sizeof(float), stream), "plain recon memset");
    if (st != TN_OK) return st;
    if (n == 0) { *loss_out = 0.0f; return TN_OK; }
    plain_recon_kernel<<<(n + 127) / 128, 128, 0, stream>>>(n, rs, ss, activation, min_transmittance, inv_nrays,
                                                            grad_scale, batch->counts, batch->offsets, bg_rgb,
                                                            target_rgba, density, rgb, dt, loss, dL_ddensity, dL_drgb);
    st = check_launch("tn_plain_recon_loss_sync");
    if (st != TN_OK) return st;
    float total = 0.0f;
    for (int c = 0; c < 4; ++c) {
        thrust::device_ptr<float> p(loss + (size_t)c * rs);
        total += thrust::reduce(thrust::cuda::par.on(stream), p, p + n, 0.0f, thrust::plus<float>());
    }
    *loss_out = inv_nrays * total;
    return TN_OK;
}

// mipNeRF360_distortion_loss_forward_backward launch structure (src/core/nerf-network.cu:605-666).
int tn_plain_distortion_sync(tn_stream_t stream, const tn_ray_batch* batch, int activation, float lambda,
                             const float* density, const float* m_norm, const float* dt_norm, float* ray_scratch,
                             float* sample_scratch, float* ray_loss, float* dL_ddensity, float* loss_out) {
    int st = check_batch(batch);
    if (st != TN_OK) return st;
    TN_NONNULL(density); TN_NONNULL(m_norm); TN_NONNULL(dt_norm); TN_NONNULL(ray_scratch); TN_NONNULL(sample_scratch);
    TN_NONNULL(ray_loss); TN_NONNULL(dL_ddensity); TN_NONNULL(loss_out);
    TN_REQUIRE(batch->n_rays_dev == nullptr, TN_E_INVALID, "plain path takes a host ray count");
    const uint32_t n = batch->n_rays, rs = batch->ray_stride, ss = batch->sample_stride;
    st = cuda_status(cudaMemsetAsync(dL_ddensity, 0, (size_t)ss * sizeof(float), stream), "plain distortion memset");
    if (st != TN_OK) return st;
    if (n == 0) { *loss_out = 0.0f; return TN_OK; }
    const uint32_t nb = (n + 127) / 128;
    plain_dist_fwd_kernel<<<nb, 128, 0, stream>>>(n, rs, activation, lambda, batch->counts, batch->offsets, density,
                                                  m_norm, dt_norm, ray_scratch, ray_loss, sample_scratch,
                                                  sample_scratch + ss);
    plain_dist_bwd_kernel<<<nb, 128, 0, stream>>>(n, rs, activation, lambda, batch->counts, batch->offsets, density,
                                                  ray_scratch, m_norm, dt_norm, sample_scratch, sample_scratch + ss,
                                                  dL_ddensity);
    st = check_launch("tn_plain_distortion_sync");
    if (st != TN_OK) return st;
    thrust::device_ptr<float> p(ray_loss);
    const float total = thrust::reduce(thrust::cuda::par.on(stream), p, p + n, 0.0f, thrust::plus<float>());
    *loss_out = (1.0f / (float)n) * total;
    return TN_OK;
}

int tn_plain_grad_epilogue(tn_stream_t stream, uint32_t n_samples, float loss_scale, const float* dL_rec,
                           const float* dL_dist, const float* t, float* grad_out) {
    TN_NONNULL(dL_rec); TN_NONNULL(grad_out);
    if (n_samples == 0) return TN_OK;
    const uint32_t nb = (n_samples + 127) / 128;
    plain_copy_gradients_kernel<<<nb, 128, 0, stream>>>(n_samples, loss_scale, dL_rec, grad_out);
    if (dL_dist) plain_copy_gradients_kernel<<<nb, 128, 0, stream>>>(n_samples, loss_scale, dL_dist, grad_out);
    if (t) plain_distance_scaling_kernel<<<nb, 128, 0, stream>>>(n_samples, t, grad_out);
    return check_launch("tn_plain_grad_epilogue");
}

}  // extern "C"
