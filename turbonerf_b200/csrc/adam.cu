// Adam over [hash grid | MLP] parameters (reference ngp_adam_step,
// src/core/adam-optimizer.cuh:48-96).
//
// Fused path: each thread owns four consecutive parameters and moves them with 16-byte
// loads and stores. The gradient quad is read first; a quad of hash-grid parameters whose
// four gradients are all zero is skipped without touching weights, moments or step
// counters (the reference's per-parameter "zero gradient => return" rule, applied to whole
// quads before any other load is issued). Mixed quads update only their active lanes.
// The kernel loops over the quads with a grid stride, so that the training controller can run
// it on a subset of the SMs (a small grid of 1024-thread blocks) beside the next step's march.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "tn_internal.cuh"

namespace tn {

struct AdamArgs {
    uint32_t n, n_grid, n_net_end;
    float inv_loss_scale, lr, beta1, beta2, eps, l2;
    float log2_beta1, log2_beta2;  // log2 of beta1 / beta2 (host double, rounded once)
    const float* lr_dev;  // when set, the learning rate is read from device memory (graph replays)
    const uint32_t* enable;  // when set, the update runs only if *enable != 0 (a pending update)
};

// One parameter of ngp_adam_step (adam-optimizer.cuh:69-95). The bias corrections beta^step
// are evaluated as exp2(step * log2(beta)) with log2(beta) prepared on the host, and the two
// divisions of the update are merged into one.
__device__ __forceinline__ void adam_one(const AdamArgs& a, float base_lr, uint32_t i, float g, float& w, float& m,
                                         float& v, uint32_t& step) {
    if (i >= a.n_grid && i < a.n_net_end) g += a.l2 * w;
    m = a.beta1 * m + (1.0f - a.beta1) * g;
    v = a.beta2 * v + (1.0f - a.beta2) * (g * g);
    step += 1u;
    const float s = (float)step;
    const float c1 = 1.0f - exp2f(s * a.log2_beta1);
    const float c2 = 1.0f - exp2f(s * a.log2_beta2);
    w = w - base_lr * sqrtf(c2) * m / (c1 * (sqrtf(v) + a.eps));
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
adam_vec4_kernel(AdamArgs a, float* __restrict__ w, float* __restrict__ wcopy, const float* __restrict__ grad,
                 float* __restrict__ m, float* __restrict__ v, uint32_t* __restrict__ steps) {
    if (a.enable && *a.enable == 0u) return;
    const uint32_t stride = gridDim.x * BLOCK;
    for (uint32_t q = blockIdx.x * BLOCK + threadIdx.x; q < (a.n + 3u) / 4u; q += stride) {
    const uint32_t i0 = q * 4u;
    if (i0 + 4u <= a.n) {
        float4 g = __ldcs(reinterpret_cast<const float4*>(grad) + q);
        g.x *= a.inv_loss_scale; g.y *= a.inv_loss_scale; g.z *= a.inv_loss_scale; g.w *= a.inv_loss_scale;
        const bool act0 = !(i0 + 0u < a.n_grid && g.x == 0.0f);
        const bool act1 = !(i0 + 1u < a.n_grid && g.y == 0.0f);
        const bool act2 = !(i0 + 2u < a.n_grid && g.z == 0.0f);
        const bool act3 = !(i0 + 3u < a.n_grid && g.w == 0.0f);
        if (!(act0 | act1 | act2 | act3)) continue;
        const float base_lr = a.lr_dev ? *a.lr_dev : a.lr;
        float4 wv = reinterpret_cast<float4*>(w)[q];
        float4 mv = reinterpret_cast<float4*>(m)[q];
        float4 vv = reinterpret_cast<float4*>(v)[q];
        uint4 sv = reinterpret_cast<uint4*>(steps)[q];
        if (act0) adam_one(a, base_lr, i0 + 0u, g.x, wv.x, mv.x, vv.x, sv.x);
        if (act1) adam_one(a, base_lr, i0 + 1u, g.y, wv.y, mv.y, vv.y, sv.y);
        if (act2) adam_one(a, base_lr, i0 + 2u, g.z, wv.z, mv.z, vv.z, sv.z);
        if (act3) adam_one(a, base_lr, i0 + 3u, g.w, wv.w, mv.w, vv.w, sv.w);
        reinterpret_cast<float4*>(w)[q] = wv;
        reinterpret_cast<float4*>(m)[q] = mv;
        reinterpret_cast<float4*>(v)[q] = vv;
        reinterpret_cast<uint4*>(steps)[q] = sv;
        if (wcopy) reinterpret_cast<float4*>(wcopy)[q] = wv;
    } else {
        const float base_lr = a.lr_dev ? *a.lr_dev : a.lr;
        for (uint32_t i = i0; i < a.n; ++i) {
            const float g = grad[i] * a.inv_loss_scale;
            if (i < a.n_grid && g == 0.0f) continue;
            float wi = w[i], mi = m[i], vi = v[i];
            uint32_t si = steps[i];
            adam_one(a, base_lr, i, g, wi, mi, vi, si);
            w[i] = wi; m[i] = mi; v[i] = vi; steps[i] = si;
            if (wcopy) wcopy[i] = wi;
        }
    }
    }
}

__global__ void adam_scalar_kernel(AdamArgs a, float* __restrict__ w, float* __restrict__ wcopy,
                                   const float* __restrict__ grad, float* __restrict__ m, float* __restrict__ v,
                                   uint32_t* __restrict__ steps) {
    const uint32_t i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= a.n || (a.enable && *a.enable == 0u)) return;
    const float g = grad[i] * a.inv_loss_scale;
    if (i < a.n_grid && g == 0.0f) return;
    float wi = w[i], mi = m[i], vi = v[i];
    uint32_t si = steps[i];
    adam_one(a, a.lr_dev ? *a.lr_dev : a.lr, i, g, wi, mi, vi, si);
    w[i] = wi; m[i] = mi; v[i] = vi; steps[i] = si;
    if (wcopy) wcopy[i] = wi;
}

// Reference structure: one thread per parameter, the gradient divided by the loss scale.
__global__ void plain_adam_kernel(AdamArgs a, float* __restrict__ wfp, float* __restrict__ wcopy,
                                  const float* __restrict__ grads, float* __restrict__ m1, float* __restrict__ m2,
                                  uint32_t* __restrict__ steps) {
    const uint32_t i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i >= a.n) return;
    float gradient = grads[i] / (1.0f / a.inv_loss_scale);
    if (i < a.n_grid && gradient == 0.0f) return;
    const float weight_fp = wfp[i];
    if (i >= a.n_grid && i < a.n_net_end) gradient += a.l2 * weight_fp;
    const float gsq = gradient * gradient;
    const float fm = m1[i] = a.beta1 * m1[i] + (1.0f - a.beta1) * gradient;
    const float sm = m2[i] = a.beta2 * m2[i] + (1.0f - a.beta2) * gsq;
    const uint32_t cs = ++steps[i];
    float lr = a.lr_dev ? *a.lr_dev : a.lr;
    lr *= sqrtf(1.0f - powf(a.beta2, (float)cs)) / (1.0f - powf(a.beta1, (float)cs));
    const float eff = lr / (sqrtf(sm) + a.eps);
    const float nw = weight_fp - eff * fm;
    wfp[i] = nw;
    if (wcopy) wcopy[i] = nw;
}

static int adam_args(uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale, float lr, float beta1,
                     float beta2, float eps, float l2, AdamArgs& a) {
    TN_REQUIRE(loss_scale != 0.0f, TN_E_INVALID, "loss_scale must be non-zero");
    TN_REQUIRE((uint64_t)n_grid + n_mlp <= n, TN_E_INVALID, "n_grid + n_mlp exceeds n");
    a.n = n;
    a.n_grid = n_grid;
    a.n_net_end = n_grid + n_mlp;
    a.inv_loss_scale = 1.0f / loss_scale;
    a.lr = lr;
    a.beta1 = beta1;
    a.beta2 = beta2;
    a.eps = eps;
    a.l2 = l2;
    a.log2_beta1 = (float)std::log2((double)beta1);
    a.log2_beta2 = (float)std::log2((double)beta2);
    a.lr_dev = nullptr;
    a.enable = nullptr;
    return TN_OK;
}

int launch_adam(cudaStream_t stream, bool plain, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale,
                float lr, const float* lr_dev, float beta1, float beta2, float epsilon, float l2_reg, float* weights,
                float* weights_copy, const float* gradients, float* first_moments, float* second_moments,
                uint32_t* param_steps, const AdamPlacement& place) {
    TN_NONNULL(weights); TN_NONNULL(gradients); TN_NONNULL(first_moments); TN_NONNULL(second_moments);
    TN_NONNULL(param_steps);
    AdamArgs a;
    int st = adam_args(n, n_grid, n_mlp, loss_scale, lr, beta1, beta2, epsilon, l2_reg, a);
    if (st != TN_OK) return st;
    a.lr_dev = lr_dev;
    a.enable = place.enable;
    if (n == 0) return TN_OK;
    if (plain) {
        plain_adam_kernel<<<(n + 127) / 128, 128, 0, stream>>>(a, weights, weights_copy, gradients, first_moments,
                                                               second_moments, param_steps);
        return check_launch("tn_plain_adam_step");
    }
    const bool aligned = (((uintptr_t)weights | (uintptr_t)gradients | (uintptr_t)first_moments |
                           (uintptr_t)second_moments | (uintptr_t)param_steps | (uintptr_t)weights_copy) & 15u) == 0;
    if (aligned && place.max_blocks) {
        // a few large blocks, each alone on its SM when reserve_smem is over half an SM's shared memory
        if (place.reserve_smem > 48 * 1024) {
            static const int optin_status = allow_optin_smem((const void*)adam_vec4_kernel<1024>);
            if (optin_status != TN_OK) return optin_status;
        }
        const uint32_t quads = (n + 3) / 4;
        const uint32_t blocks = std::max(1u, std::min(place.max_blocks, (quads + 1023) / 1024));
        adam_vec4_kernel<1024><<<blocks, 1024, place.reserve_smem, stream>>>(a, weights, weights_copy, gradients,
                                                                          first_moments, second_moments, param_steps);
    } else if (aligned) {
        const uint32_t quads = (n + 3) / 4;
        adam_vec4_kernel<256><<<(quads + 255) / 256, 256, 0, stream>>>(a, weights, weights_copy, gradients,
                                                                       first_moments, second_moments, param_steps);
    } else {
        adam_scalar_kernel<<<(n + 255) / 256, 256, 0, stream>>>(a, weights, weights_copy, gradients, first_moments,
                                                                second_moments, param_steps);
    }
    return check_launch("tn_adam_step");
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_adam_step(tn_stream_t stream, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale, float lr,
                 float beta1, float beta2, float epsilon, float l2_reg, float* weights, float* weights_copy,
                 const float* gradients, float* first_moments, float* second_moments, uint32_t* param_steps) {
    return launch_adam(stream, false, n, n_grid, n_mlp, loss_scale, lr, nullptr, beta1, beta2, epsilon, l2_reg,
                       weights, weights_copy, gradients, first_moments, second_moments, param_steps, AdamPlacement{});
}

int tn_plain_adam_step(tn_stream_t stream, uint32_t n, uint32_t n_grid, uint32_t n_mlp, float loss_scale, float lr,
                       float beta1, float beta2, float epsilon, float l2_reg, float* weights, float* weights_copy,
                       const float* gradients, float* first_moments, float* second_moments, uint32_t* param_steps) {
    return launch_adam(stream, true, n, n_grid, n_mlp, loss_scale, lr, nullptr, beta1, beta2, epsilon, l2_reg,
                       weights, weights_copy, gradients, first_moments, second_moments, param_steps, AdamPlacement{});
}

}  // extern "C"
