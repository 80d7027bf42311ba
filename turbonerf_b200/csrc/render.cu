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
};

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
    const float offx = __fadd_rn(__fmul_rn(cam.shift_x, (float)cam.width), -cam.principal_x);
    const float offy = __fadd_rn(__fmul_rn(cam.shift_y, (float)cam.height), -cam.principal_y);
    const float vx = __fdiv_rn(__fadd_rn(__fadd_rn((float)px, offx), 0.5f), cam.focal_x);
    const float vy = __fdiv_rn(__fadd_rn(__fadd_rn((float)py, offy), 0.5f), cam.focal_y);
    const float vz = 1.0f;
    const float vlen = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz)));
    const float* m = cam.transform;  // row-major 3 x 4: rotation | translation
    const float gx = __fadd_rn(__fadd_rn(__fmul_rn(m[0], vx), __fmul_rn(m[1], vy)), __fmul_rn(m[2], vz));
    const float gy = __fadd_rn(__fadd_rn(__fmul_rn(m[4], vx), __fmul_rn(m[5], vy)), __fmul_rn(m[6], vz));
    const float gz = __fadd_rn(__fadd_rn(__fmul_rn(m[8], vx), __fmul_rn(m[9], vy)), __fmul_rn(m[10], vz));
    const float gl = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy)), __fmul_rn(gz, gz)));
    const float dx = __fdiv_rn(gx, gl), dy = __fdiv_rn(gy, gl), dz = __fdiv_rn(gz, gl);
    float ox = __fadd_rn(m[3], __fmul_rn(cam.near, __fmul_rn(vlen, dx)));
    float oy = __fadd_rn(m[7], __fmul_rn(cam.near, __fmul_rn(vlen, dy)));
    float oz = __fadd_rn(m[11], __fmul_rn(cam.near, __fmul_rn(vlen, dz)));
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

// One sample of a ray at t: whether the network is queried there (filter_and_localize_samples_for_
// nerf_kernel and assign_normalized_network_inputs_kernel, rendering-kernels.cu:336-478, identity
// transform) and its network inputs.
struct RenderSample {
    bool valid;
    float ux, uy, uz;  // unit-cube position, clamped to [0, 1]
    float dt_net;      // step in units of the training box size
};

__device__ __forceinline__ RenderSample render_sample(const RenderArgs& A, const RayMarch& r, float t, float dt,
                                                      float dir_len) {
    RenderSample o;
    float x, y, z;
    ray_point(r, t, x, y, z);
    o.dt_net = __fmul_rn(A.inv_train_size, __fmul_rn(dir_len, dt));
    const float ux = __fdiv_rn(__fadd_rn(x, -A.train_bbox.min_x), A.train_size_x);
    const float uy = __fdiv_rn(__fadd_rn(y, -A.train_bbox.min_y), A.train_size_y);
    const float uz = __fdiv_rn(__fadd_rn(z, -A.train_bbox.min_z), A.train_size_z);
    o.valid = false;
    if (bbox_contains(A.render_bbox, x, y, z)) {
        const int k = grid_level_at(A.g, x, y, z, o.dt_net);
        o.valid = ((A.g.bits[voxel_morton(A.g, k, x, y, z)] >> k) & 1u) && ux >= 0.0f && ux <= 1.0f &&
                  uy >= 0.0f && uy <= 1.0f && uz >= 0.0f && uz <= 1.0f;
    }
    o.ux = clamp_ref(ux, 0.0f, 1.0f);
    o.uy = clamp_ref(uy, 0.0f, 1.0f);
    o.uz = clamp_ref(uz, 0.0f, 1.0f);
    return o;
}

// count (EMIT = false: counts[j]) or emit (EMIT = true: packed network inputs at offsets[j], and
// the ray's t advanced) the valid samples of the next `steps` steps of each live ray
template <bool EMIT>
__global__ void render_march_kernel(RenderArgs A, uint32_t n, uint32_t n_live, uint32_t steps,
                                    const uint32_t* __restrict__ live, const float* __restrict__ ori,
                                    const float* __restrict__ dir, float* __restrict__ ray_t,
                                    uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                                    uint32_t cap, float* __restrict__ s_pos, float* __restrict__ s_dir,
                                    float* __restrict__ s_dt, uint32_t* flags) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_live) return;
    const uint32_t i = live[j];
    RayMarch r;
    r.ox = ori[i]; r.oy = ori[i + n]; r.oz = ori[i + 2 * (size_t)n];
    r.dx = dir[i]; r.dy = dir[i + n]; r.dz = dir[i + 2 * (size_t)n];
    const float dir_len =
        __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(r.dx, r.dx), __fmul_rn(r.dy, r.dy)), __fmul_rn(r.dz, r.dz)));
    const float nx = __fmaf_rn(0.5f, r.dx, 0.5f), ny = __fmaf_rn(0.5f, r.dy, 0.5f), nz = __fmaf_rn(0.5f, r.dz, 0.5f);
    float t = ray_t[i];
    uint32_t c = 0, o = EMIT ? offsets[j] : 0u;
    for (uint32_t s = 0; s < steps; ++s) {
        const float dt = get_dt(t, A.cone, A.dt_min, A.dt_max);
        const RenderSample smp = render_sample(A, r, t, dt, dir_len);
        if (smp.valid) {
            if (EMIT) {
                if (o < cap) {
                    s_pos[o] = smp.ux; s_pos[o + cap] = smp.uy; s_pos[o + 2 * (size_t)cap] = smp.uz;
                    s_dir[o] = nx; s_dir[o + cap] = ny; s_dir[o + 2 * (size_t)cap] = nz;
                    s_dt[o] = smp.dt_net;
                } else {
                    raise_flag(flags, ERR_CAPACITY);
                }
                ++o;
            }
            ++c;
        }
        t = __fadd_rn(t, dt);
    }
    if (EMIT) ray_t[i] = t;
    else counts[j] = c;
}

// composite_samples_kernel (rendering-kernels.cu:530-618) after accumulate_nerf_samples_kernel
// (:480-528) for one NeRF: each live ray composites its samples of this iteration in order.
// keep[j] = 1 while the ray stays live: transmittance not below min_transmittance and t not past
// t_max (kill_terminated_rays_kernel, :620-637).
__global__ void render_composite_kernel(RenderArgs A, uint32_t n_live, const uint32_t* __restrict__ live,
                                        const uint32_t* __restrict__ counts, const uint32_t* __restrict__ offsets,
                                        uint32_t cap, const float* __restrict__ density, const float* __restrict__ rgb,
                                        const float* __restrict__ s_dt, const float* __restrict__ ray_t,
                                        const float* __restrict__ ray_tmax, float* __restrict__ trans,
                                        float* __restrict__ out, uint32_t* __restrict__ keep) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_live) return;
    const uint32_t i = live[j];
    float T = trans[i];
    float orr = 0.0f, og = 0.0f, ob = 0.0f, oa = 0.0f;
    bool alive = true;
    const uint32_t o = offsets[j];
    const uint32_t c = o < cap ? min(counts[j], cap - o) : 0u;
    for (uint32_t k = 0; k < c; ++k) {
        const uint32_t s = o + k;
        const float alpha = render_alpha(__fmul_rn(render_sigma(A.act, density[s]), s_dt[s]));
        // one NeRF's sample colour: (c alpha) / alpha, zero when alpha <= 1e-4
        const float inv_a = alpha > 0.0001f ? __fdiv_rn(1.0f, alpha) : 0.0f;
        const float cr = __fmul_rn(__fmul_rn(rgb[s], alpha), inv_a);
        const float cg = __fmul_rn(__fmul_rn(rgb[s + cap], alpha), inv_a);
        const float cb = __fmul_rn(__fmul_rn(rgb[s + 2 * (size_t)cap], alpha), inv_a);
        const float a = fminf(alpha, 1.0f);
        const float w = __fmul_rn(a, T);
        orr = __fadd_rn(orr, __fmul_rn(w, cr));
        og = __fadd_rn(og, __fmul_rn(w, cg));
        ob = __fadd_rn(ob, __fmul_rn(w, cb));
        oa = __fadd_rn(oa, w);
        T = __fmul_rn(T, __fadd_rn(1.0f, -a));
        if (T < A.min_t) {
            alive = false;
            break;
        }
    }
    trans[i] = T;
    float4* px = reinterpret_cast<float4*>(out) + i;
    float4 v = *px;
    v.x += orr; v.y += og; v.z += ob; v.w += oa;
    *px = v;
    keep[j] = (alive && !(ray_t[i] > ray_tmax[i])) ? 1u : 0u;
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
    const uint32_t batch = desc->batch_size ? desc->batch_size : (1u << 20);  // renderer default batch
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

    // workspace: rays [o 3 | d 3 | t | t_max | T] x n floats; pixel lists [live | live2 | counts |
    // offsets | keep | idx] x n u32; counters (16 u32); samples [pos 3 | dir 3 | dt | density | rgb 3]
    // x cap floats
    const size_t ray_words = (size_t)9 * n, list_words = (size_t)6 * n, smp_words = (size_t)11 * cap;
    st = ensure_render_ws(ctx, (ray_words + list_words + 16 + smp_words) * 4);
    if (st != TN_OK) return st;
    float* rays = reinterpret_cast<float*>(ctx->render_ws);
    float *ori = rays, *dir = rays + 3 * (size_t)n, *ray_t = rays + 6 * (size_t)n, *ray_tmax = rays + 7 * (size_t)n,
          *trans = rays + 8 * (size_t)n;
    uint32_t* u32 = reinterpret_cast<uint32_t*>(rays + ray_words);
    uint32_t *live = u32, *live2 = u32 + n, *counts = u32 + 2 * (size_t)n, *offsets = u32 + 3 * (size_t)n,
             *keep = u32 + 4 * (size_t)n;
    int32_t* idx = reinterpret_cast<int32_t*>(u32 + 5 * (size_t)n);
    uint32_t* counters = u32 + list_words;  // [0] live rays, [1..4] batch info, [5] kept rays
    uint32_t* info = counters + 1;
    float* smp = reinterpret_cast<float*>(counters + 16);
    float *s_pos = smp, *s_dir = smp + 3 * (size_t)cap, *s_dt = smp + 6 * (size_t)cap,
          *s_density = smp + 7 * (size_t)cap, *s_rgb = smp + 8 * (size_t)cap;

    tn_render_stats S{};
    st = cuda_status(cudaMemsetAsync(out_rgba, 0, (size_t)n * 16, stream), "tn_render(clear)");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(counters, 0, 64, stream), "tn_render(counters)");
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
    const uint32_t max_iters = 1u << 20;
    while (st == TN_OK && n_live > 0 && S.iterations < max_iters) {
        const uint32_t steps = std::max(batch / n_live, 1u);  // renderer.cu:301
        const int grid = (int)((n_live + 255) / 256);
        render_march_kernel<false><<<grid, 256, 0, stream>>>(A, n, n_live, steps, live, ori, dir, ray_t, counts,
                                                              nullptr, cap, nullptr, nullptr, nullptr, ctx->flags);
        st = check_launch("tn_render(count)");
        if (st == TN_OK) st = tn_scan_offsets(ctx, stream, n_live, counts, offsets, 0xffffffffu, info);
        if (st == TN_OK) {
            render_march_kernel<true><<<grid, 256, 0, stream>>>(A, n, n_live, steps, live, ori, dir, ray_t, counts,
                                                                 offsets, cap, s_pos, s_dir, s_dt, ctx->flags);
            st = check_launch("tn_render(emit)");
        }
        if (st == TN_OK) st = net->forward(net->user, stream, cap, info + 1, cap, s_pos, s_dir, s_density, s_rgb);
        if (st == TN_OK) {
            render_composite_kernel<<<grid, 256, 0, stream>>>(A, n_live, live, counts, offsets, cap, s_density, s_rgb,
                                                              s_dt, ray_t, ray_tmax, trans, out_rgba, keep);
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
        S.steps += (uint64_t)steps * n_live;
        ++S.iterations;
        n_live = host[4];
        std::swap(live, live2);
    }
    if (st == TN_OK && n_live > 0) st = fail(TN_E_DEVICE, "tn_render: rays still live after %u iterations", max_iters);
    uint32_t flags = 0;
    if (st == TN_OK) st = tn_ctx_check(ctx, stream, &flags);
    if (st == TN_OK && (flags & TN_FLAG_CAPACITY)) st = fail(TN_E_CAPACITY, "tn_render: sample capacity exceeded");
    if (stats) *stats = S;
    return st;
}

}  // extern "C"
