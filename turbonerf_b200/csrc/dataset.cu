// Training rays from a dataset of posed images: the reference's
// initialize_training_rays_and_pixels_kernel and deactivate_rays_with_alpha_threshold_kernel
// (src/utils/training-batch-kernels.cuh:82-208), called by Trainer::generate_next_training_batch
// (src/core/trainer.cu:40-100), in one kernel.
//
// Ray i belongs to image (uint32)(i / (n_rays / n_images)) (float arithmetic, as the reference);
// its pixel position is p = n_pixels * u_i with u_i uniform in [0, 1): x = fmod(p, width),
// y = p / width, the ray through (x, y) of the image's pinhole camera. The ray is clipped to the
// training box (t = max(0, t_min + 1e-5), t_max = min(far - near, box exit); dead when it misses
// or t_max < t), its target is the image's RGBA8 texel at index min(floor(p), n_pixels - 1) / 255,
// and with alpha selection on (threshold < 1 and probability < 1) a ray whose target alpha is
// below the threshold dies when its second draw v_i exceeds the probability.
#include "tn_internal.cuh"

namespace tn {

struct DatasetArgs {
    uint32_t n_rays, rs;
    uint32_t n_images, n_pixels;
    int32_t width;
    float rays_per_image;  // (float)n_rays / (float)n_images
    tn_bbox bbox;
    float alpha_threshold, alpha_probability;
    int alpha_selection;
};

__global__ void dataset_rays_kernel(DatasetArgs A, const tn_camera* __restrict__ cameras,
                                    const uint8_t* __restrict__ images, const float* __restrict__ random,
                                    float* __restrict__ pix_rgba, uint32_t* __restrict__ img_id,
                                    float* __restrict__ ori, float* __restrict__ dir, float* __restrict__ ray_t,
                                    float* __restrict__ ray_tmax, uint8_t* __restrict__ alive) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.n_rays) return;
    // (the reference indexes image n_images when the float quotient rounds up to it; clamped here)
    const uint32_t image = min((uint32_t)__fdiv_rn((float)i, A.rays_per_image), A.n_images - 1u);
    const float p = __fmul_rn((float)A.n_pixels, random[i]);
    const float w = (float)A.width;
    const float x = fmodf(p, w), y = __fdiv_rn(p, w);
    const tn_camera cam = cameras[image];
    float ox, oy, oz, dx, dy, dz;
    pinhole_ray(cam, x, y, ox, oy, oz, dx, dy, dz);
    // BoundingBox::get_ray_t_intersections (bounding-box.cuh:27-51)
    const tn_bbox& b = A.bbox;
    const float ix = __fdiv_rn(1.0f, dx), iy = __fdiv_rn(1.0f, dy), iz = __fdiv_rn(1.0f, dz);
    float t1x = __fmul_rn(__fadd_rn(b.min_x, -ox), ix), t2x = __fmul_rn(__fadd_rn(b.max_x, -ox), ix);
    float t1y = __fmul_rn(__fadd_rn(b.min_y, -oy), iy), t2y = __fmul_rn(__fadd_rn(b.max_y, -oy), iy);
    float t1z = __fmul_rn(__fadd_rn(b.min_z, -oz), iz), t2z = __fmul_rn(__fadd_rn(b.max_z, -oz), iz);
    if (t1x > t2x) { const float s = t1x; t1x = t2x; t2x = s; }
    if (t1y > t2y) { const float s = t1y; t1y = t2y; t2y = s; }
    if (t1z > t2z) { const float s = t1z; t1z = t2z; t2z = s; }
    const float tmin = fmaxf(t1x, fmaxf(t1y, t1z)), tmax = fminf(t2x, fminf(t2y, t2z));
    const float t_max = fminf(__fadd_rn(cam.far, -cam.near), tmax);
    const float t = fmaxf(0.0f, __fadd_rn(tmin, 1e-5f));
    bool ok = tmax >= tmin && !(t_max < t);
    // the target texel
    const uint32_t k = min((uint32_t)p, A.n_pixels - 1u);
    const uchar4 px = reinterpret_cast<const uchar4*>(images)[(size_t)A.n_pixels * image + k];
    const float ta = __fdiv_rn((float)px.w, 255.0f);
    if (ok && A.alpha_selection && ta < A.alpha_threshold && random[i + A.rs] > A.alpha_probability) ok = false;
    const size_t rs = A.rs;
    pix_rgba[i] = __fdiv_rn((float)px.x, 255.0f);
    pix_rgba[i + rs] = __fdiv_rn((float)px.y, 255.0f);
    pix_rgba[i + 2 * rs] = __fdiv_rn((float)px.z, 255.0f);
    pix_rgba[i + 3 * rs] = ta;
    ori[i] = ox; ori[i + rs] = oy; ori[i + 2 * rs] = oz;
    dir[i] = dx; dir[i + rs] = dy; dir[i + 2 * rs] = dz;
    ray_t[i] = ok ? t : 0.0f;
    ray_tmax[i] = ok ? t_max : 0.0f;
    alive[i] = ok ? 1 : 0;
    if (img_id) img_id[i] = image;
}

// The draws of one step's dataset rays, from the counter-based generator of the synthetic
// producer: random[i] (pixel), random[i + rs] (alpha selection), and the background colour bg.
__global__ void dataset_draws_kernel(uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* __restrict__ step_dev,
                                     float* __restrict__ random, float* __restrict__ bg) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t st = 0x40000000u + 2u * (step_dev ? *step_dev : 0u);
    random[i] = rng_uniform(seed, st, i, 0);
    random[i + rs] = rng_uniform(seed, st, i, 1);
    for (int c = 0; c < 3; ++c) bg[i + c * (size_t)rs] = rng_uniform(seed, st, i, 20 + c);
}

int check_dataset(uint32_t n_images, int32_t width, int32_t height) {
    TN_REQUIRE(n_images > 0, TN_E_INVALID, "dataset: no images");
    TN_REQUIRE(width > 0 && height > 0, TN_E_INVALID, "dataset: image size %d x %d", width, height);
    TN_REQUIRE((uint64_t)width * (uint64_t)height < (1ull << 31), TN_E_CAPACITY, "dataset: image of %d x %d pixels",
               width, height);
    return TN_OK;
}

int launch_dataset_rays(cudaStream_t stream, uint32_t n_rays, uint32_t rs, uint32_t n_images, int32_t width,
                        int32_t height, const tn_camera* cameras, const uint8_t* images, const tn_bbox& bbox,
                        const float* random, float alpha_threshold, float alpha_probability, float* pix_rgba,
                        uint32_t* img_id, float* ori, float* dir, float* ray_t, float* ray_tmax, uint8_t* alive) {
    if (n_rays == 0) return TN_OK;
    DatasetArgs A;
    A.n_rays = n_rays;
    A.rs = rs;
    A.n_images = n_images;
    A.n_pixels = (uint32_t)width * (uint32_t)height;
    A.width = width;
    A.rays_per_image = (float)n_rays / (float)n_images;
    A.bbox = bbox;
    A.alpha_threshold = alpha_threshold;
    A.alpha_probability = alpha_probability;
    A.alpha_selection = alpha_threshold < 1.0f && alpha_probability < 1.0f;  // trainer.cu:86
    dataset_rays_kernel<<<(n_rays + 255) / 256, 256, 0, stream>>>(A, cameras, images, random, pix_rgba, img_id, ori,
                                                                  dir, ray_t, ray_tmax, alive);
    return check_launch("dataset rays");
}

int launch_dataset_draws(cudaStream_t stream, uint32_t n, uint32_t rs, uint32_t seed, const uint32_t* step_dev,
                         float* random, float* bg) {
    if (n == 0) return TN_OK;
    dataset_draws_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, rs, seed, step_dev, random, bg);
    return check_launch("dataset draws");
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_dataset_rays(tn_stream_t stream, uint32_t n_rays, uint32_t ray_stride, uint32_t n_images, int32_t width,
                    int32_t height, const tn_camera* cameras, const uint8_t* images, const tn_bbox* bbox,
                    const float* random, float alpha_threshold, float alpha_probability, float* pix_rgba,
                    uint32_t* img_id, float* ori, float* dir, float* ray_t, float* ray_t_max, uint8_t* alive) {
    TN_NONNULL(cameras); TN_NONNULL(images); TN_NONNULL(bbox); TN_NONNULL(random); TN_NONNULL(pix_rgba);
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(ray_t); TN_NONNULL(ray_t_max); TN_NONNULL(alive);
    const int st = check_dataset(n_images, width, height);
    if (st != TN_OK) return st;
    TN_REQUIRE(ray_stride >= n_rays, TN_E_INVALID, "ray_stride %u < n_rays %u", ray_stride, n_rays);
    TN_REQUIRE(((uintptr_t)images & 3u) == 0, TN_E_INVALID, "images must be 4-byte aligned (RGBA8 texels)");
    return launch_dataset_rays(stream, n_rays, ray_stride, n_images, width, height, cameras, images, *bbox, random,
                               alpha_threshold, alpha_probability, pix_rgba, img_id, ori, dir, ray_t, ray_t_max, alive);
}

}  // extern "C"
