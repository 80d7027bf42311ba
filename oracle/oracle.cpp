// TEST INFRASTRUCTURE ONLY — CPU oracle for the TurboNeRF per-step training hot path.
//
// This file is a CPU restatement of the reference kernels. It is the checker the
// parity tests compare the CUDA library against, and the timed CPU baseline
// reported by bench.py. Nothing in the product (turbonerf_b200/) links or calls it.
//
// Parity status: UNPINNED. The reference ships no tests, golden vectors or
// fixtures, and its kernels cannot be compiled here (the tiny-cuda-nn and pybind11
// submodules are empty). This restatement is therefore pinned only by its own
// line-by-line correspondence to the reference source (each function cites the
// file:line it follows), by central finite differences of its analytic gradients,
// and by closed-form special cases (tests/test_oracle.py).
//
// Precision rules:
//  * integer outputs (march counts, offsets, emitted sample positions, occupancy
//    bits and densities) are computed in FP32 with the reference's operation order;
//    this file must be compiled with -ffp-contract=off so that no a*b+c is fused;
//  * float outputs of the compositor, distortion loss, gradient epilogue and Adam
//    are computed in FP64 (exp instead of the fast __expf intrinsic).
//
// Layout follows the reference: structure-of-arrays with an explicit stride, so
// component c of item i lives at buf[c*stride + i]
// (src/workspaces/training-workspace.cuh:87-112).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

extern "C" {

// ---------------------------------------------------------------------------
// Morton code (tiny-cuda-nn morton3D / morton3D_invert, un-vendored submodule,
// pinned version unknown). Restated from the definition used at
// src/core/occupancy-grid.cuh:162 and :173-175: x goes to bit 0, y to bit 1,
// z to bit 2 of each 3-bit group. Written bit by bit on purpose (the CUDA side
// uses the multiply/mask form; the tests check they agree).
// ---------------------------------------------------------------------------
uint32_t orc_morton3d(uint32_t x, uint32_t y, uint32_t z) {
    uint32_t r = 0;
    for (int b = 0; b < 10; ++b) {
        r |= ((x >> b) & 1u) << (3 * b);
        r |= ((y >> b) & 1u) << (3 * b + 1);
        r |= ((z >> b) & 1u) << (3 * b + 2);
    }
    return r;
}

uint32_t orc_morton3d_invert(uint32_t v) {
    uint32_t r = 0;
    for (int b = 0; b < 11; ++b) r |= ((v >> (3 * b)) & 1u) << b;
    return r;
}

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------------------
// Scalar helpers
// ---------------------------------------------------------------------------

struct Bbox { float min_x, min_y, min_z, max_x, max_y, max_z; };

struct Grid {
    int n_levels;
    int res;
    float base;            // level k covers base * 2^k world units (base = 1: reference)
    const uint8_t* bits;   // byte per Morton cell, bit k = level k
};

// BoundingBox::contains, src/models/bounding-box.cuh:70-74 (inclusive on both faces)
static inline bool bbox_contains(const Bbox& b, float x, float y, float z) {
    return x >= b.min_x && x <= b.max_x && y >= b.min_y && y <= b.max_y && z >= b.min_z && z <= b.max_z;
}

// tcnn::clamp(val, lo, hi) as used by get_dt, src/utils/raymarching-utils.cuh:7-14
static inline float clampf_ref(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}

static inline float get_dt(float t, float cone, float dt_min, float dt_max) {
    return clampf_ref(t * cone, dt_min, dt_max);
}

// OccupancyGrid::get_level_size, src/core/occupancy-grid.cuh:139-141 (base generalises 1.0)
static inline float level_size(const Grid& g, int k) { return g.base * (float)(1 << k); }

// Quantise one coordinate for get_voxel_morton_index (src/core/occupancy-grid.cuh:155-159).
// The reference casts (x*s + 0.5f)*R straight to uint32; for points outside the level
// that index leaves [0, R) and reads outside the bitfield. Here it is clamped to the
// edge cell, which is identical whenever the reference stays in bounds.
static inline uint32_t cell_coord(float x, float s, float res_f, int res) {
    const float f = (x * s + 0.5f) * res_f;
    if (!(f >= 0.0f)) return 0u;
    if (f >= res_f) return (uint32_t)(res - 1);
    return (uint32_t)f;
}

static inline uint32_t voxel_morton(const Grid& g, int k, float x, float y, float z) {
    const float s = 1.0f / level_size(g, k);
    const float res_f = (float)g.res;
    return orc_morton3d(cell_coord(x, s, res_f, g.res), cell_coord(y, s, res_f, g.res), cell_coord(z, s, res_f, g.res));
}

// OccupancyGrid::is_occupied_at, src/core/occupancy-grid.cuh:185-207
static inline bool is_occupied(const Grid& g, int k, float x, float y, float z) {
    return (g.bits[voxel_morton(g, k, x, y, z)] & (uint8_t)(1u << k)) != 0;
}

// OccupancyGrid::get_grid_level_at, src/core/occupancy-grid.cuh:232-248
static inline int grid_level_at(const Grid& g, float x, float y, float z, float dt) {
    const float inv_res = 1.0f / (float)g.res;
    for (int k = 0; k < g.n_levels; ++k) {
        const float ls = level_size(g, k);
        const float half = 0.5f * ls;
        const float cell = ls * inv_res;
        const bool covers = std::fabs(x) < half && std::fabs(y) < half && std::fabs(z) < half;
        if (covers && cell > dt) return k;
    }
    return g.n_levels - 1;
}

// __fdiv_ru: IEEE single division rounded toward +infinity. q = RN(a/b) leaves an
// exactly representable remainder a - q*b (computed exactly by fma); a remainder with
// the sign of b means the true quotient lies above q.
static inline float fdiv_ru(float a, float b) {
    float q = a / b;
    if (!std::isfinite(q)) return q;
    const float r = std::fma(-q, b, a);
    if (r != 0.0f && ((r > 0.0f) == (b > 0.0f))) q = std::nextafter(q, INFINITY);
    return q;
}

float orc_fdiv_ru(float a, float b) { return fdiv_ru(a, b); }

// OccupancyGrid::get_dt_to_next_voxel, src/core/occupancy-grid.cuh:259-282
static inline float dt_to_next_voxel(const Grid& g, float px, float py, float pz,
                                     float dx, float dy, float dz,
                                     float idx, float idy, float idz,
                                     float dt_min, int level) {
    const float ls = level_size(g, level);
    const float ils = 1.0f / ls;
    const float res_f = (float)g.res;
    const float inv_res = 1.0f / res_f;
    const float x = (px * ils + 0.5f) * res_f;
    const float y = (py * ils + 0.5f) * res_f;
    const float z = (pz * ils + 0.5f) * res_f;
    const float k = inv_res * ls;
    const float tx = k * ((std::floor(0.5f * std::copysign(1.0f, dx) + x + 0.5f) - x) * idx);
    const float ty = k * ((std::floor(0.5f * std::copysign(1.0f, dy) + y + 0.5f) - y) * idy);
    const float tz = k * ((std::floor(0.5f * std::copysign(1.0f, dz) + z + 0.5f) - z) * idz);
    const float t_target = std::fmax(dt_min, std::fmin(std::fmin(tx, ty), tz));
    return fdiv_ru(t_target, dt_min) * dt_min;
}

// ---------------------------------------------------------------------------
// Ray set-up: the bounding-box clip of initialize_training_rays_and_pixels_kernel,
// src/utils/training-batch-kernels.cuh:122-150 (the camera and pixel parts are not
// on this path). get_ray_t_intersections: src/models/bounding-box.cuh:27-51.
// ---------------------------------------------------------------------------
void orc_rays_init_bbox(int64_t n, int64_t stride, const Bbox* bbox, float t_far,
                        const float* ori, const float* dir,
                        float* ray_t, float* ray_t_max, uint8_t* alive) {
    const Bbox b = *bbox;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const float ox = ori[i], oy = ori[i + stride], oz = ori[i + 2 * stride];
        const float dx = dir[i], dy = dir[i + stride], dz = dir[i + 2 * stride];
        const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
        float t1x = (b.min_x - ox) * ix, t2x = (b.max_x - ox) * ix;
        float t1y = (b.min_y - oy) * iy, t2y = (b.max_y - oy) * iy;
        float t1z = (b.min_z - oz) * iz, t2z = (b.max_z - oz) * iz;
        if (t1x > t2x) std::swap(t1x, t2x);
        if (t1y > t2y) std::swap(t1y, t2y);
        if (t1z > t2z) std::swap(t1z, t2z);
        const float tmin = std::fmax(t1x, std::fmax(t1y, t1z));
        const float tmax = std::fmin(t2x, std::fmin(t2y, t2z));
        if (!(tmax >= tmin)) { alive[i] = 0; ray_t[i] = 0.0f; ray_t_max[i] = 0.0f; continue; }
        const float t_max = std::fmin(t_far, tmax);
        const float t = std::fmax(0.0f, tmin + 1e-5f);
        if (t_max < t) { alive[i] = 0; ray_t[i] = 0.0f; ray_t_max[i] = 0.0f; continue; }
        ray_t[i] = t;
        ray_t_max[i] = t_max;
        alive[i] = 1;
    }
}

// ---------------------------------------------------------------------------
// march_and_count_steps_per_ray_kernel, src/utils/training-batch-kernels.cuh:212-298
// max_steps = 0 reproduces the reference (no cap); otherwise counting stops at the cap.
// Returns the number of rays that hit the iteration guard (0 when all finished).
// ---------------------------------------------------------------------------
int64_t orc_march_count(int64_t n_rays, int64_t stride, const Bbox* bbox,
                        int n_levels, int res, float base, const uint8_t* bitfield,
                        float cone, float dt_min, float dt_max, uint32_t max_steps,
                        uint32_t max_iters,
                        const float* ori, const float* dir, const float* ray_t, const float* ray_t_max,
                        uint8_t* alive, uint32_t* n_steps) {
    const Bbox b = *bbox;
    const Grid g{n_levels, res, base, bitfield};
    int64_t n_guard = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : n_guard)
    for (int64_t i = 0; i < n_rays; ++i) {
        if (!alive[i]) { n_steps[i] = 0; continue; }
        const float ox = ori[i], oy = ori[i + stride], oz = ori[i + 2 * stride];
        const float dx = dir[i], dy = dir[i + stride], dz = dir[i + 2 * stride];
        const float idx = 1.0f / dx, idy = 1.0f / dy, idz = 1.0f / dz;
        uint32_t n = 0, iters = 0;
        float t = ray_t[i];
        const float t_max = ray_t_max[i];
        while (t < t_max) {
            if (++iters > max_iters) { ++n_guard; break; }
            const float x = ox + t * dx, y = oy + t * dy, z = oz + t * dz;
            if (!bbox_contains(b, x, y, z)) break;
            const float dt = get_dt(t, cone, dt_min, dt_max);
            const int k = grid_level_at(g, x, y, z, dt);
            if (is_occupied(g, k, x, y, z)) {
                t += dt;
                ++n;
                if (max_steps != 0 && n >= max_steps) break;
            } else {
                t += dt_to_next_voxel(g, x, y, z, dx, dy, dz, idx, idy, idz, dt_min, k);
            }
        }
        if (n == 0) alive[i] = 0;
        n_steps[i] = n;
    }
    return n_guard;
}

// ---------------------------------------------------------------------------
// Offsets and batch cut, src/core/trainer.cu:133-183 with find_last_lt_presorted
// (src/utils/parallel-utils.cuh:31-58): offsets = exclusive scan of n_steps;
// n_rays = (last index whose offset < batch_size); n_samples = offsets[n_rays].
// Returns 0 on success, -5 when no ray fits, -6 when no sample is produced.
// ---------------------------------------------------------------------------
int orc_scan_cut(int64_t n, const uint32_t* n_steps, uint32_t batch_size,
                 uint32_t* offsets, uint32_t* n_rays_out, uint32_t* n_samples_out) {
    uint64_t acc = 0;
    for (int64_t i = 0; i < n; ++i) { offsets[i] = (uint32_t)acc; acc += n_steps[i]; }
    int64_t last = -1;
    for (int64_t i = n - 1; i >= 0; --i) if (offsets[i] < batch_size) { last = i; break; }
    const int64_t max_idx = last - 1;
    if (max_idx < 0) { *n_rays_out = 0; *n_samples_out = 0; return -5; }
    *n_rays_out = (uint32_t)(max_idx + 1);
    *n_samples_out = offsets[max_idx + 1];
    if (*n_samples_out < 1) return -6;
    return 0;
}

// assign_normalized_ray_sample, src/utils/training-batch-kernels.cuh:305-331
static inline void assign_sample(int64_t ss, int64_t s, float x, float y, float z,
                                 float dx, float dy, float dz, float dt, float inv_aabb,
                                 float* pos, float* sdir, float* sdt) {
    sdt[s] = inv_aabb * dt;
    pos[s] = clampf_ref(x * inv_aabb + 0.5f, 0.0f, 1.0f);
    pos[s + ss] = clampf_ref(y * inv_aabb + 0.5f, 0.0f, 1.0f);
    pos[s + 2 * ss] = clampf_ref(z * inv_aabb + 0.5f, 0.0f, 1.0f);
    sdir[s] = 0.5f * dx + 0.5f;
    sdir[s + ss] = 0.5f * dy + 0.5f;
    sdir[s + 2 * ss] = 0.5f * dz + 0.5f;
}

// ---------------------------------------------------------------------------
// march_and_generate_network_positions_kernel, src/utils/training-batch-kernels.cuh:339-481
// ---------------------------------------------------------------------------
void orc_march_emit(int64_t n_rays, int64_t ray_stride, int64_t sample_stride, const Bbox* bbox,
                    float inv_aabb, int n_levels, int res, float base, const uint8_t* bitfield,
                    float cone, float dt_min, float dt_max,
                    const uint32_t* ray_img_id, const float* ori, const float* dir,
                    const float* ray_t, const uint32_t* offsets, const uint8_t* alive,
                    const uint32_t* n_steps,
                    uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir,
                    float* out_dt, float* out_m_norm, float* out_dt_norm) {
    const Bbox b = *bbox;
    const Grid g{n_levels, res, base, bitfield};
    const int64_t rs = ray_stride, ss = sample_stride;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_rays; ++i) {
        if (!alive[i]) continue;
        const uint32_t ns = n_steps[i];
        const uint32_t off = offsets[i];
        const uint32_t img = ray_img_id ? ray_img_id[i] : 0u;
        const float ox = ori[i], oy = ori[i + rs], oz = ori[i + 2 * rs];
        const float dx = dir[i], dy = dir[i + rs], dz = dir[i + 2 * rs];
        const float idx = 1.0f / dx, idy = 1.0f / dy, idz = 1.0f / dz;
        float t = ray_t[i];
        const float t_min = t;
        float t_max = t;
        uint32_t taken = 0;
        while (taken < ns) {
            const float x = ox + t * dx, y = oy + t * dy, z = oz + t * dz;
            const float dt = get_dt(t, cone, dt_min, dt_max);
            const int64_t s = (int64_t)off + taken;
            if (!bbox_contains(b, x, y, z)) {
                out_t[s] = t;
                out_m_norm[s] = t + 0.5f * dt;
                out_dt_norm[s] = dt;
                if (out_img_id) out_img_id[s] = img;
                assign_sample(ss, s, x, y, z, dx, dy, dz, dt, inv_aabb, out_pos, out_dir, out_dt);
                ++taken;
                continue;
            }
            const int k = grid_level_at(g, x, y, z, dt);
            if (is_occupied(g, k, x, y, z)) {
                out_t[s] = t;
                out_m_norm[s] = t + 0.5f * dt;
                out_dt_norm[s] = dt;
                if (out_img_id) out_img_id[s] = img;
                t += dt;
                t_max = t;
                assign_sample(ss, s, x, y, z, dx, dy, dz, dt, inv_aabb, out_pos, out_dir, out_dt);
                ++taken;
            } else {
                t += dt_to_next_voxel(g, x, y, z, dx, dy, dz, idx, idy, idz, dt_min, k);
            }
        }
        const float t_span = std::max(t_max - t_min, 1e-6f);
        for (uint32_t j = 0; j < taken; ++j) {
            const int64_t s = (int64_t)off + j;
            out_m_norm[s] = clampf_ref((out_m_norm[s] - t_min) / t_span, 0.0f, 1.0f);
            out_dt_norm[s] /= t_span;
        }
    }
}

// ---------------------------------------------------------------------------
// generate_nonzero_compaction_indices, src/utils/stream-compaction.cuh:120-139:
// ascending list of the indices whose value is non-zero.
// ---------------------------------------------------------------------------
int64_t orc_compact_nonzero(int64_t n, const uint32_t* values, int32_t* out) {
    int64_t c = 0;
    for (int64_t i = 0; i < n; ++i) if (values[i] != 0) out[c++] = (int32_t)i;
    return c;
}

// ---------------------------------------------------------------------------
// density_to_sigma / sigma_to_alpha, src/utils/common-network-kernels.cuh:7-25 (FP64).
// activation 0: the input already is sigma (d sigma / d input = 1);
// activation 1: the reference's exp(min(d, 12) - 1) with d sigma / d density taken as
// sigma (the clamp is ignored in the backward, training-kernels-fused.cuh:325).
// ---------------------------------------------------------------------------
static inline double act_sigma(int act, double d) {
    return act == 0 ? d : std::exp(std::min(d, 12.0) - 1.0);
}
static inline double act_dsigma(int act, double sigma) { return act == 0 ? 1.0 : sigma; }

static inline double huber_fwd(double x) { const double a = std::fabs(x); return a < 1.0 ? 0.5 * x * x : a - 0.5; }
static inline double huber_bwd(double x) { return std::fabs(x) < 1.0 ? x : std::copysign(1.0, x); }

// ---------------------------------------------------------------------------
// fused_reconstruction_forward_backward_kernel, src/utils/training-kernels-fused.cuh:381-498,
// with density_to_ray_rgba_forward (:227-264), density_to_ray_rgba_backward (:269-341)
// and the smooth-L1 helpers (:344-379). FP64.
//   ray_rgba  [4][ray_stride]  composited RGBA before the background blend
//   loss      [4][ray_stride]  per-channel smooth-L1 loss
//   dL_ddensity [sample]       gradient w.r.t. the network density output
//   dL_drgb   [3][sample_stride] gradient w.r.t. the colour output (x grad_scale)
//   n_used    [ray]            samples composited before the transmittance cut
//   ambiguous [ray]            1 when a transmittance check lies within amb_eps (relative)
//                              of min_transmittance, i.e. FP32 rounding may flip the cut
// Samples after the cut get zero gradients (the reference memsets both buffers first,
// src/core/nerf-network.cu:562-571).
// ---------------------------------------------------------------------------
void orc_recon_fwd_bwd(int64_t n_rays, int64_t ray_stride, int64_t sample_stride,
                       const uint32_t* counts, const uint32_t* offsets, int act,
                       const float* density, const float* rgb, const float* dt,
                       const float* target_rgba, const float* bg_rgb,
                       double inv_nrays, double grad_scale, double min_t, double amb_eps,
                       double* ray_rgba, double* loss, double* dL_ddensity, double* dL_drgb,
                       uint32_t* n_used, uint8_t* ambiguous, const uint32_t* fixed_used) {
    const int64_t rs = ray_stride, ss = sample_stride;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        const int64_t o = offsets[i];
        for (uint32_t j = 0; j < n; ++j) {
            dL_ddensity[o + j] = 0.0;
            dL_drgb[o + j] = dL_drgb[o + j + ss] = dL_drgb[o + j + 2 * ss] = 0.0;
        }
        // forward
        double r = 0, g = 0, bb = 0, a = 0, trans = 1.0;
        uint32_t used = 0;
        uint8_t amb = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * (double)dt[o + j]);
            const double w = trans * alpha;
            r += w * rgb[o + j];
            g += w * rgb[o + j + ss];
            bb += w * rgb[o + j + 2 * ss];
            a += w;
            trans *= (1.0 - alpha);
            ++used;
            if (std::fabs(trans - min_t) <= amb_eps * min_t) amb = 1;
            if (fixed_used ? used >= fixed_used[i] : trans < min_t) break;
        }
        n_used[i] = used;
        ambiguous[i] = amb;
        ray_rgba[i] = r; ray_rgba[i + rs] = g; ray_rgba[i + 2 * rs] = bb; ray_rgba[i + 3 * rs] = a;
        // background blend applied to the target and the prediction
        const double gt_r = target_rgba[i], gt_g = target_rgba[i + rs], gt_b = target_rgba[i + 2 * rs], gt_a = target_rgba[i + 3 * rs];
        const double br = bg_rgb[i], bgc = bg_rgb[i + rs], bbl = bg_rgb[i + 2 * rs];
        const double gt_ac = 1.0 - gt_a;
        const double gtr = gt_r * gt_a + br * gt_ac, gtg = gt_g * gt_a + bgc * gt_ac, gtb = gt_b * gt_a + bbl * gt_ac;
        const double ac = 1.0 - a;
        const double pr = r * a + br * ac, pg = g * a + bgc * ac, pb = bb * a + bbl * ac;
        const double dr = pr - gtr, dg = pg - gtg, db = pb - gtb, da = ac - gt_ac;
        loss[i] = huber_fwd(dr); loss[i + rs] = huber_fwd(dg); loss[i + 2 * rs] = huber_fwd(db); loss[i + 3 * rs] = huber_fwd(da);
        const double gR = inv_nrays * huber_bwd(dr), gG = inv_nrays * huber_bwd(dg), gB = inv_nrays * huber_bwd(db);
        // backward (same loop and cut as the forward)
        const double cdr = r - br, cdg = g - bgc, cdb = bb - bbl;
        double cr = r, cg = g, cb = bb, ca = a;
        trans = 1.0;
        for (uint32_t j = 0; j < used; ++j) {
            const double sr = rgb[o + j], sg = rgb[o + j + ss], sb = rgb[o + j + 2 * ss];
            const double sdt = dt[o + j];
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * sdt);
            const double w = trans * alpha;
            const double k = trans - w;
            cr -= w * sr; cg -= w * sg; cb -= w * sb; ca -= w;
            double dRr = sdt * (k * sr - cr), dRg = sdt * (k * sg - cg), dRb = sdt * (k * sb - cb);
            const double dRa = sdt * (k - ca);
            dRr = dRr * a + cdr * dRa;
            dRg = dRg * a + cdg * dRa;
            dRb = dRb * a + cdb * dRa;
            const double dL_dsigma = gR * dRr + gG * dRg + gB * dRb;
            dL_ddensity[o + j] = dL_dsigma * act_dsigma(act, sigma);
            const double dRc = w * a;
            dL_drgb[o + j] = grad_scale * gR * dRc;
            dL_drgb[o + j + ss] = grad_scale * gG * dRc;
            dL_drgb[o + j + 2 * ss] = grad_scale * gB * dRc;
            trans *= 1.0 - alpha;
        }
    }
}

// Smooth-L1 reconstruction loss of the same blend, RGB channels only (the alpha term is
// reported but not differentiated by the reference). Used by the finite-difference test.
double orc_recon_loss_rgb(int64_t n_rays, int64_t ray_stride, int64_t sample_stride,
                          const uint32_t* counts, const uint32_t* offsets, int act,
                          const double* density, const double* rgb, const double* dt,
                          const double* target_rgba, const double* bg_rgb,
                          double inv_nrays, double min_t, const uint32_t* fixed_used) {
    const int64_t rs = ray_stride, ss = sample_stride;
    double total = 0.0;
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        const int64_t o = offsets[i];
        double r = 0, g = 0, bb = 0, a = 0, trans = 1.0;
        for (uint32_t j = 0; j < n; ++j) {
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * dt[o + j]);
            const double w = trans * alpha;
            r += w * rgb[o + j]; g += w * rgb[o + j + ss]; bb += w * rgb[o + j + 2 * ss]; a += w;
            trans *= (1.0 - alpha);
            if (fixed_used ? (j + 1 >= fixed_used[i]) : (trans < min_t)) break;
        }
        const double gt_a = target_rgba[i + 3 * rs];
        const double br = bg_rgb[i], bgc = bg_rgb[i + rs], bbl = bg_rgb[i + 2 * rs];
        const double gtr = target_rgba[i] * gt_a + br * (1 - gt_a);
        const double gtg = target_rgba[i + rs] * gt_a + bgc * (1 - gt_a);
        const double gtb = target_rgba[i + 2 * rs] * gt_a + bbl * (1 - gt_a);
        const double pr = r * a + br * (1 - a), pg = g * a + bgc * (1 - a), pb = bb * a + bbl * (1 - a);
        total += huber_fwd(pr - gtr) + huber_fwd(pg - gtg) + huber_fwd(pb - gtb);
    }
    return inv_nrays * total;
}

// ---------------------------------------------------------------------------
// Generic compositor forward and vector-Jacobian product (FP64), the adjoint that the
// torch.autograd.Function wraps: given dL/dRGBA per ray, dL/dsigma and dL/drgb per
// sample, with the same transmittance cut as density_to_ray_rgba_forward
// (src/utils/training-kernels-fused.cuh:227-264).
// ---------------------------------------------------------------------------
// Sample counts at which an FP32 compositor may legitimately stop a ray. The reference breaks
// after the first sample whose transmittance falls below min_t
// (src/utils/training-kernels-fused.cuh:255, 337). A transmittance within a relative `band` of
// min_t is decided by rounding: FP32 and FP64 may take different sides of it. So a ray may stop
// after any sample whose transmittance lies inside the band, and at the latest after the first
// sample clearly below it (or after its last sample). For each ray this lists those counts
// (the FP64 cut among them; at most max_alt values, ascending; `overflow` counts the rays that
// had more).
int64_t orc_cut_branches(int64_t n_rays, const uint32_t* counts, const uint32_t* offsets, int act,
                         const float* density, const float* dt, double min_t, double band, int max_alt,
                         uint32_t* n_alt, uint32_t* alt) {
    int64_t overflow = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : overflow)
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        const int64_t o = offsets[i];
        uint32_t k = 0;
        bool over = false;
        auto add = [&](uint32_t u) {
            if (k > 0 && alt[i * max_alt + k - 1] == u) return;
            if ((int)k < max_alt) alt[i * max_alt + k++] = u;
            else over = true;
        };
        double trans = 1.0;
        uint32_t used = 0;
        bool stopped = false;
        for (uint32_t j = 0; j < n && !stopped; ++j) {
            const double sigma = act_sigma(act, density[o + j]);
            trans *= std::exp(-sigma * (double)dt[o + j]);
            ++used;
            if (std::fabs(trans - min_t) <= band * min_t) add(used);
            if (trans < min_t * (1.0 - band)) { add(used); stopped = true; }
        }
        if (!stopped) add(used);
        n_alt[i] = k;
        overflow += over ? 1 : 0;
    }
    return overflow;
}

void orc_composite_fwd(int64_t n_rays, int64_t ray_stride, int64_t sample_stride,
                       const uint32_t* counts, const uint32_t* offsets, int act,
                       const float* density, const float* rgb, const float* dt, double min_t,
                       double* ray_rgba, uint32_t* n_used, const uint32_t* fixed_used) {
    const int64_t rs = ray_stride, ss = sample_stride;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        const int64_t o = offsets[i];
        double r = 0, g = 0, bb = 0, a = 0, trans = 1.0;
        uint32_t used = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * (double)dt[o + j]);
            const double w = trans * alpha;
            r += w * rgb[o + j]; g += w * rgb[o + j + ss]; bb += w * rgb[o + j + 2 * ss]; a += w;
            trans *= (1.0 - alpha);
            ++used;
            if (fixed_used ? used >= fixed_used[i] : trans < min_t) break;
        }
        ray_rgba[i] = r; ray_rgba[i + rs] = g; ray_rgba[i + 2 * rs] = bb; ray_rgba[i + 3 * rs] = a;
        if (n_used) n_used[i] = used;
    }
}

void orc_composite_vjp(int64_t n_rays, int64_t ray_stride, int64_t sample_stride,
                       const uint32_t* counts, const uint32_t* offsets, int act,
                       const float* density, const float* rgb, const float* dt, double min_t,
                       const double* grad_rgba, double* dL_ddensity, double* dL_drgb, const uint32_t* fixed_used) {
    const int64_t rs = ray_stride, ss = sample_stride;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        const int64_t o = offsets[i];
        std::vector<double> w(n), T(n + 1), sig(n);
        uint32_t used = 0;
        double trans = 1.0;
        for (uint32_t j = 0; j < n; ++j) {
            sig[j] = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sig[j] * (double)dt[o + j]);
            T[j] = trans;
            w[j] = trans * alpha;
            trans *= (1.0 - alpha);
            T[j + 1] = trans;
            ++used;
            if (fixed_used ? used >= fixed_used[i] : trans < min_t) break;
        }
        const double gr = grad_rgba[i], gg = grad_rgba[i + rs], gb = grad_rgba[i + 2 * rs], ga = grad_rgba[i + 3 * rs];
        double sr = 0, sg = 0, sb = 0, sa = 0;   // suffix sums over j > current
        for (int64_t j = (int64_t)n - 1; j >= 0; --j) {
            if ((uint32_t)j >= used) {
                dL_ddensity[o + j] = 0.0;
                dL_drgb[o + j] = dL_drgb[o + j + ss] = dL_drgb[o + j + 2 * ss] = 0.0;
                continue;
            }
            const double cr = rgb[o + j], cg = rgb[o + j + ss], cb = rgb[o + j + 2 * ss];
            const double d = dt[o + j];
            const double tn = T[j + 1];
            const double ds = gr * d * (tn * cr - sr) + gg * d * (tn * cg - sg) + gb * d * (tn * cb - sb) + ga * d * (tn - sa);
            dL_ddensity[o + j] = ds * act_dsigma(act, sig[j]);
            dL_drgb[o + j] = gr * w[j];
            dL_drgb[o + j + ss] = gg * w[j];
            dL_drgb[o + j + 2 * ss] = gb * w[j];
            sr += w[j] * cr; sg += w[j] * cg; sb += w[j] * cb; sa += w[j];
        }
    }
}

// ---------------------------------------------------------------------------
// mipNeRF360_distortion_loss_forward_kernel (src/utils/training-kernels-fused.cuh:13-120)
// and _backward_kernel (:123-224), FP64. lambda replaces
// NeRFConstants::mipNeRF360_distortion_loss_lambda (src/utils/nerf-constants.cuh:17).
// grad_ray (nullable) scales each ray's gradient (the reference uses 1 for every ray).
// ---------------------------------------------------------------------------
void orc_distortion_fwd_bwd(int64_t n_rays, const uint32_t* counts, const uint32_t* offsets, int act,
                            const float* density, const float* m_norm, const float* dt_norm,
                            double lambda, const double* grad_ray,
                            double* ray_loss, double* dL_ddensity) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        if (n == 0) { ray_loss[i] = 0.0; continue; }
        const int64_t o = offsets[i];
        std::vector<double> w_cs(n), wm_cs(n);
        double cw = 0, cwm = 0, cdtw2 = 0, cwmw = 0, cwwm = 0, trans = 1, pw = 0, pwm = 0;
        double b0 = 0, b1 = 0, uni = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double d = dt_norm[o + j];
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * d);
            const double w = alpha * trans;
            const double m = m_norm[o + j];
            const double wm = w * m;
            const double a0 = wm * pw, a1 = w * pwm, a2 = d * w * w;
            cw += w; cwm += wm; cdtw2 += a2; cwmw += a0; cwwm += a1;
            w_cs[j] = cw; wm_cs[j] = cwm;
            b0 += a0; b1 += a1; uni += a2;
            pw = cw; pwm = cwm;
            trans *= (1.0 - alpha);
        }
        const double k = lambda / (double)n;
        ray_loss[i] = k * ((1.0 / 3.0) * uni + 2.0 * (b0 - b1));
        const double gscale = grad_ray ? grad_ray[i] : 1.0;
        trans = 1; pw = 0; pwm = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double d = dt_norm[o + j];
            const double sigma = act_sigma(act, density[o + j]);
            const double alpha = 1.0 - std::exp(-sigma * d);
            const double T = trans;
            const double w = alpha * T;
            const double m = m_norm[o + j];
            const double wm = w * m;
            const double wcs = w_cs[j], wmcs = wm_cs[j];
            const double dw = T * d * (1.0 - alpha);
            const double dwm = m * dw;
            const double tw = T - w;
            cw -= w; cwm -= wm; cdtw2 -= d * w * w; cwmw -= wm * pw; cwwm -= w * pwm;
            const double db0 = dwm * pw + d * (cwm * (wcs + tw) - 2.0 * cwmw);
            const double db1 = dw * pwm + d * (cw * (m * tw + wmcs) - 2.0 * cwwm);
            const double du = 2.0 * d * (d * w * tw - cdtw2);
            const double dsig = k * (2.0 * (db0 - db1) + (1.0 / 3.0) * du);
            dL_ddensity[o + j] = gscale * dsig * act_dsigma(act, sigma);
            pw = wcs; pwm = wmcs;
            trans *= (1.0 - alpha);
        }
    }
}

// Distortion loss of one batch (sum over rays of the per-ray loss), FP64, for the
// finite-difference test.
double orc_distortion_loss_sum(int64_t n_rays, const uint32_t* counts, const uint32_t* offsets, int act,
                               const double* density, const double* m_norm, const double* dt_norm,
                               double lambda) {
    double total = 0.0;
    for (int64_t i = 0; i < n_rays; ++i) {
        const uint32_t n = counts[i];
        if (n == 0) continue;
        const int64_t o = offsets[i];
        double trans = 1, pw = 0, pwm = 0, b0 = 0, b1 = 0, uni = 0, cw = 0, cwm = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const double d = dt_norm[o + j];
            const double alpha = 1.0 - std::exp(-act_sigma(act, density[o + j]) * d);
            const double w = alpha * trans;
            const double wm = w * m_norm[o + j];
            b0 += wm * pw; b1 += w * pwm; uni += d * w * w;
            cw += w; cwm += wm; pw = cw; pwm = cwm;
            trans *= (1.0 - alpha);
        }
        total += (lambda / (double)n) * ((1.0 / 3.0) * uni + 2.0 * (b0 - b1));
    }
    return total;
}

// ---------------------------------------------------------------------------
// Gradient merge, src/core/nerf-network.cu:734-758: copy_gradients_kernel<1,true>
// (src/utils/common-network-kernels.cuh:41-62) for the reconstruction and distortion
// gradients, then apply_gradient_distance_scaling_kernel
// (src/utils/training-kernels-fused.cuh:500-515). FP64.
// ---------------------------------------------------------------------------
void orc_grad_epilogue(int64_t n_samples, double loss_scale, const double* dL_rec, const double* dL_dist,
                       const float* sample_t, double* grad_out) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_samples; ++i) {
        double g = grad_out[i] + loss_scale * dL_rec[i];
        if (dL_dist) g += loss_scale * dL_dist[i];
        if (sample_t) {
            const double t = sample_t[i];
            if (t < 1.0) g *= t * t;
        }
        grad_out[i] = g;
    }
}

// ---------------------------------------------------------------------------
// Occupancy grid (FP32, bit-exact).
// generate_grid_cell_network_sample_points_kernel, src/utils/occupancy-grid-kernels.cu:38-76
// with get_voxel_xyz_from_morton_index (src/core/occupancy-grid.cuh:167-182).
// rand3 is [3][rand_stride]; out_pos is [3][pos_stride].
// ---------------------------------------------------------------------------
void orc_occupancy_sample_points(int64_t n, int res, float base, const int32_t* levels, const uint32_t* cells,
                                 const float* rand3, int64_t rand_stride, float inv_aabb,
                                 float* out_pos, int64_t pos_stride) {
    const float inv_res = 1.0f / (float)res;
    const int half_res = res / 2;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const int k = levels[i];
        const uint32_t idx = cells[i];
        const float ls = base * (float)(1 << k);
        const float vs = ls * inv_res;
        const int ix = (int)orc_morton3d_invert(idx >> 0);
        const int iy = (int)orc_morton3d_invert(idx >> 1);
        const int iz = (int)orc_morton3d_invert(idx >> 2);
        const float vx = (float)(ix - half_res) * vs;
        const float vy = (float)(iy - half_res) * vs;
        const float vz = (float)(iz - half_res) * vs;
        const float x = vx + rand3[i] * vs;
        const float y = vy + rand3[i + rand_stride] * vs;
        const float z = vz + rand3[i + 2 * rand_stride] * vs;
        out_pos[i] = (x * inv_aabb) + 0.5f;
        out_pos[i + pos_stride] = (y * inv_aabb) + 0.5f;
        out_pos[i + 2 * pos_stride] = (z * inv_aabb) + 0.5f;
    }
}

// decay_occupancy_grid_values_kernel (src/utils/occupancy-grid-kernels.cu:16-34), then
// update_occupancy_with_density_kernel (:79-115) over a list of (level, cell) updates,
// then update_occupancy_grid_bits_kernel (:118-141) and the popcount of
// src/utils/bit-utils.cuh:52-94. The sigma of each update is act(value) in FP32;
// act 1 uses expf(fminf(d,12)-1) (the reference's __expf differs in the last bits, so
// bit-exact parity is claimed for act 0 only). Duplicate (level, cell) pairs take the
// maximum of all their values. Returns the number of set bits.
uint64_t orc_occupancy_update(int n_levels, int res, float* density, uint8_t* bitfield,
                              int64_t n_updates, const int32_t* levels, const uint32_t* cells,
                              const float* values, const float* rand_select, int act,
                              int sample_all, float decay, float threshold) {
    const int64_t V = (int64_t)res * res * res;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < V * n_levels; ++c) density[c] *= decay;
    for (int64_t u = 0; u < n_updates; ++u) {
        const int k = levels[u];
        const uint32_t idx = cells[u];
        if (!sample_all) {
            const float r = rand_select[u];
            if (r > 0.5f) continue;
            if (!(r < 0.25f)) {
                if (!(bitfield[idx] & (uint8_t)(1u << k))) continue;
            }
        }
        const float sigma = act == 0 ? values[u] : std::exp(std::fmin(values[u], 12.0f) - 1.0f);
        float* p = density + (int64_t)k * V + idx;
        *p = std::fmax(sigma, *p);
    }
    uint64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int64_t c = 0; c < V; ++c) {
        uint8_t bits = 0;
        for (int k = 0; k < n_levels; ++k) {
            const uint8_t b = density[(int64_t)k * V + c] > threshold ? 1 : 0;
            bits |= (uint8_t)(b << k);
        }
        bitfield[c] = bits;
        total += (uint64_t)__builtin_popcount(bits);
    }
    return total;
}

uint64_t orc_popcount(int64_t n, const uint8_t* bytes) {
    uint64_t total = 0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int64_t i = 0; i < n; ++i) total += (uint64_t)__builtin_popcount(bytes[i]);
    return total;
}

// ---------------------------------------------------------------------------
// ngp_adam_step, src/core/adam-optimizer.cuh:48-96 (FP64). Parameters [0, n_grid) are the
// hash grid (skipped entirely when their gradient is zero), [n_grid, n_grid + n_mlp) the
// network weights (L2 applies), the rest get plain Adam. weights_copy (nullable) receives
// the low-precision copy.
// ---------------------------------------------------------------------------
void orc_adam_step(int64_t n, int64_t n_grid, int64_t n_mlp, double loss_scale, double lr,
                   double beta1, double beta2, double eps, double l2,
                   double* w, const float* grad, double* m, double* v, uint32_t* steps, double* weights_copy) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double g = (double)grad[i] / loss_scale;
        if (i < n_grid && g == 0.0) continue;
        const double wf = w[i];
        if (i >= n_grid && i < n_grid + n_mlp) g += l2 * wf;
        m[i] = beta1 * m[i] + (1.0 - beta1) * g;
        v[i] = beta2 * v[i] + (1.0 - beta2) * g * g;
        const uint32_t s = ++steps[i];
        const double lri = lr * std::sqrt(1.0 - std::pow(beta2, (double)s)) / (1.0 - std::pow(beta1, (double)s));
        const double nw = wf - (lri / (std::sqrt(v[i]) + eps)) * m[i];
        w[i] = nw;
        if (weights_copy) weights_copy[i] = nw;
    }
}

// ---------------------------------------------------------------------------
// Synthetic scene field (the stand-in for the tiny-cuda-nn network, same definition as
// the library's producer): density = sum of isotropic Gaussian blobs, rgb = sigmoid of
// three sinusoids of the world position. blobs is [n_blobs][5] = (cx, cy, cz, s, peak);
// waves is [3][4] = (ax, ay, az, phase). Positions are normalised network inputs in
// [0,1]^3 ([3][stride]); world = (pos - 0.5) * aabb_size. FP64.
// ---------------------------------------------------------------------------
static inline void blob_at(float px, float py, float pz, float aabb_size, int n_blobs, const float* blobs,
                           const float* waves, double* sigma, double* rgb, int64_t rgb_stride) {
    const double x = ((double)px - 0.5) * aabb_size;
    const double y = ((double)py - 0.5) * aabb_size;
    const double z = ((double)pz - 0.5) * aabb_size;
    double s = 0.0;
    for (int b = 0; b < n_blobs; ++b) {
        const double ddx = x - blobs[5 * b], ddy = y - blobs[5 * b + 1], ddz = z - blobs[5 * b + 2];
        const double sd = blobs[5 * b + 3];
        s += blobs[5 * b + 4] * std::exp(-(ddx * ddx + ddy * ddy + ddz * ddz) / (2.0 * sd * sd));
    }
    *sigma = s;
    if (rgb) {
        for (int c = 0; c < 3; ++c) {
            const double a = waves[4 * c] * x + waves[4 * c + 1] * y + waves[4 * c + 2] * z + waves[4 * c + 3];
            rgb[c * rgb_stride] = 1.0 / (1.0 + std::exp(-std::sin(a)));
        }
    }
}

void orc_blob_field(int64_t n, int64_t stride, const float* pos, float aabb_size,
                    int n_blobs, const float* blobs, const float* waves,
                    double* sigma_out, double* rgb_out, int64_t out_stride) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
        blob_at(pos[i], pos[i + stride], pos[i + 2 * stride], aabb_size, n_blobs, blobs, waves, sigma_out + i,
                rgb_out ? rgb_out + i : nullptr, out_stride);
}

// ---------------------------------------------------------------------------
// Inference render of one NeRF with the synthetic field as its network (the reference
// Renderer::perform_task, src/core/renderer.cu:172-646, for one NeRF with an identity
// transform), one ray at a time. Ray generation: Camera::global_ray_at_pixel_xy without
// lens distortion (src/models/camera.cuh:94-137); box clip: prepare_for_linear_
// raymarching_kernel (src/utils/rendering-kernels.cu:175-262); sample validity and network
// inputs: filter_and_localize_samples_for_nerf_kernel and assign_normalized_network_
// inputs_kernel (:336-478); compositing: accumulate_nerf_samples_kernel and
// composite_samples_kernel (:480-618); kill_terminated_rays_kernel (:620-637).
//
// Positions, steps and validity in FP32 with the reference's operation order (so the
// set of queried samples is exact); field, opacity and compositing in FP64. The reference
// marches rays in rounds of max(batch / live rays, 1) steps and drops a ray past t_max only
// after its round; this restatement stops at the first step past t_max, which gives the
// same image as long as no valid sample lies beyond t_max before the ray leaves the render
// box. Flags per pixel (ambiguous[i], OR of):
//   1  a valid sample lies past t_max inside the render box (the image then depends on
//      the round schedule);
//   2  the transmittance came within 0.1% of min_transmittance (FP32 and FP64 may end
//      the ray one sample apart);
//   4  a sample opacity came within 0.001% of the colour cut 1e-4.
// out_rgba: interleaved premultiplied RGBA. Returns the number of queried samples.
// ---------------------------------------------------------------------------
struct Camera {
    int32_t width, height;
    float near_, far_;
    float focal_x, focal_y;
    float principal_x, principal_y;
    float shift_x, shift_y;
    float transform[12];  // row-major 3 x 4 [R | t], camera to world
};

// Camera::global_ray_at_pixel_xy, src/models/camera.cuh:94-137, without lens distortion.
static inline void pinhole_ray(const Camera& cam, float x, float y, float& ox, float& oy, float& oz, float& dx,
                               float& dy, float& dz) {
    const float offx = cam.shift_x * (float)cam.width - cam.principal_x;
    const float offy = cam.shift_y * (float)cam.height - cam.principal_y;
    const float* m = cam.transform;
    const float vx = (x + offx + 0.5f) / cam.focal_x;
    const float vy = (y + offy + 0.5f) / cam.focal_y;
    const float vz = 1.0f;
    const float vlen = std::sqrt(vx * vx + vy * vy + vz * vz);
    const float gx = m[0] * vx + m[1] * vy + m[2] * vz;
    const float gy = m[4] * vx + m[5] * vy + m[6] * vz;
    const float gz = m[8] * vx + m[9] * vy + m[10] * vz;
    const float gl = std::sqrt(gx * gx + gy * gy + gz * gz);
    dx = gx / gl;
    dy = gy / gl;
    dz = gz / gl;
    ox = m[3] + cam.near_ * (vlen * dx);
    oy = m[7] + cam.near_ * (vlen * dy);
    oz = m[11] + cam.near_ * (vlen * dz);
}

int64_t orc_render(const Camera* cam, const Bbox* render_bbox, const Bbox* train_bbox, int n_levels, int res,
                   float base, const uint8_t* bits, float dt_min, float cone, double min_t, int n_blobs,
                   const float* blobs, const float* waves, float aabb_size, double* out_rgba, uint8_t* ambiguous) {
    const Grid g{n_levels, res, base, bits};
    const Bbox box = *render_bbox, tb = *train_bbox;
    const int64_t n = (int64_t)cam->width * cam->height;
    const float dt_max = 8.0f * dt_min;
    const float sx = tb.max_x - tb.min_x, sy = tb.max_y - tb.min_y, sz = tb.max_z - tb.min_z;
    const float inv_size = 1.0f / sx;
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
    for (int64_t i = 0; i < n; ++i) {
        double* o4 = out_rgba + 4 * i;
        o4[0] = o4[1] = o4[2] = o4[3] = 0.0;
        ambiguous[i] = 0;
        const uint32_t py = (uint32_t)(i / cam->width), px = (uint32_t)(i % cam->width);
        float ox, oy, oz, dx, dy, dz;
        pinhole_ray(*cam, (float)px, (float)py, ox, oy, oz, dx, dy, dz);
        const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
        float t1x = (box.min_x - ox) * ix, t2x = (box.max_x - ox) * ix;
        float t1y = (box.min_y - oy) * iy, t2y = (box.max_y - oy) * iy;
        float t1z = (box.min_z - oz) * iz, t2z = (box.max_z - oz) * iz;
        if (t1x > t2x) std::swap(t1x, t2x);
        if (t1y > t2y) std::swap(t1y, t2y);
        if (t1z > t2z) std::swap(t1z, t2z);
        const float bmin = std::fmax(t1x, std::fmax(t1y, t1z)), bmax = std::fmin(t2x, std::fmin(t2y, t2z));
        const bool volume = box.max_x > box.min_x && box.max_y > box.min_y && box.max_z > box.min_z;
        if (!(volume && bmax >= bmin)) continue;
        const float t0 = std::fmax(bmin, 1e-4f);
        ox = ox + t0 * dx;
        oy = oy + t0 * dy;
        oz = oz + t0 * dz;
        const float tmax = std::fmin(bmax, cam->far_ - cam->near_);
        const float dir_len = std::sqrt(dx * dx + dy * dy + dz * dz);
        double T = 1.0;
        float t = 0.0f;
        bool past = false;
        for (int64_t guard = 0; guard < (1 << 24); ++guard) {
            const float dt = get_dt(t, cone, dt_min, dt_max);
            const float x = ox + t * dx, y = oy + t * dy, z = oz + t * dz;
            if (past && !bbox_contains(box, x, y, z)) break;
            const float dt_net = inv_size * (dir_len * dt);
            bool valid = false;
            float u[3] = {(x - tb.min_x) / sx, (y - tb.min_y) / sy, (z - tb.min_z) / sz};
            if (bbox_contains(box, x, y, z)) {
                const int k = grid_level_at(g, x, y, z, dt_net);
                valid = is_occupied(g, k, x, y, z) && u[0] >= 0.0f && u[0] <= 1.0f && u[1] >= 0.0f &&
                        u[1] <= 1.0f && u[2] >= 0.0f && u[2] <= 1.0f;
            }
            if (valid && past) {
                ambiguous[i] |= 1;
                break;
            }
            if (valid) {
                for (int c = 0; c < 3; ++c) u[c] = clampf_ref(u[c], 0.0f, 1.0f);
                double sigma, rgb[3];
                blob_at(u[0], u[1], u[2], aabb_size, n_blobs, blobs, waves, &sigma, rgb, 1);
                ++total;
                const double alpha = -std::expm1(-sigma * (double)dt_net);
                if (std::fabs(alpha - 1e-4) <= 1e-9) ambiguous[i] |= 4;
                const double inv_a = alpha > 1e-4 ? 1.0 / alpha : 0.0;
                const double a = std::fmin(alpha, 1.0);
                const double w = a * T;
                for (int c = 0; c < 3; ++c) o4[c] += w * (rgb[c] * alpha * inv_a);
                o4[3] += w;
                T *= 1.0 - a;
                if (std::fabs(T - min_t) <= 1e-3 * min_t) ambiguous[i] |= 2;
                if (T < min_t) break;
            }
            t = t + dt;
            if (t > tmax) past = true;
        }
    }
    return total;
}

// ---------------------------------------------------------------------------
// Training rays from posed RGBA8 images: initialize_training_rays_and_pixels_kernel and
// deactivate_rays_with_alpha_threshold_kernel, src/utils/training-batch-kernels.cuh:82-208, with
// n_rays_per_image = n_rays / n_images (src/core/trainer.cu:60). random: [2][rs] (pixel draw,
// alpha-selection draw). Outputs [c][rs]; a ray that misses the box keeps alive = 0 and its other
// outputs are unspecified (the reference leaves them untouched). Returns the number of live rays.
// ---------------------------------------------------------------------------
int64_t orc_dataset_rays(int64_t n_rays, int64_t rs, int64_t n_images, int width, int height, const Camera* cameras,
                         const uint8_t* images, const Bbox* bbox, const float* random, float alpha_threshold,
                         float alpha_probability, float* pix_rgba, uint32_t* img_id, float* ori, float* dir,
                         float* ray_t, float* ray_t_max, uint8_t* alive) {
    const uint32_t n_pixels = (uint32_t)width * (uint32_t)height;
    const float rays_per_image = (float)n_rays / (float)n_images;
    const bool selection = alpha_threshold < 1.0f && alpha_probability < 1.0f;
    const Bbox b = *bbox;
    int64_t live = 0;
#pragma omp parallel for schedule(static) reduction(+ : live)
    for (int64_t i = 0; i < n_rays; ++i) {
        alive[i] = 0;
        const uint32_t image = std::min((uint32_t)((float)i / rays_per_image), (uint32_t)n_images - 1u);
        const float p = (float)n_pixels * random[i];
        const float w = (float)width;
        const float x = std::fmod(p, w), y = p / w;
        float ox, oy, oz, dx, dy, dz;
        pinhole_ray(cameras[image], x, y, ox, oy, oz, dx, dy, dz);
        const float ix = 1.0f / dx, iy = 1.0f / dy, iz = 1.0f / dz;
        float t1x = (b.min_x - ox) * ix, t2x = (b.max_x - ox) * ix;
        float t1y = (b.min_y - oy) * iy, t2y = (b.max_y - oy) * iy;
        float t1z = (b.min_z - oz) * iz, t2z = (b.max_z - oz) * iz;
        if (t1x > t2x) std::swap(t1x, t2x);
        if (t1y > t2y) std::swap(t1y, t2y);
        if (t1z > t2z) std::swap(t1z, t2z);
        const float tmin = std::fmax(t1x, std::fmax(t1y, t1z)), tmax = std::fmin(t2x, std::fmin(t2y, t2z));
        if (!(tmax >= tmin)) continue;
        const Camera& cam = cameras[image];
        const float t_max = std::fmin(cam.far_ - cam.near_, tmax);
        const float t = std::fmax(0.0f, tmin + 1e-5f);
        if (t_max < t) continue;
        const size_t k = std::min((size_t)p, (size_t)n_pixels - 1);
        const uint8_t* px = images + 4 * ((size_t)n_pixels * image + k);
        const float rgba[4] = {(float)px[0] / 255.0f, (float)px[1] / 255.0f, (float)px[2] / 255.0f,
                               (float)px[3] / 255.0f};
        for (int c = 0; c < 4; ++c) pix_rgba[i + c * rs] = rgba[c];
        ori[i] = ox; ori[i + rs] = oy; ori[i + 2 * rs] = oz;
        dir[i] = dx; dir[i + rs] = dy; dir[i + 2 * rs] = dz;
        ray_t[i] = t;
        ray_t_max[i] = t_max;
        img_id[i] = image;
        if (selection && rgba[3] < alpha_threshold && random[i + rs] > alpha_probability) continue;
        alive[i] = 1;
        ++live;
    }
    return live;
}


// ---- hash-grid encoding and the linear heads (the tiny-cuda-nn boundary) -------------------
// tcnn's HashGrid is not in the reference tree (the submodule is empty); this is the published
// multiresolution hash encoding (Mueller et al. 2022, section 3) with the reference's settings
// (src/core/nerf-network.cu:27-124): level l of resolution res[l] maps x in [0,1] to the cell
// floor(x res) (clamped to [0, res - 1]) and f = x res - cell; the 8 corners' weights are
// ((w_x w_y) w_z) with w = f or 1 - f (bit 0: x + 1, bit 1: y + 1, bit 2: z + 1); a level whose
// (res + 1)^3 vertices fit in its 2^log2_t entries indexes them directly (x + (res + 1) (y +
// (res + 1) z)), the others by (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod 2^log2_t. The
// forward is FP32 in the same operation order as the library (features bit for bit), with the
// corners' products summed by fused multiply-adds in corner order; the backward is FP64.
static inline uint32_t orc_hg_index(uint32_t res, int dense, int log2_t, uint32_t x, uint32_t y, uint32_t z) {
    if (dense) {
        const uint32_t r = res + 1u;
        return x + r * (y + r * z);
    }
    return ((x * 1u) ^ (y * 2654435761u) ^ (z * 805459861u)) & ((1u << log2_t) - 1u);
}

static inline void orc_hg_corners(uint32_t res, int dense, int log2_t, float px, float py, float pz,
                                  uint32_t idx[8], float w[8]) {
    const float p[3] = {px, py, pz};
    uint32_t i[3];
    float f[3], g[3];
    for (int d = 0; d < 3; ++d) {
        const float s = p[d] * (float)res;
        const float fl = std::fmin(std::fmax(std::floor(s), 0.0f), (float)(res - 1u));
        i[d] = (uint32_t)fl;
        f[d] = s - fl;
        g[d] = 1.0f - f[d];
    }
    for (int k = 0; k < 8; ++k) {
        const int bx = k & 1, by = (k >> 1) & 1, bz = (k >> 2) & 1;
        idx[k] = orc_hg_index(res, dense, log2_t, i[0] + bx, i[1] + by, i[2] + bz);
        const float wxy = (bx ? f[0] : g[0]) * (by ? f[1] : g[1]);
        w[k] = wxy * (bz ? f[2] : g[2]);
    }
}

// feat[2 l + c][stride] for n positions pos[3][pstride]; params [L][2^log2_t][2].
void orc_hashgrid_encode(int n_levels, int log2_t, const uint32_t* res, const int* dense, int64_t n, int64_t pstride,
                         int64_t stride, const float* pos, const float* params, float* feat) {
    const size_t T = (size_t)1 << log2_t;
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < n; ++s) {
        for (int l = 0; l < n_levels; ++l) {
            uint32_t idx[8];
            float w[8];
            orc_hg_corners(res[l], dense[l], log2_t, pos[s], pos[s + pstride], pos[s + 2 * pstride], idx, w);
            const float* P = params + (size_t)l * T * 2;
            float a0 = 0.0f, a1 = 0.0f;
            for (int k = 0; k < 8; ++k) {
                a0 = std::fmaf(w[k], P[2 * (size_t)idx[k]], a0);
                a1 = std::fmaf(w[k], P[2 * (size_t)idx[k] + 1], a1);
            }
            feat[(size_t)(2 * l) * stride + s] = a0;
            feat[(size_t)(2 * l + 1) * stride + s] = a1;
        }
    }
}

// grads[l][entry][c] += w_k dfeat[2 l + c][s] over every live sample and corner (FP64, serial);
// touched[l 2^log2_t + entry] = 1 for every entry a sample touches.
void orc_hashgrid_backward(int n_levels, int log2_t, const uint32_t* res, const int* dense, int64_t n,
                           int64_t pstride, int64_t stride, const float* pos, const double* dfeat, double* grads,
                           uint8_t* touched) {
    const size_t T = (size_t)1 << log2_t;
    for (int64_t s = 0; s < n; ++s) {
        for (int l = 0; l < n_levels; ++l) {
            uint32_t idx[8];
            float w[8];
            orc_hg_corners(res[l], dense[l], log2_t, pos[s], pos[s + pstride], pos[s + 2 * pstride], idx, w);
            const double g0 = dfeat[(size_t)(2 * l) * stride + s], g1 = dfeat[(size_t)(2 * l + 1) * stride + s];
            for (int k = 0; k < 8; ++k) {
                const size_t e = (size_t)l * T + idx[k];
                grads[2 * e] += (double)w[k] * g0;
                grads[2 * e + 1] += (double)w[k] * g1;
                if (touched) touched[e] = 1;
            }
        }
    }
}

// Linear heads (FP64): z_o = b_o + W_o . f over nf features ([nf][stride]); head parameters
// [4][nf + 1] (weights, then the bias): density = z_0, rgb_c = sigmoid(z_{c+1}).
void orc_hash_heads_forward(int nf, int64_t n, int64_t stride, const float* feat, const float* head, double* density,
                            double* rgb, int64_t ostride) {
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < n; ++s) {
        for (int o = 0; o < 4; ++o) {
            double z = head[o * (nf + 1) + nf];
            for (int j = 0; j < nf; ++j) z += (double)head[o * (nf + 1) + j] * (double)feat[(size_t)j * stride + s];
            if (o == 0) density[s] = z;
            else if (rgb) rgb[(size_t)(o - 1) * ostride + s] = 1.0 / (1.0 + std::exp(-z));
        }
    }
}

// The heads' backward (FP64): dfeat[nf][stride] and the head parameters' gradients [4][nf + 1]
// (summed over the n samples) from dL/d density and dL/d rgb ([3][stride]).
void orc_hash_heads_backward(int nf, int64_t n, int64_t stride, const float* feat, const float* head,
                             const double* dL_ddensity, const double* dL_drgb, double* dfeat, double* dhead) {
    for (int k = 0; k < 4 * (nf + 1); ++k) dhead[k] = 0.0;
    for (int64_t s = 0; s < n; ++s) {
        double dz[4];
        dz[0] = dL_ddensity[s];
        for (int c = 0; c < 3; ++c) {
            double z = head[(c + 1) * (nf + 1) + nf];
            for (int j = 0; j < nf; ++j)
                z += (double)head[(c + 1) * (nf + 1) + j] * (double)feat[(size_t)j * stride + s];
            const double y = 1.0 / (1.0 + std::exp(-z));
            dz[c + 1] = dL_drgb[(size_t)c * stride + s] * y * (1.0 - y);
        }
        for (int j = 0; j < nf; ++j) {
            double g = 0.0;
            for (int o = 0; o < 4; ++o) g += dz[o] * (double)head[o * (nf + 1) + j];
            dfeat[(size_t)j * stride + s] = g;
        }
        for (int o = 0; o < 4; ++o) {
            for (int j = 0; j < nf; ++j) dhead[o * (nf + 1) + j] += dz[o] * (double)feat[(size_t)j * stride + s];
            dhead[o * (nf + 1) + nf] += dz[o];
        }
    }
}

}  // extern "C"
