// Autotuner of the hot path's launch shapes (tn_tuning). Every shape only changes how a stage's
// work is split over blocks, warps and lanes, so the tuner can try them all on the caller's own
// inputs: per candidate, one warm-up call and TUNE_REPS timed calls (CUDA events on the caller's
// stream around each call), the median kept. The fastest candidate replaces the context's
// current shape only when it is faster by more than the noise margin. Each tuner ends by running
// its stage once more with the chosen shape, so its outputs are those of one ordinary call.
//
// The reference has no counterpart: its kernels run with fixed shapes (tiny-cuda-nn's
// linear_kernel launches).
#include <algorithm>
#include <vector>

#include "tn_internal.cuh"

namespace tn {
namespace {

constexpr int TUNE_REPS = 7;
// a candidate replaces the current shape only when its median is below this fraction of it
constexpr float TUNE_MARGIN = 0.98f;

constexpr uint32_t COUNT_CANDIDATES[] = {32, 64, 128, 256};
constexpr uint32_t EMIT_WARPS[] = {1, 2, 4, 8, 16};
constexpr uint32_t EMIT_RPW[] = {1, 2, 4};
constexpr uint32_t LOSS_CANDIDATES[] = {2, 4, 8};
constexpr uint32_t COMPACT_CANDIDATES[] = {128, 256, 512, 1024, 2048};
constexpr int N_EMIT = 15;

struct Events {
    cudaEvent_t e[2 * TUNE_REPS] = {};
    int status = TN_OK;
    Events() {
        for (auto& x : e)
            if (status == TN_OK) status = cuda_status(cudaEventCreate(&x), "autotune: event");
    }
    ~Events() {
        for (auto x : e)
            if (x) cudaEventDestroy(x);
    }
};

// Median time (ms) of one call of run(): a warm-up call, then TUNE_REPS calls, each after pre()
// (which is not timed).
template <class Pre, class Run>
int median_ms(cudaStream_t s, Pre& pre, Run& run, float* ms) {
    Events ev;
    if (ev.status != TN_OK) return ev.status;
    int st = pre();
    if (st == TN_OK) st = run();
    for (int r = 0; r < TUNE_REPS && st == TN_OK; ++r) {
        st = pre();
        if (st == TN_OK) st = cuda_status(cudaEventRecord(ev.e[2 * r], s), "autotune: record");
        if (st == TN_OK) st = run();
        if (st == TN_OK) st = cuda_status(cudaEventRecord(ev.e[2 * r + 1], s), "autotune: record");
    }
    if (st != TN_OK) return st;
    st = cuda_status(cudaStreamSynchronize(s), "autotune: sync");
    if (st != TN_OK) return st;
    float t[TUNE_REPS];
    for (int r = 0; r < TUNE_REPS; ++r) {
        st = cuda_status(cudaEventElapsedTime(&t[r], ev.e[2 * r], ev.e[2 * r + 1]), "autotune: elapsed");
        if (st != TN_OK) return st;
    }
    std::sort(t, t + TUNE_REPS);
    *ms = t[TUNE_REPS / 2];
    return TN_OK;
}

// Times the n candidates (apply(c) installs candidate c in the context) and installs the
// chosen one: the fastest, unless the current one (index cur, -1 when it is not a candidate)
// is within the margin.
template <class Apply, class Pre, class Run>
int pick(cudaStream_t s, int n, int cur, Apply&& apply, Pre&& pre, Run&& run, tn_tune_report* rep) {
    std::vector<float> t(n);
    for (int c = 0; c < n; ++c) {
        apply(c);
        const int st = median_ms(s, pre, run, &t[c]);
        if (st != TN_OK) {
            if (cur >= 0) apply(cur);
            return st;
        }
    }
    int fastest = 0;
    for (int c = 1; c < n; ++c)
        if (t[c] < t[fastest]) fastest = c;
    const int chosen = (cur >= 0 && !(t[fastest] < TUNE_MARGIN * t[cur])) ? cur : fastest;
    apply(chosen);
    if (rep) {
        rep->n_candidates = (uint32_t)n;
        rep->before_ms = t[cur >= 0 ? cur : chosen];
        rep->best_ms = t[chosen];
    }
    return TN_OK;
}

template <size_t N>
int index_of(const uint32_t (&list)[N], uint32_t v) {
    for (size_t i = 0; i < N; ++i)
        if (list[i] == v) return (int)i;
    return -1;
}

int emit_index(const tn_tuning& t) {
    const int w = index_of(EMIT_WARPS, t.emit_warps_per_block), r = index_of(EMIT_RPW, t.emit_rays_per_warp);
    return (w < 0 || r < 0) ? -1 : w * 3 + r;
}

void set_emit(tn_ctx* ctx, int c) {
    ctx->tune.emit_warps_per_block = EMIT_WARPS[c / 3];
    ctx->tune.emit_rays_per_warp = EMIT_RPW[c % 3];
}

int no_pre() { return TN_OK; }

int not_capturing(cudaStream_t s, const char* who) {
    TN_REQUIRE(!stream_capturing(s), TN_E_STATE, "%s: the stream is being captured (tune before capture)", who);
    return TN_OK;
}

}  // namespace
}  // namespace tn

using namespace tn;

extern "C" {

int tn_autotune_march(tn_ctx* ctx, tn_stream_t stream, const tn_grid_desc* grid, const uint8_t* bitfield,
                      const tn_bbox* bbox, const tn_march_desc* march, float inv_aabb_size, uint32_t n_rays,
                      uint32_t ray_stride, const uint32_t* ray_img_id, const float* ori, const float* dir,
                      const float* ray_t, const float* ray_t_max, uint8_t* alive, uint32_t* n_steps,
                      uint32_t batch_size, uint32_t* batch_info, uint32_t sample_stride, uint32_t* offsets,
                      uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                      float* out_m_norm, float* out_dt_norm, tn_tune_report* count_report,
                      tn_tune_report* emit_report) {
    TN_NONNULL(ctx);
    int st = not_capturing(stream, "tn_autotune_march");
    if (st != TN_OK) return st;
    auto count = [&] {
        return tn_march_count(ctx, stream, grid, bitfield, bbox, march, n_rays, ray_stride, nullptr, ori, dir, ray_t,
                              ray_t_max, alive, n_steps, batch_size, batch_info);
    };
    auto emit = [&] {
        return tn_march_emit(ctx, stream, grid, bitfield, bbox, march, inv_aabb_size, n_rays, ray_stride,
                             sample_stride, batch_info, ray_img_id, ori, dir, ray_t, alive, n_steps, offsets,
                             out_img_id, out_t, out_pos, out_dir, out_dt, out_m_norm, out_dt_norm);
    };
    // With SMs kept aside, count blocks hold an SM each: only block sizes whose blocks all fit
    // on the remaining SMs at once are candidates.
    std::vector<uint32_t> cands;
    for (uint32_t c : COUNT_CANDIDATES)
        if (!ctx->tune.side_sms || (n_rays + c - 1) / c <= (uint32_t)num_sms() - ctx->tune.side_sms)
            cands.push_back(c);
    if (cands.empty()) cands.push_back(COUNT_CANDIDATES[3]);
    int cur = -1;
    for (size_t i = 0; i < cands.size(); ++i)
        if (cands[i] == ctx->tune.count_rays_per_block) cur = (int)i;
    // the count modifies only `alive`, and only to clear rays without samples: calling it again
    // gives the same outputs
    st = pick(stream, (int)cands.size(), cur, [&](int c) { ctx->tune.count_rays_per_block = cands[c]; }, no_pre,
              count, count_report);
    if (st == TN_OK) st = count();  // the emit candidates read this count's block prefixes
    if (st == TN_OK)
        st = pick(stream, N_EMIT, emit_index(ctx->tune), [&](int c) { set_emit(ctx, c); }, no_pre, emit,
                  emit_report);
    if (st == TN_OK) st = emit();
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_autotune_march");
    return st;
}

int tn_autotune_multi(tn_ctx* ctx, tn_stream_t stream, uint32_t n_scenes, const tn_scene* scenes,
                      uint32_t ray_stride, const uint32_t* ray_img_id, const float* ori, const float* dir,
                      const float* ray_t, const float* ray_t_max, uint8_t* alive, uint32_t* n_steps,
                      uint32_t* scene_samples, uint32_t* batch_info, uint32_t sample_stride, uint32_t* offsets,
                      uint32_t* out_img_id, float* out_t, float* out_pos, float* out_dir, float* out_dt,
                      float* out_m_norm, float* out_dt_norm, tn_tune_report* count_report,
                      tn_tune_report* emit_report) {
    TN_NONNULL(ctx);
    int st = not_capturing(stream, "tn_autotune_multi");
    if (st != TN_OK) return st;
    auto count = [&] {
        return tn_multi_march_count(ctx, stream, n_scenes, scenes, ray_stride, ori, dir, ray_t, ray_t_max, alive,
                                    n_steps, scene_samples, batch_info);
    };
    auto emit = [&] {
        return tn_multi_march_emit(ctx, stream, n_scenes, scenes, ray_stride, sample_stride, ray_img_id, ori, dir,
                                   ray_t, alive, n_steps, offsets, out_img_id, out_t, out_pos, out_dir, out_dt,
                                   out_m_norm, out_dt_norm);
    };
    st = pick(stream, 4, index_of(COUNT_CANDIDATES, ctx->tune.multi_chunk_rays),
              [&](int c) { ctx->tune.multi_chunk_rays = COUNT_CANDIDATES[c]; }, no_pre, count, count_report);
    if (st == TN_OK) st = count();
    if (st == TN_OK)
        st = pick(stream, N_EMIT, emit_index(ctx->tune), [&](int c) { set_emit(ctx, c); }, no_pre, emit,
                  emit_report);
    if (st == TN_OK) st = emit();
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_autotune_multi");
    return st;
}

int tn_autotune_losses(tn_ctx* ctx, tn_stream_t stream, const tn_ray_batch* batch, int activation,
                       float min_transmittance, float inv_nrays, const uint32_t* inv_nrays_from_dev,
                       float grad_scale, float lambda, const float* density, const float* rgb, const float* dt,
                       const float* m_norm, const float* dt_norm, const float* t, const float* target_rgba,
                       const float* bg_rgb, float* ray_rgba, float* grad_density, float* dL_drgb, float* loss_sums,
                       tn_tune_report* report) {
    TN_NONNULL(ctx);
    TN_NONNULL(batch);
    TN_NONNULL(grad_density);
    int st = not_capturing(stream, "tn_autotune_losses");
    if (st != TN_OK) return st;
    // grad_density is accumulated into: every call starts from the caller's values
    const size_t bytes = (size_t)batch->sample_stride * sizeof(float);
    float* saved = nullptr;
    st = cuda_status(cudaMalloc(&saved, bytes ? bytes : 4), "tn_autotune_losses: scratch");
    if (st != TN_OK) return st;
    st = cuda_status(cudaMemcpyAsync(saved, grad_density, bytes, cudaMemcpyDeviceToDevice, stream),
                     "tn_autotune_losses: save");
    auto restore = [&] {
        return cuda_status(cudaMemcpyAsync(grad_density, saved, bytes, cudaMemcpyDeviceToDevice, stream),
                           "tn_autotune_losses: restore");
    };
    auto run = [&] {
        return tn_train_losses(ctx, stream, batch, activation, min_transmittance, inv_nrays, inv_nrays_from_dev,
                               grad_scale, lambda, density, rgb, dt, m_norm, dt_norm, t, target_rgba, bg_rgb,
                               ray_rgba, grad_density, dL_drgb, loss_sums);
    };
    if (st == TN_OK)
        st = pick(stream, 3, index_of(LOSS_CANDIDATES, ctx->tune.loss_rays_per_block),
                  [&](int c) { ctx->tune.loss_rays_per_block = LOSS_CANDIDATES[c]; }, restore, run, report);
    if (st == TN_OK) st = restore();
    if (st == TN_OK) st = run();
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_autotune_losses");
    cudaStreamSynchronize(stream);
    cudaFree(saved);
    return st;
}

int tn_autotune_compact(tn_ctx* ctx, tn_stream_t stream, uint32_t n, const uint32_t* values, int32_t* out,
                        uint32_t* count_dev, tn_tune_report* report) {
    TN_NONNULL(ctx);
    int st = not_capturing(stream, "tn_autotune_compact");
    if (st != TN_OK) return st;
    auto run = [&] { return tn_compact_nonzero(ctx, stream, n, values, out, count_dev); };
    st = pick(stream, 5, index_of(COMPACT_CANDIDATES, ctx->tune.compact_tile),
              [&](int c) { ctx->tune.compact_tile = COMPACT_CANDIDATES[c]; }, no_pre, run, report);
    if (st == TN_OK) st = run();
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_autotune_compact");
    return st;
}

}  // extern "C"
