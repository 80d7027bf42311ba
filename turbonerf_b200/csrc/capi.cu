// Context, error reporting and scratch management of the turbo_hot C ABI.
#include <initializer_list>

#include "tn_internal.cuh"

namespace tn {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return TN_OK;
    return fail(TN_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_launch(const char* what) { return cuda_status(cudaGetLastError(), what); }

bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return false;
    return st != cudaStreamCaptureStatusNone;
}

int allow_optin_smem(const void* func) {
    cudaFuncAttributes fa;
    int dev = 0, optin = 0;
    cudaError_t e = cudaFuncGetAttributes(&fa, func);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    return cuda_status(e, "shared memory opt-in");
}

size_t exclusive_smem() {
    static size_t cached = 0;
    if (cached == 0) {
        int dev = 0, per_sm = 0, reserved = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
        // two blocks would need 2 * (excl + reserved) > per_sm
        cached = (size_t)(per_sm - 2 * reserved) / 2 + 1024;
    }
    return cached;
}

int num_sms() {
    static int cached = 0;
    if (cached == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
        if (cached <= 0) cached = 148;
    }
    return cached;
}

template <typename T>
static int ensure(T*& ptr, size_t& cap, size_t n, const char* what) {
    if (n <= cap) return TN_OK;
    size_t want = cap ? cap : 1024;
    while (want < n) want *= 2;
    T* fresh = nullptr;
    cudaError_t e = cudaMalloc(&fresh, want * sizeof(T));
    if (e != cudaSuccess) return fail(TN_E_CUDA, "%s: cudaMalloc(%zu) failed: %s (reserve scratch with tn_ctx_reserve "
                                      "before capturing a graph)", what, want * sizeof(T), cudaGetErrorString(e));
    cudaMemset(fresh, 0, want * sizeof(T));
    if (ptr) cudaFree(ptr);
    ptr = fresh;
    cap = want;
    return TN_OK;
}

int ensure_block_u32(tn_ctx* ctx, size_t n) { return ensure(ctx->block_u32, ctx->block_u32_cap, n, "scratch(u32)"); }
int ensure_block_f32(tn_ctx* ctx, size_t n) { return ensure(ctx->block_f32, ctx->block_f32_cap, n, "scratch(f32)"); }
int ensure_mip(tn_ctx* ctx, size_t bytes) { return ensure(ctx->mip, ctx->mip_cap, bytes, "scratch(mip)"); }
int ensure_slots(tn_ctx* ctx, size_t n) { return ensure(ctx->slots, ctx->slots_cap, n, "scratch(slots)"); }
int ensure_render_ws(tn_ctx* ctx, size_t bytes) { return ensure(ctx->render_ws, ctx->render_ws_cap, bytes, "scratch(render)"); }

int validate_grid(const tn_grid_desc* grid) {
    TN_REQUIRE(grid != nullptr, TN_E_NULL, "grid descriptor is NULL");
    TN_REQUIRE(grid->n_levels >= 1 && grid->n_levels <= 8, TN_E_LEVELS, "n_levels = %d outside 1..8", grid->n_levels);
    const int r = grid->resolution;
    TN_REQUIRE(r >= 2 && r <= 1024 && (r & (r - 1)) == 0, TN_E_INVALID, "resolution %d must be a power of two in 2..1024", r);
    TN_REQUIRE(grid->base_size > 0.0f, TN_E_INVALID, "base_size must be positive");
    return TN_OK;
}

}  // namespace tn

using namespace tn;

extern "C" {

int tn_version(void) { return 1; }

const char* tn_last_error(void) { return g_last_error.c_str(); }

int tn_ctx_create(tn_ctx** out) {
    TN_NONNULL(out);
    *out = nullptr;
    tn_ctx* ctx = new tn_ctx();
    cudaGetDevice(&ctx->device);
    int st = cuda_status(cudaMalloc(&ctx->flags, sizeof(uint32_t)), "tn_ctx_create flags");
    if (st == TN_OK) st = cuda_status(cudaMalloc(&ctx->tickets, TICKET_COUNT * sizeof(uint32_t)), "tn_ctx_create tickets");
    if (st == TN_OK) st = cuda_status(cudaMemset(ctx->flags, 0, sizeof(uint32_t)), "tn_ctx_create memset");
    if (st == TN_OK) st = cuda_status(cudaMemset(ctx->tickets, 0, TICKET_COUNT * sizeof(uint32_t)), "tn_ctx_create memset");
    if (st == TN_OK) st = ensure_block_u32(ctx, 4096);
    if (st == TN_OK) st = ensure_block_f32(ctx, 4096);
    if (st == TN_OK) st = cuda_status(cudaDeviceSynchronize(), "tn_ctx_create sync");
    if (st != TN_OK) {
        tn_ctx_destroy(ctx);
        return st;
    }
    *out = ctx;
    return TN_OK;
}

int tn_ctx_destroy(tn_ctx* ctx) {
    if (!ctx) return TN_OK;
    cudaFree(ctx->flags);
    cudaFree(ctx->tickets);
    cudaFree(ctx->block_u32);
    cudaFree(ctx->block_f32);
    cudaFree(ctx->mip);
    cudaFree(ctx->slots);
    cudaFree(ctx->render_ws);
    delete ctx;
    return TN_OK;
}

int tn_ctx_reserve(tn_ctx* ctx, uint32_t max_rays, uint32_t max_samples) {
    TN_NONNULL(ctx);
    // One u32 per count block (32 rays at the smallest tuned size) plus per-block float partials.
    const size_t blocks = (size_t)max_rays / 32 + (size_t)max_samples / 1024 + 1024;
    int st = ensure_block_u32(ctx, 2 * blocks);
    if (st == TN_OK) st = ensure_block_f32(ctx, 8 * blocks);
    // march scratch: the 128^3 coarse mip with its occupied boxes and 8 bit-planes (33,024 B +
    // 8 x 256 KiB), and the step-position slots (16 Mi floats at most)
    if (st == TN_OK) st = ensure_mip(ctx, 33024u + 8u * 262144u);
    if (st == TN_OK && max_rays) {
        size_t per = (16u << 20) / max_rays;
        if (per > 1024) per = 1024;
        if (per < 16) per = 16;
        st = ensure_slots(ctx, per * max_rays);
    }
    if (st == TN_OK) st = cuda_status(cudaDeviceSynchronize(), "tn_ctx_reserve");
    return st;
}

int tn_ctx_check(tn_ctx* ctx, tn_stream_t stream, uint32_t* flags_out) {
    TN_NONNULL(ctx);
    uint32_t h = 0;
    int st = cuda_status(cudaMemcpyAsync(&h, ctx->flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream), "tn_ctx_check");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(stream), "tn_ctx_check sync");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(ctx->flags, 0, sizeof(uint32_t), stream), "tn_ctx_check clear");
    if (flags_out) *flags_out = h;
    return st;
}

int tn_ctx_flags_ptr(tn_ctx* ctx, uint32_t** flags_dev) {
    TN_NONNULL(ctx);
    TN_NONNULL(flags_dev);
    *flags_dev = ctx->flags;
    return TN_OK;
}

}  // extern "C"

extern "C" {

void tn_tuning_default(tn_tuning* out) {
    if (out) *out = tn_tuning{64, 8, 1, 4, 128, 64, 0};
}

static bool one_of(uint32_t v, std::initializer_list<uint32_t> allowed) {
    for (uint32_t a : allowed)
        if (v == a) return true;
    return false;
}

int tn_tuning_validate(const tn_tuning* t) {
    TN_NONNULL(t);
    TN_REQUIRE(one_of(t->count_rays_per_block, {32, 64, 128, 256}), TN_E_INVALID,
               "tuning: count_rays_per_block %u not in {32, 64, 128, 256}", t->count_rays_per_block);
    TN_REQUIRE(one_of(t->emit_warps_per_block, {1, 2, 4, 8, 16}), TN_E_INVALID,
               "tuning: emit_warps_per_block %u not in {1, 2, 4, 8, 16}", t->emit_warps_per_block);
    TN_REQUIRE(one_of(t->emit_rays_per_warp, {1, 2, 4}), TN_E_INVALID,
               "tuning: emit_rays_per_warp %u not in {1, 2, 4}", t->emit_rays_per_warp);
    TN_REQUIRE(one_of(t->loss_rays_per_block, {2, 4, 8}), TN_E_INVALID,
               "tuning: loss_rays_per_block %u not in {2, 4, 8}", t->loss_rays_per_block);
    TN_REQUIRE(one_of(t->compact_tile, {128, 256, 512, 1024, 2048}), TN_E_INVALID,
               "tuning: compact_tile %u not in {128, 256, 512, 1024, 2048}", t->compact_tile);
    TN_REQUIRE(one_of(t->multi_chunk_rays, {32, 64, 128, 256}), TN_E_INVALID,
               "tuning: multi_chunk_rays %u not in {32, 64, 128, 256}", t->multi_chunk_rays);
    TN_REQUIRE(t->side_sms < 1024u, TN_E_INVALID, "tuning: side_sms %u not below 1024", t->side_sms);
    return TN_OK;
}

int tn_ctx_set_tuning(tn_ctx* ctx, const tn_tuning* t) {
    TN_NONNULL(ctx);
    const int st = tn_tuning_validate(t);
    if (st != TN_OK) return st;
    TN_REQUIRE(t->side_sms < (uint32_t)num_sms(), TN_E_INVALID, "tuning: side_sms %u leaves no SM of %d", t->side_sms,
               num_sms());
    ctx->tune = *t;
    return TN_OK;
}

int tn_ctx_get_tuning(tn_ctx* ctx, tn_tuning* out) {
    TN_NONNULL(ctx);
    TN_NONNULL(out);
    *out = ctx->tune;
    return TN_OK;
}

}  // extern "C"
