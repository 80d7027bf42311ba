// Training-step controller (reference NeRFTrainingController + Trainer,
// src/controllers/nerf-training-controller.cu:27-226, src/core/trainer.cu:39-349).
//
// One step = rays -> march count + device batch cut -> march emit -> network forward ->
// reconstruction + distortion losses with the gradient merge -> network backward ->
// [occupancy re-sampling of random cells] -> Adam.
//
// Count-ahead schedule (tn_tuning side_sms > 0, the trainer's default when the SMs allow it):
// a step is split into its head (the rays and the march count with the batch cut) and its tail
// (emit, network forward, losses, network backward, Adam, and the step's occupancy update).
// The march count is bound by the latency of its longest ray (a dependent chain of a few
// hundred steps), not by bandwidth, and fills only part of the GPU; so each step's tail runs
// beside the next step's head: the next step's rays and count start at once, on
// count_rays_per_block-ray blocks that each hold an SM alone (see exclusive_smem), while Adam
// runs on the other side_sms SMs. The count must see the bitfield of this step's occupancy
// update, as in the reference's order; the tail before this one computed it already, once the
// grid had settled and this step's occupancy query was made: the update leaves every cell at
// max(decay * density, the values of its selected queries), so its bits are the decayed grid
// against the threshold with the selected queried cells above it or-ed in (exact, as a
// comparison of the same products). The update itself then only writes the densities back.
// The first tail of a run (no tail before it) rebuilds the bitfield first and starts the
// count after it. The two steps in flight use two
// sets of ray buffers and two march contexts (slots, per-block scan totals, error word). Every
// step computes what the in-order schedule computes, bit for bit: the head of step N+1 reads
// only its own rays and the grid after step N's update, and the tail of step N reads only its
// own set. A head computed ahead for the trainer's own rays is dropped when anything it read
// changes (grid, dataset, launch shapes, a load or reset); a head of caller rays (the
// pipelined caller-ray call) is completed by its tail before the trainer's state is read.
//
// Fused path: every stage is one of the library's fused kernels; every step-dependent
// scalar (step index, learning rate, occupancy selection policy, ray and sample counts)
// lives in device memory, so the whole step is captured once into a CUDA graph and
// replayed without any host synchronisation.
// Plain path: the reference's launch structure (thrust scans, blocking device->host reads of
// the sample count and the losses, separate memsets and epilogue kernels, dense Adam).
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "tn_internal.cuh"

namespace tn {

struct StepState {
    unsigned long long samples_total;  // samples processed by all steps so far
    unsigned long long rays_total;     // rays used by all steps so far
    uint32_t step_count;   // started steps; also the key of the next step's rays
    uint32_t cur_step;     // index of the running step
    float lr;              // decayed learning rate of the running step
    uint32_t sample_all;   // occupancy selection policy: 1 while cur_step < 256
    uint32_t batch_info[4];  // batch cut of the last completed step
    uint32_t n_occupied;
    float loss_sums[2];
    uint32_t err;          // error bits of the completed steps not yet read (TN_FLAG_*)
    uint32_t next_sample_all;  // the selection policy of the step after the running one
    uint32_t pad[2];
};

// End of a step's tail: its batch cut becomes the state's, the totals grow, and the error bits
// of the step's march context move into the state (the context's word is left clear for the
// head that will use it next).
__global__ void step_end_kernel(StepState* s, const uint32_t* __restrict__ info, uint32_t* ctx_flags) {
    for (int k = 0; k < 4; ++k) s->batch_info[k] = info[k];
    s->samples_total += info[1];
    s->rays_total += info[0];
    s->err |= *ctx_flags;
    *ctx_flags = 0u;
}

__global__ void step_begin_kernel(StepState* s, float base_lr, float lr_decay) {
    const uint32_t k = s->step_count;
    s->cur_step = k;
    s->lr = base_lr / (1.0f + lr_decay * (float)k);
    s->sample_all = k < 256u ? 1u : 0u;
    s->next_sample_all = k + 1u < 256u ? 1u : 0u;
    s->step_count = k + 1u;
}

// Built-in synthetic network: blob field forward, fixed gradients backward.
struct SynthNet {
    float* blobs = nullptr;
    float* waves = nullptr;
    uint32_t n_blobs = 0;
    float aabb = 1.0f;
};

static int synth_forward(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                         const float* pos, const float*, float* density, float* rgb) {
    SynthNet* s = static_cast<SynthNet*>(user);
    if (!s->blobs) return fail(TN_E_STATE, "synthetic network has no field (call tn_trainer_set_synthetic_field)");
    return tn_synth_field(stream, n, n_dev, stride, pos, s->aabb, s->n_blobs, s->blobs, s->waves, density, rgb, stride);
}

static int synth_density(void* user, tn_stream_t stream, uint32_t n, const uint32_t* n_dev, uint32_t stride,
                         const float* pos, float* density) {
    SynthNet* s = static_cast<SynthNet*>(user);
    if (!s->blobs) return fail(TN_E_STATE, "synthetic network has no field (call tn_trainer_set_synthetic_field)");
    return tn_synth_field(stream, n, n_dev, stride, pos, s->aabb, s->n_blobs, s->blobs, s->waves, density, nullptr,
                          stride);
}

}  // namespace tn

using namespace tn;

// One set of per-step ray buffers with the march context that counted them: two steps are in
// flight at once in the count-ahead schedule (the tail of one, the head of the next).
struct RaySet {
    float *ori = nullptr, *dir = nullptr, *target = nullptr, *bg = nullptr;  // one allocation, [3|3|4|3][R]
    float *ray_t = nullptr, *ray_tmax = nullptr;
    uint8_t* alive = nullptr;
    uint32_t *n_steps = nullptr, *offsets = nullptr;
    uint32_t* info = nullptr;      // device batch_info[4] of this set's count
    float* ds_random = nullptr;    // [2][R] dataset draws of this set's rays (with a dataset)
    // the occupancy query of this set's step: random cells, their points, the network's values
    int32_t* occ_levels = nullptr;
    uint32_t* occ_cells = nullptr;
    float *occ_rand3 = nullptr, *occ_rsel = nullptr, *occ_pos = nullptr, *occ_values = nullptr;
    tn_ctx* ctx = nullptr;
};

// Step graphs: in-order step (head + tail of one step), tail of this step + head of the next,
// head alone, tail alone; per ray source (own, caller) and per ray set of the tail.
enum StepKind : int { K_HT = 0, K_TH = 1, K_H = 2, K_T = 3, K_KINDS = 4 };

struct tn_trainer {
    tn_trainer_desc d{};
    tn_network net{};
    SynthNet synth;
    void* hashnet = nullptr;  // the built-in hash-grid network, when it is the trainer's network
    cudaStream_t stream = nullptr;
    // the occupancy query and update beside the training chain, and the next step's head
    cudaStream_t aux = nullptr, cstream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_emit = nullptr, ev_occ = nullptr, ev_occ_all = nullptr, ev_head = nullptr;
    RaySet set[2];
    int cur = 0;               // set of the last completed step (the aliases below point into it)
    bool spec_own = false;     // set cur ^ 1 holds the head of the next step, computed from own rays
    bool pending_ext = false;  // set cur ^ 1 holds the head of a requested caller-ray step, tail not run
    tn_ctx* ctx = nullptr;     // set[cur].ctx
    std::vector<void*> allocs;
    uint32_t R = 0, B = 0, V = 0, P = 0, M = 0, chunk = 0;
    float aabb = 1.0f;
    // rays of the last completed step (aliases of set[cur])
    float *ori, *dir, *ray_t, *ray_tmax, *target, *bg;
    uint8_t* alive;
    uint32_t *n_steps, *offsets;
    // samples
    float *s_t, *s_pos, *s_dir, *s_dt, *s_mnorm, *s_dtnorm;
    float *net_density, *net_rgb, *grad_density, *dl_drgb;
    // plain-path scratch
    float *loss4, *dl_rec, *dl_dist, *ray5, *sample2, *ray_loss;
    uint8_t* count_scratch;
    // grid: densities, and the bitfield of the last completed step (an alias of bits_buf). With
    // an occupancy update in every step the bitfield is double-buffered, so that a step's update
    // can rebuild it while the step's emit pass still reads the one its count used: the step in
    // set s reads bits_buf[s ^ 1] and writes bits_buf[s].
    float* density;
    uint8_t* bits;
    uint8_t* bits_buf[2] = {nullptr, nullptr};
    // occupancy re-sampling of the last completed step (aliases of set[cur])
    int32_t* occ_levels;
    uint32_t* occ_cells;
    float *occ_rand3, *occ_rsel, *occ_pos, *occ_values;
    // params
    float *w, *g, *m, *v;
    uint32_t* steps;
    // step state
    StepState* state = nullptr;
    StepState* state_host = nullptr;  // pinned
    // pipelined caller-ray steps: each step's state and error word copied to pinned slots
    // (alternating), read by the host one call later
    StepState* ring_state = nullptr;  // pinned [2]
    volatile uint32_t* ring_flag = nullptr;  // pinned [2]: step count of the state in the slot
    uint64_t ring_calls = 0;          // pipelined calls since the last synchronous read
    // pipelined steps copy their host rays into the idle ray set on a copy stream, beside the
    // step in flight
    cudaStream_t h2d = nullptr;
    // a dataset of posed images as the ray source (tn_trainer_set_dataset)
    tn_camera* ds_cameras = nullptr;
    uint8_t* ds_images = nullptr;
    uint32_t ds_n = 0;
    int32_t ds_w = 0, ds_h = 0;
    float alpha_threshold = 1.0f, alpha_probability = 1.0f;
    cudaEvent_t ev_staged[2] = {nullptr, nullptr};
    // [kind][ray source: own, caller][ray set of the tail, or of the head for K_H][bits of the
    // tail's occupancy update computed ahead]
    cudaGraph_t graph[K_KINDS][2][2][2] = {};
    cudaGraphExec_t graph_exec[K_KINDS][2][2][2] = {};
    bool warm[K_KINDS][2][2][2] = {};     // ran once eagerly (lazy resources initialised)
    // bits_ahead[s]: the bitfield the occupancy update of the step in set s writes is already in
    // tail_bits(s), computed by the tail before it (its head then marches without waiting for
    // the update); set by a tail with a next step, consumed by that step's tail, cleared when a
    // head computed ahead is dropped
    bool bits_ahead[2] = {false, false};
    uint32_t graph_kernels[K_KINDS][2] = {};  // kernels captured in one graph of each kind and ray source
    uint32_t graph_nodes[K_KINDS][2] = {};
    uint32_t fused_steps_enqueued = 0;
    uint32_t host_step = 0;
    tn_training_metrics last{};

    void select(int p) {
        cur = p;
        RaySet& q = set[p];
        ori = q.ori; dir = q.dir; target = q.target; bg = q.bg;
        ray_t = q.ray_t; ray_tmax = q.ray_tmax; alive = q.alive; n_steps = q.n_steps; offsets = q.offsets;
        occ_levels = q.occ_levels; occ_cells = q.occ_cells; occ_rand3 = q.occ_rand3; occ_rsel = q.occ_rsel;
        occ_pos = q.occ_pos; occ_values = q.occ_values;
        ctx = q.ctx;
        bits = bits_buf[M > 0 ? p : 0];
    }
    // the bitfield the step in set s marches on, and the one its occupancy update writes
    uint8_t* head_bits(int s) const { return bits_buf[M > 0 ? s ^ 1 : 0]; }
    uint8_t* tail_bits(int s) const { return bits_buf[M > 0 ? s : 0]; }
    bool lookahead() const { return d.path == TN_PATH_FUSED && ctx->tune.side_sms > 0; }

    template <typename T>
    int alloc(T*& p, size_t n) {
        p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) return fail(TN_E_CUDA, "tn_trainer: cudaMalloc(%zu): %s", n * sizeof(T), cudaGetErrorString(e));
        allocs.push_back(p);
        return cudaMemsetAsync(p, 0, n * sizeof(T), stream) == cudaSuccess ? TN_OK : fail(TN_E_CUDA, "memset");
    }

    tn_grid_desc grid() const { return d.grid; }
    // dt_max = aabb_size * dt_min (reference src/core/trainer.cu:102-104)
    tn_march_desc march() const {
        tn_march_desc m{d.cone_angle, d.min_step_size, aabb * d.min_step_size, d.max_steps_per_ray, 0};
        return m;
    }
};

namespace {

// Stage boundaries of one fused step (for per-stage timing with events).
enum Stage : int { ST_RAYS = 0, ST_COUNT, ST_EMIT, ST_FORWARD, ST_LOSSES, ST_BACKWARD, ST_ADAM, ST_OCC_QUERY, ST_OCCUPANCY, ST_N };

// The rays of the step keyed by the state's step_count (the index the next step_begin gives
// the step) when the caller supplies none: from the dataset when one is set, else the built-in
// synthetic rays. Written into set q.
static int enqueue_own_rays(tn_trainer* tr, cudaStream_t s, RaySet& q) {
    const tn_trainer_desc& d = tr->d;
    const uint32_t* key = &tr->state->step_count;
    if (tr->ds_n) {
        int st = launch_dataset_draws(s, tr->R, tr->R, d.seed, key, q.ds_random, q.bg);
        if (st == TN_OK)
            st = launch_dataset_rays(s, tr->R, tr->R, tr->ds_n, tr->ds_w, tr->ds_h, tr->ds_cameras, tr->ds_images,
                                     d.bbox, q.ds_random, tr->alpha_threshold, tr->alpha_probability, q.target,
                                     nullptr, q.ori, q.dir, q.ray_t, q.ray_tmax, q.alive);
        return st;
    }
    return launch_synth_rays(s, tr->R, tr->R, d.seed, key, d.ray_radius, d.ray_jitter, d.bbox, 3.0e38f, q.ori, q.dir,
                             q.target, q.bg, q.ray_t, q.ray_tmax, q.alive);
}

// Occupancy query of one step (the step keyed by *key): random cells, their sample points, the
// density network, into set q's query buffers.
static int enqueue_occupancy_query(tn_trainer* tr, cudaStream_t s, const tn_grid_desc& grid, RaySet& q,
                                   const uint32_t* key) {
    const tn_trainer_desc& d = tr->d;
    int st = launch_synth_cells(s, tr->M, d.seed, key, grid.n_levels, tr->V, q.occ_levels, q.occ_cells, q.occ_rand3,
                                tr->M, q.occ_rsel);
    if (st == TN_OK)
        st = tn_occupancy_sample_points(s, &grid, tr->M, q.occ_levels, q.occ_cells, q.occ_rand3, tr->M,
                                        1.0f / tr->aabb, q.occ_pos, tr->M);
    if (st == TN_OK) st = tr->net.density(tr->net.user, s, tr->M, nullptr, tr->M, q.occ_pos, q.occ_values);
    return st;
}

// Occupancy update of the step in set pi: decay + max-update of the queried cells (the selection
// rule reads the bitfield the step marched on), bitfield rebuild into the step's output bitfield.
// With bits_done the rebuild runs first and records the event, and the decayed densities are
// written back after it (the next step's march waits only for the bits).
// With bits_ready the step's output bitfield was computed ahead (enqueue_occupancy_bits_ahead)
// and the update only writes the densities back and counts.
static int enqueue_occupancy_update(tn_trainer* tr, cudaStream_t s, const tn_grid_desc& grid, int pi,
                                    cudaEvent_t bits_done = nullptr, bool bits_ready = false) {
    const tn_trainer_desc& d = tr->d;
    RaySet& p = tr->set[pi];
    return launch_occupancy_update(p.ctx, s, &grid, tr->density, tr->head_bits(pi), tr->M, p.occ_levels, p.occ_cells,
                                   p.occ_values, p.occ_rsel, tr->net.activation, 0, &tr->state->sample_all, nullptr,
                                   d.occupancy_decay, d.occupancy_threshold, &tr->state->n_occupied,
                                   tr->tail_bits(pi), bits_done, bits_ready);
}

// The bitfield the occupancy update of the step in set qi will write, from its query (already in
// set qi) and the settled densities, into the step's output bitfield; the step's selection
// policy is the state's next_sample_all (the running step's step_begin has run, the step's has
// not). Nothing changes the densities or the query before that update runs.
static int enqueue_occupancy_bits_ahead(tn_trainer* tr, cudaStream_t s, const tn_grid_desc& grid, int qi) {
    const tn_trainer_desc& d = tr->d;
    RaySet& q = tr->set[qi];
    return launch_occupancy_bits_ahead(s, &grid, tr->density, tr->head_bits(qi), tr->tail_bits(qi), tr->M,
                                       q.occ_levels, q.occ_cells, q.occ_values, q.occ_rsel, tr->net.activation,
                                       &tr->state->next_sample_all, d.occupancy_decay, d.occupancy_threshold);
}

// Head of a step: its rays (own, or the caller's already in set q, clipped to the box) and the
// march count with the batch cut into set q's buffers and context.
static int enqueue_head_rays(tn_trainer* tr, cudaStream_t s, bool external, int qi) {
    const tn_trainer_desc& d = tr->d;
    RaySet& q = tr->set[qi];
    return external ? tn_rays_init_bbox(s, tr->R, tr->R, &d.bbox, 3.0e38f, q.ori, q.dir, q.ray_t, q.ray_tmax, q.alive)
                    : enqueue_own_rays(tr, s, q);
}

static int enqueue_head_count(tn_trainer* tr, cudaStream_t s, int qi) {
    const tn_trainer_desc& d = tr->d;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    RaySet& q = tr->set[qi];
    return tn_march_count(q.ctx, s, &grid, tr->head_bits(qi), &d.bbox, &march, tr->R, tr->R, nullptr, q.ori, q.dir,
                          q.ray_t, q.ray_tmax, q.alive, q.n_steps, tr->B, q.info);
}

static int enqueue_head(tn_trainer* tr, cudaStream_t s, bool external, int qi) {
    int st = enqueue_head_rays(tr, s, external, qi);
    return st == TN_OK ? enqueue_head_count(tr, s, qi) : st;
}

// Tail of the step whose head is in set pi: step_begin, emit, network forward, the fused losses,
// network backward and Adam; on the second stream the step's occupancy update (from the query
// made with its head), which writes the step's output bitfield while the emit pass still reads
// the one the count used (or only the densities, when the bitfield was computed ahead). With
// next >= 0 the head of the following step (rays from next_external / own rays) runs on the
// third stream into set next, its count once the output bitfield is there, Adam keeps to
// side_sms SMs beside it, and the following step's occupancy query runs after Adam (the
// density network reads the updated parameters), followed by the bitfield its update will
// write. ring >= 0 copies the finished step's state into that pinned slot before the head is
// joined.
static int enqueue_tail(tn_trainer* tr, int pi, int next, bool next_external, int ring) {
    const tn_trainer_desc& d = tr->d;
    cudaStream_t s = tr->stream, so = tr->aux, cs = tr->cstream;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    const bool occ = tr->M > 0;
    const bool ahead = occ && tr->bits_ahead[pi];
    RaySet& p = tr->set[pi];
    step_begin_kernel<<<1, 1, 0, s>>>(tr->state, d.learning_rate, d.learning_rate_decay);
    int st = check_launch("step_begin");
    if (st == TN_OK && (occ || next >= 0)) st = cuda_status(cudaEventRecord(tr->ev_fork, s), "fork");
    // the occupancy update; its bitfield computed ahead by the previous tail, or beside a next
    // head split: ev_occ once the bitfield is rebuilt
    if (st == TN_OK && occ) {
        st = cuda_status(cudaStreamWaitEvent(so, tr->ev_fork, 0), "fork");
        if (st == TN_OK)
            st = enqueue_occupancy_update(tr, so, grid, pi, next >= 0 && !ahead ? tr->ev_occ : nullptr, ahead);
        if (st == TN_OK) st = cuda_status(cudaEventRecord(tr->ev_occ_all, so), "occupancy done");
    }
    // the next step's head: its rays at once, its march count on the step's output bitfield
    // (ready at once when it was computed ahead)
    if (st == TN_OK && next >= 0) {
        st = cuda_status(cudaStreamWaitEvent(cs, tr->ev_fork, 0), "head start");
        if (st == TN_OK) st = enqueue_head_rays(tr, cs, next_external, next);
        if (st == TN_OK && occ && !ahead) st = cuda_status(cudaStreamWaitEvent(cs, tr->ev_occ, 0), "grid rebuilt");
        if (st == TN_OK) st = enqueue_head_count(tr, cs, next);
        if (st == TN_OK) st = cuda_status(cudaEventRecord(tr->ev_head, cs), "head done");
    }
    uint32_t* info = p.info;
    if (st == TN_OK)
        st = tn_march_emit(p.ctx, s, &grid, tr->head_bits(pi), &d.bbox, &march, 1.0f / tr->aabb, tr->R, tr->R, tr->B,
                           info, nullptr, p.ori, p.dir, p.ray_t, p.alive, p.n_steps, p.offsets, nullptr, tr->s_t,
                           tr->s_pos, tr->s_dir, tr->s_dt, tr->s_mnorm, tr->s_dtnorm);
    if (st == TN_OK)
        st = tr->net.forward(tr->net.user, s, tr->B, info + 1, tr->B, tr->s_pos, tr->s_dir, tr->net_density,
                             tr->net_rgb);
    // the merged density gradient is written over grad_density (no zeroing pass)
    tn_ray_batch rb{tr->R, tr->R, tr->B, 0, p.n_steps, p.offsets, info};
    if (st == TN_OK)
        st = train_losses(p.ctx, s, &rb, tr->net.activation, d.min_transmittance, 0.0f, info, d.loss_scale,
                          d.use_distortion_loss ? d.distortion_lambda : 0.0f, tr->net_density, tr->net_rgb, tr->s_dt,
                          tr->s_mnorm, tr->s_dtnorm, tr->s_t, p.target, p.bg, nullptr, tr->grad_density, tr->dl_drgb,
                          tr->state->loss_sums, false);
    if (st == TN_OK && tr->net.backward)
        st = tr->net.backward(tr->net.user, s, tr->B, info + 1, tr->B, tr->s_pos, tr->s_dir, tr->grad_density,
                              tr->dl_drgb, tr->g);
    if (st == TN_OK) {
        AdamPlacement place;
        if (next >= 0 && p.ctx->tune.side_sms) {
            place.max_blocks = p.ctx->tune.side_sms;
            place.reserve_smem = exclusive_smem();
        }
        st = launch_adam(s, false, tr->P, d.n_grid_params, d.n_mlp_params, d.loss_scale, d.learning_rate,
                         &tr->state->lr, d.beta1, d.beta2, d.epsilon, d.l2_reg, tr->w, nullptr, tr->g, tr->m, tr->v,
                         tr->steps, place);
    }
    if (st == TN_OK && occ) st = cuda_status(cudaStreamWaitEvent(s, tr->ev_occ_all, 0), "occupancy joined");
    // the following step's occupancy query, keyed by its index (step_count after this step_begin)
    if (st == TN_OK && occ && next >= 0) st = enqueue_occupancy_query(tr, s, grid, tr->set[next], &tr->state->step_count);
    // and the bitfield its occupancy update will write, so that the head after it need not wait
    if (st == TN_OK && occ && next >= 0) st = enqueue_occupancy_bits_ahead(tr, s, grid, next);
    if (st == TN_OK) {
        step_end_kernel<<<1, 1, 0, s>>>(tr->state, info, p.ctx->flags);
        st = check_launch("step_end");
    }
    // The finished step's state to the pinned ring slot, then its step count to the slot's pinned
    // flag word: the copies run in stream order, so once the host sees the flag the state has
    // landed. The host polls the flag (tn_trainer_train_step_rays_pipelined) while the next
    // step's head may still be marching.
    if (st == TN_OK && ring >= 0) {
        st = cuda_status(cudaMemcpyAsync(&tr->ring_state[ring], tr->state, sizeof(StepState), cudaMemcpyDeviceToHost,
                                         s), "state to ring");
        if (st == TN_OK)
            st = cuda_status(cudaMemcpyAsync(const_cast<uint32_t*>(&tr->ring_flag[ring]), &tr->state->step_count,
                                             sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "ring flag");
        if (st == TN_OK) st = cuda_status(cudaMemsetAsync(&tr->state->err, 0, sizeof(uint32_t), s), "err clear");
    }
    if (st == TN_OK && next >= 0) st = cuda_status(cudaStreamWaitEvent(s, tr->ev_head, 0), "head joined");
    return st;
}

// One fused step in order on the trainer's stream with events between its stages (stage
// timing): head and tail of the step in set pi, nothing beside it.
static int enqueue_profiled_step(tn_trainer* tr, int pi, cudaEvent_t* ev) {
    const tn_trainer_desc& d = tr->d;
    cudaStream_t s = tr->stream;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    RaySet& p = tr->set[pi];
    cudaEventRecord(ev[0], s);
    int st = enqueue_own_rays(tr, s, p);
    cudaEventRecord(ev[ST_RAYS + 1], s);
    if (st == TN_OK)
        st = tn_march_count(p.ctx, s, &grid, tr->head_bits(pi), &d.bbox, &march, tr->R, tr->R, nullptr, p.ori, p.dir,
                            p.ray_t, p.ray_tmax, p.alive, p.n_steps, tr->B, p.info);
    cudaEventRecord(ev[ST_COUNT + 1], s);
    if (st == TN_OK) {
        step_begin_kernel<<<1, 1, 0, s>>>(tr->state, d.learning_rate, d.learning_rate_decay);
        st = check_launch("step_begin");
    }
    if (st == TN_OK)
        st = tn_march_emit(p.ctx, s, &grid, tr->head_bits(pi), &d.bbox, &march, 1.0f / tr->aabb, tr->R, tr->R, tr->B,
                           p.info, nullptr, p.ori, p.dir, p.ray_t, p.alive, p.n_steps, p.offsets, nullptr, tr->s_t,
                           tr->s_pos, tr->s_dir, tr->s_dt, tr->s_mnorm, tr->s_dtnorm);
    cudaEventRecord(ev[ST_EMIT + 1], s);
    if (st == TN_OK)
        st = tr->net.forward(tr->net.user, s, tr->B, p.info + 1, tr->B, tr->s_pos, tr->s_dir, tr->net_density,
                             tr->net_rgb);
    cudaEventRecord(ev[ST_FORWARD + 1], s);
    tn_ray_batch rb{tr->R, tr->R, tr->B, 0, p.n_steps, p.offsets, p.info};
    if (st == TN_OK)
        st = train_losses(p.ctx, s, &rb, tr->net.activation, d.min_transmittance, 0.0f, p.info, d.loss_scale,
                          d.use_distortion_loss ? d.distortion_lambda : 0.0f, tr->net_density, tr->net_rgb, tr->s_dt,
                          tr->s_mnorm, tr->s_dtnorm, tr->s_t, p.target, p.bg, nullptr, tr->grad_density, tr->dl_drgb,
                          tr->state->loss_sums, false);
    cudaEventRecord(ev[ST_LOSSES + 1], s);
    if (st == TN_OK && tr->net.backward)
        st = tr->net.backward(tr->net.user, s, tr->B, p.info + 1, tr->B, tr->s_pos, tr->s_dir, tr->grad_density,
                              tr->dl_drgb, tr->g);
    cudaEventRecord(ev[ST_BACKWARD + 1], s);
    if (st == TN_OK)
        st = launch_adam(s, false, tr->P, d.n_grid_params, d.n_mlp_params, d.loss_scale, d.learning_rate,
                         &tr->state->lr, d.beta1, d.beta2, d.epsilon, d.l2_reg, tr->w, nullptr, tr->g, tr->m, tr->v,
                         tr->steps, AdamPlacement{});
    cudaEventRecord(ev[ST_ADAM + 1], s);
    if (st == TN_OK && tr->M > 0) st = enqueue_occupancy_query(tr, s, grid, p, &tr->state->cur_step);
    cudaEventRecord(ev[ST_OCC_QUERY + 1], s);
    if (st == TN_OK && tr->M > 0) st = enqueue_occupancy_update(tr, s, grid, pi);
    cudaEventRecord(ev[ST_OCCUPANCY + 1], s);
    if (st == TN_OK) {
        step_end_kernel<<<1, 1, 0, s>>>(tr->state, p.info, p.ctx->flags);
        st = check_launch("step_end");
    }
    return st;
}

// Enqueues one kind of step (ray source: own or caller rays) with set p as the set of its
// tail (K_HT, K_TH, K_T) or of its head (K_H). The first run of each variant is eager (it also
// initialises every lazily created resource); later runs replay a graph captured once.
static int enqueue_kind(tn_trainer* tr, int kind, bool external, int p, int ring) {
    const int src = external ? 1 : 0;
    // a head run here queries afresh, so only a lone tail (K_TH, K_T) finds its set's bits
    // computed ahead; a tail consumes them, and a tail with a next step computes the next's
    if (kind == K_H || kind == K_HT) tr->bits_ahead[p] = false;
    const int ahead = tr->M > 0 && tr->bits_ahead[p] ? 1 : 0;
    auto advance = [&](int st) -> int {
        if (st == TN_OK && kind != K_H) tr->bits_ahead[p] = false;
        if (st == TN_OK && kind == K_TH && tr->M > 0) tr->bits_ahead[p ^ 1] = true;
        return st;
    };
    // a head without a tail before it also makes its step's occupancy query (a tail runs the
    // next step's query after its Adam update); before its step_begin, the step's key is
    // step_count
    auto head_alone = [&]() -> int {
        int st = enqueue_head(tr, tr->stream, external, p);
        if (st == TN_OK && tr->M > 0)
            st = enqueue_occupancy_query(tr, tr->stream, tr->grid(), tr->set[p], &tr->state->step_count);
        return st;
    };
    auto body = [&]() -> int {
        switch (kind) {
            case K_HT: {
                const int st = head_alone();
                return st == TN_OK ? enqueue_tail(tr, p, -1, false, ring) : st;
            }
            case K_TH: return enqueue_tail(tr, p, p ^ 1, external, ring);
            case K_H: return head_alone();
            default: return enqueue_tail(tr, p, -1, false, ring);
        }
    };
    // a ring copy is baked into a graph: the pipelined caller-ray steps copy into slot p
    if (!tr->d.use_cuda_graph || !tr->warm[kind][src][p][ahead] || (ring >= 0 && ring != p)) {
        tr->warm[kind][src][p][ahead] = true;
        return advance(body());
    }
    cudaGraphExec_t& ex = tr->graph_exec[kind][src][p][ahead];
    if (!ex) {
        int st = cuda_status(cudaStreamBeginCapture(tr->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        if (st != TN_OK) return st;
        const int est = body();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(tr->stream, &g);
        if (est != TN_OK) {
            if (g) cudaGraphDestroy(g);
            return est;
        }
        st = cuda_status(e, "end capture");
        if (st == TN_OK) st = cuda_status(cudaGraphInstantiate(&ex, g, 0), "instantiate");
        if (st != TN_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        tr->graph[kind][src][p][ahead] = g;
        size_t n_nodes = 0;
        cudaGraphGetNodes(g, nullptr, &n_nodes);
        std::vector<cudaGraphNode_t> nodes(n_nodes);
        cudaGraphGetNodes(g, nodes.data(), &n_nodes);
        uint32_t kernels = 0;
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            cudaGraphNodeGetType(nd, &t);
            kernels += t == cudaGraphNodeTypeKernel;
        }
        tr->graph_kernels[kind][src] = kernels;
        tr->graph_nodes[kind][src] = (uint32_t)n_nodes;
    }
    return advance(cuda_status(cudaGraphLaunch(ex, tr->stream), "graph launch"));
}

// Drops a head computed ahead from own rays (what it read is about to change, or the next
// step takes caller rays): its work is done by the time the stream is idle, and the error bits
// it raised belong to no step.
static int drop_spec(tn_trainer* tr) {
    if (!tr->spec_own) return TN_OK;
    tr->spec_own = false;
    tr->bits_ahead[0] = tr->bits_ahead[1] = false;  // the dropped step's update never runs
    int st = cuda_status(cudaStreamSynchronize(tr->stream), "drop head");
    if (st == TN_OK)
        st = cuda_status(cudaMemsetAsync(tr->set[tr->cur ^ 1].ctx->flags, 0, sizeof(uint32_t), tr->stream),
                         "drop head flags");
    return st;
}

// Runs the tail of a requested caller-ray step whose head is in set cur ^ 1.
static int finish_pending(tn_trainer* tr) {
    if (!tr->pending_ext) return TN_OK;
    tr->pending_ext = false;
    const int q = tr->cur ^ 1;
    int st = enqueue_kind(tr, K_T, true, q, -1);
    if (st != TN_OK) return st;
    tr->select(q);
    ++tr->fused_steps_enqueued;
    return TN_OK;
}

// Brings the trainer to a step boundary with nothing in flight ahead of it: a requested step is
// completed; a head computed ahead is kept (keep_spec) or dropped.
static int settle(tn_trainer* tr, bool keep_spec = false) {
    int st = finish_pending(tr);
    if (st == TN_OK && !keep_spec) st = drop_spec(tr);
    return st;
}

int run_plain_step(tn_trainer* tr, bool external_rays, tn_training_metrics* out) {
    const tn_trainer_desc& d = tr->d;
    cudaStream_t s = tr->stream;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    const uint32_t k = tr->host_step;
    const float lr = d.learning_rate / (1.0f + d.learning_rate_decay * (float)k);
    // the step's rays (own rays keyed by the step's index, the state's step_count before
    // step_begin), then step_begin
    int st = external_rays ? tn_rays_init_bbox(s, tr->R, tr->R, &d.bbox, 3.0e38f, tr->ori, tr->dir, tr->ray_t,
                                               tr->ray_tmax, tr->alive)
                           : enqueue_own_rays(tr, s, tr->set[tr->cur]);
    if (st == TN_OK) {
        step_begin_kernel<<<1, 1, 0, s>>>(tr->state, d.learning_rate, d.learning_rate_decay);
        st = check_launch("step_begin");
    }
    if (st == TN_OK)
        st = tn_plain_march_count(s, &grid, tr->bits, &d.bbox, &march, tr->R, tr->R, tr->ori, tr->dir, tr->ray_t,
                                  tr->ray_tmax, tr->alive, tr->n_steps);
    uint32_t nr = 0, ns = 0;
    if (st == TN_OK) st = tn_plain_scan_cut_sync(s, tr->R, tr->n_steps, tr->offsets, tr->B, &nr, &ns);
    if (st == TN_OK)
        st = tn_plain_march_emit(s, &grid, tr->bits, &d.bbox, &march, 1.0f / tr->aabb, nr, tr->R, tr->B, nullptr,
                                 tr->ori, tr->dir, tr->ray_t, tr->offsets, tr->alive, tr->n_steps, nullptr, tr->s_t,
                                 tr->s_pos, tr->s_dir, tr->s_dt, tr->s_mnorm, tr->s_dtnorm);
    if (st == TN_OK)
        st = tr->net.forward(tr->net.user, s, ns, nullptr, tr->B, tr->s_pos, tr->s_dir, tr->net_density, tr->net_rgb);
    tn_ray_batch rb{nr, tr->R, tr->B, 0, tr->n_steps, tr->offsets, nullptr};
    float rec = 0.0f, dist = 0.0f;
    if (st == TN_OK)
        st = tn_plain_recon_loss_sync(s, &rb, tr->net.activation, d.min_transmittance, 1.0f / (float)nr, d.loss_scale,
                                      tr->net_density, tr->net_rgb, tr->s_dt, tr->target, tr->bg, tr->loss4,
                                      tr->dl_rec, tr->dl_drgb, &rec);
    if (st == TN_OK && d.use_distortion_loss)
        st = tn_plain_distortion_sync(s, &rb, tr->net.activation, d.distortion_lambda, tr->net_density, tr->s_mnorm,
                                      tr->s_dtnorm, tr->ray5, tr->sample2, tr->ray_loss, tr->dl_dist, &dist);
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(tr->grad_density, 0, (size_t)tr->B * 4, s), "grad memset");
    if (st == TN_OK)
        st = tn_plain_grad_epilogue(s, ns, d.loss_scale, tr->dl_rec, d.use_distortion_loss ? tr->dl_dist : nullptr,
                                    tr->s_t, tr->grad_density);
    if (st == TN_OK && tr->net.backward)
        st = tr->net.backward(tr->net.user, s, ns, nullptr, tr->B, tr->s_pos, tr->s_dir, tr->grad_density, tr->dl_drgb,
                              tr->g);
    if (st == TN_OK)
        st = launch_adam(s, true, tr->P, d.n_grid_params, d.n_mlp_params, d.loss_scale, lr, nullptr, d.beta1, d.beta2,
                         d.epsilon, d.l2_reg, tr->w, nullptr, tr->g, tr->m, tr->v, tr->steps);
    if (st == TN_OK && tr->M > 0) {
        st = launch_synth_cells(s, tr->M, d.seed, &tr->state->cur_step, grid.n_levels, tr->V, tr->occ_levels,
                                tr->occ_cells, tr->occ_rand3, tr->M, tr->occ_rsel);
        if (st == TN_OK)
            st = tn_occupancy_sample_points(s, &grid, tr->M, tr->occ_levels, tr->occ_cells, tr->occ_rand3, tr->M,
                                            1.0f / tr->aabb, tr->occ_pos, tr->M);
        if (st == TN_OK) st = tr->net.density(tr->net.user, s, tr->M, nullptr, tr->M, tr->occ_pos, tr->occ_values);
        uint32_t nocc = 0;
        if (st == TN_OK)
            st = tn_plain_occupancy_update_sync(s, &grid, tr->density, tr->bits, tr->M, tr->occ_levels, tr->occ_cells,
                                                tr->occ_values, tr->occ_rsel, tr->net.activation, k < 256 ? 1 : 0,
                                                d.occupancy_decay, d.occupancy_threshold, tr->count_scratch, &nocc);
    }
    if (st == TN_OK) {
        uint32_t info[4] = {nr, ns, 0, 0};
        st = cuda_status(cudaMemcpyAsync(tr->set[tr->cur].info, info, sizeof(info), cudaMemcpyHostToDevice, s),
                         "batch info");
        if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "plain info sync");
        if (st == TN_OK) {
            step_end_kernel<<<1, 1, 0, s>>>(tr->state, tr->set[tr->cur].info, tr->ctx->flags);
            st = check_launch("step_end");
        }
    }
    if (st != TN_OK) return st;
    tr->host_step = k + 1;
    tr->last.step = k + 1;
    tr->last.n_rays = nr;
    tr->last.n_samples = ns;
    tr->last.loss = rec + dist;
    if (out) {
        st = cuda_status(cudaStreamSynchronize(s), "plain step sync");
        *out = tr->last;
    }
    return st;
}

// Metrics of a step from its state (with its error bits), as read back to the host.
int metrics_from(tn_trainer* tr, const StepState& h, tn_training_metrics* out) {
    const uint32_t flags = h.err;
    if (flags & TN_FLAG_NO_RAYS) return fail(TN_E_NO_RAYS, "No rays were generated for this training batch");
    if (flags & TN_FLAG_NO_SAMPLES) return fail(TN_E_NO_SAMPLES, "No samples were generated for this training batch");
    if (flags) return fail(TN_E_DEVICE, "device error flags 0x%x", flags);
    tr->last.step = h.step_count;
    tr->last.n_rays = h.batch_info[0];
    tr->last.n_samples = h.batch_info[1];
    tr->last.loss = h.loss_sums[0] + h.loss_sums[1];
    if (out) *out = tr->last;
    return TN_OK;
}

// Waits for the trainer's stream and reads the state of the last completed step; its error bits
// (every step's since the last read) are cleared.
int read_state(tn_trainer* tr, tn_training_metrics* out) {
    int st = cuda_status(cudaMemcpyAsync(tr->state_host, tr->state, sizeof(StepState), cudaMemcpyDeviceToHost, tr->stream),
                         "state read");
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(&tr->state->err, 0, sizeof(uint32_t), tr->stream), "err clear");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "state sync");
    if (st != TN_OK) return st;
    tr->ring_calls = 0;  // every earlier step is complete; its error bits were in the state
    return metrics_from(tr, *tr->state_host, out);
}

}  // namespace

extern "C" {

int tn_trainer_default_desc(tn_trainer_desc* o) {
    TN_NONNULL(o);
    std::memset(o, 0, sizeof(*o));
    o->grid = tn_grid_desc{1, 128, 1.0f, 0};
    o->bbox = tn_bbox{-0.5f, -0.5f, -0.5f, 0.5f, 0.5f, 0.5f};
    o->batch_size = 2u << 21;            // NeRFConstants::batch_size
    o->n_rays_per_step = 1u << 14;
    o->min_step_size = 0.00169145586f;   // NeRFConstants::min_step_size
    o->cone_angle = 1.0f / 256.0f;       // NeRFConstants::cone_angle
    o->max_steps_per_ray = 0;
    o->min_transmittance = 1e-4f;        // NeRFConstants::min_transmittance
    o->use_distortion_loss = 0;
    o->distortion_lambda = 0.01f;        // NeRFConstants::mipNeRF360_distortion_loss_lambda
    o->loss_scale = 1.0f;
    o->occupancy_decay = 0.95f;          // NeRFConstants::occupancy_decay
    o->occupancy_threshold = 0.01f * 0.00169145586f;  // NeRFConstants::occupancy_threshold
    o->occupancy_cells_per_step = 0;
    o->n_grid_params = 16u * (1u << 19) * 2u;
    o->n_mlp_params = 7168;
    o->learning_rate = 1e-2f;            // nerf-network.cu:173-178
    o->learning_rate_decay = 3.3e-5f;    // NeRFConstants::learning_rate_decay
    o->beta1 = 0.9f;
    o->beta2 = 0.999f;                   // adam-optimizer.cuh:240
    o->epsilon = 1e-15f;
    o->l2_reg = 1e-6f;
    o->path = TN_PATH_FUSED;
    o->use_cuda_graph = 1;
    o->seed = 0x7B0u;
    o->ray_radius = 4.0f;
    o->ray_jitter = 0.05f;
    return TN_OK;
}

int tn_trainer_create(tn_trainer** out, const tn_trainer_desc* desc, const tn_network* net) {
    TN_NONNULL(out);
    TN_NONNULL(desc);
    *out = nullptr;
    int st = validate_grid(&desc->grid);
    if (st != TN_OK) return st;
    TN_REQUIRE(desc->path == TN_PATH_FUSED || desc->path == TN_PATH_PLAIN, TN_E_INVALID, "unknown path %d", desc->path);
    TN_REQUIRE(desc->batch_size >= 2 && desc->n_rays_per_step >= 2, TN_E_INVALID, "batch_size and n_rays_per_step must be >= 2");
    TN_REQUIRE(desc->bbox.max_x > desc->bbox.min_x, TN_E_INVALID, "empty bounding box");
    if (net) {
        TN_REQUIRE(net->forward && net->density, TN_E_NULL, "tn_network needs forward and density callbacks");
    }
    tn_trainer* tr = new tn_trainer();
    tr->d = *desc;
    tr->aabb = desc->bbox.max_x - desc->bbox.min_x;
    tr->synth.aabb = tr->aabb;
    if (net) {
        tr->net = *net;
    } else {
        tr->net.user = &tr->synth;
        tr->net.activation = TN_ACT_SIGMA;
        tr->net.forward = synth_forward;
        tr->net.backward = nullptr;
        tr->net.density = synth_density;
    }
    st = cuda_status(cudaStreamCreateWithFlags(&tr->stream, cudaStreamNonBlocking), "stream");
    if (st == TN_OK) st = cuda_status(cudaStreamCreateWithFlags(&tr->aux, cudaStreamNonBlocking), "aux stream");
    if (st == TN_OK) st = cuda_status(cudaStreamCreateWithFlags(&tr->cstream, cudaStreamNonBlocking), "head stream");
    if (st == TN_OK) st = cuda_status(cudaStreamCreateWithFlags(&tr->h2d, cudaStreamNonBlocking), "copy stream");
    for (cudaEvent_t* e : {&tr->ev_fork, &tr->ev_emit, &tr->ev_occ, &tr->ev_occ_all, &tr->ev_head,
                           &tr->ev_staged[0], &tr->ev_staged[1]})
        if (st == TN_OK) st = cuda_status(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "step events");
    for (int k = 0; k < 2 && st == TN_OK; ++k) st = tn_ctx_create(&tr->set[k].ctx);
    const uint32_t R = desc->n_rays_per_step, B = desc->batch_size;
    const uint32_t res = (uint32_t)desc->grid.resolution;
    const uint32_t V = res * res * res, L = (uint32_t)desc->grid.n_levels;
    const uint32_t P = desc->n_grid_params + desc->n_mlp_params;
    tr->R = R; tr->B = B; tr->V = V; tr->P = P; tr->M = desc->occupancy_cells_per_step;
    tr->chunk = std::min(B, V);
    const uint32_t occ_n = std::max(tr->M, tr->chunk);
    for (int k = 0; k < 2 && st == TN_OK; ++k) st = tn_ctx_reserve(tr->set[k].ctx, R, B);
    // Count-ahead by default: the march count in 256-ray blocks, one per SM, and the other SMs
    // for Adam beside it, when that leaves at least 16 of them.
    if (st == TN_OK && desc->path == TN_PATH_FUSED) {
        const int side = num_sms() - (int)((R + 255) / 256);
        if (side >= 16) {
            for (int k = 0; k < 2; ++k) {
                tr->set[k].ctx->tune.count_rays_per_block = 256;
                tr->set[k].ctx->tune.side_sms = (uint32_t)side;
            }
        }
    }
#define ALLOC(p, n) if (st == TN_OK) st = tr->alloc(p, (size_t)(n))
    // each set's input rays in one allocation, [ori 3R | dir 3R | target 4R | bg 3R]
    for (int k = 0; k < 2; ++k) {
        RaySet& q = tr->set[k];
        ALLOC(q.ori, 13 * (size_t)R);
        if (st == TN_OK) {
            q.dir = q.ori + 3 * (size_t)R;
            q.target = q.ori + 6 * (size_t)R;
            q.bg = q.ori + 10 * (size_t)R;
        }
        ALLOC(q.ray_t, R); ALLOC(q.ray_tmax, R);
        ALLOC(q.alive, R); ALLOC(q.n_steps, R); ALLOC(q.offsets, R); ALLOC(q.info, 4);
    }
    ALLOC(tr->s_t, B); ALLOC(tr->s_pos, 3 * B); ALLOC(tr->s_dir, 3 * B); ALLOC(tr->s_dt, B); ALLOC(tr->s_mnorm, B);
    ALLOC(tr->s_dtnorm, B); ALLOC(tr->net_density, B); ALLOC(tr->net_rgb, 3 * B); ALLOC(tr->grad_density, B);
    ALLOC(tr->dl_drgb, 3 * B);
    if (desc->path == TN_PATH_PLAIN) {
        ALLOC(tr->loss4, 4 * R); ALLOC(tr->dl_rec, B); ALLOC(tr->dl_dist, B); ALLOC(tr->ray5, 5 * R);
        ALLOC(tr->sample2, 2 * B); ALLOC(tr->ray_loss, R);
    }
    ALLOC(tr->count_scratch, V / 4);
    ALLOC(tr->density, (size_t)L * V); ALLOC(tr->bits_buf[0], V);
    if (tr->M > 0) {
        ALLOC(tr->bits_buf[1], V);
    } else {
        tr->bits_buf[1] = tr->bits_buf[0];
    }
    for (int k = 0; k < 2; ++k) {
        RaySet& q = tr->set[k];
        ALLOC(q.occ_levels, occ_n); ALLOC(q.occ_cells, occ_n); ALLOC(q.occ_rand3, 3 * (size_t)occ_n);
        ALLOC(q.occ_rsel, occ_n); ALLOC(q.occ_pos, 3 * (size_t)occ_n); ALLOC(q.occ_values, occ_n);
    }
    ALLOC(tr->w, P); ALLOC(tr->g, P); ALLOC(tr->m, P); ALLOC(tr->v, P); ALLOC(tr->steps, P);
    ALLOC(tr->state, 1);
#undef ALLOC
    if (st == TN_OK) tr->select(0);
    if (st == TN_OK) st = cuda_status(cudaMallocHost(&tr->state_host, sizeof(StepState)), "pinned state");
    if (st == TN_OK) st = cuda_status(cudaMallocHost(&tr->ring_state, 2 * sizeof(StepState)), "pinned state ring");
    if (st == TN_OK) {
        uint32_t* f = nullptr;
        st = cuda_status(cudaMallocHost(&f, 2 * sizeof(uint32_t)), "pinned ring flags");
        tr->ring_flag = f;
    }
    // reference initial grid: every bit set, densities zero (occupancy-grid.cuh:81-85)
    for (int k = 0; k < 2 && st == TN_OK; ++k)
        st = cuda_status(cudaMemsetAsync(tr->bits_buf[k], 0xFF, V, tr->stream), "bitfield init");
    if (st == TN_OK) st = launch_synth_params(tr->stream, P, desc->n_grid_params, desc->seed, tr->w);
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "trainer init");
    if (st != TN_OK) {
        tn_trainer_destroy(tr);
        return st;
    }
    *out = tr;
    return TN_OK;
}

static void drop_graphs(tn_trainer* tr);

int tn_trainer_destroy(tn_trainer* tr) {
    if (!tr) return TN_OK;
    if (tr->stream) cudaStreamSynchronize(tr->stream);
    drop_graphs(tr);
    if (tr->hashnet) hashnet_destroy(tr->hashnet);
    for (void* p : tr->allocs) cudaFree(p);
    if (tr->synth.blobs) cudaFree(tr->synth.blobs);
    if (tr->synth.waves) cudaFree(tr->synth.waves);
    if (tr->state_host) cudaFreeHost(tr->state_host);
    if (tr->ring_state) cudaFreeHost(tr->ring_state);
    if (tr->ring_flag) cudaFreeHost(const_cast<uint32_t*>(tr->ring_flag));
    for (int k = 0; k < 2; ++k)
        if (tr->set[k].ctx) tn_ctx_destroy(tr->set[k].ctx);
    if (tr->h2d) cudaStreamSynchronize(tr->h2d);
    for (cudaEvent_t e : {tr->ev_fork, tr->ev_emit, tr->ev_occ, tr->ev_occ_all, tr->ev_head,
                          tr->ev_staged[0], tr->ev_staged[1]})
        if (e) cudaEventDestroy(e);
    if (tr->h2d) cudaStreamDestroy(tr->h2d);
    if (tr->aux) cudaStreamDestroy(tr->aux);
    if (tr->cstream) cudaStreamDestroy(tr->cstream);
    if (tr->stream) cudaStreamDestroy(tr->stream);
    delete tr;
    return TN_OK;
}

int tn_trainer_set_synthetic_field(tn_trainer* tr, uint32_t n_blobs, const float* blobs, const float* waves) {
    TN_NONNULL(tr); TN_NONNULL(blobs); TN_NONNULL(waves);
    TN_REQUIRE(n_blobs >= 1 && n_blobs <= 256, TN_E_INVALID, "n_blobs %u outside 1..256", n_blobs);
    bool captured = false;
    for (auto& k : tr->graph_exec)
        for (auto& r : k)
            for (auto& q : r)
                for (auto& e : q) captured = captured || e != nullptr;
    TN_REQUIRE(!captured, TN_E_STATE, "the field must be set before the first captured step");
    if (tr->synth.blobs) cudaFree(tr->synth.blobs);
    if (tr->synth.waves) cudaFree(tr->synth.waves);
    tr->synth.blobs = tr->synth.waves = nullptr;
    int st = cuda_status(cudaMalloc(&tr->synth.blobs, 5 * n_blobs * sizeof(float)), "blobs");
    if (st == TN_OK) st = cuda_status(cudaMalloc(&tr->synth.waves, 12 * sizeof(float)), "waves");
    if (st == TN_OK) st = cuda_status(cudaMemcpy(tr->synth.blobs, blobs, 5 * n_blobs * sizeof(float), cudaMemcpyHostToDevice), "blobs copy");
    if (st == TN_OK) st = cuda_status(cudaMemcpy(tr->synth.waves, waves, 12 * sizeof(float), cudaMemcpyHostToDevice), "waves copy");
    tr->synth.n_blobs = n_blobs;
    return st;
}

int tn_trainer_set_grid(tn_trainer* tr, const float* density, const uint8_t* bitfield) {
    TN_NONNULL(tr);
    const size_t L = (size_t)tr->d.grid.n_levels;
    int st = settle(tr);  // a head computed ahead read the old grid
    if (density) st = cuda_status(cudaMemcpyAsync(tr->density, density, L * tr->V * sizeof(float), cudaMemcpyHostToDevice, tr->stream), "density copy");
    if (st == TN_OK && bitfield) st = cuda_status(cudaMemcpyAsync(tr->bits, bitfield, tr->V, cudaMemcpyHostToDevice, tr->stream), "bits copy");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "set_grid sync");
    return st;
}

int tn_trainer_use_hashgrid(tn_trainer* tr, const tn_hashgrid_desc* desc) {
    TN_NONNULL(tr);
    TN_REQUIRE(tr->d.path == TN_PATH_FUSED, TN_E_STATE, "the hash-grid network runs on the fused path");
    uint64_t n_hash = 0;
    uint32_t n_head = 0;
    int st = tn_hashgrid_n_params(desc, &n_hash, &n_head);
    if (st != TN_OK) return st;
    TN_REQUIRE(n_hash == tr->d.n_grid_params, TN_E_INVALID,
               "hash-grid entries take %llu parameters, the trainer's grid section %u",
               (unsigned long long)n_hash, tr->d.n_grid_params);
    TN_REQUIRE(n_head <= tr->d.n_mlp_params, TN_E_INVALID, "the heads take %u parameters, the trainer's MLP section %u",
               n_head, tr->d.n_mlp_params);
    st = settle(tr);
    if (st != TN_OK) return st;
    tn_network net{};
    void* handle = nullptr;
    st = hashnet_create(desc, tr->w, tr->B, std::max(tr->M, 1u), &net, &handle);
    if (st != TN_OK) return st;
    if (tr->hashnet) hashnet_destroy(tr->hashnet);
    tr->hashnet = handle;
    tr->net = net;
    drop_graphs(tr);  // the captured graphs hold the previous network's launches
    return cuda_status(cudaMemsetAsync(tr->g, 0, (size_t)tr->P * 4, tr->stream), "hash-grid: gradients");
}

int tn_trainer_init_synthetic_gradients(tn_trainer* tr, float std, uint32_t* n_touched_out) {
    TN_NONNULL(tr);
    const int fst = settle(tr);
    if (fst != TN_OK) return fst;
    const tn_trainer_desc& d = tr->d;
    cudaStream_t s = tr->stream;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    // one batch of samples from the current grid (rays of step 0)
    int st = cuda_status(cudaMemsetAsync(tr->state, 0, sizeof(StepState), s), "state clear");
    if (st == TN_OK)
        st = enqueue_own_rays(tr, s, tr->set[tr->cur]);
    uint32_t* info = tr->set[tr->cur].info;
    if (st == TN_OK)
        st = tn_march_count(tr->ctx, s, &grid, tr->bits, &d.bbox, &march, tr->R, tr->R, nullptr, tr->ori, tr->dir,
                            tr->ray_t, tr->ray_tmax, tr->alive, tr->n_steps, tr->B, info);
    if (st == TN_OK)
        st = tn_march_emit(tr->ctx, s, &grid, tr->bits, &d.bbox, &march, 1.0f / tr->aabb, tr->R, tr->R, tr->B, info,
                           nullptr, tr->ori, tr->dir, tr->ray_t, tr->alive, tr->n_steps, tr->offsets, nullptr, tr->s_t,
                           tr->s_pos, tr->s_dir, tr->s_dt, tr->s_mnorm, tr->s_dtnorm);
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(tr->g, 0, (size_t)tr->P * 4, s), "grad clear");
    // the reference's encoding: 16 levels, 2 features, 2^19 entries, base 16, max 2048 * aabb
    const int levels = 16, feats = 2;
    uint32_t log2_t = 19;
    while (log2_t > 0 && (uint64_t)levels * feats * (1ull << log2_t) > d.n_grid_params) --log2_t;
    const double n_max = 2048.0 * std::max(1.0, (double)tr->aabb);
    const float scale = (float)std::exp((std::log(n_max) - std::log(16.0)) / 15.0);
    if (st == TN_OK)
        st = launch_synth_hash_grads(s, tr->B, info + 1, tr->B, tr->s_pos, levels, log2_t, feats, 16.0f, scale, d.seed,
                                     std, tr->g);
    // every MLP weight gets a gradient too
    if (st == TN_OK && d.n_mlp_params) {
        std::vector<float> hg(d.n_mlp_params);
        uint32_t x = d.seed * 2654435761u + 1u;
        for (auto& v : hg) {
            x ^= x << 13; x ^= x >> 17; x ^= x << 5;
            v = std * (((float)(x >> 8) / 16777216.0f) * 2.0f - 1.0f) * 1.7320508f;
        }
        st = cuda_status(cudaMemcpyAsync(tr->g + d.n_grid_params, hg.data(), hg.size() * 4, cudaMemcpyHostToDevice, s), "mlp grads");
        if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "mlp grads sync");
    }
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(tr->state, 0, sizeof(StepState), s), "state clear");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "init grads sync");
    if (st == TN_OK && n_touched_out) {
        std::vector<float> hg(d.n_grid_params);
        st = cuda_status(cudaMemcpy(hg.data(), tr->g, hg.size() * 4, cudaMemcpyDeviceToHost), "grad read");
        uint32_t c = 0;
        for (float v : hg) c += v != 0.0f;
        *n_touched_out = c;
    }
    uint32_t flags = 0;
    if (st == TN_OK) st = tn_ctx_check(tr->ctx, s, &flags);
    return st;
}

// One fused step. Own rays with the count-ahead schedule: the head of this step was computed
// ahead by the previous step (or runs first here), and this step's tail runs beside the next
// step's head. Otherwise (caller rays, already copied into set cur ^ 1, or side_sms = 0) the
// head and the tail of the step run in order.
static int fused_step(tn_trainer* tr, bool external, tn_training_metrics* metrics) {
    int st = finish_pending(tr);
    if (st != TN_OK) return st;
    const int q = tr->cur ^ 1;
    if (!external && tr->lookahead()) {
        if (!tr->spec_own) st = enqueue_kind(tr, K_H, false, q, -1);
        if (st == TN_OK) st = enqueue_kind(tr, K_TH, false, q, -1);
        tr->spec_own = st == TN_OK;
    } else {
        st = drop_spec(tr);
        if (st == TN_OK) st = enqueue_kind(tr, K_HT, external, q, -1);
    }
    if (st != TN_OK) return st;
    tr->select(q);
    ++tr->fused_steps_enqueued;
    if (metrics) return read_state(tr, metrics);
    return TN_OK;
}

static int train_step_impl(tn_trainer* tr, bool external, tn_training_metrics* metrics) {
    if (tr->d.path == TN_PATH_PLAIN) return run_plain_step(tr, external, metrics);
    return fused_step(tr, external, metrics);
}

int tn_trainer_train_step(tn_trainer* tr, tn_training_metrics* metrics) {
    TN_NONNULL(tr);
    return train_step_impl(tr, false, metrics);
}

int tn_trainer_train_step_rays(tn_trainer* tr, uint32_t n_rays, const float* ori, const float* dir,
                               const float* target_rgba, const float* bg_rgb, tn_training_metrics* metrics) {
    TN_NONNULL(tr); TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(target_rgba); TN_NONNULL(bg_rgb);
    TN_REQUIRE(n_rays == tr->R, TN_E_INVALID, "tn_trainer_train_step_rays: n_rays must equal n_rays_per_step (%u)", tr->R);
    int st = settle(tr);
    if (st != TN_OK) return st;
    // the plain path steps in the current set; the fused path takes the step's head into the other
    RaySet& q = tr->set[tr->d.path == TN_PATH_PLAIN ? tr->cur : tr->cur ^ 1];
    cudaStream_t s = tr->stream;
    const size_t row = (size_t)n_rays * sizeof(float);
    st = cuda_status(cudaMemcpy2DAsync(q.ori, row, ori, row, row, 3, cudaMemcpyHostToDevice, s), "rays H2D");
    if (st == TN_OK) st = cuda_status(cudaMemcpy2DAsync(q.dir, row, dir, row, row, 3, cudaMemcpyHostToDevice, s), "rays H2D");
    if (st == TN_OK) st = cuda_status(cudaMemcpy2DAsync(q.target, row, target_rgba, row, row, 4, cudaMemcpyHostToDevice, s), "rays H2D");
    if (st == TN_OK) st = cuda_status(cudaMemcpy2DAsync(q.bg, row, bg_rgb, row, row, 3, cudaMemcpyHostToDevice, s), "rays H2D");
    if (st != TN_OK) return st;
    return train_step_impl(tr, true, metrics);
}

int tn_trainer_train_step_rays_pipelined(tn_trainer* tr, uint32_t n_rays, const float* ori, const float* dir,
                                         const float* target_rgba, const float* bg_rgb,
                                         tn_training_metrics* previous) {
    TN_NONNULL(tr); TN_NONNULL(previous);
    TN_NONNULL(ori); TN_NONNULL(dir); TN_NONNULL(target_rgba); TN_NONNULL(bg_rgb);
    TN_REQUIRE(tr->d.path == TN_PATH_FUSED, TN_E_STATE, "pipelined steps run on the fused path");
    TN_REQUIRE(n_rays == tr->R, TN_E_INVALID, "tn_trainer_train_step_rays_pipelined: n_rays must equal n_rays_per_step (%u)",
               tr->R);
    int st = drop_spec(tr);
    if (st != TN_OK) return st;
    cudaStream_t s = tr->stream;
    // The new step's head goes into the set that no step in flight uses: with a step pending,
    // the set of the last completed step (the pending step's tail runs on the other one, and
    // the previous call waited for the step before it). The host rays are copied straight into
    // it on the copy stream, beside whatever the step stream is still running; the step waits
    // for the copy.
    const bool has_prev = tr->pending_ext;
    const int p = tr->cur ^ 1;
    RaySet& dst = tr->set[has_prev ? tr->cur : p];
    const int slot = (int)(tr->ring_calls & 1u);
    const size_t R = n_rays;
    const float* src[4] = {ori, dir, target_rgba, bg_rgb};
    float* to[4] = {dst.ori, dst.dir, dst.target, dst.bg};
    const size_t len[4] = {3 * R, 3 * R, 4 * R, 3 * R};
    for (int k = 0; k < 4 && st == TN_OK; ++k)
        st = cuda_status(cudaMemcpyAsync(to[k], src[k], len[k] * sizeof(float), cudaMemcpyHostToDevice, tr->h2d),
                         "rays H2D");
    if (st == TN_OK) st = cuda_status(cudaEventRecord(tr->ev_staged[slot], tr->h2d), "staged");
    if (st == TN_OK) st = cuda_status(cudaStreamWaitEvent(s, tr->ev_staged[slot], 0), "wait staged");
    if (st != TN_OK) return st;
    ++tr->ring_calls;
    if (!has_prev) {
        // first call: the step's head only; its tail runs beside the next call's head
        st = enqueue_kind(tr, K_H, true, p, -1);
        if (st != TN_OK) return st;
        tr->pending_ext = true;
        *previous = tn_training_metrics{};
        return TN_OK;
    }
    // the pending step's tail beside this step's head; its state is copied to ring slot p
    constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    tr->ring_flag[p] = kEmpty;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    st = enqueue_kind(tr, K_TH, true, p, p);
    if (st != TN_OK) return st;
    tr->select(p);
    ++tr->fused_steps_enqueued;
    // wait for the pending step only (this step's head may still be marching): the slot's flag,
    // or the end of everything queued, whichever comes first; a failed stream ends the wait. The
    // flag is read many times between two queries of the stream.
    while (tr->ring_flag[p] == kEmpty) {
        for (int spin = 0; spin < 256 && tr->ring_flag[p] == kEmpty; ++spin) std::this_thread::yield();
        if (tr->ring_flag[p] != kEmpty) break;
        const cudaError_t q = cudaStreamQuery(s);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) return cuda_status(q, "previous step");
    }
    std::atomic_thread_fence(std::memory_order_seq_cst);
    if (tr->ring_flag[p] == kEmpty) return fail(TN_E_CUDA, "previous step: its state never arrived");
    return metrics_from(tr, tr->ring_state[p], previous);
}

// Holds a stream until the host has enqueued everything behind it (at most a second), so that
// the stages after it run back to back, as in the captured step, without gaps for host launches.
struct StreamGate {
    std::mutex mu;
    std::condition_variable cv;
    bool open = false;
    static void CUDART_CB wait(void* self) {
        auto* g = static_cast<StreamGate*>(self);
        std::unique_lock<std::mutex> lock(g->mu);
        g->cv.wait_for(lock, std::chrono::seconds(1), [g] { return g->open; });
    }
    void release() {
        {
            std::lock_guard<std::mutex> lock(mu);
            open = true;
        }
        cv.notify_all();
    }
};

int tn_trainer_profile_step(tn_trainer* tr, float* stage_ms, uint32_t max_stages, uint32_t* n_stages) {
    TN_NONNULL(tr); TN_NONNULL(stage_ms);
    TN_REQUIRE(tr->d.path == TN_PATH_FUSED, TN_E_STATE, "stage timing covers the fused path");
    // the timed step runs alone and in order
    const int fst = settle(tr);
    if (fst != TN_OK) return fst;
    const int q = tr->cur ^ 1;
    cudaEvent_t ev[ST_N + 1];
    for (auto& e : ev) cudaEventCreate(&e);
    StreamGate gate;
    int st = cuda_status(cudaLaunchHostFunc(tr->stream, StreamGate::wait, &gate), "profile gate");
    if (st == TN_OK) st = enqueue_profiled_step(tr, q, ev);
    gate.release();
    if (st == TN_OK) st = cuda_status(cudaEventSynchronize(ev[ST_N]), "profile sync");
    else cudaStreamSynchronize(tr->stream);  // the gate must not outlive this frame
    const uint32_t n = std::min<uint32_t>(max_stages, ST_N);
    for (uint32_t k = 0; k < n && st == TN_OK; ++k) cudaEventElapsedTime(&stage_ms[k], ev[k], ev[k + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (st == TN_OK) tr->select(q);
    ++tr->fused_steps_enqueued;
    if (n_stages) *n_stages = n;
    return st;
}

// Releases the captured step graphs; the next steps run eagerly once and capture them again
// (after a change of launch shapes, ray source or alpha selection).
static void drop_graphs(tn_trainer* tr) {
    for (int k = 0; k < K_KINDS; ++k)
        for (int r = 0; r < 2; ++r)
            for (int p = 0; p < 2; ++p)
                for (int a = 0; a < 2; ++a) {
                    if (tr->graph_exec[k][r][p][a]) cudaGraphExecDestroy(tr->graph_exec[k][r][p][a]);
                    if (tr->graph[k][r][p][a]) cudaGraphDestroy(tr->graph[k][r][p][a]);
                    tr->graph_exec[k][r][p][a] = nullptr;
                    tr->graph[k][r][p][a] = nullptr;
                    tr->warm[k][r][p][a] = false;
                }
}

int tn_trainer_set_dataset(tn_trainer* tr, uint32_t n_images, int32_t width, int32_t height, const tn_camera* cameras,
                           const uint8_t* images) {
    TN_NONNULL(tr); TN_NONNULL(cameras); TN_NONNULL(images);
    int st = check_dataset(n_images, width, height);
    if (st != TN_OK) return st;
    st = settle(tr);  // a head computed ahead took the old ray source
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "tn_trainer_set_dataset");
    if (st != TN_OK) return st;
    const size_t texels = (size_t)n_images * (size_t)width * (size_t)height;
    tn_camera* cams = nullptr;
    uint8_t* imgs = nullptr;
    st = tr->alloc(cams, n_images);
    if (st == TN_OK) st = tr->alloc(imgs, 4 * texels);
    for (int k = 0; k < 2; ++k)
        if (st == TN_OK && !tr->set[k].ds_random) st = tr->alloc(tr->set[k].ds_random, 2 * (size_t)tr->R);
    if (st == TN_OK)
        st = cuda_status(cudaMemcpyAsync(cams, cameras, n_images * sizeof(tn_camera), cudaMemcpyHostToDevice, tr->stream),
                         "dataset cameras");
    if (st == TN_OK)
        st = cuda_status(cudaMemcpyAsync(imgs, images, 4 * texels, cudaMemcpyHostToDevice, tr->stream), "dataset images");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "dataset upload");
    if (st != TN_OK) return st;
    tr->ds_cameras = cams;
    tr->ds_images = imgs;
    tr->ds_n = n_images;
    tr->ds_w = width;
    tr->ds_h = height;
    drop_graphs(tr);  // the next step captures the dataset rays
    return TN_OK;
}

int tn_trainer_set_alpha_selection(tn_trainer* tr, float threshold, float probability) {
    TN_NONNULL(tr);
    TN_REQUIRE(threshold == threshold && probability == probability, TN_E_INVALID, "alpha selection: NaN");
    if (threshold == tr->alpha_threshold && probability == tr->alpha_probability) return TN_OK;
    const int st = settle(tr);  // a head computed ahead selected its rays with the old values
    if (st != TN_OK) return st;
    tr->alpha_threshold = threshold;
    tr->alpha_probability = probability;
    drop_graphs(tr);  // kernel parameters of the captured step
    return cuda_status(cudaStreamSynchronize(tr->stream), "tn_trainer_set_alpha_selection");
}

int tn_trainer_autotune(tn_trainer* tr, tn_tune_report* reports) {
    TN_NONNULL(tr);
    TN_REQUIRE(tr->d.path == TN_PATH_FUSED, TN_E_STATE, "tn_trainer_autotune: the fused path only");
    const int fst = settle(tr);  // the tuners rewrite the march context's scratch
    if (fst != TN_OK) return fst;
    cudaStream_t s = tr->stream;
    const tn_trainer_desc& d = tr->d;
    const tn_grid_desc grid = tr->grid();
    const tn_march_desc march = tr->march();
    int st = cuda_status(cudaStreamSynchronize(s), "tn_trainer_autotune");
    // before the first step the ray buffers are empty: generate the first step's rays
    if (st == TN_OK && tr->fused_steps_enqueued == 0)
        st = enqueue_own_rays(tr, s, tr->set[tr->cur]);
    uint32_t* info = tr->set[tr->cur].info;
    tn_tune_report rep[3] = {};
    if (st == TN_OK)
        st = tn_autotune_march(tr->ctx, s, &grid, tr->bits, &d.bbox, &march, 1.0f / tr->aabb, tr->R, tr->R, nullptr,
                               tr->ori, tr->dir, tr->ray_t, tr->ray_tmax, tr->alive, tr->n_steps, tr->B, info, tr->B,
                               tr->offsets, nullptr, tr->s_t, tr->s_pos, tr->s_dir, tr->s_dt, tr->s_mnorm,
                               tr->s_dtnorm, &rep[0], &rep[1]);
    if (st == TN_OK)
        st = tr->net.forward(tr->net.user, s, tr->B, info + 1, tr->B, tr->s_pos, tr->s_dir, tr->net_density,
                             tr->net_rgb);
    if (st == TN_OK) st = cuda_status(cudaMemsetAsync(tr->grad_density, 0, (size_t)tr->B * 4, s), "grad memset");
    tn_ray_batch rb{tr->R, tr->R, tr->B, 0, tr->n_steps, tr->offsets, info};
    if (st == TN_OK)
        st = tn_autotune_losses(tr->ctx, s, &rb, tr->net.activation, d.min_transmittance, 0.0f, info, d.loss_scale,
                                d.use_distortion_loss ? d.distortion_lambda : 0.0f, tr->net_density, tr->net_rgb,
                                tr->s_dt, tr->s_mnorm, tr->s_dtnorm, tr->s_t, tr->target, tr->bg, nullptr,
                                tr->grad_density, tr->dl_drgb, tr->state->loss_sums, &rep[2]);
    // both march contexts take the chosen shapes
    if (st == TN_OK) st = tn_ctx_set_tuning(tr->set[tr->cur ^ 1].ctx, &tr->ctx->tune);
    drop_graphs(tr);  // the captured step graphs hold the previous shapes
    if (reports)
        for (int k = 0; k < 3; ++k) reports[k] = rep[k];
    return st;
}

int tn_trainer_flush(tn_trainer* tr) {
    TN_NONNULL(tr);
    int st = settle(tr, true);
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "tn_trainer_flush");
    return st;
}

namespace {

// The AABB scale of the reference's header: the edge of the training box (a whole number there).
uint32_t turbo_aabb_scale(const tn_trainer* tr) { return (uint32_t)std::lround(tr->aabb); }

struct FileCloser {
    FILE* f;
    ~FileCloser() { if (f) std::fclose(f); }
};

}  // namespace

int tn_trainer_save(tn_trainer* tr, const char* path, const char* dataset_path) {
    TN_NONNULL(tr); TN_NONNULL(path);
    int st = settle(tr, true);
    if (st != TN_OK) return st;
    const size_t P = tr->P, V = tr->V, LV = (size_t)tr->d.grid.n_levels * V;
    std::vector<float> w(P), m(P), v(P), density(LV);
    std::vector<uint32_t> steps(P);
    std::vector<uint8_t> bits(V);
    cudaStream_t s = tr->stream;
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        if (st == TN_OK) st = cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s), "save read");
    };
    d2h(w.data(), tr->w, P * 4); d2h(m.data(), tr->m, P * 4); d2h(v.data(), tr->v, P * 4);
    d2h(steps.data(), tr->steps, P * 4); d2h(density.data(), tr->density, LV * 4); d2h(bits.data(), tr->bits, V);
    d2h(tr->state_host, tr->state, sizeof(StepState));
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "save sync");
    if (st != TN_OK) return st;
    const StepState& h = *tr->state_host;
    TurboHeader hd{};
    std::strncpy(hd.project_name, "TurboNeRF", sizeof(hd.project_name));
    if (dataset_path) std::strncpy(hd.dataset_path, dataset_path, sizeof(hd.dataset_path) - 1);
    hd.version = 0;
    hd.n_color_params = tr->d.n_mlp_params;
    hd.n_density_params = tr->d.n_grid_params;
    hd.n_appearance_embedding_params = 0;
    hd.n_occ_grid_bits = (uint32_t)V;
    hd.aabb_scale = turbo_aabb_scale(tr);
    hd.n_appearances = 0;
    TurboResume r{};
    std::memcpy(r.magic, "TNRESUME", 8);
    r.version = 1;
    r.n_levels = (uint32_t)tr->d.grid.n_levels;
    r.resolution = (uint32_t)tr->d.grid.resolution;
    r.n_grid_params = tr->d.n_grid_params;
    r.n_mlp_params = tr->d.n_mlp_params;
    r.step_count = h.step_count;
    r.samples_total = h.samples_total;
    r.rays_total = h.rays_total;
    FileCloser fc{std::fopen(path, "wb")};
    if (!fc.f) return fail(TN_E_INVALID, "cannot create %s", path);
    bool ok = std::fwrite(&hd, sizeof(hd), 1, fc.f) == 1 && std::fwrite(w.data(), 4, P, fc.f) == P &&
              std::fwrite(bits.data(), 1, V, fc.f) == V && std::fwrite(&r, sizeof(r), 1, fc.f) == 1 &&
              std::fwrite(m.data(), 4, P, fc.f) == P && std::fwrite(v.data(), 4, P, fc.f) == P &&
              std::fwrite(steps.data(), 4, P, fc.f) == P && std::fwrite(density.data(), 4, LV, fc.f) == LV;
    ok = std::fclose(fc.f) == 0 && ok;
    fc.f = nullptr;
    return ok ? TN_OK : fail(TN_E_INVALID, "writing %s failed", path);
}

int tn_trainer_load(tn_trainer* tr, const char* path) {
    TN_NONNULL(tr); TN_NONNULL(path);
    TurboHeader hd;
    TurboResume r;
    bool has = false;
    uint64_t size = 0;
    int st = read_turbo_file(path, &hd, &r, &has, &size);
    if (st != TN_OK) return st;
    const size_t P = tr->P, V = tr->V, LV = (size_t)tr->d.grid.n_levels * V;
    TN_REQUIRE(hd.n_density_params == tr->d.n_grid_params && hd.n_color_params == tr->d.n_mlp_params &&
                   hd.n_appearance_embedding_params == 0,
               TN_E_INVALID, "%s holds %u + %u + %u parameters; the trainer has %u (hash grid) + %u (MLP)", path,
               hd.n_density_params, hd.n_color_params, hd.n_appearance_embedding_params, tr->d.n_grid_params,
               tr->d.n_mlp_params);
    TN_REQUIRE(hd.n_occ_grid_bits == V, TN_E_INVALID, "%s holds a %u-byte bitfield; the trainer's grid has %zu cells",
               path, hd.n_occ_grid_bits, V);
    TN_REQUIRE(hd.aabb_scale == turbo_aabb_scale(tr), TN_E_INVALID, "%s: AABB scale %u, the trainer's box is %u",
               path, hd.aabb_scale, turbo_aabb_scale(tr));
    if (has) {
        TN_REQUIRE(r.n_levels == (uint32_t)tr->d.grid.n_levels && r.resolution == (uint32_t)tr->d.grid.resolution &&
                       r.n_grid_params == tr->d.n_grid_params && r.n_mlp_params == tr->d.n_mlp_params,
                   TN_E_INVALID, "%s: resume block of a %u-level %u^3 grid; the trainer has %d levels of %d^3", path,
                   r.n_levels, r.resolution, tr->d.grid.n_levels, tr->d.grid.resolution);
        const uint64_t need = sizeof(TurboHeader) + 4ull * P + V + sizeof(TurboResume) + 12ull * P + 4ull * LV;
        TN_REQUIRE(size >= need, TN_E_INVALID, "%s: resume block truncated (%llu bytes of %llu)", path,
                   (unsigned long long)size, (unsigned long long)need);
    }
    std::vector<float> w(P), m, v, density;
    std::vector<uint32_t> steps;
    std::vector<uint8_t> bits(V);
    FileCloser fc{std::fopen(path, "rb")};
    if (!fc.f) return fail(TN_E_INVALID, "cannot open %s", path);
    bool ok = std::fseek(fc.f, (long)sizeof(TurboHeader), SEEK_SET) == 0 && std::fread(w.data(), 4, P, fc.f) == P &&
              std::fread(bits.data(), 1, V, fc.f) == V;
    if (ok && has) {
        m.resize(P); v.resize(P); steps.resize(P); density.resize(LV);
        ok = std::fseek(fc.f, (long)sizeof(TurboResume), SEEK_CUR) == 0 && std::fread(m.data(), 4, P, fc.f) == P &&
             std::fread(v.data(), 4, P, fc.f) == P && std::fread(steps.data(), 4, P, fc.f) == P &&
             std::fread(density.data(), 4, LV, fc.f) == LV;
    }
    if (!ok) return fail(TN_E_INVALID, "reading %s failed", path);
    // a requested step completes on the old state; a head computed ahead read the old grid
    st = settle(tr);
    cudaStream_t s = tr->stream;
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "load sync");
    auto h2d = [&](void* dst, const void* src, size_t bytes) {
        if (st == TN_OK) st = cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s), "load write");
    };
    h2d(tr->w, w.data(), P * 4);
    h2d(tr->bits, bits.data(), V);
    StepState& h = *tr->state_host;
    h = StepState{};
    if (has) {
        h2d(tr->m, m.data(), P * 4); h2d(tr->v, v.data(), P * 4); h2d(tr->steps, steps.data(), P * 4);
        h2d(tr->density, density.data(), LV * 4);
        h.step_count = r.step_count;
        h.samples_total = r.samples_total;
        h.rays_total = r.rays_total;
        h.cur_step = r.step_count ? r.step_count - 1u : 0u;
    }
    h2d(tr->state, &h, sizeof(StepState));
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "load sync");
    if (st != TN_OK) return st;
    tr->host_step = h.step_count;
    tr->last = tn_training_metrics{};
    tr->last.step = h.step_count;
    tr->ring_calls = 0;
    return TN_OK;
}

// NeRFTrainingController::reset_training (src/controllers/nerf-training-controller.cu:108-120):
// the reference frees the network's training data, the occupancy grid, the parameters and the
// workspace, then runs setup_data again, which re-creates them as at the start of training
// (parameters from the fixed seed, fresh optimizer state, every grid bit set, densities zero,
// training_step = 0). Here the buffers are kept and rewritten to that state; the captured step
// graphs stay valid, since they only hold the buffers' addresses. A pending caller-ray step
// completes first and a head counted ahead is dropped. The gradient source of the built-in
// stand-in network (its fixed synthetic gradients) is the network's, not the trainer's, and is
// kept.
int tn_trainer_reset(tn_trainer* tr) {
    TN_NONNULL(tr);
    cudaStream_t s = tr->stream;
    int st = settle(tr);
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->h2d), "reset sync");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->aux), "reset sync");
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "reset sync");
    const size_t P = tr->P, V = tr->V, LV = (size_t)tr->d.grid.n_levels * V;
    auto clear = [&](void* p, int value, size_t bytes) {
        if (st == TN_OK) st = cuda_status(cudaMemsetAsync(p, value, bytes, s), "reset clear");
    };
    clear(tr->bits, 0xFF, V);  // occupancy-grid.cuh:81-85
    clear(tr->density, 0, LV * 4);
    clear(tr->m, 0, P * 4);
    clear(tr->v, 0, P * 4);
    clear(tr->steps, 0, P * 4);
    clear(tr->state, 0, sizeof(StepState));
    for (int k = 0; k < 2; ++k) clear(tr->set[k].ctx->flags, 0, sizeof(uint32_t));
    if (st == TN_OK) st = launch_synth_params(s, (uint32_t)P, tr->d.n_grid_params, tr->d.seed, tr->w);
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "reset sync");
    if (st != TN_OK) return st;
    tr->host_step = 0;
    tr->last = tn_training_metrics{};
    tr->ring_calls = 0;
    return TN_OK;
}

int tn_trainer_render(tn_trainer* tr, const tn_camera* camera, const tn_bbox* render_bbox, float min_step_size,
                      uint32_t batch_size, float* out_rgba, tn_render_stats* stats) {
    TN_NONNULL(tr);
    int st = settle(tr, true);
    if (st != TN_OK) return st;
    tn_render_desc rd{};
    rd.grid = tr->d.grid;
    rd.bitfield = tr->bits;
    rd.training_bbox = tr->d.bbox;
    rd.render_bbox = render_bbox ? *render_bbox : tr->d.bbox;
    rd.dt_min = min_step_size > 0.0f ? min_step_size : tr->d.min_step_size;
    rd.cone_angle = tr->d.cone_angle;
    rd.min_transmittance = tr->d.min_transmittance;
    rd.batch_size = batch_size;
    return tn_render(tr->ctx, tr->stream, &rd, camera, &tr->net, out_rgba, stats);
}

int tn_trainer_get_tuning(tn_trainer* tr, tn_tuning* out) {
    TN_NONNULL(tr);
    return tn_ctx_get_tuning(tr->ctx, out);
}

int tn_trainer_set_tuning(tn_trainer* tr, const tn_tuning* t) {
    TN_NONNULL(tr);
    int st = settle(tr);  // a head computed ahead ran with the old shapes
    if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "tn_trainer_set_tuning");
    for (int k = 0; k < 2 && st == TN_OK; ++k) st = tn_ctx_set_tuning(tr->set[k].ctx, t);
    if (st == TN_OK) drop_graphs(tr);
    return st;
}

int tn_trainer_stat(tn_trainer* tr, int which, uint64_t* out) {
    TN_NONNULL(tr); TN_NONNULL(out);
    switch (which) {
        // the step graph of own rays (tail beside the next head, or the in-order step) and of
        // caller rays (the pipelined or the synchronous call)
        case 0: *out = tr->graph_kernels[tr->lookahead() ? K_TH : K_HT][0]; return TN_OK;
        case 1: *out = tr->graph_kernels[K_TH][1] ? tr->graph_kernels[K_TH][1] : tr->graph_kernels[K_HT][1]; return TN_OK;
        case 2: *out = tr->graph_nodes[tr->lookahead() ? K_TH : K_HT][0]; return TN_OK;
        case 3:
        case 4:
        case 5: {
            int st = settle(tr, true);  // a requested step counts once its tail has run
            if (st == TN_OK)
                st = cuda_status(cudaMemcpyAsync(tr->state_host, tr->state, sizeof(StepState), cudaMemcpyDeviceToHost,
                                                 tr->stream), "stat");
            if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(tr->stream), "stat sync");
            if (st != TN_OK) return st;
            *out = which == 3 ? tr->state_host->samples_total
                 : which == 4 ? tr->state_host->rays_total : tr->state_host->step_count;
            return TN_OK;
        }
        default: return fail(TN_E_INVALID, "unknown trainer stat %d", which);
    }
}

int tn_trainer_sync_metrics(tn_trainer* tr, tn_training_metrics* metrics) {
    TN_NONNULL(tr);
    if (tr->d.path == TN_PATH_PLAIN) {
        int st = cuda_status(cudaStreamSynchronize(tr->stream), "sync");
        if (metrics) *metrics = tr->last;
        return st;
    }
    const int st = settle(tr, true);  // a requested caller-ray step runs its tail first
    return st == TN_OK ? read_state(tr, metrics) : st;
}

int tn_trainer_update_occupancy_grid(tn_trainer* tr, uint32_t training_step, tn_occupancy_metrics* metrics) {
    TN_NONNULL(tr);
    const int fst = settle(tr);  // a head computed ahead read the grid this rewrites
    if (fst != TN_OK) return fst;
    const tn_trainer_desc& d = tr->d;
    cudaStream_t s = tr->stream;
    const tn_grid_desc grid = tr->grid();
    const int sample_all = training_step < 256 ? 1 : 0;
    const bool plain = d.path == TN_PATH_PLAIN;
    int st = TN_OK;
    if (plain) st = launch_plain_occ_decay(s, &grid, tr->density, d.occupancy_decay);
    for (int level = 0; level < grid.n_levels && st == TN_OK; ++level) {
        for (uint32_t start = 0; start < tr->V && st == TN_OK; start += tr->chunk) {
            const uint32_t n = std::min(tr->chunk, tr->V - start);
            st = launch_synth_level_cells(s, n, start, level, d.seed, 0x20000000u + training_step, tr->occ_levels,
                                          tr->occ_cells, tr->occ_rand3, n, tr->occ_rsel);
            if (st == TN_OK)
                st = tn_occupancy_sample_points(s, &grid, n, tr->occ_levels, tr->occ_cells, tr->occ_rand3, n,
                                                1.0f / tr->aabb, tr->occ_pos, n);
            if (st == TN_OK) st = tr->net.density(tr->net.user, s, n, nullptr, n, tr->occ_pos, tr->occ_values);
            if (st == TN_OK) {
                st = plain ? launch_plain_occ_update(s, &grid, tr->density, tr->bits, n, tr->occ_levels, tr->occ_cells,
                                                     tr->occ_values, tr->occ_rsel, tr->net.activation, sample_all)
                           : launch_occupancy_scatter(s, &grid, tr->density, tr->bits, n, tr->occ_levels, tr->occ_cells,
                                                      tr->occ_values, tr->occ_rsel, tr->net.activation, sample_all,
                                                      d.occupancy_decay);
            }
        }
    }
    uint32_t nocc = 0;
    if (st == TN_OK) {
        if (plain) {
            st = launch_plain_occ_bits_sync(s, &grid, tr->density, tr->bits, d.occupancy_threshold, tr->count_scratch,
                                            &nocc);
        } else {
            st = launch_occupancy_sweep(s, &grid, tr->density, tr->bits, d.occupancy_decay, d.occupancy_threshold,
                                        &tr->state->n_occupied);
            if (st == TN_OK)
                st = cuda_status(cudaMemcpyAsync(&tr->state_host->n_occupied, &tr->state->n_occupied, 4,
                                                 cudaMemcpyDeviceToHost, s), "n_occupied");
            if (st == TN_OK) st = cuda_status(cudaStreamSynchronize(s), "occupancy sync");
            nocc = tr->state_host->n_occupied;
        }
    }
    if (st == TN_OK && metrics) {
        metrics->n_occupied = nocc;
        metrics->n_total = (uint32_t)grid.n_levels * tr->V;  // reference: n_levels * 128^3
    }
    return st;
}

int tn_trainer_stream(tn_trainer* tr, tn_stream_t* out) {
    TN_NONNULL(tr); TN_NONNULL(out);
    *out = tr->stream;
    return TN_OK;
}

int tn_trainer_buffer(tn_trainer* tr, int which, void** ptr, uint64_t* bytes) {
    TN_NONNULL(tr); TN_NONNULL(ptr);
    // the state the caller reads includes every requested step
    int fst = settle(tr, true);
    if (fst == TN_OK) fst = cuda_status(cudaStreamSynchronize(tr->stream), "tn_trainer_buffer");
    if (fst != TN_OK) return fst;
    const uint64_t R = tr->R, B = tr->B, V = tr->V, P = tr->P, L = (uint64_t)tr->d.grid.n_levels;
    void* p = nullptr;
    uint64_t n = 0;
    switch (which) {
        case 0: p = tr->w; n = 4 * P; break;
        case 1: p = tr->g; n = 4 * P; break;
        case 2: p = tr->m; n = 4 * P; break;
        case 3: p = tr->v; n = 4 * P; break;
        case 4: p = tr->steps; n = 4 * P; break;
        case 5: p = tr->density; n = 4 * L * V; break;
        case 6: p = tr->bits; n = V; break;
        case 7: p = tr->s_t; n = 4 * B; break;
        case 8: p = tr->s_pos; n = 12 * B; break;
        case 9: p = tr->s_dt; n = 4 * B; break;
        case 10: p = tr->offsets; n = 4 * R; break;
        case 11: p = tr->n_steps; n = 4 * R; break;
        case 12: p = tr->state->batch_info; n = 16; break;
        case 13: p = tr->net_density; n = 4 * B; break;
        case 14: p = tr->net_rgb; n = 12 * B; break;
        case 15: p = tr->grad_density; n = 4 * B; break;
        case 16: p = tr->dl_drgb; n = 12 * B; break;
        case 17: p = tr->ori; n = 12 * R; break;
        case 18: p = tr->dir; n = 12 * R; break;
        case 19: p = tr->ray_t; n = 4 * R; break;
        case 20: p = tr->ray_tmax; n = 4 * R; break;
        case 21: p = tr->alive; n = R; break;
        case 22: p = tr->target; n = 16 * R; break;
        case 23: p = tr->bg; n = 12 * R; break;
        case 24: p = tr->s_mnorm; n = 4 * B; break;
        case 25: p = tr->s_dtnorm; n = 4 * B; break;
        case 26: p = tr->set[tr->cur].ds_random; n = p ? 8 * R : 0; break;
        case 27: p = tr->occ_levels; n = 4ull * tr->M; break;
        case 28: p = tr->occ_cells; n = 4ull * tr->M; break;
        case 29: p = tr->occ_values; n = 4ull * tr->M; break;
        case 30: p = tr->occ_rsel; n = 4ull * tr->M; break;
        case 31: {  // the hash-grid network's touched-entry list and its count
            const uint32_t* list = nullptr;
            const uint32_t* count = tr->hashnet ? hashnet_touched(tr->hashnet, &list) : nullptr;
            p = const_cast<uint32_t*>(list);
            n = list ? 4ull * (tr->d.n_grid_params / 2) : 0;
            (void)count;
            break;
        }
        case 32: {
            p = tr->hashnet ? const_cast<uint32_t*>(hashnet_touched(tr->hashnet, nullptr)) : nullptr;
            n = p ? 4 : 0;
            break;
        }
        default: return fail(TN_E_INVALID, "unknown trainer buffer %d", which);
    }
    *ptr = p;
    if (bytes) *bytes = n;
    return TN_OK;
}

}  // extern "C"
