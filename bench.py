"""Benchmark of the TurboNeRF training hot path on B200: samples/s of the full train step.

Workload (one step): 2^14 synthetic rays (origins on a radius-4 sphere, directions toward
the centre + N(0, 0.05)) through a 5-cascade 128^3 occupancy grid built from an 8-blob
Gaussian field (base size 1: extents 1..16) -> march count + batch cut at 2^18 samples ->
march emit -> field (network stand-in) -> reconstruction + distortion (lambda 1e-3) loss
forward/backward with the gradient merge -> Adam (beta1 0.9, beta2 0.99, eps 1e-15,
lr 1e-2) over 16 x 2^19 x 2 hash-grid + 7168 MLP parameters with fixed sparse synthetic
gradients -> occupancy EMA (decay 0.95, threshold 0.01, 2^16 random cells re-sampled).

Prints ONE JSON line. `value` = samples/s of the fused, CUDA-graph-captured step with
inputs resident in HBM; `e2e` = the same through Trainer.train_step_rays_pipelined() with each
step's host rays copied in and its metrics copied back and read by the host (one step later, the
last one inside the timed region); `plain` = the one-kernel-per-stage path.
`--impl reference` times the reference's own kernels compiled on the host cores (oracle/_ref,
OpenMP) on the same workload instead, or the oracle's restatement where that library is not
built.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "train-step samples/s fused vs plain on 1 B200 (grad err ≤1e-4); % HBM roofline"
WORKLOAD = "full single-scene train step, CUDA graph: 5x128^3 cascades, 2^18 samples/step from 2^14 rays"
BATCH = 1 << 18
RAYS = 1 << 14
OCC_CELLS = 1 << 16
N_GRID = 16 * (1 << 19) * 2
N_MLP = 7168
LAMBDA = 1e-3
THRESHOLD = 0.01


def _env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _scene(seed):
    from turbonerf_b200 import scenes
    return scenes.march_scene_cascaded(seed=seed, n_rays=64, n_levels=5)


def _trainer(scene, path, seed):
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    tr = Trainer(SyntheticNeRF.from_scene(scene), path=path, use_cuda_graph=(path == "fused"), n_rays_per_step=RAYS,
                 occupancy_cells_per_step=OCC_CELLS, distortion_lambda=LAMBDA, occupancy_threshold=THRESHOLD,
                 n_grid_params=N_GRID, n_mlp_params=N_MLP, beta2=0.99, seed=seed)
    tr.use_distortion_loss = True
    tr.setup_data(batch_size=BATCH, synthetic_grad_std=1e-3)
    return tr


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region (read only). NVML is
    polled every 2 ms from a thread, so even a region of a few ms gets samples; without NVML,
    nvidia-smi at its shortest interval. The device is found by its PCI bus id."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []  # (sm MHz, max MHz, set of reasons)
        self.stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.index)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except pynvml.NVMLError:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _poll(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self.stop.is_set():
            sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, mx, {k for k, b in bits.items() if r & b}))
            time.sleep(0.002)

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.nvml.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 2.0:
                time.sleep(0.001)
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:
                time.sleep(0.005)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.nvml:
            self.stop.set()
            self.nvml.join(timeout=2)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        for s_mhz, m_mhz, rs in self.samples:
            sm.append(s_mhz)
            mx = max(mx, m_mhz)
            reasons |= rs
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(self.NAMES):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml" if self.samples else "nvidia-smi"}


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def stage_bytes(n_rays_gen, n_rays, n_samples, n_touched, levels=5, volume=128 ** 3):
    """Algorithmic HBM bytes of each fused stage for one step (what the stage must move)."""
    P = N_GRID + N_MLP
    return {
        "rays": n_rays_gen * (12 + 12 + 16 + 12 + 9),                    # write ori, dir, target, bg, t, t_max, alive
        "march_count": n_rays_gen * (24 + 8 + 1 + 4),                    # read o, d, t, t_max, alive; write count
        "march_emit": n_rays_gen * 37 + n_samples * 40,                  # ray reads + 10 floats per sample
        "network_forward": n_samples * (12 + 16),                        # read pos, write sigma + rgb
        "losses": n_samples * (4 + 12 + 4 + 4 + 4 + 4 + 8 + 12) + n_rays * 36,
        "network_backward": 0,
        "occupancy_query": OCC_CELLS * (4 + 4 + 12 + 4 + 12 + 4),       # cells, levels, rand3, select; pos; sigma
        "occupancy": levels * volume * 8 + volume + OCC_CELLS * 48,      # sweep RMW + bits + scatter inputs
        "adam": 4 * P + 32 * (n_touched + N_MLP),                        # gradient read + RMW of touched params
    }


STAGES = ["rays", "march_count", "march_emit", "network_forward", "losses", "network_backward", "adam",
          "occupancy_query", "occupancy"]

# DRAM bytes (read + write) of one launch of each stage's main kernel on this workload, measured
# with ncu (dram__bytes_read.sum + dram__bytes_write.sum, one pass, after the warm-up steps).
NCU_TRAFFIC = {"march_count": 1_138_944, "march_emit": 1_285_376, "losses": 9_637_888, "adam": 304_766_208,
               "occupancy": 50_338_304}
# The same for the compositor tile kernels on the 2^22-sample batch (the `--workload compositor`
# capture: DRAM read + write of the first forward and the first VJP launch).
NCU_TRAFFIC_COMPOSITE = {"composite_fwd_tiles": 87_796_224, "composite_bwd_tiles": 113_915_904}


class L2Flush:
    """Flushes the L2 (126 MB) between timed launches, outside the timed region: a 256 MB write,
    then a 256 MB read of a second buffer. The read evicts the dirty lines of the write, so the
    timed launch does not pay for writing them back (as under ncu, whose cache control leaves
    clean caches); its DRAM traffic is its own."""

    def __init__(self):
        import torch
        self.w = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
        self.r = torch.ones(64 << 20, dtype=torch.float32, device="cuda")
        self.s = torch.empty((), dtype=torch.float32, device="cuda")

    def __call__(self):
        import torch
        self.w.fill_(1.0)
        torch.sum(self.r, dim=0, out=self.s)


def compositor_rooflines(peak, reps=20):
    """Roofline of the compositor's tile kernels (forward, VJP) on the compositor workload at 2^22
    samples (truncated geometric counts, mean 64, at most 1024: 65,571 rays): the L2 (126 MB) is
    flushed before every timed launch (L2Flush, outside the events), each launch timed with
    CUDA events, the median kept (a launch that meets another tenant's work on the shared GPU
    does not move it). Algorithmic bytes: forward 20 B/sample + 32 B/ray, VJP 36 B/sample
    + 24 B/ray."""
    import torch
    from turbonerf_b200 import hotpath as hp, scenes
    sb = scenes.make_sample_batch(0x7B5, 1 << 22, mean=64.0, max_count=1024)
    n, ss = sb.n_rays, sb.n_samples
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    counts, offsets = d(sb.counts.view(np.int32)), d(sb.offsets.view(np.int32))
    sig, rgb, dt = d(sb.sigma), d(sb.rgb), d(sb.dt)
    rb = hp.ray_batch(counts, offsets, n, n, ss)
    ctx = hp.Context(n, ss)
    g_rgba = torch.full((4 * n,), 1e-3, device="cuda")
    fo = hp.composite_fwd(ctx, rb, sig, rgb, dt)
    bo = hp.composite_bwd(ctx, rb, sig, rgb, dt, fo["depth"], fo["n_used"], g_rgba)
    flush = L2Flush()
    kernels = {
        "composite_fwd_tiles": (lambda: hp.composite_fwd(ctx, rb, sig, rgb, dt, out=fo), 20 * ss + 32 * n),
        "composite_bwd_tiles": (lambda: hp.composite_bwd(ctx, rb, sig, rgb, dt, fo["depth"], fo["n_used"], g_rgba,
                                                         out=bo), 36 * ss + 24 * n),
    }
    out = []
    for name, (fn, alg) in kernels.items():
        for _ in range(3):
            fn()
        times = []
        for _ in range(reps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = float(np.median(times))
        gbs = alg / (ms * 1e-3) / 1e9
        out.append({"kernel": name, "workload": f"compositor, 2^22 samples over {n} rays (mean 64), L2 flushed",
                    "bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s", "frac": round(gbs / peak, 4),
                    "traffic": NCU_TRAFFIC_COMPOSITE[name], "alg_bytes": int(alg), "ms": round(ms, 4)})
    assert ctx.check() == 0
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = _env_rank()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    from turbonerf_b200.replicas import barrier, job_throughput, replica_seed
    seed = replica_seed(0x7B0, rank)

    scene = _scene(0x7B0)
    tr = _trainer(scene, "fused", seed)
    stream = torch.cuda.ExternalStream(tr.stream_handle())
    # launch shapes of the march and the loss kernel, chosen on this trainer's own batch
    tuned = tr.autotune() if not args.no_autotune else {"tuning": tr.tuning}

    for _ in range(max(args.warmup, 3)):
        tr.train_step_async()
    tr.sync_metrics()
    s0 = tr.stat(3)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            tr.train_step_async()
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    last = tr.sync_metrics()
    samples = tr.stat(3) - s0
    rays_used = last.n_rays
    kernels_per_step = tr.stat(0)
    value, ms_max, _ = job_throughput(ms, samples, dev)

    # per-stage timing (eager step with events between stages), averaged
    prof = []
    for _ in range(5):
        prof.append(tr.profile_step())
    stage_ms = [float(np.median([p[i] for p in prof])) for i in range(len(STAGES))]
    m = tr.sync_metrics()

    result = None
    if rank == 0:
        peak, peak_kind = _peaks()
        sb = stage_bytes(RAYS, m.n_rays, m.n_samples, tr.n_touched_grads)
        stages = {}
        for i, name in enumerate(STAGES):
            b = sb[name]
            gbs = b / (stage_ms[i] / 1e3) / 1e9 if stage_ms[i] > 0 else 0.0
            stages[name] = {"ms": round(stage_ms[i], 4), "alg_bytes": int(b), "achieved_gbs": round(gbs, 1),
                            "frac": round(gbs / peak, 4)}
        dom = max(STAGES, key=lambda k: stages[k]["ms"])
        roofline = {"bound": "hbm", "kernel": dom, "achieved": stages[dom]["achieved_gbs"], "peak": peak,
                    "unit": "GB/s", "frac": round(stages[dom]["achieved_gbs"] / peak, 4),
                    "traffic": NCU_TRAFFIC.get(dom), "peak_source": peak_kind}
        result = dict(value=value, ms=ms_max, samples=samples, rays=rays_used, kernels=kernels_per_step,
                      clocks=clk.summary(), stages=stages, roofline=roofline, n_touched=tr.n_touched_grads,
                      last=dict(n_rays=m.n_rays, n_samples=m.n_samples, loss=m.loss),
                      rooflines=compositor_rooflines(peak))

    # e2e: public API with host rays (pinned) copied in and metrics read back every step
    from turbonerf_b200 import scenes
    rng = np.random.default_rng(seed + 1)
    n_batches = 4
    host = []
    for _ in range(n_batches):
        r = scenes.sphere_rays(rng, RAYS)
        tgt = np.concatenate([rng.uniform(0, 1, 3 * RAYS), np.ones(RAYS)]).astype(np.float32)
        bg = rng.uniform(0, 1, 3 * RAYS).astype(np.float32)
        host.append([torch.from_numpy(a).pin_memory() for a in (r.ori, r.dir, tgt, bg)])
    for i in range(max(args.warmup, 3)):
        tr.train_step_rays(*host[i % n_batches])
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0 = tr.stat(3)
    e0.record(stream)
    wall0 = time.perf_counter()
    # each call enqueues its step (rays in, state out) and reads the previous step's metrics;
    # the last step's metrics are read inside the timed region
    for i in range(args.steps):
        tr.train_step_rays_pipelined(*host[i % n_batches])
    last_m = tr.sync_metrics()
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - wall0
    e_ms = e0.elapsed_time(e1)
    e_samples = tr.stat(3) - s0
    assert last_m.step == tr.stat(5)
    e2e_value, _, _ = job_throughput(max(e_ms, wall * 1e3), e_samples, dev)
    tr.teardown()

    # plain path (reference launch structure) on the same workload
    plain = None
    if rank == 0 and not args.no_plain:
        trp = _trainer(scene, "plain", seed)
        for _ in range(max(args.warmup, 3)):
            trp.train_step()
        torch.cuda.synchronize()
        ps = torch.cuda.ExternalStream(trp.stream_handle())
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ss0 = trp.stat(3)
        k_plain = max(5, args.steps // 4)
        p0.record(ps)
        for _ in range(k_plain):
            trp.train_step()
        p1.record(ps)
        p1.synchronize()
        p_ms = p0.elapsed_time(p1)
        p_samples = trp.stat(3) - ss0
        plain = {"value": p_samples / (p_ms / 1e3), "ms_per_step": p_ms / k_plain, "steps": k_plain}
        trp.teardown()

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    cpu = None if args.no_cpu else cpu_baseline(seconds=args.cpu_seconds)
    others = None
    if world == 1 and not args.no_configs:
        try:
            others = other_configs(args)
        except Exception as e:  # a side measurement never takes the headline line with it
            others = {"error": f"{type(e).__name__}: {e}"}
    bi = RAYS * 4 * (3 + 3 + 4 + 3)
    line = {
        "metric": METRIC, "value": round(result["value"], 1), "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(result["ms"] / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch_size_samples": BATCH, "rays_per_step": RAYS, "cascades": 5,
                   "grid": "128^3", "occupancy_cells_per_step": OCC_CELLS, "hash_params": N_GRID, "mlp_params": N_MLP,
                   "distortion_lambda": LAMBDA, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (Adam state 268 MB + grid 42 MB touched per step)",
                   "samples_last_step": result["last"]["n_samples"], "rays_last_step": result["last"]["n_rays"],
                   "touched_hash_grads": result["n_touched"], "launch_shapes": tuned["tuning"],
                   "autotuned": not args.no_autotune},
        "e2e": {"value": round(e2e_value, 1), "unit": "samples/s", "h2d_bytes_per_step": bi, "d2h_bytes_per_step": 76},
        "gpu_launches": int(result["kernels"]) * args.steps,
        "roofline": result["roofline"],
        "rooflines": result["rooflines"],
        "stages": result["stages"],
        "clocks": result["clocks"],
        "plain": plain,
        "speedup_vs_plain": round(result["value"] / plain["value"], 2) if plain else None,
        "cpu_baseline": cpu,
        "other_configs": others,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# CPU: the oracle's restatement of the reference, one train step of the same workload
# ---------------------------------------------------------------------------------------
class CpuStep:
    def __init__(self, seed=0x7B0):
        import oracle
        from turbonerf_b200 import scenes
        self.o = oracle
        self.sc = _scene(0x7B0)
        self.rng = np.random.default_rng(seed)
        P = N_GRID + N_MLP
        g = np.zeros(P, np.float32)
        # same sparsity class as the GPU run: a fixed random half of the hash entries touched
        touched = self.rng.random(N_GRID) < 0.5
        g[:N_GRID][touched] = self.rng.normal(0, 1e-3, int(touched.sum())).astype(np.float32)
        g[N_GRID:] = self.rng.normal(0, 1e-3, N_MLP).astype(np.float32)
        self.grad = g
        self.adam = dict(w=self.rng.uniform(-1e-4, 1e-4, P), m=np.zeros(P), v=np.zeros(P),
                         steps=np.zeros(P, np.uint32))
        self.density = self.sc.grid.density.copy()
        self.bits = self.sc.grid.bitfield.copy()
        self.k = 0

    def step(self):
        from turbonerf_b200 import scenes
        o, sc = self.o, self.sc
        rays = scenes.rays_init_bbox(scenes.sphere_rays(self.rng, RAYS), sc.bbox)
        grid = dict(n_levels=5, res=128, base=1.0, bitfield=self.bits)
        march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=0)
        ns, alive, _ = o.march_count(rays.as_dict(), grid, march)
        st, off, nr, nsamp = o.scan_cut(ns, BATCH)
        em = o.march_emit(rays.as_dict(), grid, march, off, ns, alive, nr, BATCH, 1.0 / sc.aabb_size)
        sig, rgb = o.blob_field(em["pos"], BATCH, BATCH, sc.aabb_size, sc.field.blobs, sc.field.waves)
        tgt = np.concatenate([self.rng.uniform(0, 1, 3 * nr), np.ones(nr)]).astype(np.float32)
        bg = self.rng.uniform(0, 1, 3 * nr).astype(np.float32)
        counts = ns[:nr]
        rec = o.recon_fwd_bwd(counts, off[:nr], sig.astype(np.float32), rgb.astype(np.float32), em["dt"], tgt, bg,
                              nr, BATCH)
        _, ddist = o.distortion_fwd_bwd(counts, off[:nr], sig.astype(np.float32), em["m_norm"], em["dt_norm"], LAMBDA,
                                        BATCH)
        o.grad_epilogue(nsamp, 1.0, rec["dL_ddensity"][:nsamp], ddist[:nsamp], em["t"][:nsamp], np.zeros(nsamp))
        lv = self.rng.integers(0, 5, OCC_CELLS).astype(np.int32)
        cells = self.rng.integers(0, 128 ** 3, OCC_CELLS).astype(np.uint32)
        r3 = self.rng.random(3 * OCC_CELLS).astype(np.float32)
        pos = o.occupancy_sample_points(lv, cells, r3, OCC_CELLS, 128, 1.0, 1.0 / sc.aabb_size, OCC_CELLS)
        vals, _ = o.blob_field(pos, OCC_CELLS, OCC_CELLS, sc.aabb_size, sc.field.blobs, sc.field.waves, want_rgb=False)
        self.density, self.bits, _ = o.occupancy_update(self.density, self.bits, 5, 128, lv, cells,
                                                        vals.astype(np.float32), self.rng.random(OCC_CELLS).astype(
                                                            np.float32), sample_all=self.k < 256,
                                                        threshold=THRESHOLD)
        lr = 1e-2 / (1.0 + 3.3e-5 * self.k)
        o.adam_step(self.adam, self.grad, N_GRID, N_MLP, lr=lr, beta2=0.99)
        self.k += 1
        return nsamp


class RefCpuStep(CpuStep):
    """The same train step through the reference's own kernels compiled on the host
    (oracle/_ref: TurboNeRF's kernel sources, unchanged, with OpenMP over its CUDA threads):
    march count and emit, fused reconstruction loss forward/backward, distortion loss forward
    and backward, the gradient merge, the occupancy decay and threshold, the popcount and
    Adam. Between them, as in the reference's host code: the exclusive scan and batch cut (the
    reference: thrust), the stand-in network (the blob field), and the occupancy max-update of
    the sampled cells (the reference's kernel for it cannot be compiled on the host: its
    update_sigma_at returns nothing from a float function)."""

    def __init__(self, seed=0x7B0):
        super().__init__(seed)
        from oracle import ref
        self.r = ref
        self.w32 = self.adam["w"].astype(np.float32)
        P = self.w32.size
        self.m32, self.v32, self.s32 = np.zeros(P, np.float32), np.zeros(P, np.float32), np.zeros(P, np.uint32)
        self.w_copy = np.zeros(P, np.float32)

    def step(self):
        from turbonerf_b200 import scenes
        o, r, sc = self.o, self.r, self.sc
        rays = scenes.rays_init_bbox(scenes.sphere_rays(self.rng, RAYS), sc.bbox)
        rd = rays.as_dict()
        grid = dict(n_levels=5, res=128, base=1.0, bitfield=self.bits)
        march = dict(bbox=np.float32(sc.bbox), cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max)
        ns, alive = r.march_count(rd, grid, march)
        st, off, nr, nsamp = o.scan_cut(ns, BATCH)
        em = r.march_emit(rd, grid, march, off, ns, alive, nr, BATCH, 1.0 / sc.aabb_size)
        sig, rgb = o.blob_field(em["pos"], BATCH, BATCH, sc.aabb_size, sc.field.blobs, sc.field.waves)
        dens = (np.log(np.maximum(sig, 1e-30)) + 1.0).astype(np.float32)  # network density of that sigma
        tgt = np.zeros(4 * BATCH, np.float32)
        tgt[:3 * BATCH] = self.rng.uniform(0, 1, 3 * BATCH).astype(np.float32)
        tgt[3 * BATCH:3 * BATCH + nr] = 1.0
        bg = self.rng.uniform(0, 1, 3 * BATCH).astype(np.float32)
        counts = ns[:nr]
        rec = r.fused_reconstruction(counts, off[:nr], dens, rgb.astype(np.float32), em["dt"], tgt, bg, nr, BATCH)
        _, ddist = r.distortion(counts, off[:nr], dens, em["m_norm"], em["dt_norm"], BATCH)
        r.grad_merge(nsamp, 1.0, rec["dL_ddensity"], ddist, em["t"], np.zeros(BATCH, np.float32))
        # occupancy: decay (reference) -> sampled cells' max-update -> threshold (reference)
        lv = self.rng.integers(0, 5, OCC_CELLS).astype(np.int32)
        cells = self.rng.integers(0, 128 ** 3, OCC_CELLS).astype(np.uint32)
        r3 = self.rng.random(3 * OCC_CELLS).astype(np.float32)
        pos = o.occupancy_sample_points(lv, cells, r3, OCC_CELLS, 128, 1.0, 1.0 / sc.aabb_size, OCC_CELLS)
        vals, _ = o.blob_field(pos, OCC_CELLS, OCC_CELLS, sc.aabb_size, sc.field.blobs, sc.field.waves, want_rgb=False)
        d = np.ascontiguousarray(self.density, np.float32).ravel()
        r.occupancy_decay(d, 5, 128, 0.95)
        rs = self.rng.random(OCC_CELLS)
        sel = np.ones(OCC_CELLS, bool) if self.k < 256 else (rs < 0.25) | (
            (rs <= 0.5) & ((self.bits[cells] >> lv) & 1).astype(bool))
        idx = lv[sel].astype(np.int64) * 128 ** 3 + cells[sel]
        np.maximum.at(d, idx, vals[sel].astype(np.float32))
        self.density = d
        r.occupancy_bits(d, self.bits, 5, 128, THRESHOLD)
        r.popcount(self.bits)
        lr = 1e-2 / (1.0 + 3.3e-5 * self.k)
        r.adam_step(self.w32, self.grad, self.m32, self.v32, self.s32, N_GRID, N_MLP, lr, inplace=True,
                    weights_copy=self.w_copy)
        self.k += 1
        return nsamp


def _cpu_step():
    """The reference's own kernels on the host when they are built (kind "reference"), else the
    oracle's restatement (kind "port")."""
    import oracle
    oracle.build()
    from oracle import ref
    if ref.available():
        return RefCpuStep(), "reference", ref.num_threads()
    return CpuStep(), "port", oracle.num_threads()


def cpu_baseline(seconds=12.0):
    cs, kind, cores = _cpu_step()
    cs.step()  # warm-up (first touch of the buffers)
    t0 = time.perf_counter()
    samples, steps = 0, 0
    while True:
        samples += cs.step()
        steps += 1
        if time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    what = "the reference's kernels compiled on the host" if kind == "reference" else "the CPU oracle"
    return {"value": round(samples / el, 1), "unit": "samples/s", "cores": cores, "kind": kind,
            "sample": f"{steps} full train steps of the same workload on {what} (OpenMP), {el:.1f} s"}


def run_reference(args):
    rank, world, _ = _env_rank()
    if rank != 0:
        return
    cs, kind, cores = _cpu_step()
    for _ in range(max(args.warmup, 1)):
        cs.step()
    t0 = time.perf_counter()
    samples = 0
    k = max(1, args.steps)
    for _ in range(k):
        samples += cs.step()
    el = time.perf_counter() - t0
    v = samples / el
    what = "the reference's kernels compiled on the host" if kind == "reference" else "the CPU oracle"
    line = {
        "metric": METRIC, "value": round(v, 1), "unit": "samples/s", "n_gpus": world, "steps": k,
        "warmup": args.warmup, "ms_per_step": round(el / k * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if kind == "reference" else "f64/f32", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD, "batch_size_samples": BATCH, "rays_per_step": RAYS, "cascades": 5,
                   "parallelism": "cpu"},
        "cpu_baseline": {"value": round(v, 1), "unit": "samples/s", "cores": cores, "kind": kind,
                         "sample": f"{k} full train steps on {what} (OpenMP, {cores} threads)"},
        "e2e": {"value": round(v, 1), "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def backward_memory_result(args):
    """Backward memory study: 2^22 samples over about 2^16 rays (truncated geometric counts,
    mean 64, at most 1024; sigma and rgb as in the compositor workload), compositor + distortion
    loss forward and backward, two ways:
      * recompute: the compositor keeps only per-ray state (RGBA, optical depth, samples used)
        and its backward rebuilds transmittance by a reverse scan; the distortion loss runs as
        one fused forward/backward pass;
      * store: the compositor forward also stores every sample's transmittance and weight and
        its backward reads them; the distortion loss stores its per-sample running sums between
        a forward and a backward kernel (the reference's structure).
    Reports, per variant, the device memory its buffers add beyond the shared inputs (allocator
    peak) and the time of forward + backward (CUDA events, after warm-up). Both variants'
    gradients are checked against the FP64 oracle by tests/test_gpu_backward_memory.py."""
    import torch
    from turbonerf_b200 import hotpath as hp, scenes

    torch.cuda.set_device(0)
    sb = scenes.make_sample_batch(0x7B5, 1 << 22, mean=64.0, max_count=1024)
    n, ss = sb.n_rays, sb.n_samples
    lam = 1e-3
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    counts = dev(sb.counts.view(np.int32))
    offsets = dev(sb.offsets.view(np.int32))
    sig, rgb, dt, mn, dtn = (dev(a) for a in (sb.sigma, sb.rgb, sb.dt, sb.m_norm, sb.dt_norm))
    g_rgba = dev(np.random.default_rng(5).normal(size=4 * n).astype(np.float32))
    rb = hp.ray_batch(counts, offsets, n, n, ss)
    ctx = hp.Context()
    ctx.reserve(n, ss)
    variants = {
        "recompute": lambda: hp.backward_recompute(ctx, rb, sig, rgb, dt, mn, dtn, g_rgba, lam),
        "store": lambda: hp.backward_store(ctx, rb, sig, rgb, dt, mn, dtn, g_rgba, lam),
    }
    result = {}
    for name, fn in variants.items():
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        base = torch.cuda.memory_allocated()
        torch.cuda.reset_peak_memory_stats()
        out = fn()
        torch.cuda.synchronize()
        extra = torch.cuda.max_memory_allocated() - base
        del out
        reps = max(args.steps // 10, 5)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        result[name] = {"extra_device_bytes": int(extra), "ms": round(ms, 4),
                        "samples_per_s": round(ss / (ms / 1e3), 1)}
    line = {"workload": "compositor + distortion backward, recompute vs store: 2^22 samples, "
                        f"{n} rays (truncated geometric, mean 64, max 1024)",
            "n_samples": ss, "n_rays": n, "dtype": "f32", "data": "synthetic",
            "store_minus_recompute_bytes": result["store"]["extra_device_bytes"] -
                                           result["recompute"]["extra_device_bytes"], **result}
    return line


def run_backward_memory(args):
    print(json.dumps(backward_memory_result(args)), flush=True)


def _multi_scene_gpu(params, resolution=128, threshold=THRESHOLD):
    """Scenes of the multi-scene workload with their occupancy grids built on the device: per
    level, the field's density at every cell centre (Morton order) thresholded into that
    level's bit."""
    import torch
    from turbonerf_b200 import hotpath as hp, scenes
    ms = scenes.make_multi_scene(params, resolution=resolution, grids=False)
    V = resolution ** 3
    m = np.arange(V, dtype=np.uint32)
    unit = np.stack([(scenes.morton3d_invert(m >> np.uint32(c)).astype(np.float64) - resolution / 2 + 0.5) / resolution
                     for c in range(3)])  # [3][V]: centres of a level of size 1
    unit_d = torch.from_numpy(unit).cuda()
    table, grids = [], []
    for sc, b, p in zip(ms.scenes, ms.ray_begin, params):
        base = float(np.float32(p["aabb"]) / np.float32(1 << (p["n_levels"] - 1)))
        bits = torch.zeros(V, dtype=torch.uint8, device="cuda")
        blobs = torch.from_numpy(sc.field.blobs).cuda()
        waves = torch.from_numpy(sc.field.waves).cuda()
        for k in range(p["n_levels"]):
            ls = float(np.float32(base) * np.float32(1 << k))
            pos = (unit_d * ls).float().contiguous().view(-1)
            sigma, _ = hp.synth_field(pos, V, V, p["aabb"], blobs, waves, want_rgb=False)
            bits |= (sigma > threshold).to(torch.uint8) << k
        g = hp.GridSpec(p["n_levels"], resolution, base)
        mk = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
        table.append(dict(grid=g, bitfield=bits, bbox=sc.bbox, march=mk, inv_aabb=1.0 / sc.aabb_size,
                          ray_begin=int(b), n_rays=sc.rays.n))
    return ms, table


def _multi_scene_losses(args, ctx, ctx_s, table_in, R, ss, n_steps, offsets, samples):
    """The fused losses (tn_train_losses, lambda 1e-3, distance scaling) over the packed samples of
    every scene: one launch over all rays (its grid is every resident warp, each taking rays of all
    scenes in turn) against one launch per scene, each captured in a CUDA graph and replayed. The
    network outputs are seeded stand-ins (sigma = exp(N(0, 2)) clipped to 1e4, rgb U[0, 1]);
    targets and backgrounds U[0, 1]."""
    import torch
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(0x7C5)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    sig = d(np.clip(np.exp(rng.normal(0.0, 2.0, ss)), 0.0, 1e4).astype(np.float32))
    rgb = d(rng.uniform(0.0, 1.0, 3 * ss).astype(np.float32))
    tgt = d(rng.uniform(0.0, 1.0, 4 * R).astype(np.float32))
    bg = d(rng.uniform(0.0, 1.0, 3 * R).astype(np.float32))
    gd = torch.zeros(ss, device="cuda")
    drgb = torch.zeros(3 * ss, device="cuda")
    sums = torch.zeros(2 * (len(table_in) + 1), device="cuda")
    fields = (samples["dt"], samples["m_norm"], samples["dt_norm"], samples["t"])
    rb_all = hp.ray_batch(n_steps, offsets, R, R, ss)
    rbs = [hp.ray_batch(n_steps[ti["ray_begin"]:], offsets[ti["ray_begin"]:], ti["n_rays"], R, ss) for ti in table_in]

    def one_launch():
        hp.train_losses(ctx, rb_all, sig, rgb, *fields, tgt, bg, gd, inv_nrays=1.0 / R, lam=1e-3, dL_drgb=drgb,
                        loss_sums=sums[:2])

    def one_per_scene():
        for k, (ti, rb) in enumerate(zip(table_in, rbs)):
            b = ti["ray_begin"]
            hp.train_losses(ctx_s, rb, sig, rgb, *fields, tgt[b:], bg[b:], gd, inv_nrays=1.0 / ti["n_rays"],
                            lam=1e-3, dL_drgb=drgb, loss_sums=sums[2 * k + 2:2 * k + 4])

    out = {"n_rays": R, "n_samples": ss - 64}
    for name, fn in (("one_launch", one_launch), ("per_scene", one_per_scene)):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        for _ in range(3):
            g.replay()
        reps = max(args.steps, 10)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            g.replay()
        e1.record()
        e1.synchronize()
        ms_ = e0.elapsed_time(e1) / reps
        out[name] = {"ms": round(ms_, 4), "samples_per_s": round((ss - 64) / (ms_ / 1e3), 1)}
        del g
    assert ctx.check() == 0 and ctx_s.check() == 0
    out["one_launch_speedup"] = round(out["per_scene"]["ms"] / out["one_launch"]["ms"], 3)
    return out


def multi_scene_result(args, labels=("as_drawn", "scaled_2e19_samples")):
    """Batched multi-scene march: 16 scenes, each its own blob field (8-32 blobs), 1-5 cascades
    of 128^3 and an AABB of size 0.5-16, ray counts log-uniform in 2^10..2^16, rays from a
    sphere of radius 4A/3 toward the centre (cone stepping 1/256). Times the march count +
    emit of every scene (no batch cut) two ways, each captured in a CUDA graph and replayed:
      * persistent: one work-stealing count launch and one emit launch for all scenes;
      * per-scene: tn_march_count + tn_march_emit once per scene.
    A second workload scales every scene's ray count by one factor so that the batch holds
    about 2^19 samples. Each workload then times the fused losses over the packed samples of all
    scenes, one launch against one per scene (_multi_scene_losses). Per-scene counts and samples of
    the persistent launch, and the losses over all scenes, are checked against the oracle by
    tests/test_gpu_multi_scene.py."""
    import torch
    from turbonerf_b200 import hotpath as hp, scenes

    torch.cuda.set_device(0)
    params = scenes.multi_scene_params(seed=0x7C3, n_scenes=16, ray_lo=1 << 10, ray_hi=1 << 16)
    out = {"workload": "batched multi-scene march count + emit: 16 scenes, 8-32 blobs, 1-5 cascades of 128^3, "
                       "AABB 0.5-16, rays log-uniform 2^10..2^16", "dtype": "f32", "data": "synthetic"}
    for label, scale in (("as_drawn", None), ("scaled_2e19_samples", 1 << 19)):
        if label not in labels:
            continue
        ps = [dict(p) for p in params]
        if scale is not None:
            f = scale / max(out["as_drawn"]["n_samples"], 1)
            for p in ps:
                p["n_rays"] = max(1, int(round(p["n_rays"] * f)))
        ms, table_in = _multi_scene_gpu(ps)
        table = hp.scene_table(table_in)
        R = ms.rays.n
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        ori, dr, t, tmax, alive = d(ms.rays.ori), d(ms.rays.dir), d(ms.rays.t), d(ms.rays.t_max), d(ms.rays.alive)
        ctx = hp.Context()
        n_steps, scene_samples, info = hp.multi_march_count(ctx, table, R, ori, dr, t, tmax, alive)
        total = int(info[1].item())
        per_scene = scene_samples.cpu().numpy().astype(np.int64)
        ss = total + 64
        samples = hp.alloc_samples(ss, "cuda")
        offsets = torch.zeros(R, dtype=torch.int32, device="cuda")
        tune_rep = None
        if not args.no_autotune:
            *_, tune_rep = hp.autotune_multi(ctx, table, R, ss, ori, dr, t, tmax, alive, n_steps=n_steps,
                                             scene_samples=scene_samples, info=info, offsets=offsets,
                                             samples=samples)

        def persistent():
            hp.multi_march_count(ctx, table, R, ori, dr, t, tmax, alive, n_steps=n_steps, scene_samples=scene_samples,
                                 info=info)
            hp.multi_march_emit(ctx, table, R, ss, ori, dr, t, alive, n_steps, samples=samples, offsets=offsets)

        ctx_s = hp.Context()
        tun = ctx.tuning  # the same launch shapes on both sides
        ctx_s.tuning = dict(count_rays_per_block=tun["multi_chunk_rays"], emit_warps_per_block=tun["emit_warps_per_block"],
                            emit_rays_per_warp=tun["emit_rays_per_warp"])
        bufs = []
        for sc_in, ns_k in zip(table_in, per_scene):
            b, n = sc_in["ray_begin"], sc_in["n_rays"]
            bufs.append(dict(b=b, n=n, ss=int(ns_k) + 64, samples=hp.alloc_samples(int(ns_k) + 64, "cuda"),
                             n_steps=torch.zeros(n, dtype=torch.int32, device="cuda"),
                             offsets=torch.zeros(n, dtype=torch.int32, device="cuda"),
                             info=torch.zeros(4, dtype=torch.int32, device="cuda")))

        def one_per_scene():
            for sc_in, bf in zip(table_in, bufs):
                b, n = bf["b"], bf["n"]
                ns_k, inf = hp.march_count(ctx_s, sc_in["grid"], sc_in["bitfield"], sc_in["bbox"], sc_in["march"], n,
                                           R, ori[b:], dr[b:], t[b:], tmax[b:], alive[b:], 0xFFFFFFFF,
                                           n_steps=bf["n_steps"], batch_info=bf["info"])
                hp.march_emit(ctx_s, sc_in["grid"], sc_in["bitfield"], sc_in["bbox"], sc_in["march"],
                              sc_in["inv_aabb"], n, R, bf["ss"], inf, ori[b:], dr[b:], t[b:], alive[b:], ns_k,
                              offsets=bf["offsets"], samples=bf["samples"])

        res = {"n_rays": R, "n_samples": total, "rays_per_scene": [int(p["n_rays"]) for p in ps],
               "samples_per_scene": [int(v) for v in per_scene], "launch_shapes": ctx.tuning,
               "autotune": tune_rep}
        for name, fn in (("persistent", persistent), ("per_scene", one_per_scene)):
            for _ in range(max(args.warmup, 3)):
                fn()
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                fn()
            reps = max(args.steps, 10)
            for _ in range(3):
                g.replay()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                g.replay()
            e1.record()
            e1.synchronize()
            ms_ = e0.elapsed_time(e1) / reps
            res[name] = {"ms": round(ms_, 4), "samples_per_s": round(total / (ms_ / 1e3), 1)}
            del g
        assert ctx.check() == 0 and ctx_s.check() == 0
        res["persistent_speedup"] = round(res["per_scene"]["ms"] / res["persistent"]["ms"], 3)
        res["losses"] = _multi_scene_losses(args, ctx, ctx_s, table_in, R, ss, n_steps, offsets, samples)
        out[label] = res
    return out


def run_multi_scene(args):
    print(json.dumps(multi_scene_result(args)), flush=True)


def run_compositor(args):
    """The compositor tile kernels alone on the compositor workload (the `rooflines` object of the
    default line): 2^22 samples over 65,571 rays, L2 flushed before every timed launch."""
    import torch
    torch.cuda.set_device(0)
    peak, kind = _peaks()
    print(json.dumps({"workload": "compositor tiles, 2^22 samples", "peak_source": kind,
                      "rooflines": compositor_rooflines(peak, reps=max(args.steps // 5, 5))}), flush=True)


def run_losses(args):
    """The fused train-step loss kernel alone (tn_train_losses: reconstruction + distortion forward
    and backward + gradient merge, lambda 1e-3) on two batches of 2^18 samples shaped like the train
    step's: late in training (truncated geometric counts, mean 120, at most 240: every ray in the
    one-pass path) and early (mean 178, at most 290: some rays past 256 samples take the chunked
    path). CUDA events around 20 back-to-back launches, median of 5."""
    import torch
    from turbonerf_b200 import hotpath as hp, scenes
    torch.cuda.set_device(0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out = {"workload": "fused train-step losses, 2^18 samples", "batches": []}
    for label, mean, mx in (("late", 120.0, 240), ("early", 178.0, 290)):
        sb = scenes.make_sample_batch(0x7B4, 1 << 18, mean=mean, max_count=mx)
        n, ss = sb.n_rays, sb.n_samples
        ctx = hp.Context()
        rb = hp.ray_batch(d(sb.counts.view(np.int32)), d(sb.offsets.view(np.int32)), n, n, ss)
        ins = [d(a) for a in (sb.sigma, sb.rgb, sb.dt, sb.m_norm, sb.dt_norm, sb.t, sb.target_rgba, sb.bg_rgb)]
        gd, drgb, sums = torch.zeros(ss, device="cuda"), torch.zeros(3 * ss, device="cuda"), torch.zeros(2, device="cuda")

        def launch():
            hp.train_losses(ctx, rb, *ins, gd, inv_nrays=1.0 / n, lam=1e-3, dL_drgb=drgb, loss_sums=sums)

        for _ in range(max(args.warmup, 3)):
            launch()
        torch.cuda.synchronize()
        ts = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(20):
                launch()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) * 1e3 / 20)
        assert ctx.check() == 0
        out["batches"].append({"batch": label, "rays": n, "samples": ss, "max_count": int(sb.counts.max()),
                               "rays_over_256": int((sb.counts > 256).sum()), "us": round(float(np.median(ts)), 2)})
    print(json.dumps(out), flush=True)


def hashgrid_result(args):
    """The hash-grid encoding of the reference (16 levels of 2 features, 2^19 entries a level,
    resolutions 16..2048 x 16 for the train step's 16-unit box) on 2^18 uniform positions: the
    encode and the backward (with the touched-entry list, and without it) alone, CUDA events, median
    of 20 launches after warm-up (the 64 MB table stays in L2 between launches); then the full
    train step of the
    train-step workload with the hash-grid network (and its linear heads) as the trainer's network
    instead of the synthetic stand-in: real gradients, Adam over the entries they touch, CUDA graph,
    count-ahead schedule."""
    import torch
    from turbonerf_b200 import hotpath as hp
    from turbonerf_b200.replicas import replica_seed
    torch.cuda.set_device(0)
    spec = hp.HashgridSpec.reference(16.0)
    n_hash, n_head = spec.n_params()
    rng = np.random.default_rng(0x7C6)
    n = 1 << 18
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    pos = d(rng.uniform(0.0, 1.0, 3 * n).astype(np.float32))
    params = d(rng.uniform(-1e-4, 1e-4, n_hash).astype(np.float32))
    feat = torch.zeros(spec.n_features * n, device="cuda")
    dfeat = d(rng.normal(0.0, 1e-3, spec.n_features * n).astype(np.float32))
    grads = torch.zeros(n_hash, device="cuda")
    entries = spec.n_levels << spec.log2_hashmap_size
    bits = torch.zeros((entries + 31) // 32, dtype=torch.int32, device="cuda")
    lst = torch.zeros(entries, dtype=torch.int32, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = {"workload": "hash-grid encoding, 16 levels x 2^19 x 2, 2^18 positions", "n": n}

    def timed(fn, before=None):
        for _ in range(3):
            if before:
                before()
            fn()
        ts = []
        for _ in range(20):
            if before:
                before()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    ms = timed(lambda: hp.hashgrid_encode(spec, pos, params, n, n, out=feat))
    out["encode"] = {"ms": round(ms, 4), "samples_per_s": round(n / (ms / 1e3), 1)}

    def backward():
        import ctypes
        from turbonerf_b200.native import call
        from turbonerf_b200.hotpath import _ptr, _stream
        call("tn_hashgrid_backward", _stream(), ctypes.byref(spec.desc()), n, None, n, _ptr(pos), _ptr(dfeat),
             _ptr(grads), _ptr(bits), _ptr(lst), _ptr(count))

    ms = timed(backward, before=lambda: hp.hashgrid_clear_touched(lst, count, grads, bits))
    out["backward"] = {"ms": round(ms, 4), "samples_per_s": round(n / (ms / 1e3), 1),
                       "touched_entries": int(count.item())}
    ms = timed(lambda: hp.hashgrid_backward(spec, pos, dfeat, grads, n, n, touched=False))
    out["backward_without_list"] = {"ms": round(ms, 4), "samples_per_s": round(n / (ms / 1e3), 1)}
    # the train step with the hash-grid network
    scene = _scene(0x7B0)
    tr = _trainer(scene, "fused", replica_seed(0x7B0, 0))
    tr.use_hashgrid(spec)
    tr.autotune()
    steps = max(args.steps // 2, 10)
    for _ in range(max(args.warmup, 3)):
        tr.train_step_async()
    m0 = tr.sync_metrics()
    stream = torch.cuda.ExternalStream(tr.stream_handle())
    s0 = tr.stat(3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        tr.train_step_async()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    m = tr.sync_metrics()
    samples = tr.stat(3) - s0
    out["train_step"] = {"ms_per_step": round(ms / steps, 4), "samples_per_s": round(samples / (ms / 1e3), 1),
                         "steps": steps, "loss_first": round(float(m0.loss), 6), "loss_last": round(float(m.loss), 6),
                         "touched_entries_last_step": int(tr.buffer(32, np.uint32)[0].item())}
    tr.teardown()
    return out


def run_hashgrid(args):
    print(json.dumps(hashgrid_result(args)), flush=True)


def run_kernel_tour(args):
    """Every kernel of the library, launched at representative sizes, for profiling (for instance
    `ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum`, one pass per
    launch): the fused and plain train steps of the train-step workload (graph replay, stage
    timing, the full occupancy update), the compositor, distortion and fused losses on 2^22
    samples (65,571 rays, truncated geometric counts, mean 64), the march, scan and compaction
    entry points on 2^14 rays of the 5-cascade scene, and the batched multi-scene march of six
    small scenes. About 1.2 GB of device memory. Prints what ran."""
    import torch
    from turbonerf_b200 import hotpath as hp, native, scenes

    torch.cuda.set_device(0)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ran = []
    # training steps
    scene = _scene(0x7B0)
    tr = _trainer(scene, "fused", 0x7B0)
    for _ in range(3):
        tr.train_step()
    tr.profile_step()
    tr.update_occupancy_grid(300)
    tr.flush()
    ran.append("fused train steps (eager, graph capture and replay, stage timing, full occupancy update)")
    del tr
    trp = _trainer(scene, "plain", 0x7B0)
    trp.train_step()
    ran.append("plain train step")
    del trp
    # compositor and losses
    sb = scenes.make_sample_batch(0x7B5, 1 << 22, mean=64.0, max_count=1024)
    n, ss = sb.n_rays, sb.n_samples
    counts, offsets = d(sb.counts.view(np.int32)), d(sb.offsets.view(np.int32))
    sig, rgb, dt, mn, dtn, t = (d(a) for a in (sb.sigma, sb.rgb, sb.dt, sb.m_norm, sb.dt_norm, sb.t))
    tgt, bg = d(sb.target_rgba), d(sb.bg_rgb)
    rb = hp.ray_batch(counts, offsets, n, n, ss)
    ctx = hp.Context(n, ss)
    g_rgba = torch.full((4 * n,), 1e-3, device="cuda")
    fo = hp.composite_fwd(ctx, rb, sig, rgb, dt)
    hp.composite_bwd(ctx, rb, sig, rgb, dt, fo["depth"], fo["n_used"], g_rgba)
    st = hp.composite_fwd_store(ctx, rb, sig, rgb, dt)
    hp.composite_bwd_stored(ctx, rb, sig, rgb, dt, st["n_used"], st["t_saved"], st["w_saved"], g_rgba)
    hp.recon_loss_fwd_bwd(ctx, rb, sig, rgb, dt, tgt, bg, 1.0 / n)
    hp.distortion_fwd_bwd(ctx, rb, sig, mn, dtn, 1e-3)
    gd = torch.zeros(ss, device="cuda")
    hp.train_losses(ctx, rb, sig, rgb, dt, mn, dtn, t, tgt, bg, gd, inv_nrays=1.0 / n, lam=1e-3)
    hp.grad_epilogue(ss, 1.0, gd, gd, t, torch.zeros(ss, device="cuda"))
    ran.append(f"compositor, distortion and fused losses on {ss} samples / {n} rays")
    rbs = hp.ray_batch(counts[:4096].contiguous(), offsets[:4096].contiguous(), 4096, 4096, ss)
    hp.plain_recon_loss(rbs, sig, rgb, dt, tgt, bg, 1.0 / 4096)
    hp.plain_distortion(rbs, sig, mn, dtn, 1e-3)
    hp.plain_grad_epilogue(ss, 1.0, gd, gd, t, torch.zeros(ss, device="cuda"))
    ran.append("plain compositor and distortion on the first 4096 rays")
    del sig, rgb, dt, mn, dtn, t, gd, fo, st
    # march, scan, compaction
    sc = scenes.march_scene_cascaded(seed=0x7B0, n_rays=RAYS, n_levels=5)
    r = sc.rays
    ori, dr = d(r.ori), d(r.dir)
    hp.rays_init_bbox(ori, dr, RAYS, RAYS, sc.bbox, t_far=3.0e38)
    g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, 0)
    bits = d(sc.grid.bitfield)
    t0, tm, al = d(r.t), d(r.t_max), d(r.alive)
    mctx = hp.Context(RAYS, BATCH)
    ns, info = hp.march_count(mctx, g, bits, sc.bbox, m, RAYS, RAYS, ori, dr, t0, tm, al, BATCH)
    hp.march_emit(mctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, RAYS, RAYS, BATCH + 64, info, ori, dr, t0, al, ns)
    hp.plain_march_count(g, bits, sc.bbox, m, RAYS, RAYS, ori, dr, t0, tm, al.clone())
    hp.scan_offsets(mctx, ns, BATCH)
    hp.compact_nonzero(mctx, ns)
    hp.popcount(mctx, bits)
    off_na, info_na = torch.zeros(RAYS, dtype=torch.int32, device="cuda"), torch.zeros(4, dtype=torch.int32, device="cuda")
    native.call("tn_scan_offsets_noalloc", hp._stream(), RAYS, hp._ptr(ns), hp._ptr(off_na), BATCH, hp._ptr(info_na),
                hp._ptr(info_na[3:]))
    ran.append(f"box clip, march count and emit, plain march count, scans, compaction, popcount on {RAYS} rays")
    # batched multi-scene march
    params = scenes.multi_scene_params(seed=0x7C1, n_scenes=6, ray_lo=64, ray_hi=2048)
    ms = scenes.make_multi_scene(params, resolution=32)
    rows = [dict(grid=hp.GridSpec(s_.grid.n_levels, s_.grid.resolution, s_.grid.base_size), bitfield=d(s_.grid.bitfield),
                 bbox=s_.bbox, march=hp.MarchSpec(s_.cone_angle, s_.dt_min, s_.dt_max, s_.max_steps),
                 inv_aabb=1.0 / s_.aabb_size, ray_begin=int(b), n_rays=s_.rays.n) for s_, b in zip(ms.scenes, ms.ray_begin)]
    table = hp.scene_table(rows)
    mr = ms.rays
    mo, mdr, mt, mtm, mal = d(mr.ori), d(mr.dir), d(mr.t), d(mr.t_max), d(mr.alive)
    n_steps, _, minfo = hp.multi_march_count(mctx, table, mr.n, mo, mdr, mt, mtm, mal)
    hp.multi_march_emit(mctx, table, mr.n, int(minfo[1].item()) + 64, mo, mdr, mt, mal, n_steps)
    ran.append(f"multi-scene march count and emit: {len(rows)} scenes, {mr.n} rays")
    torch.cuda.synchronize()
    assert ctx.check() == 0 and mctx.check() == 0
    print(json.dumps({"workload": "kernel tour", "ran": ran, "data": "synthetic"}), flush=True)


def _look_at(eye, target=(0.0, 0.0, 0.0)):
    """Camera to world [3][4]: columns right, down, forward (the camera looks along +z)."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, [0.0, 1.0, 0.0])
    r /= np.linalg.norm(r)
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = r, np.cross(f, r), f, eye
    return t


def run_render(args):
    """Inference render (Renderer.submit) of the train-step scene: 5 cascades of 128^3 built
    from the 8-blob field, which also stands in for the network; the camera at (0.3, 0.8, 4.0)
    looks at the centre from inside the 16-unit training box (focal 0.7 x width). Frames of
    800 x 800 and 1920 x 1080 (--render-sizes) at sample budgets per round (--render-batches) of
    the library default (0), 2^20 (the reference default), 2^22 and 2^24. A frame is one synchronous submit (it reads the live ray count back every
    round), so frames are timed on the host clock around the call. The CPU oracle renders the
    same view at 200 x 200 on all host threads; its rays/s is the CPU baseline, and its image
    is compared with the GPU frame of the same size."""
    import torch
    import oracle
    from turbonerf_b200 import scenes
    from turbonerf_b200.renderer import Camera, CPURenderBuffer, CUDARenderBuffer, RenderRequest, Renderer

    torch.cuda.set_device(0)
    sc = _scene(0x7B0)
    tr = _trainer(sc, "fused", 0x7B0)
    eye = (0.3, 0.8, 4.0)

    def cam(w, h):
        return Camera((w, h), 0.1, 100.0, (0.7 * w, 0.7 * w), (w / 2, h / 2), (0.0, 0.0), _look_at(eye))

    out = {"workload": "inference render of the train-step scene (5x128^3 cascades, 8-blob field as the network)",
           "metric": "rays/s per frame (host clock around the synchronous submit)", "dtype": "f32",
           "data": "synthetic", "frames": []}
    buf = CUDARenderBuffer()
    sizes = [tuple(int(v) for v in wh.split("x")) for wh in args.render_sizes.split(",")]
    batches = [int(v) for v in args.render_batches.split(",")]
    for (w, h) in sizes:
        for bs in batches:
            r = Renderer(batch_size=bs)
            req = RenderRequest(cam(w, h), [tr], buf)
            for _ in range(max(args.warmup, 3)):
                r.submit(req)
            reps = max(min(args.steps, 20), 3)
            times = []
            for _ in range(reps):
                t0 = time.perf_counter()
                st = r.submit(req)
                times.append(time.perf_counter() - t0)
            ms = 1e3 * statistics.median(times)
            out["frames"].append({"width": w, "height": h, "batch_size": bs, "ms_per_frame": round(ms, 3),
                                  "rays_per_s": round(w * h / (ms / 1e3), 1),
                                  "samples_per_s": round(st["samples"] / (ms / 1e3), 1),
                                  "steps_per_s": round(st["steps"] / (ms / 1e3), 1), **st})
    if args.no_cpu:
        tr.teardown()
        print(json.dumps(out), flush=True)
        return
    # CPU oracle on a 200 x 200 frame of the same view, and the GPU frame it is compared with
    c = cam(200, 200)
    od = dict(width=200, height=200, near=c.near, far=c.far, focal=c.focal_length, principal=c.principal_point,
              shift=c.shift, transform=c.transform)
    t0 = time.perf_counter()
    ref, amb, _ = oracle.render(od, sc.bbox, sc.bbox, sc.grid.as_dict(), float(np.float32(scenes.MIN_STEP_SIZE)),
                                1.0 / 256.0, 1e-4, sc.field.blobs, sc.field.waves, sc.aabb_size)
    el = time.perf_counter() - t0
    cpu = CPURenderBuffer()
    Renderer().submit(RenderRequest(c, [tr], cpu))
    img = cpu.get_rgba().astype(np.float64)
    ok = amb == 0
    err = np.abs(img - ref)[ok] / (np.abs(ref)[ok] + 1e-6 * np.abs(ref).max())
    out["cpu_baseline"] = {"value": round(200 * 200 / el, 1), "unit": "rays/s", "cores": oracle.num_threads(),
                           "kind": "port", "sample": f"one 200 x 200 frame of the same view on the CPU oracle, {el:.2f} s"}
    out["parity_200x200"] = {"max_rel_err": float(err.max()), "ambiguous_pixels": int((~ok).sum())}
    tr.teardown()
    print(json.dumps(out), flush=True)


def run_dataset_rays(args):
    """Training rays from posed images (tn_dataset_rays; reference
    initialize_training_rays_and_pixels_kernel + deactivate_rays_with_alpha_threshold_kernel):
    100 synthetic 800 x 800 RGBA8 images (256 MB on the device, larger than L2; 40% of texels
    transparent) seen by cameras on a radius-4 sphere around the 16-unit training box, 2^20 rays
    per launch, with alpha selection off and on (threshold 0.5, probability 0.25). Each launch is
    timed with CUDA events after an L2 flush (L2Flush). Algorithmic bytes: 65 per ray (two draws and one
    texel read; RGBA, image id, origin, direction, t, t_max and alive written). The CPU oracle
    runs the same 2^20 rays; its output is compared with the GPU's bit for bit. Last, the
    train step on dataset rays (the train-step workload with the images as the ray source)."""
    import ctypes
    import torch
    import oracle
    from turbonerf_b200.native import Bbox, CameraC, call
    from turbonerf_b200.renderer import Camera
    from turbonerf_b200.trainer import Dataset, SyntheticNeRF, Trainer

    torch.cuda.set_device(0)
    n_img, w, h, n = 100, 800, 800, 1 << 20
    rng = np.random.default_rng(0x7B0)
    cams = []
    for _ in range(n_img):
        e = rng.normal(size=3)
        cams.append(Camera((w, h), 0.1, 100.0, (1111.0, 1111.0), (w / 2, h / 2), (0.0, 0.0),
                           _look_at(tuple(4.0 * e / np.linalg.norm(e)))))
    imgs = rng.integers(0, 256, (n_img, h, w, 4), dtype=np.uint8)
    imgs[..., 3] = np.where(rng.random((n_img, h, w)) < 0.4, rng.integers(0, 40, (n_img, h, w)), 255)
    half = 8.0
    bbox = (-half, -half, -half, half, half, half)
    cam_arr = (CameraC * n_img)(*[c.c_struct() for c in cams])
    cam_dev = torch.frombuffer(bytearray(bytes(cam_arr)), dtype=torch.uint8).cuda()
    img_dev = torch.from_numpy(imgs).cuda()
    rnd = torch.rand((2, n), device="cuda", generator=torch.Generator("cuda").manual_seed(0x7B0))
    f32 = lambda k: torch.empty(k, device="cuda")  # noqa: E731
    outs = dict(pix_rgba=f32(4 * n), img_id=torch.empty(n, dtype=torch.int32, device="cuda"), ori=f32(3 * n),
                dir=f32(3 * n), t=f32(n), t_max=f32(n), alive=torch.empty(n, dtype=torch.uint8, device="cuda"))
    b = Bbox(*bbox)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    stream = torch.cuda.current_stream()
    flush = L2Flush()
    peak, peak_src = _peaks()
    alg = 65 * n

    def launch(thr, prob, k=n):
        call("tn_dataset_rays", ctypes.c_void_p(stream.cuda_stream), k, n, n_img, w, h, p(cam_dev), p(img_dev),
             ctypes.byref(b), p(rnd), thr, prob, p(outs["pix_rgba"]), p(outs["img_id"]), p(outs["ori"]),
             p(outs["dir"]), p(outs["t"]), p(outs["t_max"]), p(outs["alive"]))

    res = {"workload": "training rays from 100 posed 800x800 RGBA8 images, 2^20 rays per launch, L2 flushed",
           "metric": "rays/s", "dtype": "f32", "data": "synthetic", "launches": []}
    reps = max(min(args.steps, 50), 5)
    for thr, prob in ((1.0, 1.0), (0.5, 0.25)):
        for _ in range(max(args.warmup, 3)):
            launch(thr, prob)
        ms = []
        for _ in range(reps):
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            launch(thr, prob)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        m = statistics.mean(ms)
        live = int(outs["alive"].sum().item())
        res["launches"].append({"alpha_threshold": thr, "alpha_probability": prob, "ms": round(m, 4),
                                "rays_per_s": round(n / (m / 1e3), 1), "live_rays": live,
                                "roofline": {"bound": "hbm", "achieved": round(alg / (m / 1e3) / 1e9, 1),
                                             "peak": peak, "unit": "GB/s",
                                             "frac": round(alg / (m / 1e3) / 1e9 / peak, 4),
                                             "alg_bytes": alg, "peak_source": peak_src}})
    # parity and the CPU baseline: the oracle on the same 2^20 rays as the last launch
    torch.cuda.synchronize()
    od = [dict(width=w, height=h, near=c.near, far=c.far, focal=c.focal_length, principal=c.principal_point,
               shift=c.shift, transform=c.transform) for c in cams]
    r_host = rnd.cpu().numpy()
    t0 = time.perf_counter()
    ref, live = oracle.dataset_rays(n, od, imgs, bbox, r_host, 0.5, 0.25)
    el = time.perf_counter() - t0
    got = {key: v.cpu().numpy() for key, v in outs.items()}
    alive = got["alive"].astype(bool)
    bad = int(np.count_nonzero(alive != ref["alive"].astype(bool)))
    for key in ("ori", "dir", "pix_rgba", "t", "t_max"):
        comps = got[key].size // n
        g = got[key].reshape(comps, n)[:, alive]
        r = np.asarray(ref[key], np.float32).reshape(comps, n)[:, alive]
        bad += int(np.count_nonzero(g.view(np.uint32) != r.view(np.uint32)))
    res["parity_2e20"] = {"mismatched_values": bad, "live_rays": int(live)}
    res["cpu_baseline"] = {"value": round(n / el, 1), "unit": "rays/s", "cores": oracle.num_threads(), "kind": "port",
                           "sample": f"the same 2^20 rays on the CPU oracle, {el:.3f} s"}
    del flush, img_dev
    # the train step with the images as its ray source (2^14 rays on 100 smaller images)
    sc = _scene(0x7B0)
    nerf = SyntheticNeRF.from_scene(sc)
    nerf.dataset = Dataset(cams[:20], imgs[:20])
    tr = Trainer(nerf, path="fused", n_rays_per_step=RAYS, occupancy_cells_per_step=OCC_CELLS,
                 distortion_lambda=LAMBDA, occupancy_threshold=THRESHOLD, n_grid_params=N_GRID, n_mlp_params=N_MLP,
                 beta2=0.99, seed=0x7B0)
    tr.use_distortion_loss = True
    tr.setup_data(batch_size=BATCH, synthetic_grad_std=1e-3)
    for _ in range(max(args.warmup, 3)):
        tr.train_step_async()
    torch.cuda.synchronize()
    steps = max(min(args.steps, 100), 5)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.ExternalStream(tr.stream_handle())
    e0.record(s)
    for _ in range(steps):
        tr.train_step_async()
    e1.record(s)
    e1.synchronize()
    m = tr.sync_metrics()
    ms = e0.elapsed_time(e1) / steps
    res["train_step_on_dataset_rays"] = {"ms_per_step": round(ms, 4), "samples_last_step": m.n_samples,
                                         "rays_last_step": m.n_rays,
                                         "samples_per_s": round(m.n_samples / (ms / 1e3), 1),
                                         "images": "20 of the 800x800 images"}
    tr.teardown()
    print(json.dumps(res), flush=True)


def configs_result(args):
    """GPU and CPU oracle side by side on the smaller configurations, samples/s each:
    * forward march + composite: 1 cascade of 128^3 over [-1.5, 1.5]^3, 8 blobs, 4096 rays from
      a radius-4 sphere, fixed dt = sqrt(3)/1024, at most 1024 steps; march count, emit (no
      batch cut), the blob field as the network, compositor forward;
    * compositor + distortion: 2^18 samples (truncated geometric counts, mean 48), compositor
      forward and backward with the fused distortion forward/backward (lambda 1e-3);
    * large-batch backward: the same on 2^22 samples (mean 64, at most 1024).
    GPU: CUDA events around the chain, L2 flushed before each repetition (L2Flush), mean.
    CPU: the oracle's restatement of the same stages on all host threads."""
    import torch
    import oracle
    from turbonerf_b200 import hotpath as hp, scenes

    torch.cuda.set_device(0)
    oracle.build()
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    flush = L2Flush()
    reps = max(min(args.steps, 20), 3)

    def gpu_time(fn, before=None):
        for _ in range(max(args.warmup, 3)):
            if before:
                before()
            fn()
        total = 0.0
        for _ in range(reps):
            if before:
                before()
            flush()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total / reps / 1e3

    out = {"workload": "march + composite (1 cascade, 4096 rays); compositor + distortion at 2^18 and 2^22 samples",
           "metric": "samples/s", "dtype": "f32", "data": "synthetic", "cores": oracle.num_threads(), "configs": []}
    # forward march + composite
    sc = scenes.march_scene_single(seed=0x7B0)
    r = sc.rays
    n, B = r.n, 1 << 22
    ss = B + 64
    g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
    bits, ori, dr, t0, tm, al0 = d(sc.grid.bitfield), d(r.ori), d(r.dir), d(r.t), d(r.t_max), d(r.alive)
    al = al0.clone()
    blobs, waves = d(sc.field.blobs), d(sc.field.waves)
    mctx = hp.Context(n, B)
    state = {}

    def chain0():
        ns, info = hp.march_count(mctx, g, bits, sc.bbox, m, n, n, ori, dr, t0, tm, al, 0xFFFFFFFF)
        off, smp = hp.march_emit(mctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, n, n, ss, info, ori, dr, t0, al, ns)
        sig, rgb = hp.synth_field(smp["pos"], ss, ss, sc.aabb_size, blobs, waves, n_dev=info[1:])
        rb = hp.ray_batch(ns, off, n, n, ss)
        state["fo"] = hp.composite_fwd(mctx, rb, sig, rgb, smp["dt"])
        state["info"] = info

    sec = gpu_time(chain0, before=lambda: al.copy_(al0))
    n_samp = int(state["info"][1].item())
    rd, gd = r.as_dict(), sc.grid.as_dict()
    md = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
    c0 = time.perf_counter()
    n_steps, alive, _ = oracle.march_count(rd, gd, md)
    ns_cpu = int(n_steps.astype(np.int64).sum())
    offsets = np.concatenate([[0], np.cumsum(n_steps.astype(np.int64))[:-1]]).astype(np.uint32)
    sst = ns_cpu + 64
    smp = oracle.march_emit(rd, gd, md, offsets, n_steps, alive, n, sst, 1.0 / sc.aabb_size)
    sig_c, rgb_c = oracle.blob_field(smp["pos"], sst, ns_cpu, sc.aabb_size, sc.field.blobs, sc.field.waves,
                                     out_stride=sst)
    oracle.composite_fwd(n_steps, offsets, sig_c.astype(np.float32), rgb_c.astype(np.float32), smp["dt"], n, sst)
    el = time.perf_counter() - c0
    out["configs"].append({"config": "forward march + composite, 1 x 128^3, 4096 rays", "samples": n_samp,
                           "samples_cpu": int(ns_cpu), "gpu_ms": round(sec * 1e3, 4),
                           "gpu_samples_per_s": round(n_samp / sec, 1), "cpu_s": round(el, 3),
                           "cpu_samples_per_s": round(ns_cpu / el, 1)})
    del mctx
    # compositor + distortion, forward and backward
    for label, seed, total, mean in (("compositor + distortion fwd/bwd, 2^18 samples", 0x7B1, 1 << 18, 48.0),
                                     ("large-batch backward, 2^22 samples", 0x7B5, 1 << 22, 64.0)):
        sb = scenes.make_sample_batch(seed, total, mean=mean, max_count=1024)
        nr, ns = sb.n_rays, sb.n_samples
        counts, offs = d(sb.counts.view(np.int32)), d(sb.offsets.view(np.int32))
        sig, rgb, dt, mn, dtn = (d(a) for a in (sb.sigma, sb.rgb, sb.dt, sb.m_norm, sb.dt_norm))
        rb = hp.ray_batch(counts, offs, nr, nr, ns)
        ctx = hp.Context(nr, ns)
        g_rgba = torch.full((4 * nr,), 1e-3, device="cuda")
        sec = gpu_time(lambda: hp.backward_recompute(ctx, rb, sig, rgb, dt, mn, dtn, g_rgba, 1e-3))
        c0 = time.perf_counter()
        oracle.composite_fwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, nr, ns)
        oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, np.full(4 * nr, 1e-3), nr, ns)
        oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, 1e-3, ns)
        el = time.perf_counter() - c0
        out["configs"].append({"config": label, "samples": ns, "rays": nr, "gpu_ms": round(sec * 1e3, 4),
                               "gpu_samples_per_s": round(ns / sec, 1), "cpu_s": round(el, 3),
                               "cpu_samples_per_s": round(ns / el, 1)})
        del ctx
    return out


def run_configs(args):
    print(json.dumps(configs_result(args)), flush=True)


def other_configs(args):
    """The smaller configurations beside the train step, for the default bench line: GPU and
    CPU-oracle samples/s of the forward march + composite (1 cascade, 4096 rays) and of the
    compositor + distortion forward/backward at 2^18 samples; the batched multi-scene march
    (16 scenes, 128^3, 2^10..2^16 rays a scene), persistent launch against one launch per scene,
    and its fused losses in one launch against one per scene; the train step with the hash-grid
    network instead of the synthetic stand-in; the device memory of the recompute and store
    backwards at 2^22 samples."""
    import torch
    cfg = configs_result(args)
    rows = {c["config"]: c for c in cfg["configs"]}
    out = {"cores": cfg["cores"]}
    for key, label in (("march_composite_4096_rays", "forward march + composite, 1 x 128^3, 4096 rays"),
                       ("compositor_distortion_2e18", "compositor + distortion fwd/bwd, 2^18 samples")):
        c = rows[label]
        out[key] = {"gpu_samples_per_s": c["gpu_samples_per_s"], "cpu_samples_per_s": c["cpu_samples_per_s"],
                    "samples": c["samples"], "gpu_ms": c["gpu_ms"]}
    torch.cuda.empty_cache()
    ms = multi_scene_result(args, labels=("as_drawn",))["as_drawn"]
    out["multi_scene_16"] = {"n_rays": ms["n_rays"], "n_samples": ms["n_samples"],
                             "persistent_ms": ms["persistent"]["ms"], "per_scene_ms": ms["per_scene"]["ms"],
                             "persistent_speedup": ms["persistent_speedup"],
                             "losses_one_launch_ms": ms["losses"]["one_launch"]["ms"],
                             "losses_per_scene_ms": ms["losses"]["per_scene"]["ms"],
                             "losses_one_launch_speedup": ms["losses"]["one_launch_speedup"]}
    torch.cuda.empty_cache()
    hg = hashgrid_result(args)
    out["hashgrid_network_step"] = {"samples_per_s": hg["train_step"]["samples_per_s"],
                                    "ms_per_step": hg["train_step"]["ms_per_step"],
                                    "encode_ms_2e18": hg["encode"]["ms"], "backward_ms_2e18": hg["backward"]["ms"],
                                    "backward_without_list_ms_2e18": hg["backward_without_list"]["ms"]}
    torch.cuda.empty_cache()
    bm = backward_memory_result(args)
    out["backward_memory_2e22"] = {v: {"extra_device_bytes": bm[v]["extra_device_bytes"], "ms": bm[v]["ms"]}
                                   for v in ("recompute", "store")}
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="leave the smaller configurations out of the line")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--render-sizes", default="800x800,1920x1080", help="render workload: frame sizes WxH")
    ap.add_argument("--render-batches", default="0,1048576,4194304,16777216",
                    help="render workload: sample budgets per round (0: the library default)")
    ap.add_argument("--workload", default="train-step",
                    choices=["train-step", "backward-memory", "multi-scene", "kernel-tour", "render", "dataset-rays", "configs",
                             "compositor", "losses", "hashgrid"],
                    help="backward-memory: the recompute-vs-store study of the compositor and distortion backward; "
                         "multi-scene: the batched persistent march of 16 scenes against one launch per scene; "
                         "kernel-tour: every kernel once at representative sizes, for profiling; "
                         "render: inference frames through Renderer.submit; "
                         "dataset-rays: training rays from posed images; "
                         "configs: GPU and CPU oracle on the smaller configurations; "
                         "compositor: the compositor tile kernels alone; losses: the fused loss kernel alone; "
                         "hashgrid: the hash-grid encoding and the train step with it as the network")
    args = ap.parse_args()
    if args.workload == "backward-memory":
        run_backward_memory(args)
    elif args.workload == "multi-scene":
        run_multi_scene(args)
    elif args.workload == "kernel-tour":
        run_kernel_tour(args)
    elif args.workload == "render":
        run_render(args)
    elif args.workload == "dataset-rays":
        run_dataset_rays(args)
    elif args.workload == "configs":
        run_configs(args)
    elif args.workload == "compositor":
        run_compositor(args)
    elif args.workload == "losses":
        run_losses(args)
    elif args.workload == "hashgrid":
        run_hashgrid(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
