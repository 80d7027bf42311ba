"""Tensor-level entry points of the training hot path (thin wrappers over the C ABI).

Every function takes CUDA tensors in the reference's structure-of-arrays layout and
enqueues work on torch's current stream; nothing here computes on the CPU. Tensors must be
contiguous with the dtypes named in each docstring.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from . import native
from .native import Bbox, GridDesc, MarchDesc, RayBatchDesc, call


def _ptr(t):
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("turbo_hot tensors must live on a CUDA device")
    if not t.is_contiguous():
        raise ValueError("turbo_hot tensors must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Context:
    """Owns a tn_ctx (scratch, device error word) on the current CUDA device."""

    def __init__(self, max_rays: int = 0, max_samples: int = 0):
        h = ctypes.c_void_p()
        call("tn_ctx_create", ctypes.byref(h))
        self.handle = h
        if max_rays or max_samples:
            self.reserve(max_rays, max_samples)

    def reserve(self, max_rays: int, max_samples: int) -> None:
        call("tn_ctx_reserve", self.handle, max_rays, max_samples)

    def check(self) -> int:
        """Synchronises the stream; returns and clears the device error bits."""
        f = ctypes.c_uint32(0)
        call("tn_ctx_check", self.handle, _stream(), ctypes.byref(f))
        return f.value

    @property
    def tuning(self) -> dict:
        """Launch shapes used by later calls on this context (tn_tuning fields)."""
        t = native.Tuning()
        call("tn_ctx_get_tuning", self.handle, ctypes.byref(t))
        return t.as_dict()

    @tuning.setter
    def tuning(self, values: dict) -> None:
        t = native.Tuning()
        call("tn_ctx_get_tuning", self.handle, ctypes.byref(t))
        for k, v in values.items():
            setattr(t, k, int(v))
        call("tn_ctx_set_tuning", self.handle, ctypes.byref(t))

    def close(self) -> None:
        if getattr(self, "handle", None):
            native.lib().tn_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class GridSpec:
    n_levels: int
    resolution: int = 128
    base_size: float = 1.0

    def desc(self) -> GridDesc:
        return GridDesc(self.n_levels, self.resolution, float(self.base_size), 0)

    @property
    def volume(self) -> int:
        return self.resolution ** 3


@dataclass
class MarchSpec:
    cone_angle: float
    dt_min: float
    dt_max: float
    max_steps: int = 0
    max_iterations: int = 0

    def desc(self) -> MarchDesc:
        return MarchDesc(self.cone_angle, self.dt_min, self.dt_max, self.max_steps, self.max_iterations)


def bbox_desc(b) -> Bbox:
    return Bbox(*[float(v) for v in b])


def ray_batch(counts: torch.Tensor, offsets: torch.Tensor, n_rays: int, ray_stride: int, sample_stride: int,
              n_rays_dev: torch.Tensor | None = None) -> RayBatchDesc:
    """Descriptor of a packed batch. It holds references to the tensors whose device
    pointers it carries, so they stay allocated for as long as the descriptor lives."""
    rb = RayBatchDesc(n_rays, ray_stride, sample_stride, 0, _ptr(counts), _ptr(offsets), _ptr(n_rays_dev))
    rb._keep = (counts, offsets, n_rays_dev)
    return rb


# ---- rays -------------------------------------------------------------------------------
def rays_init_bbox(ori, dir_, n_rays, ray_stride, bbox, t_far=3.0e38):
    dev = ori.device
    t = torch.zeros(ray_stride, dtype=torch.float32, device=dev)
    tmax = torch.zeros(ray_stride, dtype=torch.float32, device=dev)
    alive = torch.zeros(ray_stride, dtype=torch.uint8, device=dev)
    b = bbox_desc(bbox)
    call("tn_rays_init_bbox", _stream(), n_rays, ray_stride, ctypes.byref(b), t_far, _ptr(ori), _ptr(dir_), _ptr(t),
         _ptr(tmax), _ptr(alive))
    return t, tmax, alive


# ---- march ------------------------------------------------------------------------------
def march_count(ctx: Context, grid: GridSpec, bitfield, bbox, march: MarchSpec, n_rays: int, ray_stride: int,
                ori, dir_, ray_t, ray_t_max, alive, batch_size: int, n_rays_dev=None, n_steps=None, batch_info=None):
    """Fused count pass + device batch cut. `alive` (uint8) is updated in place.
    Returns (n_steps uint32[ray_stride], batch_info uint32[3] = n_rays_cut, n_samples, total)."""
    dev = ori.device
    if n_steps is None:
        n_steps = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if batch_info is None:
        batch_info = torch.zeros(4, dtype=torch.int32, device=dev)
    g, b, m = grid.desc(), bbox_desc(bbox), march.desc()
    call("tn_march_count", ctx.handle, _stream(), ctypes.byref(g), _ptr(bitfield), ctypes.byref(b), ctypes.byref(m),
         n_rays, ray_stride, _ptr(n_rays_dev), _ptr(ori), _ptr(dir_), _ptr(ray_t), _ptr(ray_t_max), _ptr(alive),
         _ptr(n_steps), batch_size, _ptr(batch_info))
    return n_steps, batch_info


def alloc_samples(sample_stride: int, device) -> dict:
    f = dict(dtype=torch.float32, device=device)
    return dict(img_id=torch.zeros(sample_stride, dtype=torch.int32, device=device),
                t=torch.zeros(sample_stride, **f), pos=torch.zeros(3 * sample_stride, **f),
                dir=torch.zeros(3 * sample_stride, **f), dt=torch.zeros(sample_stride, **f),
                m_norm=torch.zeros(sample_stride, **f), dt_norm=torch.zeros(sample_stride, **f))


def march_emit(ctx: Context, grid: GridSpec, bitfield, bbox, march: MarchSpec, inv_aabb: float, n_rays: int,
               ray_stride: int, sample_stride: int, batch_info, ori, dir_, ray_t, alive, n_steps, ray_img_id=None,
               offsets=None, samples=None):
    dev = ori.device
    if offsets is None:
        offsets = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if samples is None:
        samples = alloc_samples(sample_stride, dev)
    g, b, m = grid.desc(), bbox_desc(bbox), march.desc()
    call("tn_march_emit", ctx.handle, _stream(), ctypes.byref(g), _ptr(bitfield), ctypes.byref(b), ctypes.byref(m),
         inv_aabb, n_rays, ray_stride, sample_stride, _ptr(batch_info), _ptr(ray_img_id), _ptr(ori), _ptr(dir_),
         _ptr(ray_t), _ptr(alive), _ptr(n_steps), _ptr(offsets), _ptr(samples["img_id"]), _ptr(samples["t"]),
         _ptr(samples["pos"]), _ptr(samples["dir"]), _ptr(samples["dt"]), _ptr(samples["m_norm"]),
         _ptr(samples["dt_norm"]))
    return offsets, samples


def default_tuning() -> dict:
    t = native.Tuning()
    native.lib().tn_tuning_default(ctypes.byref(t))
    return t.as_dict()


def autotune_march(ctx: Context, grid: GridSpec, bitfield, bbox, march: MarchSpec, inv_aabb: float, n_rays: int,
                   ray_stride: int, ori, dir_, ray_t, ray_t_max, alive, batch_size: int, sample_stride: int,
                   ray_img_id=None, n_steps=None, batch_info=None, offsets=None, samples=None):
    """Autotuner of the march count block size and the emit shape on these rays. Returns
    (n_steps, batch_info, offsets, samples, reports): the outputs of one count + emit with the
    chosen shapes, and the count and emit tuning reports (dicts)."""
    dev = ori.device
    if n_steps is None:
        n_steps = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if batch_info is None:
        batch_info = torch.zeros(4, dtype=torch.int32, device=dev)
    if offsets is None:
        offsets = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if samples is None:
        samples = alloc_samples(sample_stride, dev)
    rc, re_ = native.TuneReport(), native.TuneReport()
    g, b, m = grid.desc(), bbox_desc(bbox), march.desc()
    call("tn_autotune_march", ctx.handle, _stream(), ctypes.byref(g), _ptr(bitfield), ctypes.byref(b),
         ctypes.byref(m), inv_aabb, n_rays, ray_stride, _ptr(ray_img_id), _ptr(ori), _ptr(dir_), _ptr(ray_t),
         _ptr(ray_t_max), _ptr(alive), _ptr(n_steps), batch_size, _ptr(batch_info), sample_stride, _ptr(offsets),
         _ptr(samples["img_id"]), _ptr(samples["t"]), _ptr(samples["pos"]), _ptr(samples["dir"]),
         _ptr(samples["dt"]), _ptr(samples["m_norm"]), _ptr(samples["dt_norm"]), ctypes.byref(rc),
         ctypes.byref(re_))
    return n_steps, batch_info, offsets, samples, {"count": rc.as_dict(), "emit": re_.as_dict()}


def autotune_compact(ctx: Context, values):
    """Autotuner of the compaction tile. Returns (indices, report)."""
    n = values.numel()
    out = torch.zeros(max(n, 1), dtype=torch.int32, device=values.device)
    cnt = torch.zeros(1, dtype=torch.int32, device=values.device)
    rep = native.TuneReport()
    call("tn_autotune_compact", ctx.handle, _stream(), n, _ptr(values), _ptr(out), _ptr(cnt), ctypes.byref(rep))
    return out[:int(cnt.item())], rep.as_dict()


def scan_offsets(ctx: Context, counts, batch_size: int):
    n = counts.numel()
    offsets = torch.zeros(n, dtype=torch.int32, device=counts.device)
    info = torch.zeros(4, dtype=torch.int32, device=counts.device)
    call("tn_scan_offsets", ctx.handle, _stream(), n, _ptr(counts), _ptr(offsets), batch_size, _ptr(info))
    return offsets, info


def compact_nonzero(ctx: Context, values):
    n = values.numel()
    out = torch.zeros(n, dtype=torch.int32, device=values.device)
    cnt = torch.zeros(1, dtype=torch.int32, device=values.device)
    call("tn_compact_nonzero", ctx.handle, _stream(), n, _ptr(values), _ptr(out), _ptr(cnt))
    return out, cnt


# ---- plain march ------------------------------------------------------------------------
def plain_march_count(grid, bitfield, bbox, march, n_rays, ray_stride, ori, dir_, ray_t, ray_t_max, alive):
    n_steps = torch.zeros(ray_stride, dtype=torch.int32, device=ori.device)
    g, b, m = grid.desc(), bbox_desc(bbox), march.desc()
    call("tn_plain_march_count", _stream(), ctypes.byref(g), _ptr(bitfield), ctypes.byref(b), ctypes.byref(m), n_rays,
         ray_stride, _ptr(ori), _ptr(dir_), _ptr(ray_t), _ptr(ray_t_max), _ptr(alive), _ptr(n_steps))
    return n_steps


def plain_scan_cut(n, n_steps, batch_size, offsets=None):
    if offsets is None:
        offsets = torch.zeros(n_steps.numel(), dtype=torch.int32, device=n_steps.device)
    nr, ns = ctypes.c_uint32(0), ctypes.c_uint32(0)
    call("tn_plain_scan_cut_sync", _stream(), n, _ptr(n_steps), _ptr(offsets), batch_size, ctypes.byref(nr),
         ctypes.byref(ns))
    return offsets, nr.value, ns.value


def plain_march_emit(grid, bitfield, bbox, march, inv_aabb, n_rays, ray_stride, sample_stride, ori, dir_, ray_t,
                     offsets, alive, n_steps, ray_img_id=None, samples=None):
    if samples is None:
        samples = alloc_samples(sample_stride, ori.device)
    g, b, m = grid.desc(), bbox_desc(bbox), march.desc()
    call("tn_plain_march_emit", _stream(), ctypes.byref(g), _ptr(bitfield), ctypes.byref(b), ctypes.byref(m), inv_aabb,
         n_rays, ray_stride, sample_stride, _ptr(ray_img_id), _ptr(ori), _ptr(dir_), _ptr(ray_t), _ptr(offsets),
         _ptr(alive), _ptr(n_steps), _ptr(samples["img_id"]), _ptr(samples["t"]), _ptr(samples["pos"]),
         _ptr(samples["dir"]), _ptr(samples["dt"]), _ptr(samples["m_norm"]), _ptr(samples["dt_norm"]))
    return samples


# ---- several scenes in one launch ----------------------------------------------------------
def scene_table(scenes):
    """scenes: sequence of dicts with grid (GridSpec), bitfield (device tensor), bbox, march
    (MarchSpec), inv_aabb, ray_begin, n_rays. Returns a ctypes array of tn_scene (keeps the
    bitfield tensors alive)."""
    from .native import SceneDesc
    arr = (SceneDesc * len(scenes))()
    keep = []
    for k, sc in enumerate(scenes):
        arr[k].grid = sc["grid"].desc()
        arr[k].bitfield = _ptr(sc["bitfield"])
        arr[k].bbox = bbox_desc(sc["bbox"])
        arr[k].march = sc["march"].desc()
        arr[k].inv_aabb_size = float(sc["inv_aabb"])
        arr[k].ray_begin = int(sc["ray_begin"])
        arr[k].n_rays = int(sc["n_rays"])
        keep.append(sc["bitfield"])
    arr._keep = keep
    return arr


def multi_march_count(ctx, table, ray_stride, ori, dir_, ray_t, ray_t_max, alive, n_steps=None, scene_samples=None,
                      info=None):
    """Count pass of every scene of `table` in one persistent launch. Returns (n_steps
    uint32[ray_stride], scene_samples uint32[n_scenes], info uint32[4] = total rays, total
    samples)."""
    n = len(table)
    dev = ori.device
    if n_steps is None:
        n_steps = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if scene_samples is None:
        scene_samples = torch.zeros(n, dtype=torch.int32, device=dev)
    if info is None:
        info = torch.zeros(4, dtype=torch.int32, device=dev)
    call("tn_multi_march_count", ctx.handle, _stream(), n, ctypes.addressof(table), ray_stride, _ptr(ori), _ptr(dir_), _ptr(ray_t),
         _ptr(ray_t_max), _ptr(alive), _ptr(n_steps), _ptr(scene_samples), _ptr(info))
    return n_steps, scene_samples, info


def multi_march_emit(ctx, table, ray_stride, sample_stride, ori, dir_, ray_t, alive, n_steps, ray_img_id=None,
                     samples=None, offsets=None):
    """Offsets and samples of every scene of `table`, packed scene after scene, after
    multi_march_count on the same context."""
    dev = ori.device
    if samples is None:
        samples = alloc_samples(sample_stride, dev)
    if offsets is None:
        offsets = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    call("tn_multi_march_emit", ctx.handle, _stream(), len(table), ctypes.addressof(table), ray_stride, sample_stride,
         _ptr(ray_img_id),
         _ptr(ori), _ptr(dir_), _ptr(ray_t), _ptr(alive), _ptr(n_steps), _ptr(offsets), _ptr(samples["img_id"]),
         _ptr(samples["t"]), _ptr(samples["pos"]), _ptr(samples["dir"]), _ptr(samples["dt"]), _ptr(samples["m_norm"]),
         _ptr(samples["dt_norm"]))
    return offsets, samples


def autotune_multi(ctx, table, ray_stride, sample_stride, ori, dir_, ray_t, ray_t_max, alive, ray_img_id=None,
                   n_steps=None, scene_samples=None, info=None, offsets=None, samples=None):
    """Autotuner of the multi-scene chunk size and emit shape. Returns (n_steps, scene_samples,
    info, offsets, samples, reports) with the outputs of one count + emit with the chosen shapes."""
    dev = ori.device
    if n_steps is None:
        n_steps = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if scene_samples is None:
        scene_samples = torch.zeros(len(table), dtype=torch.int32, device=dev)
    if info is None:
        info = torch.zeros(4, dtype=torch.int32, device=dev)
    if offsets is None:
        offsets = torch.zeros(ray_stride, dtype=torch.int32, device=dev)
    if samples is None:
        samples = alloc_samples(sample_stride, dev)
    rc, re_ = native.TuneReport(), native.TuneReport()
    call("tn_autotune_multi", ctx.handle, _stream(), len(table), ctypes.addressof(table), ray_stride,
         _ptr(ray_img_id), _ptr(ori), _ptr(dir_), _ptr(ray_t), _ptr(ray_t_max), _ptr(alive), _ptr(n_steps),
         _ptr(scene_samples), _ptr(info), sample_stride, _ptr(offsets), _ptr(samples["img_id"]), _ptr(samples["t"]),
         _ptr(samples["pos"]), _ptr(samples["dir"]), _ptr(samples["dt"]), _ptr(samples["m_norm"]),
         _ptr(samples["dt_norm"]), ctypes.byref(rc), ctypes.byref(re_))
    return n_steps, scene_samples, info, offsets, samples, {"count": rc.as_dict(), "emit": re_.as_dict()}


# ---- compositor / losses ------------------------------------------------------------------
def composite_fwd(ctx, rb: RayBatchDesc, density, rgb, dt, activation=0, min_t=1e-4, out=None):
    dev = density.device
    rs = rb.ray_stride
    if out is None:
        out = dict(rgba=torch.zeros(4 * rs, dtype=torch.float32, device=dev),
                   depth=torch.zeros(rs, dtype=torch.float32, device=dev),
                   n_used=torch.zeros(rs, dtype=torch.int32, device=dev))
    call("tn_composite_fwd", ctx.handle, _stream(), ctypes.byref(rb), activation, min_t, _ptr(density), _ptr(rgb),
         _ptr(dt), _ptr(out["rgba"]), _ptr(out["depth"]), _ptr(out["n_used"]))
    return out


def composite_bwd(ctx, rb: RayBatchDesc, density, rgb, dt, depth, n_used, grad_rgba, activation=0, out=None):
    """Compositor VJP. Returns (dL/d density, dL/d rgb); `out` = (dd, drgb) reuses buffers."""
    dev = density.device
    ss = rb.sample_stride
    if out is None:
        dd = torch.zeros(ss, dtype=torch.float32, device=dev)
        drgb = torch.zeros(3 * ss, dtype=torch.float32, device=dev)
    else:
        dd, drgb = out
    call("tn_composite_bwd", ctx.handle, _stream(), ctypes.byref(rb), activation, _ptr(density), _ptr(rgb), _ptr(dt),
         _ptr(depth), _ptr(n_used), _ptr(grad_rgba), _ptr(dd), _ptr(drgb))
    return dd, drgb


def composite_fwd_store(ctx, rb: RayBatchDesc, density, rgb, dt, activation=0, min_t=1e-4, out=None):
    """Compositor forward that also stores every composited sample's transmittance (after the
    sample) and weight, for composite_bwd_stored."""
    dev = density.device
    rs, ss = rb.ray_stride, rb.sample_stride
    if out is None:
        out = dict(rgba=torch.zeros(4 * rs, dtype=torch.float32, device=dev),
                   n_used=torch.zeros(rs, dtype=torch.int32, device=dev),
                   t_saved=torch.empty(ss, dtype=torch.float32, device=dev),
                   w_saved=torch.empty(ss, dtype=torch.float32, device=dev))
    call("tn_composite_fwd_store", ctx.handle, _stream(), ctypes.byref(rb), activation, min_t, _ptr(density),
         _ptr(rgb), _ptr(dt), _ptr(out["rgba"]), _ptr(out["n_used"]), _ptr(out["t_saved"]), _ptr(out["w_saved"]))
    return out


def composite_bwd_stored(ctx, rb: RayBatchDesc, density, rgb, dt, n_used, t_saved, w_saved, grad_rgba, activation=0,
                         out=None):
    dev = density.device
    ss = rb.sample_stride
    if out is None:
        out = (torch.zeros(ss, dtype=torch.float32, device=dev), torch.zeros(3 * ss, dtype=torch.float32, device=dev))
    dd, drgb = out
    call("tn_composite_bwd_stored", ctx.handle, _stream(), ctypes.byref(rb), activation, _ptr(density), _ptr(rgb),
         _ptr(dt), _ptr(n_used), _ptr(t_saved), _ptr(w_saved), _ptr(grad_rgba), _ptr(dd), _ptr(drgb))
    return dd, drgb


def recon_loss_fwd_bwd(ctx, rb: RayBatchDesc, density, rgb, dt, target_rgba, bg_rgb, inv_nrays, grad_scale=1.0,
                       activation=0, min_t=1e-4):
    dev = density.device
    rs, ss = rb.ray_stride, rb.sample_stride
    out = dict(ray_rgba=torch.zeros(4 * rs, dtype=torch.float32, device=dev),
               loss=torch.zeros(4 * rs, dtype=torch.float32, device=dev),
               loss_sum=torch.zeros(1, dtype=torch.float32, device=dev),
               dL_ddensity=torch.zeros(ss, dtype=torch.float32, device=dev),
               dL_drgb=torch.zeros(3 * ss, dtype=torch.float32, device=dev))
    call("tn_recon_loss_fwd_bwd", ctx.handle, _stream(), ctypes.byref(rb), activation, min_t, inv_nrays, grad_scale,
         _ptr(density), _ptr(rgb), _ptr(dt), _ptr(target_rgba), _ptr(bg_rgb), _ptr(out["ray_rgba"]), _ptr(out["loss"]),
         _ptr(out["loss_sum"]), _ptr(out["dL_ddensity"]), _ptr(out["dL_drgb"]))
    return out


def distortion_fwd_bwd(ctx, rb: RayBatchDesc, density, m_norm, dt_norm, lam, activation=0, grad_ray=None,
                       backward=True):
    dev = density.device
    out = dict(ray_loss=torch.zeros(rb.ray_stride, dtype=torch.float32, device=dev),
               loss_sum=torch.zeros(1, dtype=torch.float32, device=dev),
               dL_ddensity=torch.zeros(rb.sample_stride, dtype=torch.float32, device=dev) if backward else None)
    call("tn_distortion_fwd_bwd", ctx.handle, _stream(), ctypes.byref(rb), activation, lam, _ptr(density),
         _ptr(m_norm), _ptr(dt_norm), _ptr(grad_ray), _ptr(out["ray_loss"]), _ptr(out["loss_sum"]),
         _ptr(out["dL_ddensity"]))
    return out


def grad_epilogue(n_samples, loss_scale, dL_rec, dL_dist, t, grad_out, n_samples_dev=None):
    call("tn_grad_epilogue", _stream(), n_samples, _ptr(n_samples_dev), loss_scale, _ptr(dL_rec), _ptr(dL_dist), _ptr(t),
         _ptr(grad_out))
    return grad_out


def train_losses(ctx, rb: RayBatchDesc, density, rgb, dt, m_norm, dt_norm, t, target_rgba, bg_rgb, grad_density,
                 inv_nrays=0.0, inv_nrays_from=None, grad_scale=1.0, lam=0.0, activation=0, min_t=1e-4,
                 ray_rgba=None, dL_drgb=None, loss_sums=None):
    dev = density.device
    if dL_drgb is None:
        dL_drgb = torch.zeros(3 * rb.sample_stride, dtype=torch.float32, device=dev)
    if loss_sums is None:
        loss_sums = torch.zeros(2, dtype=torch.float32, device=dev)
    call("tn_train_losses", ctx.handle, _stream(), ctypes.byref(rb), activation, min_t, inv_nrays,
         _ptr(inv_nrays_from), grad_scale, lam, _ptr(density), _ptr(rgb), _ptr(dt), _ptr(m_norm), _ptr(dt_norm),
         _ptr(t), _ptr(target_rgba), _ptr(bg_rgb), _ptr(ray_rgba), _ptr(grad_density), _ptr(dL_drgb), _ptr(loss_sums))
    return grad_density, dL_drgb, loss_sums


def autotune_losses(ctx, rb: RayBatchDesc, density, rgb, dt, m_norm, dt_norm, t, target_rgba, bg_rgb, grad_density,
                    inv_nrays=0.0, inv_nrays_from=None, grad_scale=1.0, lam=0.0, activation=0, min_t=1e-4,
                    ray_rgba=None, dL_drgb=None, loss_sums=None):
    """Autotuner of the fused loss kernel's block size; the outputs are those of one
    train_losses call with the chosen shape. Returns (grad_density, dL_drgb, loss_sums, report)."""
    dev = density.device
    if dL_drgb is None:
        dL_drgb = torch.zeros(3 * rb.sample_stride, dtype=torch.float32, device=dev)
    if loss_sums is None:
        loss_sums = torch.zeros(2, dtype=torch.float32, device=dev)
    rep = native.TuneReport()
    call("tn_autotune_losses", ctx.handle, _stream(), ctypes.byref(rb), activation, min_t, inv_nrays,
         _ptr(inv_nrays_from), grad_scale, lam, _ptr(density), _ptr(rgb), _ptr(dt), _ptr(m_norm), _ptr(dt_norm),
         _ptr(t), _ptr(target_rgba), _ptr(bg_rgb), _ptr(ray_rgba), _ptr(grad_density), _ptr(dL_drgb), _ptr(loss_sums),
         ctypes.byref(rep))
    return grad_density, dL_drgb, loss_sums, rep.as_dict()


def plain_recon_loss(rb, density, rgb, dt, target_rgba, bg_rgb, inv_nrays, grad_scale=1.0, activation=0, min_t=1e-4):
    dev = density.device
    rs, ss = rb.ray_stride, rb.sample_stride
    loss = torch.zeros(4 * rs, dtype=torch.float32, device=dev)
    dd = torch.zeros(ss, dtype=torch.float32, device=dev)
    drgb = torch.zeros(3 * ss, dtype=torch.float32, device=dev)
    out = ctypes.c_float(0)
    call("tn_plain_recon_loss_sync", _stream(), ctypes.byref(rb), activation, min_t, inv_nrays, grad_scale,
         _ptr(density), _ptr(rgb), _ptr(dt), _ptr(target_rgba), _ptr(bg_rgb), _ptr(loss), _ptr(dd), _ptr(drgb),
         ctypes.byref(out))
    return loss, dd, drgb, out.value


def plain_distortion(rb, density, m_norm, dt_norm, lam, activation=0):
    dev = density.device
    rs, ss = rb.ray_stride, rb.sample_stride
    ray_scratch = torch.zeros(5 * rs, dtype=torch.float32, device=dev)
    sample_scratch = torch.zeros(2 * ss, dtype=torch.float32, device=dev)
    ray_loss = torch.zeros(rs, dtype=torch.float32, device=dev)
    dd = torch.zeros(ss, dtype=torch.float32, device=dev)
    out = ctypes.c_float(0)
    call("tn_plain_distortion_sync", _stream(), ctypes.byref(rb), activation, lam, _ptr(density), _ptr(m_norm),
         _ptr(dt_norm), _ptr(ray_scratch), _ptr(sample_scratch), _ptr(ray_loss), _ptr(dd), ctypes.byref(out))
    return ray_loss, dd, out.value


def plain_grad_epilogue(n_samples, loss_scale, dL_rec, dL_dist, t, grad_out):
    call("tn_plain_grad_epilogue", _stream(), n_samples, loss_scale, _ptr(dL_rec), _ptr(dL_dist), _ptr(t),
         _ptr(grad_out))
    return grad_out


# ---- occupancy ------------------------------------------------------------------------------
def occupancy_sample_points(grid: GridSpec, levels, cells, rand3, rand_stride, inv_aabb, pos_stride=None):
    n = levels.numel()
    pos_stride = pos_stride or n
    out = torch.zeros(3 * pos_stride, dtype=torch.float32, device=levels.device)
    g = grid.desc()
    call("tn_occupancy_sample_points", _stream(), ctypes.byref(g), n, _ptr(levels), _ptr(cells), _ptr(rand3),
         rand_stride, inv_aabb, _ptr(out), pos_stride)
    return out


def occupancy_update(ctx, grid: GridSpec, density, bitfield, levels, cells, values, rand_select, activation=0,
                     sample_all=False, decay=0.95, threshold=0.01, n_occupied=None):
    n = levels.numel() if levels is not None else 0
    if n_occupied is None:
        n_occupied = torch.zeros(1, dtype=torch.int32, device=density.device)
    g = grid.desc()
    call("tn_occupancy_update", ctx.handle, _stream(), ctypes.byref(g), _ptr(density), _ptr(bitfield), n,
         _ptr(levels), _ptr(cells), _ptr(values), _ptr(rand_select), activation, int(bool(sample_all)), decay,
         threshold, _ptr(n_occupied))
    return n_occupied


def plain_occupancy_update(grid: GridSpec, density, bitfield, levels, cells, values, rand_select, activation=0,
                           sample_all=False, decay=0.95, threshold=0.01, count_scratch=None):
    n = levels.numel() if levels is not None else 0
    if count_scratch is None:
        count_scratch = torch.zeros(grid.volume // 4, dtype=torch.uint8, device=density.device)
    out = ctypes.c_uint32(0)
    g = grid.desc()
    call("tn_plain_occupancy_update_sync", _stream(), ctypes.byref(g), _ptr(density), _ptr(bitfield), n,
         _ptr(levels), _ptr(cells), _ptr(values), _ptr(rand_select), activation, int(bool(sample_all)), decay,
         threshold, _ptr(count_scratch), ctypes.byref(out))
    return out.value


def popcount(ctx, bytes_):
    out = torch.zeros(1, dtype=torch.int32, device=bytes_.device)
    call("tn_popcount", ctx.handle, _stream(), bytes_.numel(), _ptr(bytes_), _ptr(out))
    return out


# ---- Adam ---------------------------------------------------------------------------------
def adam_step(weights, grads, m, v, steps, n_grid, n_mlp, lr, beta1=0.9, beta2=0.99, eps=1e-15, l2=1e-6,
              loss_scale=1.0, weights_copy=None, plain=False):
    name = "tn_plain_adam_step" if plain else "tn_adam_step"
    call(name, _stream(), weights.numel(), n_grid, n_mlp, loss_scale, lr, beta1, beta2, eps, l2, _ptr(weights),
         _ptr(weights_copy), _ptr(grads), _ptr(m), _ptr(v), _ptr(steps))


# ---- synthetic producer -----------------------------------------------------------------
def synth_field(pos, pos_stride, n, aabb_size, blobs, waves, n_dev=None, out_stride=None, want_rgb=True):
    dev = pos.device
    out_stride = out_stride or pos_stride
    sigma = torch.zeros(out_stride, dtype=torch.float32, device=dev)
    rgb = torch.zeros(3 * out_stride, dtype=torch.float32, device=dev) if want_rgb else None
    call("tn_synth_field", _stream(), n, _ptr(n_dev), pos_stride, _ptr(pos), aabb_size, blobs.shape[0], _ptr(blobs),
         _ptr(waves), _ptr(sigma), _ptr(rgb), out_stride)
    return sigma, rgb


# ---- backward variants of the memory study -------------------------------------------------
def backward_recompute(ctx, rb: RayBatchDesc, density, rgb, dt, m_norm, dt_norm, grad_rgba, lam, activation=0):
    """Compositor forward (per-ray state only) + backward that recomputes transmittance, and the
    fused distortion forward/backward. Returns (dL/d density of the compositor, dL/d rgb,
    dL/d density of the distortion loss)."""
    out = composite_fwd(ctx, rb, density, rgb, dt, activation=activation)
    dd, drgb = composite_bwd(ctx, rb, density, rgb, dt, out["depth"], out["n_used"], grad_rgba, activation=activation)
    d = distortion_fwd_bwd(ctx, rb, density, m_norm, dt_norm, lam, activation=activation)
    return dd, drgb, d["dL_ddensity"]


def backward_store(ctx, rb: RayBatchDesc, density, rgb, dt, m_norm, dt_norm, grad_rgba, lam, activation=0):
    """Compositor forward that stores per-sample transmittance and weights + backward that reads
    them, and the distortion loss as a forward kernel that stores per-sample running sums and a
    backward kernel that reads them. Same returns as backward_recompute."""
    st = composite_fwd_store(ctx, rb, density, rgb, dt, activation=activation)
    dd, drgb = composite_bwd_stored(ctx, rb, density, rgb, dt, st["n_used"], st["t_saved"], st["w_saved"], grad_rgba,
                                    activation=activation)
    _, ddist, _ = plain_distortion(rb, density, m_norm, dt_norm, lam, activation=activation)
    return dd, drgb, ddist


# ---- hash-grid encoding (the tiny-cuda-nn boundary) ----------------------------------------
@dataclass
class HashgridSpec:
    """Multiresolution hash encoding: level l of resolution floor(base_resolution *
    per_level_scale^l), 2 features a level, 2^log2_hashmap_size entries a level."""
    n_levels: int = 16
    log2_hashmap_size: int = 19
    base_resolution: float = 16.0
    per_level_scale: float = 2.0

    @classmethod
    def reference(cls, aabb_scale: float = 1.0, log2_hashmap_size: int = 19) -> "HashgridSpec":
        """The reference's density encoding (src/core/nerf-network.cu:87-106): 16 levels from 16 to
        2048 * aabb_scale."""
        import math
        n_max = 2048.0 * max(1.0, float(aabb_scale))
        return cls(16, log2_hashmap_size, 16.0, math.exp((math.log(n_max) - math.log(16.0)) / 15.0))

    def desc(self):
        return native.HashgridDesc(self.n_levels, self.log2_hashmap_size, float(self.base_resolution),
                                   float(self.per_level_scale))

    @property
    def n_features(self) -> int:
        return 2 * self.n_levels

    def n_params(self):
        """(hash entries' floats, the linear heads' floats)."""
        nh, nm = ctypes.c_uint64(0), ctypes.c_uint32(0)
        call("tn_hashgrid_n_params", ctypes.byref(self.desc()), ctypes.byref(nh), ctypes.byref(nm))
        return nh.value, nm.value

    def level(self, l: int):
        """(resolution, dense) of level l as the library computes them."""
        r, d = ctypes.c_uint32(0), ctypes.c_int(0)
        call("tn_hashgrid_level_resolution", ctypes.byref(self.desc()), l, ctypes.byref(r), ctypes.byref(d))
        return r.value, bool(d.value)


def hashgrid_encode(spec: HashgridSpec, pos, params, n, stride, n_dev=None, out=None):
    """Features [2 L][stride] (float32) of n positions pos[3][stride] in [0, 1]."""
    if out is None:
        out = torch.zeros(spec.n_features * stride, dtype=torch.float32, device=pos.device)
    call("tn_hashgrid_encode", _stream(), ctypes.byref(spec.desc()), n, _ptr(n_dev), stride, _ptr(pos), _ptr(params),
         _ptr(out))
    return out


def hashgrid_backward(spec: HashgridSpec, pos, dfeat, grads, n, stride, n_dev=None, touched=True):
    """grads += the encoding's transpose applied to dfeat [2 L][stride]. With touched: returns
    (bits, list, count) of the entries the n samples touched (fresh buffers)."""
    bits = lst = count = None
    if touched:
        entries = spec.n_levels << spec.log2_hashmap_size
        bits = torch.zeros((entries + 31) // 32, dtype=torch.int32, device=pos.device)
        lst = torch.zeros(entries, dtype=torch.int32, device=pos.device)
        count = torch.zeros(1, dtype=torch.int32, device=pos.device)
    call("tn_hashgrid_backward", _stream(), ctypes.byref(spec.desc()), n, _ptr(n_dev), stride, _ptr(pos), _ptr(dfeat),
         _ptr(grads), _ptr(bits), _ptr(lst), _ptr(count))
    return bits, lst, count


def hashgrid_clear_touched(lst, count, grads, bits, max_entries=None):
    call("tn_hashgrid_clear_touched", _stream(), _ptr(lst), _ptr(count),
         int(max_entries if max_entries is not None else lst.numel()), _ptr(grads), _ptr(bits))
