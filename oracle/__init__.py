"""TEST INFRASTRUCTURE ONLY: ctypes bindings to the CPU oracle (oracle/oracle.cpp).

The oracle restates the reference kernels of TurboNeRF's training hot path on the CPU
(FP32 with the reference's operation order for integer outputs, FP64 for float
outputs). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker or the timed CPU baseline. The reference ships no tests
or golden vectors; the restatement is pinned to the reference's own kernels compiled on the
host (oracle/ref.py, oracle/_ref) through the fixtures under tests/golden/ref_*.npz.

All arrays are numpy arrays in the reference's structure-of-arrays layout
(component c of item i at buf[c * stride + i]).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")

_lib = None


class Bbox(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")]


def build() -> str:
    """Compile oracle.cpp with the committed Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(os.path.join(_HERE, "oracle.cpp")):
            build()
        _lib = ctypes.CDLL(_SO)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _declare(L):
    i64, i32, u32, f32, f64, vp = (ctypes.c_int64, ctypes.c_int, ctypes.c_uint32,
                                   ctypes.c_float, ctypes.c_double, ctypes.c_void_p)
    sig = {
        "orc_morton3d": (u32, [u32, u32, u32]),
        "orc_hashgrid_encode": (None, [i32, i32, vp, vp, i64, i64, i64, vp, vp, vp]),
        "orc_hashgrid_backward": (None, [i32, i32, vp, vp, i64, i64, i64, vp, vp, vp, vp]),
        "orc_hash_heads_forward": (None, [i32, i64, i64, vp, vp, vp, vp, i64]),
        "orc_hash_heads_backward": (None, [i32, i64, i64, vp, vp, vp, vp, vp, vp]),
        "orc_morton3d_invert": (u32, [u32]),
        "orc_fdiv_ru": (f32, [f32, f32]),
        "orc_num_threads": (i32, []),
        "orc_set_num_threads": (None, [i32]),
        "orc_rays_init_bbox": (None, [i64, i64, ctypes.POINTER(Bbox), f32, vp, vp, vp, vp, vp]),
        "orc_march_count": (i64, [i64, i64, ctypes.POINTER(Bbox), i32, i32, f32, vp, f32, f32, f32, u32, u32,
                                  vp, vp, vp, vp, vp, vp]),
        "orc_scan_cut": (i32, [i64, vp, u32, vp, ctypes.POINTER(u32), ctypes.POINTER(u32)]),
        "orc_march_emit": (None, [i64, i64, i64, ctypes.POINTER(Bbox), f32, i32, i32, f32, vp, f32, f32, f32,
                                  vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
        "orc_compact_nonzero": (i64, [i64, vp, vp]),
        "orc_recon_fwd_bwd": (None, [i64, i64, i64, vp, vp, i32, vp, vp, vp, vp, vp, f64, f64, f64, f64,
                                     vp, vp, vp, vp, vp, vp, vp]),
        "orc_recon_loss_rgb": (f64, [i64, i64, i64, vp, vp, i32, vp, vp, vp, vp, vp, f64, f64, vp]),
        "orc_composite_fwd": (None, [i64, i64, i64, vp, vp, i32, vp, vp, vp, f64, vp, vp, vp]),
        "orc_composite_vjp": (None, [i64, i64, i64, vp, vp, i32, vp, vp, vp, f64, vp, vp, vp, vp]),
        "orc_cut_branches": (i64, [i64, vp, vp, i32, vp, vp, f64, f64, i32, vp, vp]),
        "orc_distortion_fwd_bwd": (None, [i64, vp, vp, i32, vp, vp, vp, f64, vp, vp, vp]),
        "orc_distortion_loss_sum": (f64, [i64, vp, vp, i32, vp, vp, vp, f64]),
        "orc_grad_epilogue": (None, [i64, f64, vp, vp, vp, vp]),
        "orc_occupancy_sample_points": (None, [i64, i32, f32, vp, vp, vp, i64, f32, vp, i64]),
        "orc_occupancy_update": (ctypes.c_uint64, [i32, i32, vp, vp, i64, vp, vp, vp, vp, i32, i32, f32, f32]),
        "orc_popcount": (ctypes.c_uint64, [i64, vp]),
        "orc_adam_step": (None, [i64, i64, i64, f64, f64, f64, f64, f64, f64, vp, vp, vp, vp, vp, vp]),
        "orc_blob_field": (None, [i64, i64, vp, f32, i32, vp, vp, vp, vp, i64]),
        "orc_render": (i64, [vp, ctypes.POINTER(Bbox), ctypes.POINTER(Bbox), i32, i32, f32, vp, f32, f32, f64, i32,
                             vp, vp, f32, vp, vp]),
        "orc_dataset_rays": (i64, [i64, i64, i64, i32, i32, vp, vp, ctypes.POINTER(Bbox), vp, f32, f32, vp, vp, vp,
                                   vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def bbox_struct(bbox):
    b = [float(v) for v in bbox]
    return Bbox(*b)


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def morton3d(x, y, z) -> int:
    return lib().orc_morton3d(int(x), int(y), int(z))


def morton3d_invert(v) -> int:
    return lib().orc_morton3d_invert(int(v))


def fdiv_ru(a, b) -> float:
    return lib().orc_fdiv_ru(float(a), float(b))


def rays_init_bbox(ori, dir_, stride, n, bbox, t_far=3.0e38):
    ori, dir_ = _c(ori, np.float32), _c(dir_, np.float32)
    t = np.zeros(n, np.float32)
    tmax = np.zeros(n, np.float32)
    alive = np.zeros(n, np.uint8)
    b = bbox_struct(bbox)
    lib().orc_rays_init_bbox(n, stride, ctypes.byref(b), t_far, _p(ori), _p(dir_), _p(t), _p(tmax), _p(alive))
    return t, tmax, alive


def march_count(rays, grid, march, max_iters=1 << 24):
    """rays: dict(ori, dir, t, t_max, alive, stride, n); grid: dict(n_levels, res, base, bitfield);
    march: dict(bbox, cone, dt_min, dt_max, max_steps). Returns (n_steps, alive, n_guard)."""
    n, stride = rays["n"], rays["stride"]
    alive = _c(rays["alive"], np.uint8).copy()
    n_steps = np.zeros(n, np.uint32)
    b = bbox_struct(march["bbox"])
    bits = _c(grid["bitfield"], np.uint8)
    ori, dir_ = _c(rays["ori"], np.float32), _c(rays["dir"], np.float32)
    t, tmax = _c(rays["t"], np.float32), _c(rays["t_max"], np.float32)
    guard = lib().orc_march_count(n, stride, ctypes.byref(b), grid["n_levels"], grid["res"], grid["base"],
                                  _p(bits), march["cone"], march["dt_min"], march["dt_max"],
                                  march.get("max_steps", 0), max_iters, _p(ori), _p(dir_), _p(t), _p(tmax),
                                  _p(alive), _p(n_steps))
    return n_steps, alive, guard


def scan_cut(n_steps, batch_size):
    n_steps = _c(n_steps, np.uint32)
    offsets = np.zeros(len(n_steps), np.uint32)
    nr, ns = ctypes.c_uint32(0), ctypes.c_uint32(0)
    st = lib().orc_scan_cut(len(n_steps), _p(n_steps), batch_size, _p(offsets), ctypes.byref(nr), ctypes.byref(ns))
    return st, offsets, nr.value, ns.value


def march_emit(rays, grid, march, offsets, n_steps, alive, n_rays, sample_stride, inv_aabb, img_id=None):
    stride = rays["stride"]
    ss = sample_stride
    out = {
        "img_id": np.zeros(ss, np.uint32), "t": np.zeros(ss, np.float32), "pos": np.zeros(3 * ss, np.float32),
        "dir": np.zeros(3 * ss, np.float32), "dt": np.zeros(ss, np.float32), "m_norm": np.zeros(ss, np.float32),
        "dt_norm": np.zeros(ss, np.float32),
    }
    b = bbox_struct(march["bbox"])
    bits = _c(grid["bitfield"], np.uint8)
    ori, dir_ = _c(rays["ori"], np.float32), _c(rays["dir"], np.float32)
    t = _c(rays["t"], np.float32)
    img = _c(img_id, np.uint32) if img_id is not None else None
    lib().orc_march_emit(n_rays, stride, ss, ctypes.byref(b), inv_aabb, grid["n_levels"], grid["res"], grid["base"],
                         _p(bits), march["cone"], march["dt_min"], march["dt_max"], _p(img), _p(ori), _p(dir_), _p(t),
                         _p(_c(offsets, np.uint32)), _p(_c(alive, np.uint8)), _p(_c(n_steps, np.uint32)),
                         _p(out["img_id"]), _p(out["t"]), _p(out["pos"]), _p(out["dir"]), _p(out["dt"]),
                         _p(out["m_norm"]), _p(out["dt_norm"]))
    return out


def compact_nonzero(values):
    values = _c(values, np.uint32)
    out = np.zeros(len(values), np.int32)
    c = lib().orc_compact_nonzero(len(values), _p(values), _p(out))
    return out[:c]


def recon_fwd_bwd(counts, offsets, density, rgb, dt, target_rgba, bg_rgb, ray_stride, sample_stride,
                  act=0, inv_nrays=None, grad_scale=1.0, min_t=1e-4, amb_eps=1e-4, fixed_used=None):
    """fixed_used (per ray, optional): composite exactly that many samples instead of stopping
    at the transmittance cut (to evaluate the other side of a cut that rounding decides)."""
    n = len(counts)
    if inv_nrays is None:
        inv_nrays = 1.0 / max(n, 1)
    ray_rgba = np.zeros(4 * ray_stride)
    loss = np.zeros(4 * ray_stride)
    dd = np.zeros(sample_stride)
    drgb = np.zeros(3 * sample_stride)
    used = np.zeros(n, np.uint32)
    amb = np.zeros(n, np.uint8)
    lib().orc_recon_fwd_bwd(n, ray_stride, sample_stride, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                            _p(_c(density, np.float32)), _p(_c(rgb, np.float32)), _p(_c(dt, np.float32)),
                            _p(_c(target_rgba, np.float32)), _p(_c(bg_rgb, np.float32)), inv_nrays, grad_scale,
                            min_t, amb_eps, _p(ray_rgba), _p(loss), _p(dd), _p(drgb), _p(used), _p(amb),
                            _p(_c(fixed_used, np.uint32) if fixed_used is not None else None))
    return dict(ray_rgba=ray_rgba, loss=loss, dL_ddensity=dd, dL_drgb=drgb, n_used=used, ambiguous=amb)


def recon_loss_rgb(counts, offsets, density, rgb, dt, target_rgba, bg_rgb, ray_stride, sample_stride,
                   act=0, inv_nrays=None, min_t=1e-4, fixed_used=None):
    n = len(counts)
    if inv_nrays is None:
        inv_nrays = 1.0 / max(n, 1)
    fu = _c(fixed_used, np.uint32) if fixed_used is not None else None
    return lib().orc_recon_loss_rgb(n, ray_stride, sample_stride, _p(_c(counts, np.uint32)),
                                    _p(_c(offsets, np.uint32)), act, _p(_c(density, np.float64)),
                                    _p(_c(rgb, np.float64)), _p(_c(dt, np.float64)), _p(_c(target_rgba, np.float64)),
                                    _p(_c(bg_rgb, np.float64)), inv_nrays, min_t, _p(fu))


def composite_fwd(counts, offsets, density, rgb, dt, ray_stride, sample_stride, act=0, min_t=1e-4,
                  fixed_used=None):
    n = len(counts)
    rgba = np.zeros(4 * ray_stride)
    used = np.zeros(n, np.uint32)
    lib().orc_composite_fwd(n, ray_stride, sample_stride, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                            _p(_c(density, np.float32)), _p(_c(rgb, np.float32)), _p(_c(dt, np.float32)), min_t,
                            _p(rgba), _p(used), _p(_c(fixed_used, np.uint32) if fixed_used is not None else None))
    return rgba, used


def composite_vjp(counts, offsets, density, rgb, dt, grad_rgba, ray_stride, sample_stride, act=0, min_t=1e-4,
                  fixed_used=None):
    n = len(counts)
    dd = np.zeros(sample_stride)
    drgb = np.zeros(3 * sample_stride)
    lib().orc_composite_vjp(n, ray_stride, sample_stride, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                            _p(_c(density, np.float32)), _p(_c(rgb, np.float32)), _p(_c(dt, np.float32)), min_t,
                            _p(_c(grad_rgba, np.float64)), _p(dd), _p(drgb),
                            _p(_c(fixed_used, np.uint32) if fixed_used is not None else None))
    return dd, drgb


def cut_branches(counts, offsets, density, dt, act=0, min_t=1e-4, band=1e-4, max_alt=8):
    """Per ray, the sample counts at which an FP32 compositor may legitimately stop (the FP64
    cut and every count whose transmittance after it is within `band` of min_t, up to the
    first sample clearly below). Returns (n_alt [n], alt [n, max_alt], overflow)."""
    n = len(counts)
    n_alt = np.zeros(n, np.uint32)
    alt = np.zeros((n, max_alt), np.uint32)
    over = lib().orc_cut_branches(n, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                                  _p(_c(density, np.float32)), _p(_c(dt, np.float32)), min_t, band, max_alt,
                                  _p(n_alt), _p(alt))
    return n_alt, alt, int(over)


def distortion_fwd_bwd(counts, offsets, density, m_norm, dt_norm, lam, n_samples, act=0, grad_ray=None):
    n = len(counts)
    loss = np.zeros(n)
    dd = np.zeros(max(n_samples, 1))
    gr = _c(grad_ray, np.float64) if grad_ray is not None else None
    lib().orc_distortion_fwd_bwd(n, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                                 _p(_c(density, np.float32)), _p(_c(m_norm, np.float32)), _p(_c(dt_norm, np.float32)),
                                 lam, _p(gr), _p(loss), _p(dd))
    return loss, dd


def distortion_loss_sum(counts, offsets, density, m_norm, dt_norm, lam, act=0):
    return lib().orc_distortion_loss_sum(len(counts), _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)), act,
                                         _p(_c(density, np.float64)), _p(_c(m_norm, np.float64)),
                                         _p(_c(dt_norm, np.float64)), lam)


def grad_epilogue(n_samples, loss_scale, dL_rec, dL_dist, sample_t, grad_in):
    g = _c(grad_in, np.float64).copy()
    lib().orc_grad_epilogue(n_samples, loss_scale, _p(_c(dL_rec, np.float64)),
                            _p(_c(dL_dist, np.float64) if dL_dist is not None else None),
                            _p(_c(sample_t, np.float32) if sample_t is not None else None), _p(g))
    return g


def occupancy_sample_points(levels, cells, rand3, rand_stride, res, base, inv_aabb, pos_stride):
    n = len(levels)
    out = np.zeros(3 * pos_stride, np.float32)
    lib().orc_occupancy_sample_points(n, res, base, _p(_c(levels, np.int32)), _p(_c(cells, np.uint32)),
                                      _p(_c(rand3, np.float32)), rand_stride, inv_aabb, _p(out), pos_stride)
    return out


def occupancy_update(density, bitfield, n_levels, res, levels, cells, values, rand_select, act=0,
                     sample_all=False, decay=0.95, threshold=0.01):
    d = _c(density, np.float32).copy()
    b = _c(bitfield, np.uint8).copy()
    n = len(levels)
    occ = lib().orc_occupancy_update(n_levels, res, _p(d), _p(b), n, _p(_c(levels, np.int32)),
                                     _p(_c(cells, np.uint32)), _p(_c(values, np.float32)),
                                     _p(_c(rand_select, np.float32)), act, int(bool(sample_all)), decay, threshold)
    return d, b, int(occ)


def popcount(bytes_):
    b = _c(bytes_, np.uint8)
    return int(lib().orc_popcount(len(b), _p(b)))


def adam_step(state, grad, n_grid, n_mlp, loss_scale=1.0, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-15, l2=1e-6):
    """state: dict(w=f64, m=f64, v=f64, steps=u32), updated in place."""
    n = len(state["w"])
    lib().orc_adam_step(n, n_grid, n_mlp, loss_scale, lr, beta1, beta2, eps, l2, _p(state["w"]),
                        _p(_c(grad, np.float32)), _p(state["m"]), _p(state["v"]), _p(state["steps"]), None)
    return state


def blob_field(pos, stride, n, aabb_size, blobs, waves, out_stride=None, want_rgb=True):
    out_stride = out_stride or n
    sig = np.zeros(n)
    rgb = np.zeros(3 * out_stride) if want_rgb else None
    lib().orc_blob_field(n, stride, _p(_c(pos, np.float32)), aabb_size, len(blobs), _p(_c(blobs, np.float32)),
                         _p(_c(waves, np.float32)), _p(sig), _p(rgb), out_stride)
    return sig, rgb


class Camera(ctypes.Structure):
    """Same layout as the library's tn_camera: transform = camera to world, row-major 3 x 4."""
    _fields_ = [("width", ctypes.c_int32), ("height", ctypes.c_int32), ("near", ctypes.c_float),
                ("far", ctypes.c_float), ("focal_x", ctypes.c_float), ("focal_y", ctypes.c_float),
                ("principal_x", ctypes.c_float), ("principal_y", ctypes.c_float), ("shift_x", ctypes.c_float),
                ("shift_y", ctypes.c_float), ("transform", ctypes.c_float * 12)]


def render(camera: dict, render_bbox, training_bbox, grid, dt_min, cone, min_t, blobs, waves, aabb_size):
    """Inference render of one NeRF whose network is the blob field. camera: dict(width,
    height, near, far, focal (fx, fy), principal (cx, cy), shift (sx, sy), transform [3][4]).
    Returns (rgba [h][w][4] float64, ambiguous [h][w] uint8 flags, queried samples)."""
    c = Camera()
    c.width, c.height = int(camera["width"]), int(camera["height"])
    c.near, c.far = float(camera["near"]), float(camera["far"])
    c.focal_x, c.focal_y = [float(v) for v in camera["focal"]]
    c.principal_x, c.principal_y = [float(v) for v in camera["principal"]]
    c.shift_x, c.shift_y = [float(v) for v in camera["shift"]]
    for k, v in enumerate(np.asarray(camera["transform"], np.float32)[:3, :4].reshape(-1)):
        c.transform[k] = float(v)
    n = c.width * c.height
    out = np.zeros(4 * n)
    amb = np.zeros(n, np.uint8)
    rb, tb = bbox_struct(render_bbox), bbox_struct(training_bbox)
    bits = _c(grid["bitfield"], np.uint8)
    total = lib().orc_render(ctypes.byref(c), ctypes.byref(rb), ctypes.byref(tb), grid["n_levels"], grid["res"],
                             grid["base"], _p(bits), dt_min, cone, min_t, len(blobs), _p(_c(blobs, np.float32)),
                             _p(_c(waves, np.float32)), aabb_size, _p(out), _p(amb))
    return out.reshape(c.height, c.width, 4), amb.reshape(c.height, c.width), int(total)


def camera_struct(camera: dict) -> "Camera":
    c = Camera()
    c.width, c.height = int(camera["width"]), int(camera["height"])
    c.near, c.far = float(camera["near"]), float(camera["far"])
    c.focal_x, c.focal_y = [float(v) for v in camera["focal"]]
    c.principal_x, c.principal_y = [float(v) for v in camera["principal"]]
    c.shift_x, c.shift_y = [float(v) for v in camera["shift"]]
    for k, v in enumerate(np.asarray(camera["transform"], np.float32)[:3, :4].reshape(-1)):
        c.transform[k] = float(v)
    return c


def dataset_rays(n_rays, cameras, images, bbox, random, alpha_threshold=1.0, alpha_probability=1.0):
    """Training rays from posed RGBA8 images [n][h][w][4]; random: [2][n_rays] draws. Returns a
    dict of the outputs ([c][n_rays] arrays; a dead ray's values other than alive are unspecified)
    and the live count."""
    images = _c(images, np.uint8)
    n_img, h, w = images.shape[:3]
    cams = (Camera * n_img)(*[camera_struct(c) for c in cameras])
    rs = n_rays
    out = dict(pix_rgba=np.zeros(4 * rs, np.float32), img_id=np.zeros(rs, np.uint32), ori=np.zeros(3 * rs, np.float32),
               dir=np.zeros(3 * rs, np.float32), t=np.zeros(rs, np.float32), t_max=np.zeros(rs, np.float32),
               alive=np.zeros(rs, np.uint8))
    b = bbox_struct(bbox)
    live = lib().orc_dataset_rays(n_rays, rs, n_img, w, h, cams, _p(images), ctypes.byref(b),
                                  _p(_c(random, np.float32)), alpha_threshold, alpha_probability, _p(out["pix_rgba"]),
                                  _p(out["img_id"]), _p(out["ori"]), _p(out["dir"]), _p(out["t"]), _p(out["t_max"]),
                                  _p(out["alive"]))
    return out, int(live)


# ---- hash-grid encoding and linear heads --------------------------------------------------
def hashgrid_levels(n_levels, log2_t, base_resolution, per_level_scale):
    """Per-level resolution floor(N_min b^l) (double precision, from N_min and b as the FP32 values
    the library's descriptor holds) and whether the level indexes its (res + 1)^3 vertices
    directly."""
    import math
    base, b = float(np.float32(base_resolution)), float(np.float32(per_level_scale))
    res = np.array([math.floor(base * math.pow(b, l)) for l in range(n_levels)], np.uint32)
    dense = np.array([1 if (int(r) + 1) ** 3 <= (1 << log2_t) else 0 for r in res], np.int32)
    return res, dense


def hashgrid_encode(levels, log2_t, pos, params, n, pstride=None, stride=None):
    """Features [2 L][stride] (float32, the library's operation order) of n positions [3][pstride]."""
    res, dense = levels
    pstride = pstride or n
    stride = stride or n
    feat = np.zeros(2 * len(res) * stride, np.float32)
    lib().orc_hashgrid_encode(len(res), log2_t, _p(_c(res, np.uint32)), _p(_c(dense, np.int32)), n, pstride, stride,
                              _p(_c(pos, np.float32)), _p(_c(params, np.float32)), _p(feat))
    return feat


def hashgrid_backward(levels, log2_t, pos, dfeat, n, pstride=None, stride=None):
    """(grads [L][2^log2_t][2] float64, touched [L 2^log2_t] uint8) of dL/dfeatures [2 L][stride]."""
    res, dense = levels
    pstride = pstride or n
    stride = stride or n
    L = len(res)
    grads = np.zeros(L * (1 << log2_t) * 2)
    touched = np.zeros(L * (1 << log2_t), np.uint8)
    lib().orc_hashgrid_backward(L, log2_t, _p(_c(res, np.uint32)), _p(_c(dense, np.int32)), n, pstride, stride,
                                _p(_c(pos, np.float32)), _p(_c(dfeat, np.float64)), _p(grads), _p(touched))
    return grads, touched


def hash_heads_forward(nf, feat, head, n, stride=None, ostride=None):
    """(density [n] float64, rgb [3][ostride] float64) of the linear heads [4][nf + 1]."""
    stride = stride or n
    ostride = ostride or n
    density = np.zeros(n)
    rgb = np.zeros(3 * ostride)
    lib().orc_hash_heads_forward(nf, n, stride, _p(_c(feat, np.float32)), _p(_c(head, np.float32)), _p(density),
                                 _p(rgb), ostride)
    return density, rgb


def hash_heads_backward(nf, feat, head, dL_ddensity, dL_drgb, n, stride=None):
    """(dfeat [nf][stride] float64, dhead [4][nf + 1] float64)."""
    stride = stride or n
    dfeat = np.zeros(nf * stride)
    dhead = np.zeros(4 * (nf + 1))
    lib().orc_hash_heads_backward(nf, n, stride, _p(_c(feat, np.float32)), _p(_c(head, np.float32)),
                                  _p(_c(dL_ddensity, np.float64)), _p(_c(dL_drgb, np.float64)), _p(dfeat), _p(dhead))
    return dfeat, dhead
