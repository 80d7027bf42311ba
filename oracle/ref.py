"""TEST INFRASTRUCTURE ONLY: the reference's own hot-path kernels, compiled on the host.

oracle/ref_driver.cpp compiles TurboNeRF's kernel sources unchanged from the reference tree
against the host stand-ins in oracle/refstub/ (oracle/Makefile target `ref`), into
oracle/_ref/libturbonerf_ref.so. This module binds that library with ctypes. It exists to pin
the oracle restatement (oracle/oracle.cpp) to the reference's own arithmetic:
tests/golden/make_ref_golden.py writes fixtures from it, tests/test_ref_pin.py checks the oracle
against them (and, where the reference tree is present, against the live library), and the GPU
tests check the CUDA library against the same fixtures. bench.py --impl reference times it as
the reference's CPU implementation of the train step.

The library is built only where the reference tree exists; available() says whether it is
loadable. Arrays follow the reference's structure-of-arrays layout (component c of item i at
buf[c * stride + i]).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_ref", "libturbonerf_ref.so")
REFERENCE_TREE = os.environ.get("TN_REFERENCE_TREE", "/root/reference")

_lib = None


def build() -> str | None:
    """Compiles the reference's kernels when the reference tree is present (no-op when up to
    date); returns the library path, or None without the tree."""
    if not os.path.isdir(os.path.join(REFERENCE_TREE, "src")):
        return _SO if os.path.exists(_SO) else None
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REFERENCE_TREE}"], check=True)
    return _SO


def available() -> bool:
    return os.path.exists(_SO)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            raise RuntimeError("oracle/_ref/libturbonerf_ref.so is not built (needs the reference tree)")
        L = ctypes.CDLL(_SO)
        i32, u32, u64, f32, vp = ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float, ctypes.c_void_p
        sig = {
            "ref_num_threads": (i32, []),
            "ref_march_count": (None, [u32, u32, vp, i32, i32, vp, f32, f32, f32, vp, vp, vp, vp, vp, vp]),
            "ref_march_emit": (None, [u32, u32, vp, f32, i32, i32, vp, f32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp,
                                      vp, vp, vp, vp, vp, vp, vp]),
            "ref_fused_reconstruction": (None, [u32, u32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
            "ref_distortion": (None, [u32, u32, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
            "ref_grad_merge": (None, [u32, f32, vp, vp, vp, vp]),
            "ref_occupancy_decay_bits": (None, [i32, i32, f32, f32, vp, vp]),
            "ref_occupancy_sample_points": (None, [i32, i32, u32, u32, u32, i32, f32, vp, vp]),
            "ref_occupancy_decay": (None, [i32, i32, f32, vp]),
            "ref_occupancy_bits": (None, [i32, i32, f32, vp, vp]),
            "ref_popcount": (u32, [vp, u64]),
            "ref_adam_step": (None, [u32, u32, u32, f32, f32, f32, f32, f32, f32, vp, vp, vp, vp, vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def num_threads() -> int:
    return int(lib().ref_num_threads())


def march_count(rays, grid, march):
    """march_and_count_steps_per_ray_kernel. rays: dict(ori, dir, t, t_max, alive, stride, n);
    grid: dict(n_levels, res, bitfield) (the reference's level k spans 2^k); march: dict(bbox,
    cone, dt_min, dt_max). Returns (n_steps, alive)."""
    n, stride = rays["n"], rays["stride"]
    alive = _c(rays["alive"], np.uint8).copy()
    ori = _c(rays["ori"], np.float32).copy()
    t = _c(rays["t"], np.float32).copy()
    n_steps = np.zeros(n, np.uint32)
    lib().ref_march_count(n, stride, _p(_c(march["bbox"], np.float32)), grid["n_levels"], grid["res"],
                          _p(_c(grid["bitfield"], np.uint8)), march["cone"], march["dt_min"], march["dt_max"],
                          _p(_c(rays["dir"], np.float32)), _p(_c(rays["t_max"], np.float32)), _p(alive), _p(ori),
                          _p(t), _p(n_steps))
    return n_steps, alive


def _restride(a, comps, stride, n, new_stride, dtype):
    a = _c(a, dtype)
    out = np.zeros(comps * new_stride, dtype)
    for c in range(comps):
        out[c * new_stride:c * new_stride + n] = a[c * stride:c * stride + n]
    return out


def march_emit(rays, grid, march, offsets, n_steps, alive, n_rays, sample_stride, inv_aabb, img_id=None):
    """march_and_generate_network_positions_kernel over the first n_rays rays. The reference
    uses its batch size as the stride of both the ray inputs and the sample outputs, so the
    rays are laid out at the sample stride (which must be at least n_rays) for the call."""
    stride, ss = rays["stride"], sample_stride
    if ss < n_rays:
        raise ValueError("the reference's emit needs sample_stride >= n_rays")
    out = {"img_id": np.zeros(ss, np.uint32), "t": np.zeros(ss, np.float32), "pos": np.zeros(3 * ss, np.float32),
           "dir": np.zeros(3 * ss, np.float32), "dt": np.zeros(ss, np.float32), "m_norm": np.zeros(ss, np.float32),
           "dt_norm": np.zeros(ss, np.float32)}
    n = n_rays
    img = _restride(img_id if img_id is not None else np.zeros(n, np.uint32), 1, stride if img_id is not None else n,
                    n, ss, np.uint32)
    ori = _restride(rays["ori"], 3, stride, n, ss, np.float32)
    dir_ = _restride(rays["dir"], 3, stride, n, ss, np.float32)
    t = _restride(rays["t"], 1, stride, n, ss, np.float32)
    t_max = _restride(rays["t_max"], 1, stride, n, ss, np.float32)
    off = _restride(offsets, 1, len(offsets), n, ss, np.uint32)
    al = _restride(alive, 1, len(alive), n, ss, np.uint8)
    ns = _restride(n_steps, 1, len(n_steps), n, ss, np.uint32)
    lib().ref_march_emit(n, ss, _p(_c(march["bbox"], np.float32)), inv_aabb, grid["n_levels"], grid["res"],
                         _p(_c(grid["bitfield"], np.uint8)), march["dt_min"], march["dt_max"], march["cone"], _p(img),
                         _p(ori), _p(dir_), _p(t), _p(t_max), _p(off), _p(al), _p(ns), _p(out["img_id"]),
                         _p(out["t"]), _p(out["pos"]), _p(out["dir"]), _p(out["dt"]), _p(out["m_norm"]),
                         _p(out["dt_norm"]))
    return out


def fused_reconstruction(counts, offsets, density, rgb, dt, target_rgba, random_rgb, n_rays, stride,
                         inv_nrays=None, grad_scale=1.0):
    """fused_reconstruction_forward_backward_kernel; density goes through density_to_sigma.
    Ray arrays use `stride` (the reference's batch size) for their components, as do the
    per-sample buffers. Returns dict(loss [4*stride], dL_ddensity [stride], dL_drgb [3*stride])."""
    if inv_nrays is None:
        inv_nrays = 1.0 / max(n_rays, 1)
    loss = np.zeros(4 * stride, np.float32)
    dd = np.zeros(stride, np.float32)
    dc = np.zeros(3 * stride, np.float32)
    lib().ref_fused_reconstruction(n_rays, stride, inv_nrays, grad_scale, _p(_c(counts, np.uint32)),
                                   _p(_c(offsets, np.uint32)), _p(_c(random_rgb, np.float32)),
                                   _p(_c(target_rgba, np.float32)), _p(_c(density, np.float32)),
                                   _p(_c(rgb, np.float32)), _p(_c(dt, np.float32)), _p(loss), _p(dd), _p(dc))
    return dict(loss=loss, dL_ddensity=dd, dL_drgb=dc)


def distortion(counts, offsets, density, m_norm, dt_norm, sample_stride):
    """mipNeRF360 distortion forward + backward (lambda fixed at the reference's 0.01; density
    through density_to_sigma). Returns (per-ray loss, dL/ddensity [sample_stride])."""
    n = len(counts)
    ray5 = np.zeros(5 * n, np.float32)
    loss = np.zeros(n, np.float32)
    sample2 = np.zeros(2 * sample_stride, np.float32)
    dd = np.zeros(sample_stride, np.float32)
    lib().ref_distortion(n, sample_stride, _p(_c(counts, np.uint32)), _p(_c(offsets, np.uint32)),
                         _p(_c(density, np.float32)), _p(_c(m_norm, np.float32)), _p(_c(dt_norm, np.float32)),
                         _p(ray5), _p(loss), _p(sample2), _p(dd))
    return loss, dd


def grad_merge(n_samples, scale, dl_rec, dl_dist, t, grad_in):
    """copy_gradients_kernel<1, true> (twice) then apply_gradient_distance_scaling_kernel."""
    out = _c(grad_in, np.float32).copy()
    lib().ref_grad_merge(n_samples, scale, _p(_c(dl_rec, np.float32)),
                         _p(_c(dl_dist, np.float32)) if dl_dist is not None else None, _p(_c(t, np.float32)), _p(out))
    return out


def occupancy_decay_bits(density, bitfield, n_levels, res, decay, threshold):
    """decay_occupancy_grid_values_kernel (decay != 1) then update_occupancy_grid_bits_kernel."""
    d = _c(density, np.float32).copy()
    b = _c(bitfield, np.uint8).copy()
    lib().ref_occupancy_decay_bits(n_levels, res, decay, threshold, _p(d), _p(b))
    return d, b


def occupancy_decay(density, n_levels, res, decay):
    """decay_occupancy_grid_values_kernel, in place on a float32 array."""
    lib().ref_occupancy_decay(n_levels, res, decay, _p(density))
    return density


def occupancy_bits(density, bitfield, n_levels, res, threshold):
    """update_occupancy_grid_bits_kernel, in place on the bitfield (uint8)."""
    lib().ref_occupancy_bits(n_levels, res, threshold, _p(_c(density, np.float32)), _p(bitfield))
    return bitfield


def occupancy_sample_points(n_levels, res, n_cells, stride, start, level, inv_aabb, random3):
    out = np.zeros(3 * stride, np.float32)
    lib().ref_occupancy_sample_points(n_levels, res, n_cells, stride, start, level, inv_aabb,
                                      _p(_c(random3, np.float32)), _p(out))
    return out


def popcount(bytes_) -> int:
    b = _c(bytes_, np.uint8)
    return int(lib().ref_popcount(_p(b), b.size))


def adam_step(w, grads, m, v, steps, n_grid, n_net, lr, beta1=0.9, beta2=0.99, eps=1e-15, l2=1e-6, loss_scale=1.0,
              inplace=False, weights_copy=None):
    """ngp_adam_step<float>. Returns (w, m, v, steps): updated copies, or the arrays themselves
    updated in place with inplace=True (float32 / uint32 contiguous arrays). weights_copy
    receives the network-precision copy of the weights the kernel also writes."""
    if not inplace:
        w, m, v = (_c(a, np.float32).copy() for a in (w, m, v))
        steps = _c(steps, np.uint32).copy()
    w16 = weights_copy if weights_copy is not None else np.zeros_like(w)
    lib().ref_adam_step(w.size, n_grid, n_net, loss_scale, lr, beta1, beta2, eps, l2, _p(w), _p(w16),
                        _p(_c(grads, np.float32)), _p(m), _p(v), _p(steps))
    return w, m, v, steps
