"""Shared helpers for the parity tests (numpy <-> torch, tolerance checks)."""
from __future__ import annotations

import numpy as np

# Tolerances of the parity contract: composite RGBA / losses within 1e-5 relative, gradients
# within 1e-4 relative of the FP64 oracle. Elements whose reference value is tiny compared
# with the largest one cannot carry a relative bound in FP32 (their value is a difference of
# two much larger terms), so every check also accepts an absolute error of `floor` times the
# largest reference magnitude.
RTOL_COMPOSITE = 1e-5
RTOL_GRAD = 1e-4
FLOOR = 1e-6


def dev(a, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a)
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def i32(a):
    """uint32 numpy -> int32 CUDA tensor (the library reads it as uint32)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.uint32).view(np.int32))).cuda()


def host(t, dtype=None):
    a = t.detach().cpu().numpy()
    if dtype is not None:
        a = a.view(dtype) if a.dtype.itemsize == np.dtype(dtype).itemsize else a.astype(dtype)
    return a


def assert_bitwise(gpu, ref, what):
    g = np.ascontiguousarray(gpu)
    r = np.ascontiguousarray(ref)
    assert g.shape == r.shape, f"{what}: shape {g.shape} vs {r.shape}"
    gv = g.view(np.uint32) if g.dtype.itemsize == 4 else g
    rv = r.view(np.uint32) if r.dtype.itemsize == 4 else r
    bad = np.nonzero(gv != rv)[0]
    assert bad.size == 0, f"{what}: {bad.size} of {g.size} differ; first at {bad[:5]}: gpu {g[bad[:5]]} ref {r[bad[:5]]}"


def rel_err(gpu, ref, floor=FLOOR):
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    scale = np.abs(r) + floor * (np.max(np.abs(r)) if r.size else 0.0) + 1e-300
    return np.abs(g - r) / scale


def assert_close(gpu, ref, rtol, what, floor=FLOOR, mask=None):
    e = rel_err(gpu, ref, floor)
    if mask is not None:
        e = e[mask]
    worst = float(e.max()) if e.size else 0.0
    assert worst <= rtol, f"{what}: max relative error {worst:.3e} > {rtol:.1e}"
    return worst


def assert_norm_close(gpu, ref, rtol, what, mask=None):
    """Normwise relative error of a vector: max|g - r| / max|r| <= rtol.

    Gradient entries are sums of terms of both signs (T_{j+1} c_j minus a suffix sum,
    a residual pred - target), so an entry far smaller than its terms carries no relative
    accuracy in FP32 whatever the algorithm; the error of the vector is measured against
    its largest entry instead."""
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        g, r = g[mask], r[mask]
    denom = np.max(np.abs(r)) if r.size else 0.0
    err = float(np.max(np.abs(g - r)) / denom) if denom > 0 else float(np.max(np.abs(g - r), initial=0.0))
    assert err <= rtol, f"{what}: normwise relative error {err:.3e} > {rtol:.1e}"
    return err


def assert_per_ray_norm_close(gpu, ref, counts, offsets, rtol, what, ray_mask=None, floor=FLOOR):
    """Normwise relative error of each ray's gradient vector (over that ray's samples).
    A ray whose whole gradient is below `floor` times the batch's largest entry (it
    underflows in FP32) is measured against that floor instead."""
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    batch_floor = floor * float(np.max(np.abs(r))) if r.size else 0.0
    worst = 0.0
    for i in range(len(counts)):
        if ray_mask is not None and not ray_mask[i]:
            continue
        o, c = int(offsets[i]), int(counts[i])
        if c == 0:
            continue
        rr = r[o:o + c]
        m = max(float(np.max(np.abs(rr))), batch_floor)
        if m == 0:
            continue
        worst = max(worst, float(np.max(np.abs(g[o:o + c] - rr)) / m))
    assert worst <= rtol, f"{what}: worst per-ray normwise relative error {worst:.3e} > {rtol:.1e}"
    return worst


def expand_rays(mask_rays, counts, offsets, n_samples):
    """Per-sample mask from a per-ray mask."""
    m = np.zeros(n_samples, bool)
    for r in np.nonzero(mask_rays)[0]:
        m[offsets[r]:offsets[r] + counts[r]] = True
    return m
