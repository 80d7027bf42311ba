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


# ---- the transmittance cut, decided by rounding on some rays ---------------------------------
# The reference stops compositing a ray after the first sample whose transmittance falls below
# min_transmittance (training-kernels-fused.cuh:255, 337). Where that transmittance lies within
# rounding of the threshold, an FP32 kernel and the FP64 oracle may stop one or more samples
# apart, and both answers are the reference's. oracle.cut_branches lists, per ray, every count
# at which a stop is legitimate; the helpers below evaluate the oracle at each of them and
# assemble, ray by ray, the reference closest to the GPU's result. Every ray is then checked at
# the full tolerance: a ray that matches none of its legitimate branches fails.
CUT_BAND = 1e-4


def branch_cuts(n_alt, alt):
    """fixed_used arrays, one per branch index: ray i takes its b-th legitimate count (its last
    one when it has fewer)."""
    n_alt = np.asarray(n_alt)
    B = int(n_alt.max()) if n_alt.size else 1
    idx = np.arange(len(n_alt))
    return [alt[idx, np.minimum(b, np.maximum(n_alt.astype(np.int64) - 1, 0))].astype(np.uint32) for b in range(B)]


def assert_legal_cut(gpu_used, n_alt, alt, what="n_used"):
    """The GPU's stop (samples composited per ray) is one of the ray's legitimate counts."""
    g = np.asarray(gpu_used, dtype=np.uint32)
    ok = ((alt == g[:, None]) & (np.arange(alt.shape[1])[None, :] < np.asarray(n_alt)[:, None])).any(axis=1)
    bad = np.nonzero(~ok)[0]
    assert bad.size == 0, f"{what}: {bad.size} rays stop at a count the oracle does not allow; first {bad[:5]}: " \
                          f"gpu {g[bad[:5]]}, allowed {[list(alt[i, :n_alt[i]]) for i in bad[:3]]}"


def _seg_max(x, counts, offsets):
    counts = np.asarray(counts)
    out = np.zeros(len(counts))
    nz = np.nonzero(counts > 0)[0]
    if nz.size:
        o = np.asarray(offsets, dtype=np.int64)[nz]
        end = int(o[-1] + counts[nz[-1]])
        out[nz] = np.maximum.reduceat(np.asarray(x, dtype=np.float64)[:end], o)
    return out


def pick_branches(gpu, branches, counts, offsets, ray_keys=(), sample_keys=(), ray_stride=None,
                  sample_stride=None, floor=FLOOR, carry_ray_keys=()):
    """Reference assembled ray by ray from the branch (oracle outputs at one set of cuts) closest
    to the GPU. gpu and every branch are dicts of arrays: ray_keys hold C components of
    ray_stride entries, sample_keys C components of sample_stride entries; carry_ray_keys are
    per-ray outputs taken from the chosen branch without taking part in the choice. Returns
    (assembled, choice per ray)."""
    counts = np.asarray(counts)
    offsets = np.asarray(offsets, dtype=np.int64)
    n = len(counts)
    if len(branches) == 1:
        return branches[0], np.zeros(n, np.int64)
    err = np.zeros((len(branches), n))
    for b, ref in enumerate(branches):
        e = np.zeros(n)
        for k in ray_keys:
            rs = ray_stride
            for c in range(len(ref[k]) // rs):
                r = np.asarray(ref[k][c * rs:c * rs + n], dtype=np.float64)
                g = np.asarray(gpu[k][c * rs:c * rs + n], dtype=np.float64)
                sc = np.abs(r) + floor * (np.max(np.abs(r)) if r.size else 0.0) + 1e-300
                e = np.maximum(e, np.abs(g - r) / sc)
        for k in sample_keys:
            ss = sample_stride
            for c in range(len(ref[k]) // ss):
                r = np.asarray(ref[k][c * ss:(c + 1) * ss], dtype=np.float64)
                g = np.asarray(gpu[k][c * ss:(c + 1) * ss], dtype=np.float64)
                m = np.maximum(_seg_max(np.abs(r), counts, offsets), floor * (np.max(np.abs(r)) if r.size else 0.0))
                e = np.maximum(e, _seg_max(np.abs(g - r), counts, offsets) / (m + 1e-300))
        err[b] = e
    choice = np.argmin(err, axis=0)
    out = {k: np.array(v, copy=True) for k, v in branches[0].items()}
    for i in np.nonzero(choice)[0]:
        src = branches[choice[i]]
        for k in tuple(ray_keys) + tuple(carry_ray_keys):
            for c in range(len(out[k]) // ray_stride):
                out[k][c * ray_stride + i] = src[k][c * ray_stride + i]
        o, cnt = int(offsets[i]), int(counts[i])
        for k in sample_keys:
            for c in range(len(out[k]) // sample_stride):
                a = c * sample_stride + o
                out[k][a:a + cnt] = src[k][a:a + cnt]
    return out, choice


# ---- element-wise gradient errors, reported beside the normwise gate -------------------------
# Gradients are gated normwise (max |g - ref| / max |ref|, per ray or per batch): an entry far
# smaller than the terms it is a difference of carries no relative accuracy in FP32. To keep that
# relaxation visible, every gradient check also records the worst element-wise relative error
# over the entries whose magnitude is at least ELEM_FLOOR of the largest one; conftest prints
# the table at the end of the run.
ELEM_FLOOR = 1e-3
ELEMENTWISE_REPORT: list = []


def record_elementwise(gpu, ref, what, floor=ELEM_FLOOR, mask=None):
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        g, r = g[mask], r[mask]
    if not r.size:
        return 0.0
    big = np.abs(r) >= floor * np.max(np.abs(r))
    worst = float(np.max(np.abs(g[big] - r[big]) / np.abs(r[big]))) if big.any() else 0.0
    ELEMENTWISE_REPORT.append((what, int(big.sum()), worst))
    return worst
