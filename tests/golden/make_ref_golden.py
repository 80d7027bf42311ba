"""Writes the reference-pinned fixtures tests/golden/ref_*.npz from the reference's own kernels.

The kernels are TurboNeRF's sources compiled unchanged on the host (oracle/ref_driver.cpp,
oracle/Makefile target `ref`, bound by oracle/ref.py), so every output here is the reference's
arithmetic on seeded inputs. tests/test_ref_pin.py checks that the oracle reproduces them (and,
where the reference tree is present, that they are what the reference library computes);
tests/test_gpu_ref_pin.py checks the CUDA library against them.

Large sample arrays are stored as SHA-256 digests of their bytes (each component's first
n_samples entries, in component order) beside their first values, which keeps the files small
while still pinning every bit.

Needs the reference tree (to build oracle/_ref). Regenerate with:
python tests/golden/make_ref_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from turbonerf_b200 import scenes  # noqa: E402

HEAD = 4096  # leading entries kept in full beside each digest


def digest(a, comps=1, stride=None, n=None) -> str:
    """SHA-256 of the first n entries of each of `comps` components of stride `stride`."""
    a = np.ascontiguousarray(a)
    stride = stride if stride is not None else a.size // comps
    n = n if n is not None else stride
    h = hashlib.sha256()
    for c in range(comps):
        h.update(np.ascontiguousarray(a[c * stride:c * stride + n]).tobytes())
    return h.hexdigest()


def march_inputs(n_rays=1024, seed=0x7B0):
    """The train step's scene (5 cascades of 128^3, extents 1..16, blob field, sphere rays)."""
    sc = scenes.march_scene_cascaded(seed=seed, n_rays=n_rays, n_levels=5)
    march = dict(bbox=np.float32(sc.bbox), cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=0)
    return sc, march


def march_fixture(n_rays=1024):
    sc, march = march_inputs(n_rays)
    rd = sc.rays.as_dict()
    grid = dict(n_levels=5, res=128, bitfield=sc.grid.bitfield)
    ns, alive = ref.march_count(rd, grid, march)
    n = sc.rays.n
    offsets = np.zeros(n, np.uint32)
    offsets[1:] = np.cumsum(ns[:-1], dtype=np.uint64).astype(np.uint32)
    total = int(ns.sum())
    ss = max(total, n)
    em = ref.march_emit(rd, grid, march, offsets, ns, alive, n, ss, 1.0 / sc.aabb_size)
    out = dict(ori=sc.rays.ori, dir=sc.rays.dir, t=sc.rays.t, t_max=sc.rays.t_max, alive_in=sc.rays.alive,
               bitfield=sc.grid.bitfield, bbox=np.float32(sc.bbox), cone=np.float32(march["cone"]),
               dt_min=np.float32(march["dt_min"]), dt_max=np.float32(march["dt_max"]),
               inv_aabb=np.float32(1.0 / sc.aabb_size), n_steps=ns, alive=alive, offsets=offsets,
               n_samples=np.uint32(total))
    for k, comps in (("t", 1), ("pos", 3), ("dir", 3), ("dt", 1), ("m_norm", 1), ("dt_norm", 1)):
        out["sha_" + k] = np.array(digest(em[k], comps, ss, total))
        out["head_" + k] = np.stack([em[k][c * ss:c * ss + min(HEAD, total)] for c in range(comps)])
    return out


def loss_inputs(seed, n_samples, mean, sigma_scale):
    """A compositor batch with the network's density (the reference applies density_to_sigma);
    one stride, the sample count, for the ray and sample buffers as in the reference."""
    sb = scenes.make_sample_batch(seed, n_samples, mean=mean)
    sigma = np.maximum(sb.sigma * np.float32(sigma_scale), np.float32(1e-6))
    density = (np.log(sigma) + 1.0).astype(np.float32)
    n, S = sb.n_rays, sb.n_samples
    tgt = np.zeros(4 * S, np.float32)
    bg = np.zeros(3 * S, np.float32)
    for c in range(4):
        tgt[c * S:c * S + n] = sb.target_rgba[c * n:(c + 1) * n]
    for c in range(3):
        bg[c * S:c * S + n] = sb.bg_rgb[c * n:(c + 1) * n]
    t_world = (sb.t * np.float32(0.9)).astype(np.float32)  # part of the samples below t = 1
    return sb, density, tgt, bg, t_world


def loss_fixture():
    """Reconstruction fwd/bwd, distortion fwd/bwd (lambda 0.01, the reference's constant) and
    the gradient merge with distance scaling, on a light batch and on an opaque one whose rays
    stop at the transmittance cut."""
    out = {}
    for tag, seed, sigma_scale in (("a", 0x7C0, 1.0), ("b", 0x7C1, 100.0)):
        sb, density, tgt, bg, t_world = loss_inputs(seed, 1 << 13, 48, sigma_scale)
        n, S = sb.n_rays, sb.n_samples
        rec = ref.fused_reconstruction(sb.counts, sb.offsets, density, sb.rgb, sb.dt, tgt, bg, n, S)
        dl, dd = ref.distortion(sb.counts, sb.offsets, density, sb.m_norm, sb.dt_norm, S)
        merged = ref.grad_merge(S, 1.0, rec["dL_ddensity"], dd, t_world, np.zeros(S, np.float32))
        out.update({f"{tag}_counts": sb.counts, f"{tag}_offsets": sb.offsets, f"{tag}_density": density,
                    f"{tag}_rgb": sb.rgb, f"{tag}_dt": sb.dt, f"{tag}_m_norm": sb.m_norm, f"{tag}_dt_norm": sb.dt_norm,
                    f"{tag}_t": t_world, f"{tag}_target": tgt, f"{tag}_bg": bg, f"{tag}_loss": rec["loss"],
                    f"{tag}_dL_ddensity": rec["dL_ddensity"], f"{tag}_dL_drgb": rec["dL_drgb"],
                    f"{tag}_dist_loss": dl, f"{tag}_dist_dd": dd, f"{tag}_merged": merged})
    return out


def occupancy_fixture():
    """Decay + threshold of a 3-level 32^3 grid, its popcount, and cell sample points of level 1."""
    rng = np.random.default_rng(0x7C2)
    L, res = 3, 32
    V = res ** 3
    d = np.where(rng.random((L, V)) < 0.4, rng.exponential(0.02, (L, V)), 0).astype(np.float32).ravel()
    bits = rng.integers(0, 8, V).astype(np.uint8)
    d_out, b_out = ref.occupancy_decay_bits(d, bits, L, res, 0.95, 0.01)
    n_cells, start, level = 4000, 100, 1
    rnd = rng.random(3 * n_cells).astype(np.float32)
    pts = ref.occupancy_sample_points(L, res, n_cells, n_cells, start, level, 1.0 / 4.0, rnd)
    return dict(density=d, bitfield=bits, n_levels=np.int32(L), res=np.int32(res), out_density=d_out,
                out_bitfield=b_out, n_occupied=np.uint32(ref.popcount(b_out)), n_cells=np.uint32(n_cells),
                start=np.uint32(start), level=np.int32(level), inv_aabb=np.float32(0.25), random3=rnd, points=pts)


def adam_fixture():
    """Three ngp_adam_step calls (lr 1e-2 / (1 + 3.3e-5 step), beta2 0.99) over 2^14 parameters,
    the hash grid's half of gradients zero (lazy updates)."""
    rng = np.random.default_rng(0x7C3)
    P, n_grid, n_mlp = 1 << 14, 12288, 4096
    w = rng.normal(0, 1e-2, P).astype(np.float32)
    g = rng.normal(0, 1e-3, P).astype(np.float32)
    g[:n_grid][rng.random(n_grid) < 0.5] = 0
    m, v, steps = np.zeros(P, np.float32), np.zeros(P, np.float32), np.zeros(P, np.uint32)
    lrs = [np.float32(1e-2 / (1.0 + 3.3e-5 * k)) for k in range(3)]
    W, M, Vv, S = w, m, v, steps
    for lr in lrs:
        W, M, Vv, S = ref.adam_step(W, g, M, Vv, S, n_grid, n_mlp, float(lr))
    return dict(w0=w, grads=g, n_grid=np.uint32(n_grid), n_mlp=np.uint32(n_mlp), lrs=np.float32(lrs), w=W, m=M,
                v=Vv, steps=S)


FIXTURES = (("ref_march", march_fixture), ("ref_losses", loss_fixture), ("ref_occupancy", occupancy_fixture),
            ("ref_adam", adam_fixture))


def main():
    if ref.build() is None:
        raise SystemExit("the reference tree is needed to build oracle/_ref")
    for name, fn in FIXTURES:
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn())
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
