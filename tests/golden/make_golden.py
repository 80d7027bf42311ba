"""Writes the small golden fixtures under tests/golden/ from the CPU oracle.

The reference ships no golden vectors, so these fixtures are the oracle's own outputs on
seeded inputs (the fixtures written from the reference's own kernels are ref_*.npz, made by
make_ref_golden.py). They pin the oracle against regressions (tests/test_golden.py) and give
the GPU tests a fixed expected answer (tests/test_gpu_golden.py). Regenerate with:
python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from turbonerf_b200 import scenes  # noqa: E402


def march_fixture():
    rng = np.random.default_rng(0x60)
    fld = scenes.make_blob_field(rng, 8)
    grid = scenes.build_grid(fld, n_levels=2, base_size=2.0, resolution=32)
    bbox = (-2.0, -2.0, -2.0, 2.0, 2.0, 2.0)
    rays = scenes.rays_init_bbox(scenes.sphere_rays(rng, 96, radius=3.0), bbox)
    march = dict(bbox=bbox, cone=1.0 / 256.0, dt_min=float(scenes.MIN_STEP_SIZE),
                 dt_max=float(np.float32(4.0) * scenes.MIN_STEP_SIZE), max_steps=0)
    ns, alive, _ = oracle.march_count(rays.as_dict(), grid.as_dict(), march)
    batch = int(ns.sum()) // 2
    st, off, nr, nsamp = oracle.scan_cut(ns, batch)
    em = oracle.march_emit(rays.as_dict(), grid.as_dict(), march, off, ns, alive, nr, batch + 1, 0.25)
    return dict(ori=rays.ori, dir=rays.dir, t=rays.t, t_max=rays.t_max, alive_in=rays.alive, bitfield=grid.bitfield,
                n_levels=np.int32(2), res=np.int32(32), base=np.float32(2.0), bbox=np.float32(bbox),
                cone=np.float32(march["cone"]), dt_min=np.float32(march["dt_min"]),
                dt_max=np.float32(march["dt_max"]), batch=np.uint32(batch), n_steps=ns, alive=alive, offsets=off,
                n_rays=np.uint32(nr), n_samples=np.uint32(nsamp), s_t=em["t"][:nsamp], s_pos=em["pos"].reshape(3, batch + 1)[:, :nsamp],
                s_dt=em["dt"][:nsamp], s_m_norm=em["m_norm"][:nsamp], s_dt_norm=em["dt_norm"][:nsamp])


def loss_fixture():
    """Reconstruction and distortion losses on a seeded batch. Where a ray's transmittance lies
    within rounding of the cut, the reference may stop it at more than one sample; br_* hold
    the outputs at every legitimate set of cuts (branch 0 is the FP64 cut of every ray)."""
    sb = scenes.make_sample_batch(0x61, 3000, mean=20)
    n, ss = sb.n_rays, sb.n_samples
    rec = oracle.recon_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n, ss)
    dl, dd = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, 1e-3, ss)
    n_alt, alt, _ = oracle.cut_branches(sb.counts, sb.offsets, sb.sigma, sb.dt, band=1e-4)
    br = []
    for b in range(int(n_alt.max())):
        fu = alt[np.arange(n), np.minimum(b, n_alt.astype(np.int64) - 1)]
        br.append(oracle.recon_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n,
                                       ss, fixed_used=fu))
    return dict(counts=sb.counts, offsets=sb.offsets, sigma=sb.sigma, rgb=sb.rgb, dt=sb.dt, m_norm=sb.m_norm,
                dt_norm=sb.dt_norm, target=sb.target_rgba, bg=sb.bg_rgb, ray_rgba=rec["ray_rgba"], loss=rec["loss"],
                dL_ddensity=rec["dL_ddensity"], dL_drgb=rec["dL_drgb"], n_used=rec["n_used"],
                ambiguous=rec["ambiguous"], dist_loss=dl, dist_dd=dd, n_alt=n_alt, alt=alt,
                **{"br_" + k: np.stack([r[k] for r in br]) for k in ("ray_rgba", "loss", "dL_ddensity", "dL_drgb")})


def occupancy_fixture():
    rng = np.random.default_rng(0x62)
    L, res = 3, 16
    V = res ** 3
    d = np.where(rng.random((L, V)) < 0.4, rng.exponential(0.05, (L, V)), 0).astype(np.float32)
    bits = np.zeros(V, np.uint8)
    for k in range(L):
        bits |= ((d[k] > 0.01).astype(np.uint8) << k)
    m = 3000
    lv = rng.integers(0, L, m).astype(np.int32)
    cells = rng.integers(0, V, m).astype(np.uint32)
    vals = rng.exponential(0.05, m).astype(np.float32)
    rsel = rng.random(m).astype(np.float32)
    nd, nb, nocc = oracle.occupancy_update(d, bits, L, res, lv, cells, vals, rsel)
    return dict(density=d, bitfield=bits, levels=lv, cells=cells, values=vals, rsel=rsel, out_density=nd,
                out_bitfield=nb, n_occupied=np.uint32(nocc))


def render_camera():
    """Camera of the render fixture: 24 x 16 pixels from (0.4, 0.9, 3.5) toward the centre."""
    eye = np.array([0.4, 0.9, 3.5])
    fwd = -eye / np.linalg.norm(eye)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    xf = np.stack([right, np.cross(fwd, right), fwd, eye], axis=1).astype(np.float32)
    return dict(width=24, height=16, near=0.1, far=50.0, focal=(17.0, 17.0), principal=(12.0, 8.0),
                shift=(0.0, 0.0), transform=xf)


def render_fixture():
    rng = np.random.default_rng(0x63)
    fld = scenes.make_blob_field(rng, 8)
    grid = scenes.build_grid(fld, n_levels=2, base_size=2.0, resolution=32)
    bbox = (-2.0, -2.0, -2.0, 2.0, 2.0, 2.0)
    cam = render_camera()
    rgba, amb, n = oracle.render(cam, bbox, bbox, grid.as_dict(), float(np.float32(scenes.MIN_STEP_SIZE)),
                                 1.0 / 256.0, 1e-4, fld.blobs, fld.waves, 4.0)
    return dict(bitfield=grid.bitfield, blobs=fld.blobs, waves=fld.waves,
                n_levels=np.int32(2), res=np.int32(32), base=np.float32(2.0), bbox=np.float32(bbox),
                transform=cam["transform"], rgba=rgba, ambiguous=amb, n_samples=np.int64(n))


def main():
    for name, fn in (("march_small", march_fixture), ("loss_small", loss_fixture),
                     ("occupancy_small", occupancy_fixture), ("render_small", render_fixture)):
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn())
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
