"""Batched multi-scene march (one persistent count launch, one emit launch) against the oracle
run scene by scene: per-scene counts, alive flags, sample totals, offsets and every emitted
sample value bit-exact."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise, dev, host
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


def test_multi_scene_march_bit_exact():
    from turbonerf_b200 import hotpath as hp
    params = scenes.multi_scene_params(seed=0x7C0, n_scenes=6, ray_lo=64, ray_hi=2048)
    ms = scenes.make_multi_scene(params, resolution=32)
    R = ms.rays.n
    table_in = []
    for sc, b in zip(ms.scenes, ms.ray_begin):
        g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
        m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
        table_in.append(dict(grid=g, bitfield=dev(sc.grid.bitfield), bbox=sc.bbox, march=m,
                             inv_aabb=1.0 / sc.aabb_size, ray_begin=int(b), n_rays=sc.rays.n))
    table = hp.scene_table(table_in)
    ctx = hp.Context()
    r = ms.rays
    ori, dr, t, tmax, alive = dev(r.ori), dev(r.dir), dev(r.t), dev(r.t_max), dev(r.alive)
    n_steps, scene_samples, info = hp.multi_march_count(ctx, table, R, ori, dr, t, tmax, alive)
    ss = int(host(info)[1]) + 64
    offsets, gs = hp.multi_march_emit(ctx, table, R, ss, ori, dr, t, alive, n_steps)
    assert ctx.check() == 0
    ns_g, alive_g, off_g = host(n_steps).view(np.uint32), host(alive), host(offsets).view(np.uint32)
    base = 0
    for k, (sc, b) in enumerate(zip(ms.scenes, ms.ray_begin)):
        n = sc.rays.n
        march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
        ns, al, guard = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
        assert guard == 0
        assert_bitwise(ns_g[b:b + n], ns, f"scene {k} n_steps")
        assert_bitwise(alive_g[b:b + n], al, f"scene {k} alive")
        assert int(host(scene_samples)[k]) == int(ns.sum())
        off = np.zeros(n, np.uint32)
        off[1:] = np.cumsum(ns[:-1], dtype=np.uint64).astype(np.uint32)
        assert_bitwise(off_g[b:b + n] - np.uint32(base), off, f"scene {k} offsets")
        nsamp = int(ns.sum())
        out = oracle.march_emit(sc.rays.as_dict(), sc.grid.as_dict(), march, off, ns, al, n, nsamp + 8,
                                1.0 / sc.aabb_size)
        for key in ("t", "dt", "m_norm", "dt_norm"):
            assert_bitwise(host(gs[key])[base:base + nsamp].view(np.uint32), out[key][:nsamp].view(np.uint32),
                           f"scene {k} {key}")
        for key in ("pos", "dir"):
            g3 = host(gs[key]).reshape(3, ss)[:, base:base + nsamp]
            r3 = out[key].reshape(3, nsamp + 8)[:, :nsamp]
            assert_bitwise(g3.ravel(), r3.ravel(), f"scene {k} {key}")
        base += nsamp
    assert int(host(info)[1]) == base


def test_multi_scene_at_full_size_march_and_losses():
    """At the multi-scene workload's full size: 16 scenes, each its own blob field and 1-5 cascades
    of 128^3 (grids built on the device from the field), 2^10..2^16 rays a scene (226,248 rays,
    6.6 M samples). The persistent count and the emit bit-exact against the oracle scene by scene;
    then the fused losses over the packed samples of all scenes in one launch (seeded sigma and rgb,
    lambda 1e-3, distance scaling) against the oracle's stages: the merged density gradient and
    dL/drgb within 1e-4 normwise at every legitimate transmittance cut, the loss sums within 1e-5."""
    import bench
    from tests.helpers import CUT_BAND, RTOL_GRAD, assert_norm_close, branch_cuts, pick_branches
    from turbonerf_b200 import hotpath as hp
    params = scenes.multi_scene_params(seed=0x7C3, n_scenes=16, ray_lo=1 << 10, ray_hi=1 << 16)
    ms, table_in = bench._multi_scene_gpu(params)
    table = hp.scene_table(table_in)
    ctx = hp.Context()
    r = ms.rays
    R = r.n
    ori, dr, t, tmax, alive = dev(r.ori), dev(r.dir), dev(r.t), dev(r.t_max), dev(r.alive)
    n_steps, scene_samples, info = hp.multi_march_count(ctx, table, R, ori, dr, t, tmax, alive)
    total = int(host(info)[1])
    ss = total + 64
    offsets, gs = hp.multi_march_emit(ctx, table, R, ss, ori, dr, t, alive, n_steps)
    assert ctx.check() == 0
    ns_g, alive_g, off_g = host(n_steps).view(np.uint32), host(alive), host(offsets).view(np.uint32)
    smp = {k: host(gs[k]) for k in ("t", "dt", "m_norm", "dt_norm", "pos", "dir")}
    base = 0
    for k, (sc, b, ti) in enumerate(zip(ms.scenes, ms.ray_begin, table_in)):
        n = sc.rays.n
        grid = dict(n_levels=ti["grid"].n_levels, res=ti["grid"].resolution, base=float(ti["grid"].base_size),
                    bitfield=host(ti["bitfield"]))
        march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
        ns, al, guard = oracle.march_count(sc.rays.as_dict(), grid, march)
        assert guard == 0
        assert_bitwise(ns_g[b:b + n], ns, f"scene {k} n_steps")
        assert_bitwise(alive_g[b:b + n], al, f"scene {k} alive")
        assert int(host(scene_samples)[k]) == int(ns.astype(np.int64).sum())
        off = np.zeros(n, np.uint32)
        off[1:] = np.cumsum(ns[:-1], dtype=np.uint64).astype(np.uint32)
        assert_bitwise(off_g[b:b + n] - np.uint32(base), off, f"scene {k} offsets")
        nsamp = int(ns.astype(np.int64).sum())
        out = oracle.march_emit(sc.rays.as_dict(), grid, march, off, ns, al, n, nsamp + 8, 1.0 / sc.aabb_size)
        for key in ("t", "dt", "m_norm", "dt_norm"):
            assert_bitwise(smp[key][base:base + nsamp].view(np.uint32), out[key][:nsamp].view(np.uint32),
                           f"scene {k} {key}")
        for key in ("pos", "dir"):
            g3 = smp[key].reshape(3, ss)[:, base:base + nsamp]
            r3 = out[key].reshape(3, nsamp + 8)[:, :nsamp]
            assert_bitwise(g3.ravel(), r3.ravel(), f"scene {k} {key}")
        base += nsamp
    assert total == base
    # the fused losses over every scene's rays at once
    rng = np.random.default_rng(0x7C5)
    sigma = np.zeros(ss, np.float32)
    sigma[:total] = np.clip(np.exp(rng.normal(0.0, 2.0, total)), 0.0, 1e4)
    rgb = np.zeros(3 * ss, np.float32)
    rgb[:] = rng.uniform(0.0, 1.0, 3 * ss)
    tgt = np.concatenate([rng.uniform(0, 1, 3 * R), np.ones(R)]).astype(np.float32)
    bg = rng.uniform(0, 1, 3 * R).astype(np.float32)
    grad_in = rng.normal(0, 1e-3, ss).astype(np.float32)
    lam = 1e-3
    counts, offs = ns_g, off_g
    rb = hp.ray_batch(n_steps, offsets, R, R, ss)
    gd = dev(grad_in.copy())
    gpu_gd, gpu_drgb, sums = hp.train_losses(ctx, rb, dev(sigma), dev(rgb), gs["dt"], gs["m_norm"], gs["dt_norm"],
                                             gs["t"], dev(tgt), dev(bg), gd, inv_nrays=1.0 / R, lam=lam)
    assert ctx.check() == 0
    t_world = smp["t"]
    dl, ddist = oracle.distortion_fwd_bwd(counts, offs, sigma, smp["m_norm"], smp["dt_norm"], lam, ss)
    n_alt, alt, over = oracle.cut_branches(counts, offs, sigma, smp["dt"], band=CUT_BAND)
    assert over == 0
    branches = []
    for fu in branch_cuts(n_alt, alt):
        rec = oracle.recon_fwd_bwd(counts, offs, sigma, rgb, smp["dt"], tgt, bg, R, ss, fixed_used=fu)
        rec["g"] = oracle.grad_epilogue(ss, 1.0, rec["dL_ddensity"], ddist, t_world, grad_in.astype(np.float64))
        branches.append(rec)
    # samples past the live ones are not the kernel's: compared as zeros on both sides
    gpu = dict(g=host(gpu_gd), dL_drgb=host(gpu_drgb))
    gpu["g"][total:] = 0.0
    for br in branches:
        br["g"] = np.array(br["g"], np.float64)
        br["g"][total:] = 0.0
    pick, _ = pick_branches(gpu, branches, counts, offs, sample_keys=("g", "dL_drgb"), sample_stride=ss,
                            carry_ray_keys=("loss",), ray_stride=R)
    assert_norm_close(gpu["g"], pick["g"], RTOL_GRAD, "merged density gradient, 16 scenes")
    assert_norm_close(gpu["dL_drgb"], pick["dL_drgb"], RTOL_GRAD, "dL/drgb, 16 scenes")
    s = host(sums)
    ref_rec = pick["loss"][:4 * R].sum() / R
    assert abs(s[0] - ref_rec) <= 1e-5 * abs(ref_rec)
    assert abs(s[1] - dl.mean()) <= 1e-5 * abs(dl.mean())
