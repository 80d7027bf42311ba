"""Parity of the CUDA occupancy-grid march and compaction against the CPU oracle.

Contract: per-ray counts, alive flags, offsets, the batch cut (n_rays, n_samples) and every
emitted per-sample value (t, pos, dir, dt, m_norm, dt_norm, img_id) are bit-exact.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise, dev, host, i32
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


def _gpu_inputs(sc):
    r = sc.rays
    return dict(ori=dev(r.ori), dir=dev(r.dir), t=dev(r.t), t_max=dev(r.t_max), alive=dev(r.alive))


def _specs(sc):
    from turbonerf_b200.hotpath import GridSpec, MarchSpec
    g = GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
    return g, m


def _oracle(sc, batch_size, sample_stride, img_id=None):
    march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
    ns, alive, guard = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
    assert guard == 0
    if batch_size == 0xFFFFFFFF:
        off = np.zeros(len(ns), np.uint32)
        off[1:] = np.cumsum(ns[:-1], dtype=np.uint64).astype(np.uint32)
        st, nr, nsamp = 0, len(ns), int(ns.sum())
    else:
        st, off, nr, nsamp = oracle.scan_cut(ns, batch_size)
    out = oracle.march_emit(sc.rays.as_dict(), sc.grid.as_dict(), march, off, ns, alive, nr, sample_stride,
                            1.0 / sc.aabb_size, img_id=img_id)
    return ns, alive, off, st, nr, nsamp, out


def _compare_samples(gs, out, nsamp, ss):
    for key in ("t", "dt", "m_norm", "dt_norm", "img_id"):
        assert_bitwise(host(gs[key])[:nsamp].view(np.uint32), out[key][:nsamp].view(np.uint32), key)
    for key in ("pos", "dir"):
        g = host(gs[key]).reshape(3, ss)[:, :nsamp]
        r = out[key].reshape(3, ss)[:, :nsamp]
        assert_bitwise(g.ravel(), r.ravel(), key)


@pytest.mark.parametrize("scene", ["single", "cascaded"])
def test_fused_march_bit_exact(scene):
    from turbonerf_b200 import hotpath as hp
    sc = scenes.march_scene_single() if scene == "single" else scenes.march_scene_cascaded()
    n = sc.rays.n
    batch_size = 0xFFFFFFFF if scene == "single" else 1 << 18
    ss = (sc.max_steps * n if scene == "single" else batch_size) + 64
    img_id = (np.arange(n) % 7).astype(np.uint32)
    ns_o, alive_o, off_o, st, nr_o, nsamp_o, out = _oracle(sc, batch_size, ss, img_id)
    assert st == 0 and nsamp_o > 0

    ctx = hp.Context()
    g, m = _specs(sc)
    x = _gpu_inputs(sc)
    bits = dev(sc.grid.bitfield)
    n_steps, info = hp.march_count(ctx, g, bits, sc.bbox, m, n, n, x["ori"], x["dir"], x["t"], x["t_max"], x["alive"],
                                   batch_size)
    offsets, gs = hp.march_emit(ctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, n, n, ss, info, x["ori"], x["dir"],
                                x["t"], x["alive"], n_steps, ray_img_id=i32(img_id))
    assert ctx.check() == 0
    info_h = host(info).view(np.uint32)
    assert_bitwise(host(n_steps).view(np.uint32), ns_o, "n_steps")
    assert_bitwise(host(x["alive"]), alive_o, "alive")
    assert_bitwise(host(offsets).view(np.uint32), off_o, "offsets")
    assert (int(info_h[0]), int(info_h[1])) == (nr_o, nsamp_o)
    assert int(info_h[2]) == int(ns_o.sum())
    _compare_samples(gs, out, nsamp_o, ss)


@pytest.mark.parametrize("scene", ["single", "cascaded"])
def test_plain_march_bit_exact(scene):
    from turbonerf_b200 import hotpath as hp
    sc = scenes.march_scene_single() if scene == "single" else scenes.march_scene_cascaded()
    n = sc.rays.n
    batch_size = (1 << 22) if scene == "single" else 1 << 18
    ss = batch_size + 64
    ns_o, alive_o, off_o, st, nr_o, nsamp_o, out = _oracle(sc, batch_size, ss)
    g, m = _specs(sc)
    x = _gpu_inputs(sc)
    bits = dev(sc.grid.bitfield)
    n_steps = hp.plain_march_count(g, bits, sc.bbox, m, n, n, x["ori"], x["dir"], x["t"], x["t_max"], x["alive"])
    offsets, nr, nsamp = hp.plain_scan_cut(n, n_steps, batch_size)
    gs = hp.plain_march_emit(g, bits, sc.bbox, m, 1.0 / sc.aabb_size, nr, n, ss, x["ori"], x["dir"], x["t"], offsets,
                             x["alive"], n_steps)
    assert_bitwise(host(n_steps).view(np.uint32), ns_o, "n_steps")
    assert_bitwise(host(offsets).view(np.uint32), off_o, "offsets")
    assert (nr, nsamp) == (nr_o, nsamp_o)
    gs["img_id"].zero_()
    out["img_id"][:] = 0
    _compare_samples(gs, out, nsamp_o, ss)


def test_rays_init_bbox_bit_exact():
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(5)
    for sc_rays, bbox in ((scenes.sphere_rays(rng, 5000), (-1.5, -1.5, -1.5, 1.5, 1.5, 1.5)),
                          (scenes.sphere_rays(rng, 5000, radius=2.0), (-8, -8, -8, 8, 8, 8))):
        t_o, tm_o, a_o = oracle.rays_init_bbox(sc_rays.ori, sc_rays.dir, sc_rays.stride, sc_rays.n, bbox)
        t, tm, a = hp.rays_init_bbox(dev(sc_rays.ori), dev(sc_rays.dir), sc_rays.n, sc_rays.stride, bbox)
        assert_bitwise(host(a), a_o, "alive")
        assert_bitwise(host(t), t_o, "t")
        assert_bitwise(host(tm), tm_o, "t_max")


def test_march_edge_cases():
    """Empty grid (no ray survives), full grid, a single ray, dead rays, the step cap, and
    rays that graze the box faces."""
    from turbonerf_b200 import hotpath as hp
    base = scenes.march_scene_single(n_rays=256)
    for case in ("empty", "full", "single", "dead", "cap", "graze"):
        sc = scenes.march_scene_single(n_rays=256)
        if case == "empty":
            sc.grid.bitfield[:] = 0
        elif case == "full":
            sc.grid.bitfield[:] = 0xFF
        elif case == "single":
            sc = scenes.march_scene_single(n_rays=1)
        elif case == "dead":
            sc.rays.alive[::2] = 0
        elif case == "cap":
            sc.max_steps = 7
        elif case == "graze":
            # rays along the box faces: origin on the x = +1.5 face, direction along -z
            r = sc.rays
            n = r.n
            ys = np.linspace(-1.5, 1.5, n).astype(np.float32)
            r.ori[:n] = 1.5
            r.ori[n:2 * n] = ys
            r.ori[2 * n:3 * n] = 3.0
            r.dir[:n] = 0.0
            r.dir[n:2 * n] = 0.0
            r.dir[2 * n:3 * n] = -1.0
            scenes.rays_init_bbox(r, sc.bbox)
            sc.grid.bitfield[:] = 0xFF
        n = sc.rays.n
        ss = 1024 * n + 64
        ns_o, alive_o, off_o, st, nr_o, nsamp_o, out = _oracle(sc, 0xFFFFFFFF, ss)
        ctx = hp.Context()
        g, m = _specs(sc)
        x = _gpu_inputs(sc)
        bits = dev(sc.grid.bitfield)
        n_steps, info = hp.march_count(ctx, g, bits, sc.bbox, m, n, n, x["ori"], x["dir"], x["t"], x["t_max"],
                                       x["alive"], 0xFFFFFFFF)
        offsets, gs = hp.march_emit(ctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, n, n, ss, info, x["ori"], x["dir"],
                                    x["t"], x["alive"], n_steps)
        flags = ctx.check()
        assert_bitwise(host(n_steps).view(np.uint32), ns_o, f"{case}: n_steps")
        assert_bitwise(host(offsets).view(np.uint32), off_o, f"{case}: offsets")
        if case == "empty":
            assert ns_o.sum() == 0 and flags & 8  # TN_FLAG_NO_SAMPLES
        else:
            assert flags == 0
            _compare_samples(gs, out, nsamp_o, ss)
        if case == "cap":
            assert ns_o.max() <= 7
    assert base.rays.n == 256


def test_batch_cut_matches_reference_rule():
    """tn_scan_offsets: exclusive scan and the reference cut (last ray whose offset is
    below batch_size is dropped) on ragged counts, including zeros and a batch that
    everything fits into."""
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(11)
    ctx = hp.Context()
    for n, B in ((1, 10), (2, 1), (1000, 5000), (70000, 1 << 20), (70000, 1 << 30), (129, 64)):
        counts = rng.integers(0, 40, n).astype(np.uint32)
        counts[rng.random(n) < 0.2] = 0
        st, off_o, nr_o, ns_o = oracle.scan_cut(counts, B)
        off, info = hp.scan_offsets(ctx, i32(counts), B)
        flags = ctx.check()
        assert_bitwise(host(off).view(np.uint32), off_o, f"offsets n={n}")
        info_h = host(info).view(np.uint32)
        assert int(info_h[0]) == nr_o, (n, B, info_h, nr_o)
        if st == 0:
            assert int(info_h[1]) == ns_o and flags == 0
        else:
            assert flags != 0


def test_compaction_indices():
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(3)
    ctx = hp.Context()
    for n in (1, 127, 128, 129, 5000, 300001):
        v = (rng.random(n) < 0.37).astype(np.uint32) * rng.integers(1, 9, n).astype(np.uint32)
        ref = oracle.compact_nonzero(v)
        out, cnt = hp.compact_nonzero(ctx, i32(v))
        c = int(host(cnt)[0])
        assert c == len(ref)
        assert_bitwise(host(out)[:c], ref, f"compaction n={n}")
