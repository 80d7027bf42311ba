"""Launch shapes and the autotuner on the GPU.

Contract: every valid launch shape (tn_tuning) gives bit-identical counts, offsets, samples,
per-ray colours and gradients; only the scalar loss sums may differ, by summation order. Each
autotuner leaves the outputs of one ordinary call with the shape it chose, and the trainer
trains identically (bit-exact weights) after tuning.
"""
import itertools

import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise, dev, host, i32
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu

COUNT = [32, 64, 128, 256]
EMIT = list(itertools.product([1, 2, 4, 8, 16], [1, 2, 4]))


def _march_inputs(sc):
    r = sc.rays
    return dev(r.ori), dev(r.dir), dev(r.t), dev(r.t_max), dev(r.alive)


def _march(hp, ctx, sc, batch, ss, img):
    g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
    n = sc.rays.n
    ori, dr, t, tmax, alive = _march_inputs(sc)
    bits = dev(sc.grid.bitfield)
    ns, info = hp.march_count(ctx, g, bits, sc.bbox, m, n, n, ori, dr, t, tmax, alive, batch)
    off, smp = hp.march_emit(ctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, n, n, ss, info, ori, dr, t, alive, ns,
                             ray_img_id=img)
    return dict(n_steps=host(ns), info=host(info), offsets=host(off), alive=host(alive),
                **{k: host(v) for k, v in smp.items()})


def _same(a, b, what, nsamp):
    for k in ("n_steps", "info", "offsets", "alive"):
        assert_bitwise(a[k], b[k], f"{what}: {k}")
    for k in ("t", "dt", "m_norm", "dt_norm", "img_id"):
        assert_bitwise(a[k][:nsamp], b[k][:nsamp], f"{what}: {k}")
    for k in ("pos", "dir"):
        ss = a[k].size // 3
        assert_bitwise(a[k].reshape(3, ss)[:, :nsamp], b[k].reshape(3, ss)[:, :nsamp], f"{what}: {k}")


def test_every_march_shape_is_bit_identical():
    """All 4 count block sizes x 15 emit shapes, with and without the SM reservation of
    side_sms, against the default shape, which is itself checked against the oracle (with the
    batch cut of training)."""
    from turbonerf_b200 import hotpath as hp
    sc = scenes.march_scene_cascaded()
    n = sc.rays.n
    batch = 1 << 18
    ss = batch + 64
    img = i32((np.arange(n) % 5).astype(np.uint32))
    ctx = hp.Context()
    base = _march(hp, ctx, sc, batch, ss, img)
    march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=sc.max_steps)
    ns_o, _, _ = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
    _, off_o, nr_o, nsamp = oracle.scan_cut(ns_o, batch)
    assert_bitwise(base["n_steps"].view(np.uint32), ns_o, "default shape vs oracle: n_steps")
    assert_bitwise(base["offsets"].view(np.uint32)[:nr_o], off_o[:nr_o], "default shape vs oracle: offsets")
    assert int(base["info"][1]) == nsamp
    for cg in COUNT:
        for w, rpw in EMIT:
            ctx.tuning = dict(count_rays_per_block=cg, emit_warps_per_block=w, emit_rays_per_warp=rpw,
                              side_sms=20 if (w + rpw) & 1 else 0)
            got = _march(hp, ctx, sc, batch, ss, img)
            _same(got, base, f"count {cg}, emit {w}x{rpw}", nsamp)
    assert ctx.check() == 0


def test_emit_uses_the_count_block_size_of_its_count():
    """Changing the tuning between count and emit does not break the emit: it keeps the
    grouping of the count that produced its block prefixes."""
    from turbonerf_b200 import hotpath as hp
    sc = scenes.march_scene_single(n_rays=2000)
    n = sc.rays.n
    g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
    ss = sc.max_steps * n + 64
    ctx = hp.Context()
    ref = _march(hp, ctx, sc, 0xFFFFFFFF, ss, None)
    ori, dr, t, tmax, alive = _march_inputs(sc)
    bits = dev(sc.grid.bitfield)
    ctx.tuning = dict(count_rays_per_block=256)
    ns, info = hp.march_count(ctx, g, bits, sc.bbox, m, n, n, ori, dr, t, tmax, alive, 0xFFFFFFFF)
    ctx.tuning = dict(count_rays_per_block=32, emit_rays_per_warp=4)
    off, smp = hp.march_emit(ctx, g, bits, sc.bbox, m, 1.0 / sc.aabb_size, n, n, ss, info, ori, dr, t, alive, ns)
    assert_bitwise(host(off), ref["offsets"], "offsets")
    nsamp = int(ref["info"][1])
    assert_bitwise(host(smp["t"])[:nsamp], ref["t"][:nsamp], "t")
    assert ctx.check() == 0


def test_autotune_march_leaves_one_calls_outputs():
    from turbonerf_b200 import hotpath as hp
    sc = scenes.march_scene_cascaded()
    n = sc.rays.n
    batch = 1 << 18
    ss = batch + 64
    ctx = hp.Context()
    base = _march(hp, ctx, sc, batch, ss, None)
    nsamp = int(base["info"][1])
    g = hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size)
    m = hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps)
    ori, dr, t, tmax, alive = _march_inputs(sc)
    tctx = hp.Context()
    ns, info, off, smp, reps = hp.autotune_march(tctx, g, dev(sc.grid.bitfield), sc.bbox, m, 1.0 / sc.aabb_size, n,
                                                 n, ori, dr, t, tmax, alive, batch, ss)
    got = dict(n_steps=host(ns), info=host(info), offsets=host(off), alive=host(alive),
               **{k: host(v) for k, v in smp.items()})
    _same(got, base, "after autotune", nsamp)
    assert reps["count"]["n_candidates"] == 4 and reps["emit"]["n_candidates"] == 15
    assert 0 < reps["count"]["best_ms"] <= reps["count"]["before_ms"]
    assert 0 < reps["emit"]["best_ms"] <= reps["emit"]["before_ms"]
    tun = tctx.tuning
    assert tun["count_rays_per_block"] in COUNT
    assert (tun["emit_warps_per_block"], tun["emit_rays_per_warp"]) in EMIT
    assert tctx.check() == 0


def _loss_batch():
    sb = scenes.make_sample_batch(0x7B4, 1 << 17, mean=48, max_count=1024)
    t_world = (sb.t * 0.9).astype(np.float32)
    g0 = np.random.default_rng(2).normal(0, 1e-3, sb.n_samples).astype(np.float32)
    return sb, t_world, g0


def _losses(hp, ctx, sb, t_world, g0, autotune=False):
    n = sb.n_rays
    rb = hp.ray_batch(i32(sb.counts), i32(sb.offsets), n, n, sb.n_samples)
    gd = dev(g0.copy())
    rgba = dev(np.zeros(4 * n, np.float32))
    fn = hp.autotune_losses if autotune else hp.train_losses
    out = fn(ctx, rb, dev(sb.sigma), dev(sb.rgb), dev(sb.dt), dev(sb.m_norm), dev(sb.dt_norm), dev(t_world),
             dev(sb.target_rgba), dev(sb.bg_rgb), gd, inv_nrays=1.0 / n, lam=1e-3, ray_rgba=rgba)
    return host(out[0]), host(out[1]), host(out[2]), host(rgba), (out[3] if autotune else None)


def test_every_loss_block_size_is_bit_identical():
    from turbonerf_b200 import hotpath as hp
    sb, t_world, g0 = _loss_batch()
    ctx = hp.Context()
    gd0, drgb0, sums0, rgba0, _ = _losses(hp, ctx, sb, t_world, g0)
    for w in (2, 4, 8):
        ctx.tuning = dict(loss_rays_per_block=w)
        gd, drgb, sums, rgba, _ = _losses(hp, ctx, sb, t_world, g0)
        assert_bitwise(gd, gd0, f"{w} warps: grad density")
        assert_bitwise(drgb, drgb0, f"{w} warps: dL/drgb")
        assert_bitwise(rgba, rgba0, f"{w} warps: ray rgba")
        np.testing.assert_allclose(sums, sums0, rtol=1e-5)  # the same terms summed in another order
    # the autotuner restores grad_density before every trial: it leaves one call's result
    tctx = hp.Context()
    gd, drgb, sums, rgba, rep = _losses(hp, tctx, sb, t_world, g0, autotune=True)
    assert_bitwise(gd, gd0, "autotuned: grad density")
    assert_bitwise(drgb, drgb0, "autotuned: dL/drgb")
    assert rep["n_candidates"] == 3 and tctx.tuning["loss_rays_per_block"] in (2, 4, 8)
    assert ctx.check() == 0 and tctx.check() == 0


@pytest.mark.parametrize("tile", [128, 256, 512, 1024, 2048])
def test_compaction_tiles_match_oracle(tile):
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(tile)
    ctx = hp.Context()
    ctx.tuning = dict(compact_tile=tile)
    for n, p in ((1, 1.0), (tile - 1, 0.5), (tile, 1.0), (tile + 1, 0.3), (7 * tile + 5, 0.0), (300001, 0.37),
                 (1 << 20, 0.9)):
        v = (rng.random(n) < p).astype(np.uint32) * rng.integers(1, 9, n).astype(np.uint32)
        ref = oracle.compact_nonzero(v)
        out, cnt = hp.compact_nonzero(ctx, i32(v))
        c = int(host(cnt)[0])
        assert c == len(ref), (tile, n)
        assert_bitwise(host(out)[:c], ref, f"tile {tile}, n={n}")
    assert ctx.check() == 0


def test_autotune_compact():
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(11)
    v = (rng.random(1 << 21) < 0.4).astype(np.uint32)
    ctx = hp.Context()
    idx, rep = hp.autotune_compact(ctx, i32(v))
    assert_bitwise(host(idx), oracle.compact_nonzero(v), "autotuned compaction")
    assert rep["n_candidates"] == 5 and ctx.tuning["compact_tile"] in (128, 256, 512, 1024, 2048)


def _multi(hp, ctx, ms, table, ss, tune=False):
    R = ms.rays.n
    r = ms.rays
    ori, dr, t, tmax, alive = dev(r.ori), dev(r.dir), dev(r.t), dev(r.t_max), dev(r.alive)
    if tune:
        ns, sc_s, info, off, smp, rep = hp.autotune_multi(ctx, table, R, ss, ori, dr, t, tmax, alive)
    else:
        ns, sc_s, info = hp.multi_march_count(ctx, table, R, ori, dr, t, tmax, alive)
        off, smp = hp.multi_march_emit(ctx, table, R, ss, ori, dr, t, alive, ns)
        rep = None
    out = dict(n_steps=host(ns), info=host(info), offsets=host(off), alive=host(alive),
               **{k: host(v) for k, v in smp.items()})
    return out, host(sc_s), rep


def test_multi_scene_chunks_and_autotune_bit_identical():
    from turbonerf_b200 import hotpath as hp
    params = scenes.multi_scene_params(seed=0x7C1, n_scenes=5, ray_lo=32, ray_hi=1500)
    ms = scenes.make_multi_scene(params, resolution=32)
    rows = []
    for sc, b in zip(ms.scenes, ms.ray_begin):
        rows.append(dict(grid=hp.GridSpec(sc.grid.n_levels, sc.grid.resolution, sc.grid.base_size),
                         bitfield=dev(sc.grid.bitfield), bbox=sc.bbox,
                         march=hp.MarchSpec(sc.cone_angle, sc.dt_min, sc.dt_max, sc.max_steps),
                         inv_aabb=1.0 / sc.aabb_size, ray_begin=int(b), n_rays=sc.rays.n))
    table = hp.scene_table(rows)
    ctx = hp.Context()
    base, per0, _ = _multi(hp, ctx, ms, table, 1 << 21)
    nsamp = int(base["info"][1])
    ss = nsamp + 64
    base, per0, _ = _multi(hp, ctx, ms, table, ss)
    for chunk in COUNT:
        for w, rpw in ((8, 1), (4, 2), (16, 4), (1, 1)):
            ctx.tuning = dict(multi_chunk_rays=chunk, emit_warps_per_block=w, emit_rays_per_warp=rpw)
            got, per, _ = _multi(hp, ctx, ms, table, ss)
            _same(got, base, f"chunk {chunk}, emit {w}x{rpw}", nsamp)
            assert_bitwise(per, per0, "scene samples")
    tctx = hp.Context()
    got, per, rep = _multi(hp, tctx, ms, table, ss, tune=True)
    _same(got, base, "autotuned multi-scene", nsamp)
    assert rep["count"]["n_candidates"] == 4 and tctx.tuning["multi_chunk_rays"] in COUNT
    assert ctx.check() == 0 and tctx.check() == 0


def test_trainer_autotune_trains_identically():
    """Two trainers with the same seed, one autotuned before its first step and then given
    shapes other than the defaults: after four steps (eager, then graph capture and replays)
    their weights, moments and grids are bit-identical and the step metrics agree."""
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=5)

    def make():
        tr = Trainer(SyntheticNeRF.from_scene(sc), n_rays_per_step=4096, occupancy_cells_per_step=4096,
                     distortion_lambda=1e-3, occupancy_threshold=0.01, n_grid_params=16 * (1 << 15) * 2,
                     n_mlp_params=7168, beta2=0.99, seed=0x7B0)
        tr.use_distortion_loss = True
        tr.setup_data(batch_size=1 << 16)
        return tr

    a, b = make(), make()
    res = b.autotune()
    assert set(res) == {"count", "emit", "losses", "tuning"}
    b.tuning = dict(count_rays_per_block=32 if res["tuning"]["count_rays_per_block"] != 32 else 128,
                    emit_rays_per_warp=2, loss_rays_per_block=8)
    for _ in range(4):
        ma, mb = a.train_step(), b.train_step()
        assert (ma.n_rays, ma.n_samples) == (mb.n_rays, mb.n_samples)
        assert abs(ma.loss - mb.loss) <= 1e-5 * abs(ma.loss)
    for k, what in ((0, "weights"), (2, "first moments"), (3, "second moments"), (6, "bitfield")):
        dt = np.uint8 if k == 6 else np.float32
        assert_bitwise(host(a.buffer(k, dt)), host(b.buffer(k, dt)), what)


def test_count_ahead_matches_in_order_steps():
    """The default trainer runs each step's tail (emit, network, losses, Adam, occupancy update)
    beside the next step's head (its rays and march count on the bitfield the tail before it
    computed ahead of the occupancy update). Against a trainer that runs every step in order (side_sms = 0): identical
    metrics every step and bit-identical rays, counts, parameters, moments, step counters, grid
    densities and bitfield, also after buffer reads between steps (which leave the head computed
    ahead in place), after a grid change (which drops it) and with the launch shapes changed."""
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=5)

    def make():
        tr = Trainer(SyntheticNeRF.from_scene(sc), n_rays_per_step=4096, occupancy_cells_per_step=4096,
                     distortion_lambda=1e-3, occupancy_threshold=0.01, n_grid_params=16 * (1 << 15) * 2,
                     n_mlp_params=7168, beta2=0.99, seed=0x7B0)
        tr.use_distortion_loss = True
        tr.setup_data(batch_size=1 << 16)
        return tr

    def same(a, b, tag):
        for k, what in ((0, "weights"), (2, "first moments"), (3, "second moments"), (4, "param steps"),
                        (5, "grid density"), (6, "bitfield"), (11, "n_steps"), (10, "offsets"), (17, "origins")):
            dt = np.uint8 if k == 6 else (np.uint32 if k in (4, 10, 11) else np.float32)
            assert_bitwise(host(a.buffer(k, dt)), host(b.buffer(k, dt)), f"{what} {tag}")

    a, b = make(), make()
    assert a.tuning["side_sms"] > 0, "the trainer counts ahead by default"
    b.tuning = dict(side_sms=0)
    for i in range(6):  # eager first runs, then graph capture and replays of both ray sets
        ma, mb = a.train_step(), b.train_step()
        assert (ma.step, ma.n_rays, ma.n_samples) == (mb.step, mb.n_rays, mb.n_samples)
        assert ma.loss == mb.loss
        if i == 2:
            same(a, b, "mid-run")
    same(a, b, "after six steps")
    # a grid change drops the head computed ahead from the old grid
    bits = host(a.buffer(6, np.uint8)).copy()
    bits[::7] = 0
    for t in (a, b):
        call_set_grid(t, bits)
    for _ in range(3):
        ma, mb = a.train_step(), b.train_step()
        assert (ma.step, ma.n_rays, ma.n_samples, ma.loss) == (mb.step, mb.n_rays, mb.n_samples, mb.loss)
    same(a, b, "after a grid change")
    # asynchronous steps, then the metrics
    for _ in range(3):
        a.train_step_async()
        b.train_step_async()
    ma, mb = a.sync_metrics(), b.sync_metrics()
    assert (ma.step, ma.loss) == (mb.step, mb.loss)
    same(a, b, "after asynchronous steps")
    a.teardown()
    b.teardown()


def test_count_ahead_matches_in_order_steps_across_the_selection_change():
    """The tail with a next step also computes the bitfield that the next step's occupancy update
    will write (the decayed grid against the threshold, then the queried cells it raises), so
    that the head after that step marches without waiting for the update. Selection changes
    at step 256 from every queried cell to the random rule that reads the bitfield; across it,
    the count-ahead trainer stays bit-identical to the in-order one (grid densities, bitfield,
    parameters, march counts) and gives the same metrics every step."""
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=5)

    def make():
        tr = Trainer(SyntheticNeRF.from_scene(sc), n_rays_per_step=2048, occupancy_cells_per_step=8192,
                     distortion_lambda=1e-3, occupancy_threshold=0.01, n_grid_params=16 * (1 << 14) * 2,
                     n_mlp_params=7168, beta2=0.99, seed=0x5E1)
        tr.setup_data(batch_size=1 << 15)
        return tr

    a, b = make(), make()
    assert a.tuning["side_sms"] > 0
    b.tuning = dict(side_sms=0)
    for i in range(262):
        ma, mb = a.train_step(), b.train_step()
        assert (ma.step, ma.n_rays, ma.n_samples, ma.loss) == (mb.step, mb.n_rays, mb.n_samples, mb.loss), i
        if i in (254, 255, 256, 257, 261):
            for k, what in ((0, "weights"), (5, "grid density"), (6, "bitfield"), (11, "n_steps")):
                dt = np.uint8 if k == 6 else (np.uint32 if k == 11 else np.float32)
                assert_bitwise(host(a.buffer(k, dt)), host(b.buffer(k, dt)), f"{what} after step {i}")
    a.teardown()
    b.teardown()


def call_set_grid(tr, bits):
    import ctypes
    from turbonerf_b200 import native
    native.call("tn_trainer_set_grid", tr._handle(), None, bits.ctypes.data_as(ctypes.c_void_p))
