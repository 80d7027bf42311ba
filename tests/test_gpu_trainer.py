"""The C++ training controller on the GPU: one fused train step checked stage by stage
against the oracle, fused vs plain path, graph replay vs eager, and the full-grid
occupancy update of the reference API."""
import numpy as np
import pytest

import oracle
from tests.helpers import (CUT_BAND, RTOL_GRAD, assert_bitwise, assert_norm_close, branch_cuts, pick_branches,
                           record_elementwise)
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu

R, B = 4096, 1 << 16


def _make(path="fused", graph=True, cells=4096, seed=0x7B0):
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=5)
    tr = Trainer(SyntheticNeRF.from_scene(sc), path=path, use_cuda_graph=graph, n_rays_per_step=R,
                 occupancy_cells_per_step=cells, distortion_lambda=1e-3, occupancy_threshold=0.01,
                 n_grid_params=16 * (1 << 15) * 2, n_mlp_params=7168, beta2=0.99, seed=seed)
    tr.use_distortion_loss = True
    tr.setup_data(batch_size=B)
    return sc, tr


def _h(t, dtype=np.float32):
    return t.cpu().numpy().view(dtype) if t.dtype.itemsize == np.dtype(dtype).itemsize else t.cpu().numpy()


def test_fused_step_matches_oracle_stage_by_stage():
    sc, tr = _make()
    import torch
    w0 = tr.buffer(0).clone()
    m = tr.train_step()
    torch.cuda.synchronize()
    rays = scenes.RayBatch(R, R, _h(tr.buffer(17)), _h(tr.buffer(18)), _h(tr.buffer(19)), _h(tr.buffer(20)),
                           _h(tr.buffer(21, np.uint8)))
    march = dict(bbox=sc.bbox, cone=sc.cone_angle, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=0)
    # the rays' box clip
    t_o, tm_o, a_o = oracle.rays_init_bbox(rays.ori, rays.dir, R, R, sc.bbox)
    assert_bitwise(rays.t, t_o, "ray t")
    assert_bitwise(rays.t_max, tm_o, "ray t_max")
    # march on the grid as it was before the step's occupancy update
    ns, alive, _ = oracle.march_count(dict(rays.as_dict(), alive=a_o), sc.grid.as_dict(), march)
    st, off, nr, nsamp = oracle.scan_cut(ns, B)
    assert st == 0
    assert (m.n_rays, m.n_samples) == (nr, nsamp)
    assert_bitwise(_h(tr.buffer(11), np.uint32), ns, "n_steps")
    assert_bitwise(_h(tr.buffer(10), np.uint32), off, "offsets")
    em = oracle.march_emit(dict(rays.as_dict(), alive=a_o), sc.grid.as_dict(), march, off, ns, alive, nr, B,
                           1.0 / sc.aabb_size)
    for idx, key in ((7, "t"), (9, "dt"), (24, "m_norm"), (25, "dt_norm")):
        assert_bitwise(_h(tr.buffer(idx))[:nsamp], em[key][:nsamp], key)
    assert_bitwise(_h(tr.buffer(8)).reshape(3, B)[:, :nsamp], em["pos"].reshape(3, B)[:, :nsamp], "pos")
    # losses and the merged gradient on the trainer's own network outputs
    sig, rgb = _h(tr.buffer(13)), _h(tr.buffer(14))
    tgt = _h(tr.buffer(22))
    bg = _h(tr.buffer(23))
    tgt_c = np.concatenate([tgt[c * R:c * R + nr] for c in range(4)])
    bg_c = np.concatenate([bg[c * R:c * R + nr] for c in range(3)])
    dl, ddist = oracle.distortion_fwd_bwd(ns[:nr], off[:nr], sig, em["m_norm"], em["dt_norm"], 1e-3, B)
    # every legitimate set of transmittance cuts, the closest ray by ray
    n_alt, alt, over = oracle.cut_branches(ns[:nr], off[:nr], sig, em["dt"], band=CUT_BAND)
    assert over == 0
    branches = []
    for fu in branch_cuts(n_alt, alt):
        r = oracle.recon_fwd_bwd(ns[:nr], off[:nr], sig, rgb, em["dt"], tgt_c, bg_c, nr, B, fixed_used=fu)
        r["g"] = oracle.grad_epilogue(nsamp, 1.0, r["dL_ddensity"][:nsamp], ddist[:nsamp], em["t"][:nsamp],
                                      np.zeros(nsamp))
        branches.append(r)
    gpu = dict(g=_h(tr.buffer(15))[:nsamp])
    rec, _ = pick_branches(gpu, branches, ns[:nr], off[:nr], sample_keys=("g",), sample_stride=nsamp,
                           carry_ray_keys=("loss",), ray_stride=nr)
    assert_norm_close(gpu["g"], rec["g"], RTOL_GRAD, "merged density gradient")
    record_elementwise(gpu["g"], rec["g"], "train step merged density gradient (4096 rays)")
    ref_loss = rec["loss"][:4 * nr].sum() / nr + dl.mean()
    assert abs(m.loss - ref_loss) <= 1e-5 * abs(ref_loss)
    # Adam on the fixed synthetic gradients
    g = _h(tr.buffer(1))
    state = dict(w=_h(w0).astype(np.float64), m=np.zeros(len(g)), v=np.zeros(len(g)),
                 steps=np.zeros(len(g), np.uint32))
    f32 = lambda x: float(np.float32(x))  # noqa: E731
    oracle.adam_step(state, g, 16 * (1 << 15) * 2, 7168, lr=f32(1e-2), beta1=f32(0.9), beta2=f32(0.99),
                     eps=f32(1e-15), l2=f32(1e-6))
    w = _h(tr.buffer(0)).astype(np.float64)
    assert float(np.abs(w - state["w"]).max()) <= 1e-5 * 1e-2  # against one step of lr = 1e-2
    assert_bitwise(_h(tr.buffer(4), np.uint32), state["steps"], "param steps")
    tr.teardown()


def test_fused_and_plain_paths_agree():
    sc, f = _make("fused")
    _, p = _make("plain")
    for _ in range(3):
        mf = f.train_step()
        mp = p.train_step()
        assert (mf.step, mf.n_rays, mf.n_samples) == (mp.step, mp.n_rays, mp.n_samples)
        assert abs(mf.loss - mp.loss) <= 1e-3 * abs(mp.loss)
    assert_bitwise(_h(f.buffer(6, np.uint8)), _h(p.buffer(6, np.uint8)), "bitfield after 3 steps")
    assert_bitwise(_h(f.buffer(5)), _h(p.buffer(5)), "grid density after 3 steps")
    assert_norm_close(_h(f.buffer(0)), _h(p.buffer(0)), 1e-5, "weights after 3 steps")
    assert_bitwise(_h(f.buffer(4), np.uint32), _h(p.buffer(4), np.uint32), "param steps")
    f.teardown()
    p.teardown()


def test_graph_replay_matches_eager_bitwise():
    _, a = _make("fused", graph=True)
    _, b = _make("fused", graph=False)
    for _ in range(4):
        a.train_step_async()
        b.train_step_async()
    ma, mb = a.sync_metrics(), b.sync_metrics()
    assert (ma.step, ma.n_rays, ma.n_samples) == (mb.step, mb.n_rays, mb.n_samples) == (4, ma.n_rays, ma.n_samples)
    assert ma.loss == mb.loss
    for idx in (0, 2, 3, 5, 15, 16):
        assert_bitwise(_h(a.buffer(idx)), _h(b.buffer(idx)), f"buffer {idx}")
    assert_bitwise(_h(a.buffer(6, np.uint8)), _h(b.buffer(6, np.uint8)), "bitfield")
    assert a.stat(0) >= 10  # kernels captured in one step graph
    assert a.stat(3) > 0  # samples processed so far
    a.teardown()
    b.teardown()


def test_update_occupancy_grid_fused_and_plain():
    _, f = _make("fused", cells=0)
    _, p = _make("plain", cells=0)
    for step in (3, 300):
        mf = f.update_occupancy_grid(step)
        mp = p.update_occupancy_grid(step)
        assert mf.n_total == mp.n_total == 5 * 128 ** 3
        assert mf.n_occupied == mp.n_occupied
        assert_bitwise(_h(f.buffer(5)), _h(p.buffer(5)), f"density after update at step {step}")
        assert_bitwise(_h(f.buffer(6, np.uint8)), _h(p.buffer(6, np.uint8)), "bitfield")
        assert oracle.popcount(_h(f.buffer(6, np.uint8))) == mf.n_occupied
    f.teardown()
    p.teardown()


def test_train_step_rays_host_input():
    import torch
    sc, tr = _make()
    rng = np.random.default_rng(3)
    r = scenes.sphere_rays(rng, R)
    tgt = np.concatenate([rng.uniform(0, 1, 3 * R), np.ones(R)]).astype(np.float32)
    bg = rng.uniform(0, 1, 3 * R).astype(np.float32)
    host = [torch.from_numpy(a).pin_memory() for a in (r.ori, r.dir, tgt, bg)]
    m1 = tr.train_step_rays(*host)
    m2 = tr.train_step_rays(*host)  # second call replays the captured graph
    assert m1.n_samples > 0 and m2.step == 2
    assert_bitwise(_h(tr.buffer(17)), r.ori, "uploaded origins")
    tr.teardown()


def test_pipelined_caller_ray_steps_match_synchronous_steps():
    """train_step_rays_pipelined returns each step's metrics one call later and leaves the
    trainer in the state that the synchronous calls leave: the same metrics step by step and
    the same weights, moments and grid bit for bit."""
    import torch
    rng = np.random.default_rng(5)
    batches = []
    for _ in range(3):
        r = scenes.sphere_rays(rng, R)
        tgt = np.concatenate([rng.uniform(0, 1, 3 * R), np.ones(R)]).astype(np.float32)
        bg = rng.uniform(0, 1, 3 * R).astype(np.float32)
        batches.append([torch.from_numpy(a).pin_memory() for a in (r.ori, r.dir, tgt, bg)])
    steps = 6
    _, a = _make()
    sync = [a.train_step_rays(*batches[i % 3]) for i in range(steps)]
    _, b = _make()
    piped = []
    for i in range(steps):
        m = b.train_step_rays_pipelined(*batches[i % 3])
        assert (m is None) == (i == 0)
        if m is not None:
            piped.append(m)
    piped.append(b.sync_metrics())
    assert [m.step for m in piped] == list(range(1, steps + 1))
    for ms, mp in zip(sync, piped):
        assert (ms.step, ms.n_rays, ms.n_samples) == (mp.step, mp.n_rays, mp.n_samples)
        assert np.float32(ms.loss) == np.float32(mp.loss)
    for idx, name in ((0, "weights"), (2, "first moments"), (3, "second moments"), (5, "grid density")):
        assert_bitwise(_h(a.buffer(idx)), _h(b.buffer(idx)), name)
    assert_bitwise(_h(a.buffer(6, np.uint8)), _h(b.buffer(6, np.uint8)), "bitfield")
    # a synchronous read in between starts a new pipeline
    assert b.train_step_rays_pipelined(*batches[0]) is None
    assert b.sync_metrics().step == steps + 1
    a.teardown()
    b.teardown()


def test_reset_training_starts_over():
    """reset_training (reference NeRFTrainingController::reset_training) returns the trainer to
    the state setup_data left: after a reset, three steps give the same metrics and the same
    weights, moments, step counts and grid, bit for bit, as three steps of a fresh trainer."""
    _, a = _make()
    for _ in range(3):
        a.train_step()
    a.update_occupancy_grid(3)
    a.reset_training()
    ma = [a.train_step() for _ in range(3)]
    _, b = _make()
    mb = [b.train_step() for _ in range(3)]
    for x, y in zip(ma, mb):
        assert (x.step, x.n_rays, x.n_samples) == (y.step, y.n_rays, y.n_samples)
        assert np.float32(x.loss) == np.float32(y.loss)
    for idx, name in ((0, "weights"), (2, "first moments"), (3, "second moments"), (5, "grid density")):
        assert_bitwise(_h(a.buffer(idx)), _h(b.buffer(idx)), name)
    assert_bitwise(_h(a.buffer(4), np.uint32), _h(b.buffer(4), np.uint32), "param steps")
    assert_bitwise(_h(a.buffer(6, np.uint8)), _h(b.buffer(6, np.uint8)), "bitfield")
    a.teardown()
    b.teardown()
