"""The benchmarked train step against the oracle, stage by stage, step after step.

The trainer is built exactly as bench.py builds it (bench._trainer): 2^14 rays a step through
5 cascades of 128^3 (extents 1..16), a 2^18-sample batch, 16 x 2^19 x 2 hash-grid + 7168 MLP
parameters with the fixed sparse synthetic gradients, 2^16 occupancy cells re-sampled a step,
launch shapes chosen by the autotuner, each step's tail beside the next step's rays and march
count (Adam on the side SMs), captured in CUDA graphs (replayed from the third step on). For each of three steps, from the state the step
started from:
  * rays and their box clip, march counts, alive flags, offsets, the batch cut and every emitted
    sample field: bit for bit;
  * the merged density gradient (reconstruction + distortion + distance scaling) within 1e-4
    normwise, at every legitimate transmittance cut; the step's loss within 1e-5;
  * the occupancy update (decay, max-update of the sampled cells, threshold): densities and
    bitfield bit for bit;
  * Adam: per-parameter step counts bit for bit, weights within 1e-5 of one step, moments
    within 1e-5 normwise.
"""
import numpy as np
import pytest

import oracle
from tests.helpers import (CUT_BAND, RTOL_GRAD, assert_bitwise, assert_norm_close, branch_cuts, pick_branches,
                           record_elementwise)

pytestmark = pytest.mark.gpu


def _h(tr, which, dtype=np.float32):
    return tr.buffer(which, dtype).cpu().numpy().copy()


def _state(tr):
    return dict(w=_h(tr, 0), m=_h(tr, 2), v=_h(tr, 3), steps=_h(tr, 4, np.uint32), density=_h(tr, 5),
                bits=_h(tr, 6, np.uint8))


def test_bench_train_step_matches_oracle_step_by_step():
    import bench
    from turbonerf_b200.replicas import replica_seed
    scene = bench._scene(0x7B0)
    tr = bench._trainer(scene, "fused", replica_seed(0x7B0, 0))
    tr.autotune()
    assert tr.tuning["side_sms"] > 0 and tr.use_cuda_graph  # count-ahead schedule, graph replay
    R, B = bench.RAYS, bench.BATCH
    n_grid, n_mlp = bench.N_GRID, bench.N_MLP
    grads = _h(tr, 1)
    assert (grads[:n_grid] != 0).any() and (grads[:n_grid] == 0).any()  # sparse hash-grid gradients
    march = dict(bbox=scene.bbox, cone=scene.cone_angle, dt_min=scene.dt_min, dt_max=scene.dt_max, max_steps=0)
    prev = _state(tr)
    f32 = np.float32
    for _ in range(3):
        m = tr.train_step()
        k = m.step - 1  # index of the step just taken
        # rays and box clip
        ori, dr = _h(tr, 17), _h(tr, 18)
        t_o, tm_o, a_o = oracle.rays_init_bbox(ori, dr, R, R, scene.bbox)
        assert_bitwise(_h(tr, 19), t_o, f"step {k}: ray t")
        assert_bitwise(_h(tr, 20), tm_o, f"step {k}: ray t_max")
        rays = dict(ori=ori, dir=dr, t=t_o, t_max=tm_o, alive=a_o, stride=R, n=R)
        grid = dict(n_levels=5, res=128, base=1.0, bitfield=prev["bits"])
        ns, alive, guard = oracle.march_count(rays, grid, march)
        assert guard == 0
        assert_bitwise(_h(tr, 11, np.uint32), ns, f"step {k}: n_steps")
        assert_bitwise(_h(tr, 21, np.uint8), alive, f"step {k}: alive")
        st, off, nr, nsamp = oracle.scan_cut(ns, B)
        assert st == 0 and (m.n_rays, m.n_samples) == (nr, nsamp)
        assert_bitwise(_h(tr, 10, np.uint32), off, f"step {k}: offsets")
        em = oracle.march_emit(rays, grid, march, off, ns, alive, nr, B, 1.0 / scene.aabb_size)
        for idx, key in ((7, "t"), (9, "dt"), (24, "m_norm"), (25, "dt_norm")):
            assert_bitwise(_h(tr, idx)[:nsamp], em[key][:nsamp], f"step {k}: sample {key}")
        assert_bitwise(_h(tr, 8).reshape(3, B)[:, :nsamp], em["pos"].reshape(3, B)[:, :nsamp], f"step {k}: pos")
        # losses and the merged gradient on the step's network outputs
        sig, rgb = _h(tr, 13), _h(tr, 14)
        tgt, bg = _h(tr, 22), _h(tr, 23)
        tgt_c = np.concatenate([tgt[c * R:c * R + nr] for c in range(4)])
        bg_c = np.concatenate([bg[c * R:c * R + nr] for c in range(3)])
        cnt, offs = ns[:nr], off[:nr]
        dl, ddist = oracle.distortion_fwd_bwd(cnt, offs, sig, em["m_norm"], em["dt_norm"], bench.LAMBDA, B)
        n_alt, alt, over = oracle.cut_branches(cnt, offs, sig, em["dt"], band=CUT_BAND)
        assert over == 0
        branches = []
        for fu in branch_cuts(n_alt, alt):
            r = oracle.recon_fwd_bwd(cnt, offs, sig, rgb, em["dt"], tgt_c, bg_c, nr, B, fixed_used=fu)
            r["g"] = oracle.grad_epilogue(nsamp, 1.0, r["dL_ddensity"][:nsamp], ddist[:nsamp], em["t"][:nsamp],
                                          np.zeros(nsamp))
            branches.append(r)
        gpu = dict(g=_h(tr, 15)[:nsamp])
        rec, _ = pick_branches(gpu, branches, cnt, offs, sample_keys=("g",), sample_stride=nsamp,
                               carry_ray_keys=("loss",), ray_stride=nr)
        assert_norm_close(gpu["g"], rec["g"], RTOL_GRAD, f"step {k}: merged density gradient")
        record_elementwise(gpu["g"], rec["g"], f"bench step {k}: merged density gradient")
        ref_loss = rec["loss"][:4 * nr].sum() / nr + dl.mean()
        assert abs(m.loss - ref_loss) <= 1e-5 * abs(ref_loss), f"step {k}: loss {m.loss} vs {ref_loss}"
        # occupancy update from the grid the step started with
        lv, cells = _h(tr, 27, np.int32), _h(tr, 28, np.uint32)
        vals, rsel = _h(tr, 29), _h(tr, 30)
        assert lv.size == bench.OCC_CELLS
        d_o, b_o, _ = oracle.occupancy_update(prev["density"], prev["bits"], 5, 128, lv, cells, vals, rsel,
                                              sample_all=k < 256, decay=0.95, threshold=bench.THRESHOLD)
        cur = _state(tr)
        assert_bitwise(cur["density"], d_o, f"step {k}: grid density")
        assert_bitwise(cur["bits"], b_o, f"step {k}: bitfield")
        # Adam on the fixed synthetic gradients, from the parameters the step started with
        lr = float(f32(1e-2) / (f32(1.0) + f32(3.3e-5) * f32(k)))
        st_o = dict(w=prev["w"].astype(np.float64), m=prev["m"].astype(np.float64), v=prev["v"].astype(np.float64),
                    steps=prev["steps"].copy())
        oracle.adam_step(st_o, grads, n_grid, n_mlp, lr=lr, beta1=float(f32(0.9)), beta2=float(f32(0.99)),
                         eps=float(f32(1e-15)), l2=float(f32(1e-6)))
        assert_bitwise(cur["steps"], st_o["steps"], f"step {k}: parameter steps")
        assert float(np.max(np.abs(cur["w"].astype(np.float64) - st_o["w"]))) <= 1e-5 * lr, f"step {k}: weights"
        assert_norm_close(cur["m"], st_o["m"], 1e-5, f"step {k}: first moments")
        assert_norm_close(cur["v"], st_o["v"], 1e-5, f"step {k}: second moments")
        prev = cur
    tr.teardown()
