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
