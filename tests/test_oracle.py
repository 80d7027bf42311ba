"""CPU checks that pin the oracle itself (no GPU): closed-form cases, an independent
restatement of the Morton code and of round-up division, central finite differences of
every analytic gradient, and the reference's batch-cut and occupancy rules on small
hand-made inputs. The reference ships no golden vectors, so these are the pins."""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from turbonerf_b200 import scenes


def test_morton_matches_shift_mask_form_and_inverts():
    rng = np.random.default_rng(0)
    xyz = rng.integers(0, 1024, size=(2000, 3)).astype(np.uint32)
    ref = scenes.morton3d(xyz[:, 0], xyz[:, 1], xyz[:, 2])
    for (x, y, z), m in zip(xyz[:200], ref[:200]):
        assert oracle.morton3d(x, y, z) == int(m)
        assert oracle.morton3d_invert(int(m)) == x
        assert oracle.morton3d_invert(int(m) >> 1) == y
        assert oracle.morton3d_invert(int(m) >> 2) == z
    assert np.array_equal(scenes.morton3d_invert(ref), xyz[:, 0])
    assert oracle.morton3d(1, 0, 0) == 1 and oracle.morton3d(0, 1, 0) == 2 and oracle.morton3d(0, 0, 1) == 4


def _next_up(x):
    return np.nextafter(np.float32(x), np.float32(np.inf))


def test_fdiv_ru_is_the_smallest_float_not_below_the_quotient():
    rng = np.random.default_rng(1)
    b = np.float32(0.00169145586)
    cases = list(rng.uniform(0.0017, 0.5, 3000).astype(np.float32)) + [b, np.float32(2 * b), np.float32(3 * b)]
    for a in cases:
        q = np.float32(oracle.fdiv_ru(a, b))
        exact = Fraction(float(a)) / Fraction(float(b))
        assert Fraction(float(q)) >= exact
        below = np.nextafter(q, np.float32(-np.inf))
        assert Fraction(float(below)) < exact


def test_march_closed_form_full_grid_fixed_step():
    """All cells occupied, cone angle 0: the count is the number of float32 steps
    t <- t + dt that stay below t_max and inside the box."""
    sc = scenes.march_scene_single(n_rays=64)
    sc.grid.bitfield[:] = 0xFF
    dt = np.float32(sc.dt_min)
    march = dict(bbox=sc.bbox, cone=0.0, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=0)
    ns, alive, guard = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
    assert guard == 0
    r = sc.rays
    lo, hi = np.float32(-1.5), np.float32(1.5)
    for i in range(r.n):
        t, tm = np.float32(r.t[i]), np.float32(r.t_max[i])
        o = [np.float32(r.ori[c * r.stride + i]) for c in range(3)]
        d = [np.float32(r.dir[c * r.stride + i]) for c in range(3)]
        n = 0
        while t < tm:
            p = [np.float32(o[c] + np.float32(t * d[c])) for c in range(3)]
            if not all(lo <= v <= hi for v in p):
                break
            t = np.float32(t + dt)
            n += 1
        assert ns[i] == n, (i, ns[i], n)
    assert np.all(alive[ns == 0] == 0)


def test_march_empty_grid_kills_every_ray():
    sc = scenes.march_scene_single(n_rays=64)
    sc.grid.bitfield[:] = 0
    march = dict(bbox=sc.bbox, cone=0.0, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=0)
    ns, alive, _ = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
    assert ns.sum() == 0 and alive.sum() == 0


def test_batch_cut_rule():
    # offsets [0, 3, 8]; every offset is below 100, the last ray is still dropped
    st, off, nr, ns = oracle.scan_cut(np.array([3, 5, 2], np.uint32), 100)
    assert st == 0 and list(off) == [0, 3, 8] and (nr, ns) == (2, 8)
    # offsets [0, 3, 8, 10]: the last offset below 9 is index 2 -> rays 0..1, 8 samples
    st, off, nr, ns = oracle.scan_cut(np.array([3, 5, 2, 4], np.uint32), 9)
    assert st == 0 and (nr, ns) == (2, 8)
    # a single ray can never be used (the reference throws "No rays were generated")
    st, _, nr, _ = oracle.scan_cut(np.array([7], np.uint32), 100)
    assert st == -5 and nr == 0
    # only empty rays before the cut -> no samples
    st, _, nr, ns = oracle.scan_cut(np.array([0, 0, 5], np.uint32), 100)
    assert st == -6 and ns == 0


def test_single_sample_composite_is_alpha_times_colour():
    counts = np.array([1], np.uint32)
    offs = np.array([0], np.uint32)
    sigma = np.array([2.5], np.float32)
    dt = np.array([0.1], np.float32)
    rgb = np.array([0.2, 0.4, 0.8], np.float32)
    rgba, used = oracle.composite_fwd(counts, offs, sigma, rgb, dt, 1, 1)
    alpha = 1.0 - np.exp(-2.5 * float(np.float32(0.1)))
    assert np.allclose(rgba, [0.2 * alpha, 0.4 * alpha, 0.8 * alpha, alpha], rtol=1e-6)
    assert used[0] == 1


def _small_batch(seed, n_samples=600, mean=12.0):
    sb = scenes.make_sample_batch(seed, n_samples, mean=mean)
    sb.sigma[:] = np.clip(sb.sigma, 0.0, 50.0)
    return sb


def test_recon_gradient_matches_central_differences():
    sb = _small_batch(21)
    n, ss = sb.n_rays, sb.n_samples
    ref = oracle.recon_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n, ss)
    used = ref["n_used"]
    base = dict(counts=sb.counts, offsets=sb.offsets, rgb=sb.rgb.astype(np.float64), dt=sb.dt.astype(np.float64),
                target_rgba=sb.target_rgba.astype(np.float64), bg_rgb=sb.bg_rgb.astype(np.float64), ray_stride=n,
                sample_stride=ss, fixed_used=used)
    sig = sb.sigma.astype(np.float64)
    h = 1e-3
    rng = np.random.default_rng(0)
    for j in rng.choice(ss, 60, replace=False):
        sp, sm = sig.copy(), sig.copy()
        sp[j] += h
        sm[j] -= h
        fd = (oracle.recon_loss_rgb(density=sp, **base) - oracle.recon_loss_rgb(density=sm, **base)) / (2 * h)
        an = ref["dL_ddensity"][j]
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-4 * np.abs(ref["dL_ddensity"]).max()), (j, fd, an)
    for j in rng.choice(ss, 30, replace=False):
        for c in range(3):
            rp, rm = base["rgb"].copy(), base["rgb"].copy()
            rp[c * ss + j] += h
            rm[c * ss + j] -= h
            args = dict(base)
            args["rgb"] = rp
            lp = oracle.recon_loss_rgb(density=sig, **args)
            args["rgb"] = rm
            lm = oracle.recon_loss_rgb(density=sig, **args)
            fd = (lp - lm) / (2 * h)
            an = ref["dL_drgb"][c * ss + j]
            assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-6), (j, c, fd, an)


def test_distortion_gradient_matches_central_differences():
    sb = _small_batch(22, 500, 20.0)
    lam = 1e-3
    loss, dd = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, lam, sb.n_samples)
    assert np.isclose(loss.sum(), oracle.distortion_loss_sum(sb.counts, sb.offsets, sb.sigma.astype(np.float64),
                                                             sb.m_norm.astype(np.float64),
                                                             sb.dt_norm.astype(np.float64), lam), rtol=1e-12)
    sig = sb.sigma.astype(np.float64)
    h = 1e-3
    m, dtn = sb.m_norm.astype(np.float64), sb.dt_norm.astype(np.float64)
    for j in np.random.default_rng(1).choice(sb.n_samples, 80, replace=False):
        sp, sm = sig.copy(), sig.copy()
        sp[j] += h
        sm[j] -= h
        fd = (oracle.distortion_loss_sum(sb.counts, sb.offsets, sp, m, dtn, lam) -
              oracle.distortion_loss_sum(sb.counts, sb.offsets, sm, m, dtn, lam)) / (2 * h)
        assert abs(fd - dd[j]) <= 1e-5 * max(abs(dd[j]), 1e-4 * np.abs(dd).max()), (j, fd, dd[j])


def test_composite_vjp_matches_central_differences():
    sb = _small_batch(23, 400, 10.0)
    n, ss = sb.n_rays, sb.n_samples
    g = np.random.default_rng(2).normal(size=4 * n)
    rgba0, used = oracle.composite_fwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, n, ss)
    dd, drgb = oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, g, n, ss)

    def f(sig):
        # composite in float64 with the cut held fixed at the forward's n_used
        tot = 0.0
        for r in range(n):
            o, c = int(sb.offsets[r]), int(used[r])
            T = 1.0
            acc = np.zeros(4)
            for k in range(c):
                a = 1.0 - np.exp(-sig[o + k] * float(sb.dt[o + k]))
                w = T * a
                acc += w * np.array([sb.rgb[o + k], sb.rgb[ss + o + k], sb.rgb[2 * ss + o + k], 1.0])
                T *= 1.0 - a
            tot += float(np.dot(acc, g[[r, n + r, 2 * n + r, 3 * n + r]]))
        return tot

    sig = sb.sigma.astype(np.float64)
    h = 1e-4
    for j in np.random.default_rng(3).choice(ss, 25, replace=False):
        sp, sm = sig.copy(), sig.copy()
        sp[j] += h
        sm[j] -= h
        fd = (f(sp) - f(sm)) / (2 * h)
        assert abs(fd - dd[j]) <= 1e-5 * max(abs(dd[j]), 1e-4 * np.abs(dd).max()), (j, fd, dd[j])


def test_occupancy_update_rules_small_grid():
    res, L = 4, 2
    V = res ** 3
    d = np.zeros((L, V), np.float32)
    d[0, 0] = 1.0   # occupied at level 0
    d[1, 5] = 0.5   # occupied at level 1
    bits = np.zeros(V, np.uint8)
    bits[0] |= 1
    bits[5] |= 2
    levels = np.array([0, 0, 1, 1, 0], np.int32)
    cells = np.array([0, 1, 5, 6, 0], np.uint32)
    values = np.array([0.2, 0.3, 2.0, 0.7, 3.0], np.float32)
    rsel = np.array([0.3, 0.3, 0.1, 0.9, 0.45], np.float32)
    nd, nb, nocc = oracle.occupancy_update(d, bits, L, res, levels, cells, values, rsel, threshold=0.25)
    dec = np.float32(0.95)
    assert nd[0, 0] == max(np.float32(1.0) * dec, np.float32(3.0))  # occupied -> 0.3 and 0.45 pass
    assert nd[0, 1] == 0.0                                            # unoccupied, r in (0.25, 0.5] -> skipped
    assert nd[1, 5] == np.float32(2.0)                                # r < 0.25 -> always
    assert nd[1, 6] == 0.0                                            # r > 0.5 -> skipped
    assert nb[0] == 1 and nb[5] == 2 and nocc == 2
    nd2, _, _ = oracle.occupancy_update(d, bits, L, res, levels, cells, values, rsel, sample_all=True)
    assert nd2[0, 1] == np.float32(0.3) and nd2[1, 6] == np.float32(0.7)


def test_adam_first_step_moves_by_lr_times_sign():
    n = 64
    g = np.random.default_rng(4).normal(0, 1e-3, n).astype(np.float32)
    g[:8] = 0.0
    st = dict(w=np.ones(n), m=np.zeros(n), v=np.zeros(n), steps=np.zeros(n, np.uint32))
    oracle.adam_step(st, g, n_grid=32, n_mlp=16, lr=1e-2, beta2=0.99, l2=0.0)
    assert np.all(st["w"][:8] == 1.0) and np.all(st["steps"][:8] == 0)  # zero hash gradients are skipped
    moved = st["w"][8:] - 1.0
    assert np.allclose(moved, -1e-2 * np.sign(g[8:]), rtol=1e-6)
    assert np.all(st["steps"][8:] == 1)


def test_emit_normalisation_matches_scene_helper():
    """m_norm / dt_norm written by the march emit equal the helper used to build packed
    batches (same float32 formula)."""
    sc = scenes.march_scene_single(n_rays=32)
    march = dict(bbox=sc.bbox, cone=0.0, dt_min=sc.dt_min, dt_max=sc.dt_max, max_steps=64)
    ns, alive, _ = oracle.march_count(sc.rays.as_dict(), sc.grid.as_dict(), march)
    off = np.zeros(len(ns), np.uint32)
    off[1:] = np.cumsum(ns[:-1])
    out = oracle.march_emit(sc.rays.as_dict(), sc.grid.as_dict(), march, off, ns, alive, len(ns), int(ns.sum()) + 1,
                            1.0 / 3.0)
    tot = int(ns.sum())
    world_dt = np.full(tot, np.float32(sc.dt_min), np.float32)
    m, dtn = scenes.normalize_ray_t(out["t"][:tot], world_dt, ns, off, t_start=sc.rays.t)
    assert np.array_equal(m, out["m_norm"][:tot]) and np.array_equal(dtn, out["dt_norm"][:tot])
