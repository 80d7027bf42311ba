"""Parity of the CUDA compositor, reconstruction loss, distortion loss and gradient merge
against the FP64 oracle.

Tolerances: composited RGBA per element within 1e-5 relative; loss sums within 1e-5
relative; gradient vectors within 1e-4 in the normwise relative error (max |g - ref| /
max |ref|), for the whole batch and, where the upstream gradient is fixed, for every ray
(see tests/helpers.py for why entries are not checked one by one)."""
import numpy as np
import pytest

import oracle
from tests.helpers import (CUT_BAND, RTOL_COMPOSITE, RTOL_GRAD, assert_bitwise, assert_close, assert_legal_cut,
                           assert_norm_close, assert_per_ray_norm_close, branch_cuts, dev, host, i32, pick_branches,
                           record_elementwise)
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


def _batch(n_samples, mean, seed=0x7B1, max_count=1024):
    return scenes.make_sample_batch(seed, n_samples, mean=mean, max_count=max_count)


def _rb(sb, counts_t, offsets_t):
    from turbonerf_b200.hotpath import ray_batch
    return ray_batch(counts_t, offsets_t, sb.n_rays, sb.n_rays, sb.n_samples)


def _rgb_ok(ref_rgba, gpu_rgba, n_rays, mask):
    for c in range(4):
        assert_close(gpu_rgba[c * n_rays:(c + 1) * n_rays], ref_rgba[c * n_rays:(c + 1) * n_rays], RTOL_COMPOSITE,
                     f"rgba[{c}]", mask=mask)


@pytest.mark.parametrize("mean,n_samples", [(48, 1 << 18), (3, 4096), (700, 1 << 16)])
def test_composite_forward_and_vjp(mean, n_samples):
    from turbonerf_b200 import hotpath as hp
    sb = _batch(n_samples, mean)
    n, ss = sb.n_rays, sb.n_samples
    ctx = hp.Context()
    counts, offsets = i32(sb.counts), i32(sb.offsets)
    rb = _rb(sb, counts, offsets)
    sig, rgb, dt = dev(sb.sigma), dev(sb.rgb), dev(sb.dt)
    out = hp.composite_fwd(ctx, rb, sig, rgb, dt)
    # every ray stops where the reference may stop it: at the FP64 cut, or, where the
    # transmittance lies within rounding of the threshold, at one of the other legitimate counts
    used = host(out["n_used"]).view(np.uint32)
    n_alt, alt, over = oracle.cut_branches(sb.counts, sb.offsets, sb.sigma, sb.dt, band=CUT_BAND)
    assert over == 0
    assert_legal_cut(used, n_alt, alt)
    # then every ray, the ones whose cut rounding decides included, against the oracle at that cut
    ref_rgba, _ = oracle.composite_fwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, n, ss, fixed_used=used)
    _rgb_ok(ref_rgba, host(out["rgba"]), n, None)
    g = np.random.default_rng(1).normal(size=4 * n)
    dd, drgb = hp.composite_bwd(ctx, rb, sig, rgb, dt, out["depth"], out["n_used"], dev(g.astype(np.float32)))
    ref_dd, ref_drgb = oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt,
                                            g.astype(np.float32).astype(np.float64), n, ss, fixed_used=used)
    assert_per_ray_norm_close(host(dd), ref_dd, sb.counts, sb.offsets, RTOL_GRAD, "dL/dsigma")
    for c in range(3):
        assert_per_ray_norm_close(host(drgb)[c * ss:(c + 1) * ss], ref_drgb[c * ss:(c + 1) * ss], sb.counts, sb.offsets,
                                  RTOL_GRAD, f"dL/drgb[{c}]")
    assert_norm_close(host(dd), ref_dd, RTOL_GRAD, "dL/dsigma (batch)")
    record_elementwise(host(dd), ref_dd, f"composite VJP dL/dsigma, mean {mean}")
    record_elementwise(host(drgb), ref_drgb, f"composite VJP dL/drgb, mean {mean}")
    # the store-instead-of-recompute variant: same composite, same VJP
    st = hp.composite_fwd_store(ctx, rb, sig, rgb, dt)
    assert_bitwise(host(st["n_used"]).view(np.uint32), used, "n_used (store variant)")
    _rgb_ok(ref_rgba, host(st["rgba"]), n, None)
    dd2, drgb2 = hp.composite_bwd_stored(ctx, rb, sig, rgb, dt, st["n_used"], st["t_saved"], st["w_saved"],
                                         dev(g.astype(np.float32)))
    assert_per_ray_norm_close(host(dd2), ref_dd, sb.counts, sb.offsets, RTOL_GRAD, "dL/dsigma (stored)")
    for c in range(3):
        assert_per_ray_norm_close(host(drgb2)[c * ss:(c + 1) * ss], ref_drgb[c * ss:(c + 1) * ss], sb.counts,
                                  sb.offsets, RTOL_GRAD, f"dL/drgb[{c}] (stored)")
    assert ctx.check() == 0


def test_composite_clustered_empty_and_long_rays():
    """The tile kernels split a batch between warps by samples: a warp takes the rays whose first
    sample lies in its share, in groups of up to 32. Runs of hundreds of rays without samples (all
    at one offset, so one warp takes them all, over several groups), runs of one-sample rays,
    rays of up to 2,000 samples spanning many warps' shares, and empty rays at the batch's end:
    every ray is composited and differentiated as by the oracle, and empty rays get zeros."""
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(0x7C1)
    parts = []
    for i in range(40):
        parts.append(np.zeros(int(rng.integers(50, 400)), np.uint32))
        parts.append(rng.integers(1, 3, int(rng.integers(10, 200))).astype(np.uint32))
        if i % 7 == 0:
            parts.append(rng.integers(500, 2000, 2).astype(np.uint32))
    parts.append(np.zeros(300, np.uint32))
    counts = np.concatenate(parts)
    n = len(counts)
    offsets = np.zeros(n, np.uint32)
    offsets[1:] = np.cumsum(counts[:-1], dtype=np.uint64).astype(np.uint32)
    ss = int(counts.sum())
    ss += (-ss) % 4
    sigma = np.clip(np.exp(rng.normal(0.0, 2.0, ss)), 0.0, 1e4).astype(np.float32)
    rgb = (1.0 / (1.0 + np.exp(-rng.normal(0.0, 1.0, 3 * ss)))).astype(np.float32)
    dt = (rng.uniform(0.5, 2.0, ss) * float(scenes.MIN_STEP_SIZE)).astype(np.float32)
    ctx = hp.Context()
    rb = hp.ray_batch(i32(counts), i32(offsets), n, n, ss)
    out = hp.composite_fwd(ctx, rb, dev(sigma), dev(rgb), dev(dt))
    used = host(out["n_used"]).view(np.uint32)
    n_alt, alt, over = oracle.cut_branches(counts, offsets, sigma, dt, band=CUT_BAND)
    assert over == 0
    assert_legal_cut(used, n_alt, alt)
    ref_rgba, _ = oracle.composite_fwd(counts, offsets, sigma, rgb, dt, n, ss, fixed_used=used)
    _rgb_ok(ref_rgba, host(out["rgba"]), n, None)
    empty = counts == 0
    for c in range(4):
        assert np.all(host(out["rgba"])[c * n:(c + 1) * n][empty] == 0.0)
    g = rng.normal(size=4 * n).astype(np.float32)
    dd, drgb = hp.composite_bwd(ctx, rb, dev(sigma), dev(rgb), dev(dt), out["depth"], out["n_used"], dev(g))
    ref_dd, ref_drgb = oracle.composite_vjp(counts, offsets, sigma, rgb, dt, g.astype(np.float64), n, ss,
                                            fixed_used=used)
    assert_per_ray_norm_close(host(dd), ref_dd, counts, offsets, RTOL_GRAD, "dL/dsigma")
    for c in range(3):
        assert_per_ray_norm_close(host(drgb)[c * ss:(c + 1) * ss], ref_drgb[c * ss:(c + 1) * ss], counts, offsets,
                                  RTOL_GRAD, f"dL/drgb[{c}]")
    assert ctx.check() == 0


def _recon_reference(sb, dens, act, gpu, grad_scale=1.0):
    """The oracle's reconstruction fwd/bwd at every legitimate set of cuts, assembled ray by
    ray from the branch closest to the GPU's outputs (gpu: dict of host arrays)."""
    n, ss = sb.n_rays, sb.n_samples
    n_alt, alt, over = oracle.cut_branches(sb.counts, sb.offsets, dens, sb.dt, act=act, band=CUT_BAND)
    assert over == 0
    recs = [oracle.recon_fwd_bwd(sb.counts, sb.offsets, dens, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n, ss,
                                 act=act, grad_scale=grad_scale, fixed_used=fu) for fu in branch_cuts(n_alt, alt)]
    keys = [k for k in ("ray_rgba", "loss") if k in gpu]
    skeys = [k for k in ("dL_ddensity", "dL_drgb") if k in gpu]
    ref, _ = pick_branches(gpu, recs, sb.counts, sb.offsets, ray_keys=keys, sample_keys=skeys, ray_stride=n,
                           sample_stride=ss)
    return ref, recs, n_alt


@pytest.mark.parametrize("act", [0, 1])
def test_recon_loss_fused_and_plain(act):
    from turbonerf_b200 import hotpath as hp
    sb = _batch(1 << 18, 48, seed=0x7B2)
    n, ss = sb.n_rays, sb.n_samples
    dens = sb.sigma if act == 0 else np.log(np.maximum(sb.sigma, 1e-6)).astype(np.float32) + 1.0
    ctx = hp.Context()
    counts, offsets = i32(sb.counts), i32(sb.offsets)
    rb = _rb(sb, counts, offsets)
    args = (dev(dens), dev(sb.rgb), dev(sb.dt), dev(sb.target_rgba), dev(sb.bg_rgb))
    out = hp.recon_loss_fwd_bwd(ctx, rb, *args, inv_nrays=1.0 / n, grad_scale=1.0, activation=act)
    gpu = {k: host(out[k]) for k in ("ray_rgba", "loss", "dL_ddensity", "dL_drgb")}
    ref, _, n_alt = _recon_reference(sb, dens, act, gpu)
    _rgb_ok(ref["ray_rgba"], gpu["ray_rgba"], n, None)
    for c in range(4):
        assert_norm_close(gpu["loss"][c * n:(c + 1) * n], ref["loss"][c * n:(c + 1) * n], 1e-4, f"loss[{c}]")
    ref_sum = ref["loss"][:4 * n].sum() / n
    assert abs(float(host(out["loss_sum"])[0]) - ref_sum) <= 1e-5 * abs(ref_sum)
    assert_norm_close(gpu["dL_ddensity"], ref["dL_ddensity"], RTOL_GRAD, "dL/ddensity")
    assert_norm_close(gpu["dL_drgb"], ref["dL_drgb"], RTOL_GRAD, "dL/drgb")
    assert_per_ray_norm_close(gpu["dL_ddensity"], ref["dL_ddensity"], sb.counts, sb.offsets, RTOL_GRAD,
                              "dL/ddensity per ray", floor=1e-3)
    record_elementwise(gpu["dL_ddensity"], ref["dL_ddensity"], f"reconstruction dL/ddensity, act {act}")
    # the plain path (reference structure, one thread per ray, FP32 suffix subtraction)
    loss, dd, drgb, lsum = hp.plain_recon_loss(rb, *args, inv_nrays=1.0 / n, grad_scale=1.0, activation=act)
    ref_p, _, _ = _recon_reference(sb, dens, act, {"dL_ddensity": host(dd)})
    assert abs(lsum - ref_sum) <= 1e-4 * abs(ref_sum)
    assert_norm_close(host(dd), ref_p["dL_ddensity"], 1e-3, "plain dL/ddensity")
    assert ctx.check() == 0


@pytest.mark.parametrize("mean,n_samples,max_count", [
    (48, 1 << 18, 1024), (2, 2048, 1024), (1024, 1 << 16, 1024),
    (64, 1 << 22, 1024),     # the compositor workload: several rays per warp, vector loads
    (6000, 1 << 17, 20000),  # rays beyond 64 tiles of 128 samples (tile carries replayed)
])
def test_distortion_fused_and_plain(mean, n_samples, max_count):
    from turbonerf_b200 import hotpath as hp
    sb = _batch(n_samples, mean, seed=0x7B3, max_count=max_count)
    n, ss = sb.n_rays, sb.n_samples
    lam = 1e-3
    ctx = hp.Context()
    counts, offsets = i32(sb.counts), i32(sb.offsets)
    rb = _rb(sb, counts, offsets)
    out = hp.distortion_fwd_bwd(ctx, rb, dev(sb.sigma), dev(sb.m_norm), dev(sb.dt_norm), lam)
    ref_loss, ref_dd = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, lam, ss)
    assert_norm_close(host(out["ray_loss"])[:n], ref_loss, 1e-4, "ray distortion loss")
    assert abs(float(host(out["loss_sum"])[0]) - ref_loss.mean()) <= 1e-5 * abs(ref_loss.mean())
    assert_norm_close(host(out["dL_ddensity"]), ref_dd, RTOL_GRAD, "dLdist/dsigma")
    # per ray: dL/dsigma_j = dtn_j (g_j T_{j+1} - sum_{l>j} g_l w_l) keeps one intrinsic difference,
    # so rays whose whole gradient is below 1e-3 of the batch's largest are measured against that
    assert_per_ray_norm_close(host(out["dL_ddensity"]), ref_dd, sb.counts, sb.offsets, RTOL_GRAD,
                              "dLdist/dsigma per ray", floor=1e-3)
    ray_loss, dd, lsum = hp.plain_distortion(rb, dev(sb.sigma), dev(sb.m_norm), dev(sb.dt_norm), lam)
    assert abs(lsum - ref_loss.mean()) <= 1e-3 * abs(ref_loss.mean())
    assert ctx.check() == 0


@pytest.mark.parametrize("mean,max_count,n_samples,sigma_scale,shift", [
    (48, 1024, 1 << 18, 1.0, 0),      # the training mix: most rays in registers, a few long ones
    (48, 1024, 1 << 18, 1.0, 1),      # the same with sigma 4 bytes off 16-byte alignment: scalar staging
    (178, 256, 1 << 18, 1.0, 0),      # the train step's mix: rays up to 256 samples at any offset mod 4
    (700, 1024, 1 << 16, 1.0, 0),     # rays of 2-4 super-chunks, cut early by the transmittance
    (700, 1024, 1 << 16, 1e-3, 0),    # long composites that cross super-chunks
    (6000, 9000, 1 << 16, 1e-4, 0),   # rays beyond 32 super-chunks (distortion carries replayed)
])
def test_train_losses_fused_matches_oracle_chain(mean, max_count, n_samples, sigma_scale, shift):
    """One kernel = reconstruction fwd/bwd + distortion fwd/bwd + gradient merge with
    distance scaling, against the oracle's separate stages. With every sample array 16-byte
    aligned (shift 0) the kernel stages whole 16-byte groups; a shifted sigma array takes the
    sample-by-sample staging."""
    from turbonerf_b200 import hotpath as hp
    sb = scenes.make_sample_batch(0x7B4, n_samples, mean=mean, max_count=max_count)
    sb.sigma = (sb.sigma * np.float32(sigma_scale)).astype(np.float32)
    n, ss = sb.n_rays, sb.n_samples
    lam, scale = 1e-3, 1.0
    t_world = (sb.t * 0.9).astype(np.float32)  # part of the samples below t = 1
    grad_in = np.random.default_rng(2).normal(0, 1e-3, ss).astype(np.float32)
    ctx = hp.Context()
    counts, offsets = i32(sb.counts), i32(sb.offsets)
    rb = _rb(sb, counts, offsets)
    gd = dev(grad_in.copy())
    ray_rgba = dev(np.zeros(4 * n, np.float32))
    sig_d = dev(np.concatenate([np.zeros(shift, np.float32), sb.sigma]))[shift:]
    gd, drgb, sums = hp.train_losses(ctx, rb, sig_d, dev(sb.rgb), dev(sb.dt), dev(sb.m_norm), dev(sb.dt_norm),
                                     dev(t_world), dev(sb.target_rgba), dev(sb.bg_rgb), gd, inv_nrays=1.0 / n,
                                     grad_scale=scale, lam=lam, ray_rgba=ray_rgba)
    dl, ddist = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, lam, ss)
    # the merged gradient of every legitimate set of cuts (the distortion loss has no cut)
    n_alt, alt, over = oracle.cut_branches(sb.counts, sb.offsets, sb.sigma, sb.dt, band=CUT_BAND)
    assert over == 0
    branches = []
    for fu in branch_cuts(n_alt, alt):
        r = oracle.recon_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n, ss,
                                 grad_scale=scale, fixed_used=fu)
        r["g"] = oracle.grad_epilogue(ss, scale, r["dL_ddensity"], ddist, t_world, grad_in.astype(np.float64))
        branches.append(r)
    gpu = dict(g=host(gd), dL_drgb=host(drgb), ray_rgba=host(ray_rgba))
    rec, _ = pick_branches(gpu, branches, sb.counts, sb.offsets, ray_keys=("ray_rgba",), sample_keys=("g", "dL_drgb"),
                           ray_stride=n, sample_stride=ss, carry_ray_keys=("loss",))
    assert_norm_close(gpu["g"], rec["g"], RTOL_GRAD, "merged density gradient")
    assert_norm_close(gpu["dL_drgb"], rec["dL_drgb"], RTOL_GRAD, "dL/drgb")
    record_elementwise(gpu["g"], rec["g"], f"train losses merged gradient, mean {mean}, sigma x{sigma_scale:g}")
    _rgb_ok(rec["ray_rgba"], gpu["ray_rgba"], n, None)
    s = host(sums)
    assert abs(s[0] - rec["loss"][:4 * n].sum() / n) <= 1e-5 * abs(rec["loss"][:4 * n].sum() / n)
    assert abs(s[1] - dl.mean()) <= 1e-5 * abs(dl.mean())
    assert ctx.check() == 0


def test_grad_epilogue_fused_and_plain():
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(9)
    n = 100003
    rec, dist = rng.normal(size=n).astype(np.float32), rng.normal(size=n).astype(np.float32)
    t = rng.uniform(0, 2, n).astype(np.float32)
    g0 = rng.normal(size=n).astype(np.float32)
    ref = oracle.grad_epilogue(n, 128.0, rec.astype(np.float64), dist.astype(np.float64), t, g0.astype(np.float64))
    a = hp.grad_epilogue(n, 128.0, dev(rec), dev(dist), dev(t), dev(g0.copy()))
    b = hp.plain_grad_epilogue(n, 128.0, dev(rec), dev(dist), dev(t), dev(g0.copy()))
    assert_norm_close(host(a), ref, 1e-6, "fused epilogue")
    assert_norm_close(host(b), ref, 1e-6, "plain epilogue")
