"""Gradients of both backward variants of the memory study (recompute vs store) against the
FP64 oracle, on a compositor + distortion batch with the study's count distribution (truncated
geometric, mean 64, at most 1024) at 2^16 samples."""
import numpy as np
import pytest

import oracle
from tests.helpers import RTOL_GRAD, assert_norm_close, dev, expand_rays, host, i32
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["recompute", "store"])
def test_backward_variants_match_oracle(variant):
    from turbonerf_b200 import hotpath as hp
    sb = scenes.make_sample_batch(0x7B5, 1 << 16, mean=64.0, max_count=1024)
    n, ss = sb.n_rays, sb.n_samples
    lam = 1e-3
    g = np.random.default_rng(5).normal(size=4 * n).astype(np.float32)
    ctx = hp.Context()
    rb = hp.ray_batch(i32(sb.counts), i32(sb.offsets), n, n, ss)
    fn = hp.backward_recompute if variant == "recompute" else hp.backward_store
    dd, drgb, ddist = fn(ctx, rb, dev(sb.sigma), dev(sb.rgb), dev(sb.dt), dev(sb.m_norm), dev(sb.dt_norm), dev(g), lam)
    ref_dd, ref_drgb = oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, g.astype(np.float64), n, ss)
    _, ref_dist = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, lam, ss)
    rec = oracle.recon_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.target_rgba, sb.bg_rgb, n, ss,
                               amb_eps=1e-5)
    sm = expand_rays(rec["ambiguous"] == 0, sb.counts, sb.offsets, ss)
    assert_norm_close(host(dd), ref_dd, RTOL_GRAD, f"compositor dL/dsigma ({variant})", mask=sm)
    assert_norm_close(host(drgb), ref_drgb, RTOL_GRAD, f"dL/drgb ({variant})", mask=np.tile(sm, 3))
    assert_norm_close(host(ddist), ref_dist, RTOL_GRAD, f"distortion dL/dsigma ({variant})")
    assert ctx.check() == 0
