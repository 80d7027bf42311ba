"""Gradients of both backward variants of the memory study (recompute vs store) against the
FP64 oracle, on a compositor + distortion batch with the study's count distribution (truncated
geometric, mean 64, at most 1024) at 2^16 samples."""
import numpy as np
import pytest

import oracle
from tests.helpers import (CUT_BAND, RTOL_GRAD, assert_norm_close, assert_per_ray_norm_close, branch_cuts, dev,
                           host, i32, pick_branches, record_elementwise)
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
    _, ref_dist = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, lam, ss)
    # the VJP at every legitimate set of transmittance cuts, assembled ray by ray from the closest
    n_alt, alt, over = oracle.cut_branches(sb.counts, sb.offsets, sb.sigma, sb.dt, band=CUT_BAND)
    assert over == 0
    branches = []
    for fu in branch_cuts(n_alt, alt):
        a, b = oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, g.astype(np.float64), n, ss,
                                    fixed_used=fu)
        branches.append(dict(dd=a, drgb=b))
    gpu = dict(dd=host(dd), drgb=host(drgb))
    ref, _ = pick_branches(gpu, branches, sb.counts, sb.offsets, sample_keys=("dd", "drgb"), sample_stride=ss)
    assert_norm_close(gpu["dd"], ref["dd"], RTOL_GRAD, f"compositor dL/dsigma ({variant})")
    assert_per_ray_norm_close(gpu["dd"], ref["dd"], sb.counts, sb.offsets, RTOL_GRAD,
                              f"compositor dL/dsigma per ray ({variant})")
    assert_norm_close(gpu["drgb"], ref["drgb"], RTOL_GRAD, f"dL/drgb ({variant})")
    record_elementwise(gpu["dd"], ref["dd"], f"backward {variant} compositor dL/dsigma")
    assert_norm_close(host(ddist), ref_dist, RTOL_GRAD, f"distortion dL/dsigma ({variant})")
    assert ctx.check() == 0
