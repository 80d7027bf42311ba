"""The CUDA library against the reference's own kernels (fixtures tests/golden/ref_*.npz, written
by tests/golden/make_ref_golden.py from TurboNeRF's kernel sources compiled unchanged on the host).

Bit-exact: march counts, alive flags, offsets and every emitted sample field (t, position,
direction, dt, m_norm, dt_norm) on the train step's 5-cascade scene; occupancy decay and bits,
popcount and cell sample points; Adam's per-parameter step counts. Float outputs against the
reference's FP32 arithmetic: per-ray losses and gradients within the bounds below (each side
carries FP32 rounding of a few 1e-6 against the FP64 oracle, and the reference forms its suffix
sums by subtraction). No ray of these fixtures has a transmittance within rounding of the cut
(checked), so both sides stop every ray at the same sample.
"""
import os

import numpy as np
import pytest

import oracle
from tests.golden import make_ref_golden as mrg
from tests.helpers import CUT_BAND, assert_bitwise, dev, host, i32, record_elementwise

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TOL_LOSS = 5e-5
TOL_GRAD = 5e-5


def _load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


def _normwise(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    d = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / d) if d > 0 else float(np.max(np.abs(a - b)))


def test_march_matches_reference_bit_for_bit():
    from turbonerf_b200 import hotpath as hp
    fx = _load("ref_march")
    n = fx["n_steps"].size
    total = int(fx["n_samples"])
    ss = total + 64
    g = hp.GridSpec(5, 128, 1.0)
    m = hp.MarchSpec(float(fx["cone"]), float(fx["dt_min"]), float(fx["dt_max"]), 0)
    bbox = tuple(float(v) for v in fx["bbox"])
    ctx = hp.Context(n, ss)
    alive = dev(fx["alive_in"].copy())
    ori, dr, t, tmax = dev(fx["ori"]), dev(fx["dir"]), dev(fx["t"]), dev(fx["t_max"])
    bits = dev(fx["bitfield"])
    # no batch cut: the reference's kernels march and emit every ray
    n_steps, info = hp.march_count(ctx, g, bits, bbox, m, n, n, ori, dr, t, tmax, alive, 0xFFFFFFFF)
    offsets, smp = hp.march_emit(ctx, g, bits, bbox, m, float(fx["inv_aabb"]), n, n, ss, info, ori, dr, t, alive,
                                 n_steps)
    assert ctx.check() == 0
    assert_bitwise(host(n_steps).view(np.uint32), fx["n_steps"], "n_steps")
    assert_bitwise(host(alive), fx["alive"], "alive")
    assert_bitwise(host(offsets).view(np.uint32), fx["offsets"], "offsets")
    assert int(host(info).view(np.uint32)[1]) == total
    for k, comps in (("t", 1), ("pos", 3), ("dir", 3), ("dt", 1), ("m_norm", 1), ("dt_norm", 1)):
        a = host(smp[k])
        head = np.stack([a[c * ss:c * ss + min(mrg.HEAD, total)] for c in range(comps)])
        assert_bitwise(head.ravel(), fx["head_" + k].ravel(), f"{k} (leading samples)")
        assert mrg.digest(a, comps, ss, total) == str(fx["sha_" + k]), f"{k}: digest of all {total} samples"


@pytest.mark.parametrize("tag", ["a", "b"])
def test_losses_match_reference(tag):
    from turbonerf_b200 import hotpath as hp
    fx = _load("ref_losses")
    g = lambda k: fx[f"{tag}_{k}"]  # noqa: E731
    counts, offsets, dens = g("counts"), g("offsets"), g("density")
    n, S = counts.size, g("dt").size
    n_alt, _, _ = oracle.cut_branches(counts, offsets, dens, g("dt"), act=1, band=CUT_BAND)
    assert n_alt.max() == 1  # no ray's cut is decided by rounding here
    ctx = hp.Context()
    rb = hp.ray_batch(i32(counts), i32(offsets), n, S, S)
    out = hp.recon_loss_fwd_bwd(ctx, rb, dev(dens), dev(g("rgb")), dev(g("dt")), dev(g("target")), dev(g("bg")),
                                inv_nrays=1.0 / n, grad_scale=1.0, activation=1)
    for c in range(4):
        assert _normwise(host(out["loss"])[c * S:c * S + n], g("loss")[c * S:c * S + n]) <= TOL_LOSS, f"loss[{c}]"
    assert _normwise(host(out["dL_ddensity"]), g("dL_ddensity")) <= TOL_GRAD
    assert _normwise(host(out["dL_drgb"]), g("dL_drgb")) <= TOL_GRAD
    record_elementwise(host(out["dL_ddensity"]), g("dL_ddensity"), f"reconstruction dL/ddensity vs reference ({tag})")
    d = hp.distortion_fwd_bwd(ctx, rb, dev(dens), dev(g("m_norm")), dev(g("dt_norm")), 0.01, activation=1)
    assert _normwise(host(d["ray_loss"])[:n], g("dist_loss")) <= TOL_LOSS
    assert _normwise(host(d["dL_ddensity"]), g("dist_dd")) <= TOL_GRAD
    # the fused train-step loss kernel: reconstruction + distortion + merge with distance scaling
    gd = dev(np.zeros(S, np.float32))
    gd, drgb, _ = hp.train_losses(ctx, rb, dev(dens), dev(g("rgb")), dev(g("dt")), dev(g("m_norm")),
                                  dev(g("dt_norm")), dev(g("t")), dev(g("target")), dev(g("bg")), gd,
                                  inv_nrays=1.0 / n, grad_scale=1.0, lam=0.01, activation=1)
    assert _normwise(host(gd), g("merged")) <= TOL_GRAD
    assert _normwise(host(drgb), g("dL_drgb")) <= TOL_GRAD
    assert ctx.check() == 0


def test_occupancy_popcount_points_match_reference_bit_for_bit():
    from turbonerf_b200 import hotpath as hp
    fx = _load("ref_occupancy")
    L, res = int(fx["n_levels"]), int(fx["res"])
    ctx = hp.Context()
    d, b = dev(fx["density"].copy()), dev(fx["bitfield"].copy())
    z = np.zeros(0)
    nocc = hp.occupancy_update(ctx, hp.GridSpec(L, res, 1.0), d, b, dev(z.astype(np.int32)), i32(z),
                               dev(z.astype(np.float32)), dev(z.astype(np.float32)))
    assert_bitwise(host(d), fx["out_density"], "decayed density")
    assert_bitwise(host(b), fx["out_bitfield"], "bitfield")
    assert int(host(nocc).view(np.uint32)[0]) == int(fx["n_occupied"])
    nc, start, level = int(fx["n_cells"]), int(fx["start"]), int(fx["level"])
    pts = hp.occupancy_sample_points(hp.GridSpec(L, res, 1.0), dev(np.full(nc, level, np.int32)),
                                     i32(np.arange(start, start + nc, dtype=np.uint32)), dev(fx["random3"]), nc,
                                     float(fx["inv_aabb"]), nc)
    assert_bitwise(host(pts), fx["points"], "cell sample points")


def test_adam_matches_reference():
    from turbonerf_b200 import hotpath as hp
    fx = _load("ref_adam")
    w, gr = dev(fx["w0"].copy()), dev(fx["grads"])
    P = fx["w0"].size
    m, v = dev(np.zeros(P, np.float32)), dev(np.zeros(P, np.float32))
    steps = i32(np.zeros(P, np.uint32))
    for lr in fx["lrs"]:
        hp.adam_step(w, gr, m, v, steps, int(fx["n_grid"]), int(fx["n_mlp"]), float(lr))
    assert_bitwise(host(steps).view(np.uint32), fx["steps"], "per-parameter steps")
    assert float(np.max(np.abs(host(w).astype(np.float64) - fx["w"]))) <= 2e-5 * 1e-2
    assert _normwise(host(m), fx["m"]) <= 1e-6 and _normwise(host(v), fx["v"]) <= 1e-5
