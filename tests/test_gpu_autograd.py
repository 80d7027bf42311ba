"""torch.autograd wrappers: forward values and the gradients torch computes through them
against the FP64 oracle (compositor VJP, distortion adjoint scaled per ray), plus a
central-finite-difference check of the whole autograd path in FP32 on a small batch."""
import numpy as np
import pytest

import oracle
from tests.helpers import RTOL_GRAD, assert_norm_close, assert_per_ray_norm_close
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


def _tensors(sb):
    import torch
    f = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    return (f(sb.sigma).requires_grad_(True), f(sb.rgb.reshape(3, -1)).requires_grad_(True), f(sb.dt),
            f(sb.counts.astype(np.int32)), f(sb.offsets.astype(np.int32)), f(sb.m_norm), f(sb.dt_norm))


def test_composite_autograd_matches_oracle_vjp():
    import torch
    from turbonerf_b200.autograd import composite
    sb = scenes.make_sample_batch(0x7C1, 1 << 16, mean=40)
    sig, rgb, dt, cnt, off, _, _ = _tensors(sb)
    rgba = composite(sig, rgb, dt, cnt, off)
    w = torch.from_numpy(np.random.default_rng(0).normal(size=(4, sb.n_rays)).astype(np.float32)).cuda()
    (rgba * w).sum().backward()
    ref_rgba, _ = oracle.composite_fwd(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt, sb.n_rays, sb.n_samples)
    assert_norm_close(rgba.detach().cpu().numpy().ravel(), ref_rgba, 1e-5, "rgba")
    dd, drgb = oracle.composite_vjp(sb.counts, sb.offsets, sb.sigma, sb.rgb, sb.dt,
                                    w.cpu().numpy().ravel().astype(np.float64), sb.n_rays, sb.n_samples)
    assert_per_ray_norm_close(sig.grad.cpu().numpy(), dd, sb.counts, sb.offsets, RTOL_GRAD, "dL/dsigma")
    assert_norm_close(rgb.grad.cpu().numpy().ravel(), drgb, RTOL_GRAD, "dL/drgb")


def test_distortion_autograd_matches_oracle():
    import torch
    from turbonerf_b200.autograd import distortion_loss
    sb = scenes.make_sample_batch(0x7C2, 1 << 16, mean=40)
    sig, _, _, cnt, off, m, dtn = _tensors(sb)
    loss = distortion_loss(sig, m, dtn, cnt, off, lam=1e-3)
    g = np.random.default_rng(1).uniform(0.5, 2.0, sb.n_rays)
    (loss * torch.from_numpy(g.astype(np.float32)).cuda()).sum().backward()
    ref_loss, ref_dd = oracle.distortion_fwd_bwd(sb.counts, sb.offsets, sb.sigma, sb.m_norm, sb.dt_norm, 1e-3,
                                                 sb.n_samples, grad_ray=g.astype(np.float32).astype(np.float64))
    assert_norm_close(loss.detach().cpu().numpy()[:sb.n_rays], ref_loss, 1e-4, "ray loss")
    assert_norm_close(sig.grad.cpu().numpy(), ref_dd, RTOL_GRAD, "dLdist/dsigma")


def test_composite_autograd_finite_differences():
    """Central differences through the CUDA forward itself (h relative 1e-2 of sigma, FP32)."""
    import torch
    from turbonerf_b200.autograd import composite
    rng = np.random.default_rng(5)
    counts = np.array([5, 9, 1, 16], np.int32)
    offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int32)
    S = int(counts.sum())
    sig = torch.tensor(rng.uniform(0.5, 5.0, S), dtype=torch.float32, device="cuda", requires_grad=True)
    rgb = torch.tensor(rng.uniform(0, 1, (3, S)), dtype=torch.float32, device="cuda")
    dt = torch.tensor(rng.uniform(0.01, 0.05, S), dtype=torch.float32, device="cuda")
    c, o = torch.tensor(counts, device="cuda"), torch.tensor(offs, device="cuda")
    w = torch.tensor(rng.normal(size=(4, 4)), dtype=torch.float32, device="cuda")
    (composite(sig, rgb, dt, c, o) * w).sum().backward()
    for j in range(S):
        h = 1e-2 * float(sig[j])
        with torch.no_grad():
            sp, sm = sig.detach().clone(), sig.detach().clone()
            sp[j] += h
            sm[j] -= h
            fd = ((composite(sp, rgb, dt, c, o) * w).sum() - (composite(sm, rgb, dt, c, o) * w).sum()) / (2 * h)
        assert abs(float(fd) - float(sig.grad[j])) <= 2e-3 * max(abs(float(sig.grad[j])), 1e-2), j
