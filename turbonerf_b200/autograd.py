"""torch.autograd wrappers of the hand-written compositor and distortion-loss adjoints.

`composite(sigma, rgb, dt, counts, offsets)` returns the per-ray RGBA [4, n_rays] of the
reference's compositor (density_to_ray_rgba_forward, src/utils/training-kernels-fused.cuh:
227-264). Its backward is tn_composite_bwd: transmittance is recomputed by a reverse scan
from the per-ray optical depth saved by the forward, so the only per-ray state kept between
forward and backward is (optical depth, samples composited), 8 bytes per ray, instead of a
per-sample transmittance and weight (8 bytes per sample).

`distortion_loss(sigma, m_norm, dt_norm, counts, offsets, lam)` returns the per-ray
mip-NeRF 360 distortion loss [n_rays] (training-kernels-fused.cuh:13-120); its backward
recomputes the forward scans and applies the reference's adjoint (:123-224) scaled by the
upstream per-ray gradient.

Inputs are CUDA tensors in structure-of-arrays layout: sigma, dt, m_norm, dt_norm [S];
rgb [3, S]; counts and offsets int32 [R] (offsets = exclusive scan of counts).
"""
from __future__ import annotations

import torch

from . import hotpath as hp

_contexts: dict[int, hp.Context] = {}


def _ctx(device: torch.device) -> hp.Context:
    idx = device.index if device.index is not None else torch.cuda.current_device()
    if idx not in _contexts:
        with torch.cuda.device(idx):
            _contexts[idx] = hp.Context()
    return _contexts[idx]


def _check(t: torch.Tensor, name: str, dtype=torch.float32):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    return t.contiguous()


class Composite(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma, rgb, dt, counts, offsets, min_transmittance=1e-4, activation=0):
        sigma = _check(sigma, "sigma")
        rgb = _check(rgb, "rgb")
        dt = _check(dt, "dt")
        counts = _check(counts, "counts", torch.int32)
        offsets = _check(offsets, "offsets", torch.int32)
        S, R = sigma.numel(), counts.numel()
        if rgb.numel() != 3 * S or dt.numel() != S or offsets.numel() != R:
            raise ValueError("shape mismatch: rgb [3,S], dt [S], offsets [R] expected")
        rb = hp.ray_batch(counts, offsets, R, R, S)
        out = hp.composite_fwd(_ctx(sigma.device), rb, sigma, rgb, dt, activation=activation, min_t=min_transmittance)
        ctx.save_for_backward(sigma, rgb, dt, counts, offsets, out["depth"], out["n_used"])
        ctx.activation = activation
        return out["rgba"].view(4, R)

    @staticmethod
    def backward(ctx, grad_rgba):
        sigma, rgb, dt, counts, offsets, depth, n_used = ctx.saved_tensors
        S, R = sigma.numel(), counts.numel()
        rb = hp.ray_batch(counts, offsets, R, R, S)
        g = grad_rgba.contiguous().to(torch.float32)
        dd, drgb = hp.composite_bwd(_ctx(sigma.device), rb, sigma, rgb, dt, depth, n_used, g,
                                    activation=ctx.activation)
        return dd, drgb.view_as(rgb), None, None, None, None, None


class DistortionLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma, m_norm, dt_norm, counts, offsets, lam=0.01, activation=0):
        sigma = _check(sigma, "sigma")
        m_norm = _check(m_norm, "m_norm")
        dt_norm = _check(dt_norm, "dt_norm")
        counts = _check(counts, "counts", torch.int32)
        offsets = _check(offsets, "offsets", torch.int32)
        S, R = sigma.numel(), counts.numel()
        rb = hp.ray_batch(counts, offsets, R, R, S)
        out = hp.distortion_fwd_bwd(_ctx(sigma.device), rb, sigma, m_norm, dt_norm, lam, activation=activation,
                                    backward=False)
        ctx.save_for_backward(sigma, m_norm, dt_norm, counts, offsets)
        ctx.lam = lam
        ctx.activation = activation
        return out["ray_loss"]

    @staticmethod
    def backward(ctx, grad_ray):
        sigma, m_norm, dt_norm, counts, offsets = ctx.saved_tensors
        S, R = sigma.numel(), counts.numel()
        rb = hp.ray_batch(counts, offsets, R, R, S)
        out = hp.distortion_fwd_bwd(_ctx(sigma.device), rb, sigma, m_norm, dt_norm, ctx.lam,
                                    activation=ctx.activation, grad_ray=grad_ray.contiguous().to(torch.float32))
        return out["dL_ddensity"], None, None, None, None, None, None


def composite(sigma, rgb, dt, counts, offsets, min_transmittance=1e-4, activation=0):
    return Composite.apply(sigma, rgb, dt, counts, offsets, min_transmittance, activation)


def distortion_loss(sigma, m_norm, dt_norm, counts, offsets, lam=0.01, activation=0):
    return DistortionLoss.apply(sigma, m_norm, dt_norm, counts, offsets, lam, activation)
