"""The hash-grid encoding (the tiny-cuda-nn boundary) against the oracle: features bit for bit,
the backward's gradients in FP64 within 1e-5 (atomic adds in any order), the touched-entry list
as a set, the clearing; and train steps with the hash-grid network as the trainer's network,
stage by stage against the oracle: network outputs, the heads' and the hash entries' gradients,
and the listed entries of each step (those with a nonzero gradient)."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise, assert_norm_close, dev, host

pytestmark = pytest.mark.gpu


def _spec(log2_t=19, aabb=16.0):
    from turbonerf_b200 import hotpath as hp
    return hp.HashgridSpec.reference(aabb, log2_hashmap_size=log2_t)


def _levels(spec):
    lv = oracle.hashgrid_levels(spec.n_levels, spec.log2_hashmap_size, spec.base_resolution, spec.per_level_scale)
    for l in range(spec.n_levels):
        assert spec.level(l) == (int(lv[0][l]), bool(lv[1][l])), f"level {l}"
    return lv


def _positions(rng, n):
    pos = rng.uniform(0.0, 1.0, 3 * n).astype(np.float32)
    pos[:64] = 0.0
    pos[64:128] = 1.0
    pos[128:192] = np.float32(1.0 - 2 ** -24)
    return pos


def test_encode_matches_oracle_bit_for_bit():
    from turbonerf_b200 import hotpath as hp
    spec = _spec()
    lv = _levels(spec)
    rng = np.random.default_rng(11)
    n = 1 << 16
    pos = _positions(rng, n)
    n_hash, _ = spec.n_params()
    params = rng.uniform(-1.0, 1.0, n_hash).astype(np.float32)
    feat = hp.hashgrid_encode(spec, dev(pos), dev(params), n, n)
    ref = oracle.hashgrid_encode(lv, spec.log2_hashmap_size, pos, params, n)
    assert_bitwise(host(feat), ref, "hash-grid features")


def test_backward_and_touched_entries_match_oracle():
    from turbonerf_b200 import hotpath as hp
    spec = _spec(log2_t=17)
    lv = _levels(spec)
    rng = np.random.default_rng(12)
    n = 1 << 15
    pos = _positions(rng, n)
    dfeat = rng.normal(0.0, 1.0, spec.n_features * n).astype(np.float32)
    n_hash, _ = spec.n_params()
    grads = dev(np.zeros(n_hash, np.float32))
    bits, lst, count = hp.hashgrid_backward(spec, dev(pos), dev(dfeat), grads, n, n)
    ref, touched = oracle.hashgrid_backward(lv, spec.log2_hashmap_size, pos, dfeat.astype(np.float64), n)
    g = host(grads).astype(np.float64)
    T = 1 << spec.log2_hashmap_size
    for l in range(spec.n_levels):
        sl = slice(2 * l * T, 2 * (l + 1) * T)
        assert_norm_close(g[sl], ref[sl], 1e-5, f"level {l} gradients")
    k = int(host(count)[0])
    listed = host(lst)[:k].view(np.uint32)
    assert len(np.unique(listed)) == k, "an entry listed twice"
    assert np.array_equal(np.sort(listed), np.nonzero(touched)[0].astype(np.uint32))
    b = host(bits).view(np.uint32)
    want_bits = np.packbits(touched.reshape(-1, 8)[:, ::-1], axis=1).ravel().view(np.uint8)
    assert np.array_equal(b.view(np.uint8), np.ascontiguousarray(want_bits.reshape(-1, 4)).ravel())
    # clearing the listed entries leaves zero gradients, bits and count
    hp.hashgrid_clear_touched(lst, count, grads, bits)
    assert not host(grads).any() and not host(bits).any() and int(host(count)[0]) == 0


def test_trainer_steps_with_the_hashgrid_network_match_oracle():
    from turbonerf_b200 import hotpath as hp, scenes
    from turbonerf_b200.trainer import SyntheticNeRF, Trainer
    scene = scenes.march_scene_cascaded(seed=0x7B0, n_rays=64, n_levels=5)
    log2_t = 15
    spec = hp.HashgridSpec.reference(scene.aabb_size, log2_hashmap_size=log2_t)
    n_hash, n_head = spec.n_params()
    tr = Trainer(SyntheticNeRF.from_scene(scene), path="fused", use_cuda_graph=True, n_rays_per_step=4096,
                 occupancy_cells_per_step=4096, distortion_lambda=1e-3, n_grid_params=n_hash, n_mlp_params=7168,
                 beta2=0.99, seed=0x7B1)
    tr.use_distortion_loss = True
    tr.setup_data(batch_size=1 << 16)
    tr.use_hashgrid(spec)
    lv = _levels(spec)
    B = 1 << 16
    nf = spec.n_features
    h = lambda i, dt=np.float32: tr.buffer(i, dt).cpu().numpy().copy()  # noqa: E731
    for k in range(3):
        w0 = h(0)
        m = tr.train_step()
        assert np.isfinite(m.loss)
        ns = m.n_samples
        pos = h(8)
        # forward: features bit for bit, heads in FP64
        feat = oracle.hashgrid_encode(lv, log2_t, pos, w0[:n_hash], ns, pstride=B, stride=ns)
        head = w0[n_hash:n_hash + n_head]
        dens, rgb = oracle.hash_heads_forward(nf, feat, head, ns, ostride=B)
        assert_norm_close(h(13)[:ns], dens, 1e-5, f"step {k}: network density")
        assert_norm_close(h(14).reshape(3, B)[:, :ns], rgb.reshape(3, B)[:, :ns], 1e-5, f"step {k}: network rgb")
        # backward from the step's own loss gradients
        gd = h(15)[:ns].astype(np.float64)
        drgb = np.zeros(3 * ns)
        d16 = h(16).reshape(3, B)
        for c in range(3):
            drgb[c * ns:(c + 1) * ns] = d16[c, :ns]
        dfeat, dhead = oracle.hash_heads_backward(nf, feat, head, gd, drgb, ns)
        g = h(1)
        assert_norm_close(g[n_hash:n_hash + n_head], dhead, 1e-4, f"step {k}: head gradients")
        ref, touched = oracle.hashgrid_backward(lv, log2_t, pos, dfeat, ns, pstride=B, stride=ns)
        T = 1 << log2_t
        for l in range(spec.n_levels):
            sl = slice(2 * l * T, 2 * (l + 1) * T)
            assert_norm_close(g[sl], ref[sl], 1e-4, f"step {k}: level {l} hash gradients")
        # the listed entries: those with a nonzero gradient (the ones Adam updates)
        cnt = int(h(32, np.uint32)[0])
        listed = h(31, np.uint32)[:cnt]
        nonzero = np.nonzero(g[:n_hash].reshape(-1, 2).any(axis=1))[0].astype(np.uint32)
        assert np.array_equal(np.sort(listed), nonzero), f"step {k}: listed entries"
        assert set(nonzero) <= set(np.nonzero(touched)[0]), f"step {k}: a gradient outside the touched entries"
        assert not g[n_hash + n_head:].any()
    tr.teardown()


def test_encode_and_backward_edge_cases():
    """Zero samples (no launch, outputs untouched); a device live count below n (samples past it
    untouched, no gradient from them); positions outside [0, 1] (clamped to the edge cells, as the
    oracle does)."""
    import torch
    from turbonerf_b200 import hotpath as hp
    spec = _spec(log2_t=14)
    lv = _levels(spec)
    rng = np.random.default_rng(13)
    n = 4096
    pos = rng.uniform(-0.25, 1.25, 3 * n).astype(np.float32)
    n_hash, _ = spec.n_params()
    params = rng.uniform(-1.0, 1.0, n_hash).astype(np.float32)
    sentinel = np.full(spec.n_features * n, 7.0, np.float32)
    # zero samples
    out = dev(sentinel.copy())
    hp.hashgrid_encode(spec, dev(pos), dev(params), 0, n, out=out)
    assert np.array_equal(host(out), sentinel)
    # outside [0, 1]: clamped cells, bit for bit with the oracle
    feat = hp.hashgrid_encode(spec, dev(pos), dev(params), n, n)
    assert_bitwise(host(feat), oracle.hashgrid_encode(lv, spec.log2_hashmap_size, pos, params, n), "clamped features")
    # a live count below n
    live = 1000
    n_dev = torch.tensor([live], dtype=torch.int32, device="cuda")
    out = dev(sentinel.copy())
    hp.hashgrid_encode(spec, dev(pos), dev(params), n, n, n_dev=n_dev, out=out)
    got = host(out).reshape(spec.n_features, n)
    ref = oracle.hashgrid_encode(lv, spec.log2_hashmap_size, pos, params, n).reshape(spec.n_features, n)
    assert_bitwise(got[:, :live].ravel(), ref[:, :live].ravel(), "live features")
    assert (got[:, live:] == 7.0).all(), "features past the live count were written"
    dfeat = rng.normal(0.0, 1.0, spec.n_features * n).astype(np.float32)
    grads = dev(np.zeros(n_hash, np.float32))
    bits, lst, count = hp.hashgrid_backward(spec, dev(pos), dev(dfeat), grads, n, n, n_dev=n_dev)
    d_live = dfeat.reshape(spec.n_features, n).copy()
    d_live[:, live:] = 0.0
    ref_g, touched = oracle.hashgrid_backward(lv, spec.log2_hashmap_size, pos[:].copy(), d_live.ravel().astype(np.float64),
                                              n)
    _, touched_live = oracle.hashgrid_backward(
        lv, spec.log2_hashmap_size, np.ascontiguousarray(pos.reshape(3, n)[:, :live]).ravel(),
        np.ascontiguousarray(d_live[:, :live]).ravel().astype(np.float64), live)
    assert_norm_close(host(grads).astype(np.float64), ref_g, 1e-5, "gradients of the live samples")
    k = int(host(count)[0])
    assert np.array_equal(np.sort(host(lst)[:k].view(np.uint32)), np.nonzero(touched_live)[0].astype(np.uint32))
