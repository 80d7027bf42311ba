"""The oracle's hash-grid encoding and linear heads on the CPU (test infrastructure): the
published algorithm's known answers (a position on a vertex reads that vertex's entry, through
the direct index on coarse levels and the spatial hash on fine ones), the backward as the exact
transpose of the forward, and the heads' gradients against central differences. tcnn's own
HashGrid is not in the reference tree, so nothing pins these to tcnn's outputs."""
import math

import numpy as np

import oracle

LOG2_T = 12


def _levels():
    return oracle.hashgrid_levels(6, LOG2_T, 4.0, 2.0)  # resolutions 4, 8, 16, 32, 64, 128


def test_level_resolutions_and_dense_levels():
    res, dense = _levels()
    assert list(res) == [4, 8, 16, 32, 64, 128]
    # a level indexes directly while its (res + 1)^3 vertices fit in 2^12 entries
    assert list(dense) == [1, 1, 0, 0, 0, 0]
    b = math.exp((math.log(2048.0 * 16) - math.log(16.0)) / 15.0)  # the reference's encoding, aabb 16
    res, dense = oracle.hashgrid_levels(16, 19, 16.0, b)
    assert res[0] == 16 and all(np.diff(res.astype(np.int64)) > 0) and res[-1] in (32767, 32768)
    assert dense.sum() == 4


def test_vertex_positions_read_their_entry():
    res, dense = _levels()
    T = 1 << LOG2_T
    L = len(res)
    params = np.zeros(L * T * 2, np.float32)
    params[0::2] = np.tile(np.arange(T, dtype=np.float32), L)      # feature 0: the entry's index
    params[1::2] = -np.tile(np.arange(T, dtype=np.float32), L)     # feature 1: minus it
    rng = np.random.default_rng(3)
    for l in range(L):
        N = int(res[l])
        v = rng.integers(0, N, size=(64, 3))
        pos = (v.astype(np.float64) / N).astype(np.float32)
        ok = np.all((pos * np.float32(N)).astype(np.float64) == v, axis=1)  # exactly on the vertex in FP32
        pos, v = pos[ok], v[ok]
        n = len(pos)
        feat = oracle.hashgrid_encode((res, dense), LOG2_T, np.ascontiguousarray(pos.T).ravel(), params, n)
        got = feat[2 * l * n:(2 * l + 1) * n]
        x, y, z = (v[:, k].astype(np.uint64) for k in range(3))
        if dense[l]:
            want = x + (N + 1) * (y + (N + 1) * z)
        else:
            h = (x * np.uint64(1)) ^ (y * np.uint64(2654435761)) ^ (z * np.uint64(805459861))
            want = (h & np.uint64(0xFFFFFFFF)) & np.uint64(T - 1)
        assert np.array_equal(got.astype(np.uint64), want), f"level {l}"
        assert np.array_equal(feat[(2 * l + 1) * n:(2 * l + 2) * n], -got)


def test_backward_is_the_transpose_of_the_forward():
    res, dense = _levels()
    T = 1 << LOG2_T
    rng = np.random.default_rng(4)
    n = 3000
    pos = rng.uniform(0.0, 1.0, 3 * n).astype(np.float32)
    pos[:30] = 0.0
    pos[30:60] = 1.0
    params = rng.normal(0.0, 1.0, len(res) * T * 2).astype(np.float32)
    dfeat = rng.normal(0.0, 1.0, 2 * len(res) * n)
    feat = oracle.hashgrid_encode((res, dense), LOG2_T, pos, params, n).astype(np.float64)
    grads, touched = oracle.hashgrid_backward((res, dense), LOG2_T, pos, dfeat, n)
    lhs = float(np.dot(feat, dfeat))
    rhs = float(np.dot(params.astype(np.float64), grads))
    assert abs(lhs - rhs) <= 1e-5 * (np.abs(feat).max() * np.abs(dfeat).sum())
    # an entry is touched exactly when some sample's corner lands on it
    assert set(np.nonzero(touched)[0]) >= set(np.nonzero(grads.reshape(-1, 2).any(axis=1))[0])


def test_heads_gradients_match_central_differences():
    rng = np.random.default_rng(5)
    nf, n = 8, 40
    feat = rng.normal(0.0, 0.5, nf * n).astype(np.float32)
    head = rng.normal(0.0, 0.3, 4 * (nf + 1)).astype(np.float32)
    gd = rng.normal(0.0, 1.0, n)
    grgb = rng.normal(0.0, 1.0, 3 * n)

    def loss(h, f):
        d, rgb = oracle.hash_heads_forward(nf, f, h, n)
        return float(np.dot(d, gd) + np.dot(rgb, grgb))

    dfeat, dhead = oracle.hash_heads_backward(nf, feat, head, gd, grgb, n)
    eps = 1e-3
    for k in rng.choice(len(head), 10, replace=False):
        hp_, hm_ = head.astype(np.float64).copy(), head.astype(np.float64).copy()
        hp_[k] += eps
        hm_[k] -= eps
        fd = (loss(hp_.astype(np.float32), feat) - loss(hm_.astype(np.float32), feat)) / (2 * eps)
        assert abs(fd - dhead[k]) <= 2e-2 * max(1.0, abs(dhead[k])), k
    for k in rng.choice(len(feat), 10, replace=False):
        fp, fm = feat.astype(np.float64).copy(), feat.astype(np.float64).copy()
        fp[k] += eps
        fm[k] -= eps
        fd = (loss(head, fp.astype(np.float32)) - loss(head, fm.astype(np.float32))) / (2 * eps)
        assert abs(fd - dfeat[k]) <= 2e-2 * max(1.0, abs(dfeat[k])), k
