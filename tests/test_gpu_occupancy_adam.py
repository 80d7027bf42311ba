"""Parity of the occupancy-grid EMA / bitfield rebuild (bit-exact densities, bits and
popcount) and of Adam (within 1e-5 relative of the FP64 oracle) on the GPU."""
import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise, assert_norm_close, dev, host, i32
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu


def _grid(n_levels, res=128, seed=0x7B5):
    rng = np.random.default_rng(seed)
    V = res ** 3
    d = np.where(rng.random((n_levels, V)) < 0.3, rng.exponential(0.05, (n_levels, V)), 0.0).astype(np.float32)
    bits = np.zeros(V, np.uint8)
    for k in range(n_levels):
        bits |= ((d[k] > 0.01).astype(np.uint8) << k)
    return d, bits


@pytest.mark.parametrize("sample_all,dup", [(False, False), (True, False), (False, True)])
def test_occupancy_update_bit_exact(sample_all, dup):
    from turbonerf_b200 import hotpath as hp
    L = 5
    d, bits = _grid(L)
    V = d.shape[1]
    rng = np.random.default_rng(12)
    m = 1 << 16
    levels = rng.integers(0, L, m).astype(np.int32)
    cells = rng.integers(0, V, m).astype(np.uint32)
    if dup:  # many updates of the same cells
        cells[: m // 2] = cells[m // 2:]
        levels[: m // 2] = levels[m // 2:]
    values = rng.exponential(0.05, m).astype(np.float32)
    rsel = rng.random(m).astype(np.float32)
    ref_d, ref_b, ref_n = oracle.occupancy_update(d, bits, L, 128, levels, cells, values, rsel, act=0,
                                                  sample_all=sample_all)
    grid = hp.GridSpec(L, 128, 1.0)
    ctx = hp.Context()
    dd, bb = dev(d.ravel().copy()), dev(bits.copy())
    nocc = hp.occupancy_update(ctx, grid, dd, bb, dev(levels), i32(cells), dev(values), dev(rsel), sample_all=sample_all)
    assert_bitwise(host(dd), ref_d.ravel(), "density")
    assert_bitwise(host(bb), ref_b, "bitfield")
    assert int(host(nocc)[0]) == ref_n
    # plain path
    dd2, bb2 = dev(d.ravel().copy()), dev(bits.copy())
    n2 = hp.plain_occupancy_update(grid, dd2, bb2, dev(levels), i32(cells), dev(values), dev(rsel),
                                   sample_all=sample_all)
    assert_bitwise(host(dd2), ref_d.ravel(), "plain density")
    assert_bitwise(host(bb2), ref_b, "plain bitfield")
    assert n2 == ref_n
    assert ctx.check() == 0


def test_occupancy_sample_points_and_popcount():
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(4)
    n = 50000
    levels = rng.integers(0, 5, n).astype(np.int32)
    cells = rng.integers(0, 128 ** 3, n).astype(np.uint32)
    rand3 = rng.random(3 * n).astype(np.float32)
    for base, inv_aabb in ((1.0, 1.0 / 16.0), (3.0, 1.0 / 3.0)):
        ref = oracle.occupancy_sample_points(levels, cells, rand3, n, 128, base, inv_aabb, n)
        out = hp.occupancy_sample_points(hp.GridSpec(5, 128, base), dev(levels), i32(cells), dev(rand3), n, inv_aabb)
        assert_bitwise(host(out), ref, f"sample points base={base}")
    ctx = hp.Context()
    for nb in (4, 1000, 1 << 21, (1 << 21) + 3):
        b = rng.integers(0, 256, nb).astype(np.uint8)
        assert int(host(hp.popcount(ctx, dev(b)))[0]) == oracle.popcount(b)


@pytest.mark.parametrize("plain", [False, True])
def test_adam_matches_fp64(plain):
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(8)
    n_grid, n_mlp = 1 << 20, 7168
    n = n_grid + n_mlp + 5  # a ragged tail beyond the MLP (no L2)
    w0 = rng.normal(0, 1e-2, n).astype(np.float32)
    state = dict(w=w0.astype(np.float64), m=np.zeros(n), v=np.zeros(n), steps=np.zeros(n, np.uint32))
    w, m, v = dev(w0.copy()), dev(np.zeros(n, np.float32)), dev(np.zeros(n, np.float32))
    steps = dev(np.zeros(n, np.int32))
    wcopy = dev(np.zeros(n, np.float32))
    for it in range(4):
        g = rng.normal(0, 1e-3, n).astype(np.float32)
        g[:n_grid][rng.random(n_grid) < 0.6] = 0.0  # sparse hash gradients
        lr = float(np.float32(1e-2 / (1.0 + 3.3e-5 * it)))
        # the oracle gets the same float32 hyper-parameters the kernel sees
        f32 = lambda x: float(np.float32(x))  # noqa: E731
        oracle.adam_step(state, g, n_grid, n_mlp, lr=lr, beta1=f32(0.9), beta2=f32(0.99), eps=f32(1e-15),
                         l2=f32(1e-6))
        hp.adam_step(w, dev(g), m, v, steps, n_grid, n_mlp, lr=lr, beta2=0.99, weights_copy=wcopy, plain=plain)
    assert_bitwise(host(steps).view(np.uint32), state["steps"], "per-parameter steps")
    # Adam moves a weight by about lr per step whatever the gradient's scale: the weight error
    # is measured against that step size (4 steps of lr = 1e-2)
    err_w = np.abs(host(w).astype(np.float64) - state["w"]) / (4 * 1e-2)
    assert float(err_w.max()) <= 1e-5, float(err_w.max())
    assert_norm_close(host(m), state["m"], 1e-5, "first moments")
    assert_norm_close(host(v), state["v"], 1e-5, "second moments")
    touched = state["steps"] > 0
    assert_bitwise(host(wcopy)[touched], host(w)[touched], "weights copy")
    # a never-updated parameter keeps its old copy (0 here) or, when it shares a 16-byte quad
    # with updated ones, receives its unchanged weight
    wc, ww = host(wcopy)[~touched], host(w)[~touched]
    assert np.all((wc == 0) | (wc == ww))
