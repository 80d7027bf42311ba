"""The identity behind the trainer's occupancy bitfield computed one step ahead, checked on the
oracle (CPU). An occupancy update decays every cell, raises each selected queried cell to the
maximum of its decayed density and the query's sigma, and thresholds the result. Its bitfield is
therefore the decayed grid against the threshold, or-ed with the selected queried cells whose
max(decay * density, sigma) is above it, and can be computed before the update, from the same
densities and queries, without changing them. The CUDA form of this (occ_bits_decayed_kernel and
occ_bits_raise_kernel) is checked bit for bit on the GPU through the trainer, against steps run in
order (tests/test_gpu_autotune.py)."""
import numpy as np
import pytest

import oracle


def _bits_ahead(density, bitfield, n_levels, res, levels, cells, values, rand_select, sample_all, decay, thr):
    V = res ** 3
    d = density.reshape(n_levels, V)
    decayed = d * np.float32(decay)
    bits = np.zeros(V, np.uint8)
    for k in range(n_levels):
        bits |= (decayed[k] > np.float32(thr)).astype(np.uint8) << k
    r = rand_select
    held = (bitfield[cells] >> levels.astype(np.uint8)) & 1
    sel = np.ones(len(levels), bool) if sample_all else (r < 0.25) | ((r <= 0.5) & (held == 1))
    raised = np.maximum(decayed[levels, cells], values) > np.float32(thr)
    hit = sel & raised
    np.bitwise_or.at(bits, cells[hit], (np.uint8(1) << levels[hit].astype(np.uint8)))
    return bits


@pytest.mark.parametrize("sample_all", [True, False])
def test_bitfield_ahead_equals_the_updates_bitfield(sample_all):
    rng = np.random.default_rng(0x0CC + int(sample_all))
    n_levels, res = 5, 32
    V = res ** 3
    thr, decay = 0.01 * 0.00169145586, 0.95
    for trial in range(4):
        # densities straddling the threshold after the decay, many of them exactly zero
        density = (rng.exponential(thr, n_levels * V) * (rng.random(n_levels * V) < 0.6)).astype(np.float32)
        bitfield = rng.integers(0, 1 << n_levels, V).astype(np.uint8)
        n = 20000
        levels = rng.integers(0, n_levels, n).astype(np.int32)
        cells = rng.integers(0, V, n).astype(np.uint32)
        cells[: n // 4] = cells[n // 4: n // 2]  # duplicate updates of one cell
        values = (rng.exponential(thr, n) * (rng.random(n) < 0.8)).astype(np.float32)
        rand_select = rng.random(n).astype(np.float32)
        ahead = _bits_ahead(density, bitfield, n_levels, res, levels, cells, values, rand_select, sample_all,
                            decay, thr)
        _, bits, n_occ = oracle.occupancy_update(density, bitfield, n_levels, res, levels, cells, values,
                                                 rand_select, act=0, sample_all=sample_all, decay=decay,
                                                 threshold=thr)
        np.testing.assert_array_equal(ahead, bits)
        assert n_occ == int(np.unpackbits(ahead).sum())
