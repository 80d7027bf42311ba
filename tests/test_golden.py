"""The oracle reproduces the committed golden fixtures (tests/golden/make_golden.py) exactly."""
import os

import numpy as np

import oracle
from tests.golden import make_golden

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


def _same(a, b, what):
    a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
    assert a.shape == b.shape and a.dtype == b.dtype, what
    assert np.ascontiguousarray(a).tobytes() == np.ascontiguousarray(b).tobytes(), what


def test_march_fixture_reproduces():
    fx, new = _load("march_small"), make_golden.march_fixture()
    for k in ("n_steps", "alive", "offsets", "n_rays", "n_samples", "s_t", "s_pos", "s_dt", "s_m_norm", "s_dt_norm"):
        _same(new[k], fx[k], k)


def test_loss_fixture_reproduces():
    fx, new = _load("loss_small"), make_golden.loss_fixture()
    for k in ("ray_rgba", "loss", "dL_ddensity", "dL_drgb", "n_used", "dist_loss", "dist_dd", "n_alt", "alt",
              "br_ray_rgba", "br_loss", "br_dL_ddensity", "br_dL_drgb"):
        _same(new[k], fx[k], k)
    # branch 0 is the FP64 cut of every ray; the fixture holds rays that rounding decides
    assert np.array_equal(fx["br_dL_ddensity"][0], fx["dL_ddensity"])


def test_occupancy_fixture_reproduces():
    fx, new = _load("occupancy_small"), make_golden.occupancy_fixture()
    for k in ("out_density", "out_bitfield", "n_occupied"):
        _same(new[k], fx[k], k)
    assert oracle.popcount(fx["out_bitfield"]) == int(fx["n_occupied"])


def test_render_fixture_reproduces():
    fx, new = _load("render_small"), make_golden.render_fixture()
    for k in ("rgba", "ambiguous", "n_samples", "bitfield"):
        _same(new[k], fx[k], k)
    assert int(fx["n_samples"]) > 0 and not fx["ambiguous"].any()
