"""CPU checks of the renderer's host side: the oracle's per-ray render in closed-form cases,
and the Python surface (camera validation, PNG output) without a GPU."""
import struct
import zlib

import numpy as np
import pytest

import oracle

BOX = (-1.0, -1.0, -1.0, 1.0, 1.0, 1.0)


def _grid(bits_value=0xFF, n_levels=1, res=16, base=2.0):
    return dict(n_levels=n_levels, res=res, base=base, bitfield=np.full(res ** 3, bits_value, np.uint8))


def _camera(w=24, h=16, eye=(0.0, 0.0, -3.0), far=100.0):
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = (1, 0, 0), (0, 1, 0), (0, 0, 1), eye  # looks along +z
    return dict(width=w, height=h, near=0.1, far=far, focal=(20.0, 20.0), principal=(w / 2, h / 2), shift=(0, 0),
                transform=t)


def _uniform_field(sigma, phase):
    """One blob so wide that its density is constant over the box; colours sigmoid(sin(phase))."""
    blobs = np.array([[0.0, 0.0, 0.0, 1e6, sigma]], np.float32)
    waves = np.zeros((3, 4), np.float32)
    waves[:, 3] = phase
    return blobs, waves


def test_oracle_render_uniform_medium_closed_form():
    """Constant density and colour: every hit pixel's colour is c times its opacity, and the
    opacity is 1 - exp(-sigma * path / box size) for the path through the box."""
    sigma = 3.0
    phase = np.array([0.3, -0.7, 1.1], np.float32)
    blobs, waves = _uniform_field(sigma, phase)
    cam = _camera()
    rgba, amb, n = oracle.render(cam, BOX, BOX, _grid(), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    assert n > 0 and not amb.any()
    hit = rgba[..., 3] > 0
    assert hit.sum() > 100
    c = 1.0 / (1.0 + np.exp(-np.sin(phase.astype(np.float64))))
    for k in range(3):
        np.testing.assert_allclose(rgba[..., k][hit], c[k] * rgba[..., 3][hit], rtol=1e-12)
    # the centre ray crosses the box along z: path 2, box size 2 -> optical depth sigma
    h, w = rgba.shape[:2]
    centre = rgba[h // 2, w // 2, 3]
    assert abs(centre - (1.0 - np.exp(-sigma))) < 2e-3


def test_oracle_render_empty_grid_and_misses():
    blobs, waves = _uniform_field(3.0, np.zeros(3, np.float32))
    rgba, amb, n = oracle.render(_camera(), BOX, BOX, _grid(0), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    assert n == 0 and not rgba.any()
    away = _camera(eye=(0.0, 0.0, 3.0))  # outside the box, looking away from it
    rgba, _, n = oracle.render(away, BOX, BOX, _grid(), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    assert n == 0 and not rgba.any()


def test_oracle_render_opaque_medium_stops_at_min_transmittance():
    """A very dense medium: the ray ends once the transmittance falls below the cut, so the
    opacity is 1 - T_end with T_end just under 1e-4, and few samples are taken."""
    blobs, waves = _uniform_field(2000.0, np.zeros(3, np.float32))
    cam = _camera(w=4, h=4)
    rgba, amb, n = oracle.render(cam, BOX, BOX, _grid(), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    a = rgba[..., 3]
    assert np.all(a > 1.0 - 1e-4) and np.all(a < 1.0)
    assert n < 16 * 20


def test_oracle_render_crop_box_limits_samples():
    """A render box inside the training box: only samples inside it are composited."""
    blobs, waves = _uniform_field(1.0, np.zeros(3, np.float32))
    crop = (-0.5, -0.5, -0.5, 0.5, 0.5, 0.5)
    cam = _camera()
    full, _, n_full = oracle.render(cam, BOX, BOX, _grid(), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    part, _, n_part = oracle.render(cam, crop, BOX, _grid(), np.float32(1e-3), 0.0, 1e-4, blobs, waves, 2.0)
    assert 0 < n_part < n_full
    h, w = full.shape[:2]
    # centre ray: path 1 through the crop instead of 2 through the box
    assert abs(part[h // 2, w // 2, 3] - (1.0 - np.exp(-0.5))) < 2e-3
    assert np.count_nonzero(part[..., 3]) < np.count_nonzero(full[..., 3])


def test_camera_and_png_without_gpu(tmp_path):
    from turbonerf_b200.renderer import Camera, CPURenderBuffer, RenderFlags, RenderPattern, Renderer
    with pytest.raises(NotImplementedError):
        Camera((8, 8), 0.1, 10.0, (8, 8), (4, 4), (0, 0), np.eye(4), dist_params=dict(k1=0.1))
    with pytest.raises(ValueError):
        Camera((8, 8), 0.1, 10.0, (8, 8), (4, 4), (0, 0), np.eye(3))
    cam = Camera((8, 4), 0.1, 10.0, (8, 8), (4, 2), (0.5, 0.0), np.eye(4))
    c = cam.c_struct()
    assert (c.width, c.height, c.shift_x) == (8, 4, 0.5) and list(c.transform)[:4] == [1.0, 0.0, 0.0, 0.0]
    assert Renderer().batch_size == 0 and Renderer(batch_size=4096).batch_size == 4096
    assert Renderer(pattern=RenderPattern.HexagonalGrid).pattern == RenderPattern.HexagonalGrid
    assert int(RenderFlags.Preview | RenderFlags.Final) == 3
    buf = CPURenderBuffer()
    buf.set_size(8, 4)
    buf._rgba = np.zeros((4, 8, 4), np.float32)
    buf._rgba[1, 2] = (1.0, 0.5, 0.0, 1.0)
    path = tmp_path / "img.png"
    buf.save_image(str(path))
    data = path.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h = struct.unpack(">II", data[16:24])
    assert (w, h) == (8, 4)
    idat_len = struct.unpack(">I", data[33:37])[0]
    raw = zlib.decompress(data[41:41 + idat_len])
    row = raw[1 * (1 + 32):2 * (1 + 32)]
    assert row[1 + 2 * 4:1 + 3 * 4] == bytes([255, 128, 0, 255])
