"""CPU checks of the training-ray restatement for posed images (oracle `dataset_rays`) in closed
form, and of the Python Dataset surface."""
import numpy as np
import pytest

import oracle

W, H = 8, 6
BOX = (-1.0, -1.0, -1.0, 1.0, 1.0, 1.0)


def _camera(eye, near=0.1, far=100.0):
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = (1, 0, 0), (0, 1, 0), (0, 0, 1), eye  # looks along +z
    return dict(width=W, height=H, near=near, far=far, focal=(6.0, 6.0), principal=(4.0, 3.0), shift=(0, 0),
                transform=t)


def _images(n, seed=0):
    return np.random.default_rng(seed).integers(0, 256, (n, H, W, 4), dtype=np.uint8)


def test_rays_images_and_texels():
    n = 64
    r = np.random.default_rng(1).random((2, n)).astype(np.float32)
    imgs = _images(2)
    cams = [_camera((0.0, 0.0, -3.0)), _camera((0.25, -0.1, -3.0))]
    out, live = oracle.dataset_rays(n, cams, imgs, BOX, r)
    assert 0 < live <= n
    alive = out["alive"].astype(bool)
    i = np.arange(n)
    img = np.minimum((i / np.float32(n / 2)).astype(np.int64), 1)
    p = (np.float32(W * H) * r[0]).astype(np.float64)
    x, y = np.fmod(p, W), p / W
    for k in np.nonzero(alive)[0]:
        assert out["img_id"][k] == img[k]
        eye = np.array(cams[img[k]]["transform"])[:, 3]
        v = np.array([(x[k] - 4.0 + 0.5) / 6.0, (y[k] - 3.0 + 0.5) / 6.0, 1.0])
        d = v / np.linalg.norm(v)
        np.testing.assert_allclose(out["dir"][k::n], d, atol=2e-6)
        np.testing.assert_allclose(out["ori"][k::n], eye + 0.1 * np.linalg.norm(v) * d, atol=2e-6)
        # entry through the z = -1 face (the rays point into the box from z = -3)
        o = out["ori"][k::n].astype(np.float64)
        t_in = max((-1.0 - o[2]) / d[2], 0.0) + 1e-5
        assert abs(out["t"][k] - t_in) < 1e-5
        assert out["t_max"][k] > out["t"][k]
        texel = imgs[img[k]].reshape(-1, 4)[min(int(np.float32(W * H) * r[0, k]), W * H - 1)]
        np.testing.assert_array_equal(out["pix_rgba"][k::n], texel.astype(np.float32) / np.float32(255.0))


def test_missing_rays_and_far_plane():
    r = np.random.default_rng(2).random((2, 16)).astype(np.float32)
    # looking away from the box: every ray misses
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = (1, 0, 0), (0, 1, 0), (0, 0, 1), (0.0, 0.0, 3.0)
    cam = dict(_camera((0, 0, 0)), transform=t)
    out, live = oracle.dataset_rays(16, [cam], _images(1), BOX, r)
    assert live == 0 and not out["alive"].any()
    # a far plane before the box: t_max < t kills every ray
    out, live = oracle.dataset_rays(16, [_camera((0.0, 0.0, -3.0), far=1.5)], _images(1), BOX, r)
    assert live == 0


def test_alpha_selection_drops_transparent_rays():
    n = 512
    rng = np.random.default_rng(3)
    r = rng.random((2, n)).astype(np.float32)
    imgs = _images(1, seed=4)
    cams = [_camera((0.0, 0.0, -3.0))]
    base, live0 = oracle.dataset_rays(n, cams, imgs, BOX, r)
    sel, live1 = oracle.dataset_rays(n, cams, imgs, BOX, r, alpha_threshold=0.5, alpha_probability=0.25)
    a = base["pix_rgba"][3 * n:]
    hit = base["alive"].astype(bool)
    drop = hit & (a < np.float32(0.5)) & (r[1] > np.float32(0.25))
    np.testing.assert_array_equal(sel["alive"].astype(bool), hit & ~drop)
    assert live1 == live0 - int(drop.sum()) and drop.sum() > 0
    # on only while both are below 1 (trainer.cu:86)
    _, live2 = oracle.dataset_rays(n, cams, imgs, BOX, r, alpha_threshold=0.5, alpha_probability=1.0)
    assert live2 == live0


def test_dataset_surface_checks():
    from turbonerf_b200.renderer import Camera
    from turbonerf_b200.trainer import Dataset
    cam = Camera((W, H), 0.1, 100.0, (6.0, 6.0), (4.0, 3.0), (0.0, 0.0), np.eye(4))
    ds = Dataset([cam, cam], _images(2))
    assert ds.images.shape == (2, H, W, 4) and ds.images.dtype == np.uint8
    with pytest.raises(ValueError):
        Dataset([cam], _images(2))
    with pytest.raises(ValueError):
        Dataset([cam, cam], _images(2)[..., :3])
    other = Camera((W + 1, H), 0.1, 100.0, (6.0, 6.0), (4.0, 3.0), (0.0, 0.0), np.eye(4))
    with pytest.raises(ValueError):
        Dataset([cam, other], _images(2))
