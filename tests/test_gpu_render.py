"""The inference renderer on the GPU (tn_trainer_render -> tn_render behind
`Renderer(pattern, batch_size).submit(RenderRequest(...))`) against the oracle's per-ray render
of the same scene: the trainer's occupancy grid and training box, the blob field as the network.

The sample positions and their validity are exact FP32 in both; the field, opacities and
compositing are FP32 on the GPU and FP64 in the oracle, so pixels are compared within the
composite tolerance. Pixels the oracle flags as ambiguous (transmittance or opacity within a
hair of the reference's cut-offs) are left out of the comparison."""
import numpy as np
import pytest

import oracle
from tests.helpers import FLOOR, RTOL_COMPOSITE, assert_close
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu

CONE = 1.0 / 256.0


def look_at(eye, target=(0.0, 0.0, 0.0)):
    """Camera to world [3][4]: columns right, down, forward (the camera looks along +z)."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, [0.0, 1.0, 0.0])
    r /= np.linalg.norm(r)
    d = np.cross(f, r)
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = r, d, f, eye
    return t


def _trainer(n_levels=5, cells=0, render_bbox=None, min_transmittance=1e-4, bitfield=None):
    from turbonerf_b200.trainer import BoundingBox, SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=n_levels)
    if bitfield is not None:
        sc.grid.bitfield = bitfield
    nerf = SyntheticNeRF.from_scene(sc)
    if render_bbox is not None:
        b = BoundingBox()
        b.min_x, b.min_y, b.min_z, b.max_x, b.max_y, b.max_z = render_bbox
        nerf.render_bbox = b
    tr = Trainer(nerf, n_rays_per_step=4096, occupancy_cells_per_step=cells, occupancy_threshold=0.01,
                 n_grid_params=16 * (1 << 15) * 2, min_transmittance=min_transmittance)
    tr.setup_data(batch_size=1 << 16)
    return sc, tr


def _camera(w, h, eye, far=100.0, shift=(0.0, 0.0)):
    from turbonerf_b200.renderer import Camera
    f = 0.7 * w
    return Camera((w, h), 0.1, far, (f, f), (w / 2, h / 2), shift, look_at(eye))


def _oracle_image(sc, cam, bits=None, render_bbox=None, dt_min=scenes.MIN_STEP_SIZE, min_t=1e-4):
    grid = sc.grid.as_dict()
    if bits is not None:
        grid = dict(grid, bitfield=bits)
    c = dict(width=cam.resolution[0], height=cam.resolution[1], near=cam.near, far=cam.far,
             focal=cam.focal_length, principal=cam.principal_point, shift=cam.shift, transform=cam.transform)
    return oracle.render(c, render_bbox or sc.bbox, sc.bbox, grid, float(np.float32(dt_min)), CONE, min_t,
                         sc.field.blobs, sc.field.waves, sc.aabb_size)


def _submit(tr, cam, batch_size=0, target=None, min_step_size=None):
    from turbonerf_b200.renderer import CPURenderBuffer, Renderer, RenderPattern, RenderRequest
    r = Renderer(pattern=RenderPattern.LinearChunks, batch_size=batch_size)
    if min_step_size is not None:
        r.min_step_size = min_step_size
    out = target if target is not None else CPURenderBuffer()
    done = []
    req = RenderRequest(cam, [tr], out, on_complete=lambda: done.append(True))
    stats = r.submit(req)
    assert done == [True]
    return out.get_rgba(), stats


def _compare(img, ref, amb, what):
    ok = amb == 0
    assert ok.mean() > 0.99, f"{what}: {np.count_nonzero(~ok)} ambiguous pixels"
    assert img.shape == ref.shape
    for c, name in enumerate("rgba"):
        assert_close(img[..., c][ok], ref[..., c][ok], RTOL_COMPOSITE, f"{what} {name}", floor=FLOOR)
    # pixels the rays miss stay exactly clear
    miss = ref[..., 3] == 0
    assert np.all(img[miss] == 0), what


@pytest.mark.parametrize("eye,res", [((0.3, 0.8, 4.0), (96, 64)), ((-3.0, 2.0, -2.5), (160, 120)),
                                     ((0.2, -0.1, 0.6), (64, 64))])
def test_render_matches_oracle(eye, res):
    """Views from outside the scene's blobs and from inside the training box."""
    sc, tr = _trainer()
    cam = _camera(*res, eye)
    img, stats = _submit(tr, cam)
    ref, amb, n_ref = _oracle_image(sc, cam)
    _compare(img, ref, amb, f"eye {eye}")
    assert stats["rays_hit"] == res[0] * res[1]  # every ray meets the 16-unit training box
    assert stats["samples"] >= n_ref > 0  # rays that end mid-round still sent that round's samples
    tr.teardown()


def test_render_is_schedule_independent():
    """The round size (batch_size / live rays steps) changes only the FP32 grouping of the
    per-round partial sums, not which samples are composited."""
    sc, tr = _trainer()
    cam = _camera(80, 60, (0.5, 0.6, 3.5))
    ref, amb, _ = _oracle_image(sc, cam)
    imgs = {}
    for bs in (1 << 12, 1 << 16, 1 << 22):
        imgs[bs], stats = _submit(tr, cam, batch_size=bs)
        _compare(imgs[bs], ref, amb, f"batch {bs}")
    assert stats["iterations"] < 200
    tr.teardown()


def test_render_bbox_crop_and_far_plane():
    """A render box smaller than the training box (the reference's per-NeRF crop) and a camera
    whose far plane lies beyond the box."""
    crop = (-0.6, -0.5, -0.7, 0.8, 0.6, 0.5)
    sc, tr = _trainer(render_bbox=crop)
    cam = _camera(96, 72, (1.0, 0.7, 3.0), far=50.0)
    img, stats = _submit(tr, cam)
    ref, amb, _ = _oracle_image(sc, cam, render_bbox=crop)
    _compare(img, ref, amb, "cropped")
    assert 0 < stats["rays_hit"] < 96 * 72
    tr.teardown()


def test_render_misses_and_shift():
    sc, tr = _trainer()
    from turbonerf_b200.renderer import Camera
    # rays that pass beside the box: the slab test fails, no ray is marched
    t = look_at((0.0, 20.0, 0.0), (10.0, 20.0, 0.0))
    cam = Camera((32, 24), 0.1, 100.0, (30.0, 30.0), (16.0, 12.0), (0.0, 0.0), t)
    img, stats = _submit(tr, cam)
    assert stats["rays_hit"] == 0 and stats["samples"] == 0 and not img.any()
    # looking away from the box: the reference's slab test (t_max >= t_min, bounding-box.cuh:50)
    # accepts a box behind the ray, which is then marched for one round outside the box and
    # dropped with nothing composited
    t = look_at((0.0, 0.0, 20.0), (0.0, 0.0, 40.0))
    cam = Camera((32, 24), 0.1, 100.0, (30.0, 30.0), (16.0, 12.0), (0.0, 0.0), t)
    img, stats = _submit(tr, cam)
    assert stats["rays_hit"] == 32 * 24 and stats["iterations"] == 1
    assert stats["samples"] == 0 and not img.any()
    # a shifted view (the principal point moves by shift * resolution)
    cam = _camera(64, 48, (0.3, 0.8, 4.0), shift=(0.25, -0.1))
    img, _ = _submit(tr, cam)
    ref, amb, _ = _oracle_image(sc, cam)
    _compare(img, ref, amb, "shifted")
    tr.teardown()


def test_render_after_training_uses_the_live_grid_and_min_step_size():
    """After steps that re-sample the occupancy grid, the render reads the trainer's current
    bitfield; the renderer's min_step_size sets the step."""
    sc, tr = _trainer(cells=1 << 16)
    for _ in range(3):
        tr.train_step()
    tr.update_occupancy_grid(300)
    bits = tr.buffer(6, np.uint8).cpu().numpy().copy()
    assert not np.array_equal(bits, sc.grid.bitfield)
    cam = _camera(72, 54, (0.4, 0.9, 3.8))
    img, _ = _submit(tr, cam)
    ref, amb, _ = _oracle_image(sc, cam, bits=bits)
    _compare(img, ref, amb, "trained grid")
    img2, _ = _submit(tr, cam, min_step_size=2.0 * scenes.MIN_STEP_SIZE)
    ref2, amb2, _ = _oracle_image(sc, cam, bits=bits, dt_min=2.0 * scenes.MIN_STEP_SIZE)
    _compare(img2, ref2, amb2, "double step")
    tr.teardown()


def test_cuda_render_buffer_matches_cpu_buffer_and_png():
    import torch

    from turbonerf_b200.renderer import CUDARenderBuffer
    sc, tr = _trainer()
    cam = _camera(48, 32, (0.3, 0.8, 4.0))
    img, _ = _submit(tr, cam)
    buf = CUDARenderBuffer()
    img_dev, _ = _submit(tr, cam, target=buf)
    assert isinstance(buf.rgba, torch.Tensor) and buf.rgba.is_cuda and tuple(buf.rgba.shape) == (32, 48, 4)
    assert np.array_equal(img, img_dev)
    tr.teardown()


def test_render_rejects_bad_cameras():
    from turbonerf_b200.native import TurboError
    from turbonerf_b200.renderer import Camera
    sc, tr = _trainer()
    cam = Camera((16, 16), 0.1, 10.0, (0.0, 0.0), (8, 8), (0, 0), look_at((0, 0, 4)))
    with pytest.raises(TurboError, match="focal"):
        _submit(tr, cam)
    cam = Camera((0, 16), 0.1, 10.0, (10.0, 10.0), (8, 8), (0, 0), look_at((0, 0, 4)))
    with pytest.raises(TurboError, match="empty image"):
        _submit(tr, cam)
    tr.teardown()


@pytest.mark.parametrize("density", [0.002, 0.03, 0.3])
def test_render_sample_set_is_exact_on_random_grids(density):
    """With no early termination (min_transmittance 0) every ray collects all of its valid
    samples, so the number sent to the network must equal the oracle's step-by-step count
    exactly: a sample lost or added by the empty-space skipping changes it. Random bitfields
    put occupied cells at every level next to empty ones, and the views include cameras inside
    several cascade levels."""
    rng = np.random.default_rng(int(density * 1e4))
    R = 128
    bits = np.zeros(R ** 3, np.uint8)
    for k in range(5):
        bits |= ((rng.random(R ** 3) < density).astype(np.uint8) << np.uint8(k))
    sc, tr = _trainer(min_transmittance=0.0, bitfield=bits)
    for eye in ((0.3, 0.8, 4.0), (0.05, -0.2, 0.3), (-1.7, 0.9, 1.2), (6.0, -5.0, 7.5), (12.0, 3.0, -9.0)):
        cam = _camera(48, 40, eye)
        img, stats = _submit(tr, cam, batch_size=1 << 16)
        ref, amb, n_ref = _oracle_image(sc, cam, min_t=0.0)
        assert stats["samples"] == n_ref, (eye, stats, n_ref)
        assert stats["tests"] <= stats["steps"]
        _compare(img, ref, amb, f"random grid {density} eye {eye}")
    tr.teardown()
