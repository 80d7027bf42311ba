"""Training rays from posed images on the GPU (tn_dataset_rays, and the trainer's dataset ray
source) against the oracle's restatement of the reference kernels, bit for bit: alive flags,
origins, directions, t, t_max, target texels and image ids of every live ray."""
import ctypes

import numpy as np
import pytest

import oracle
from tests.helpers import assert_bitwise
from turbonerf_b200 import scenes

pytestmark = pytest.mark.gpu

W, H = 40, 30


def look_at(eye, target=(0.0, 0.0, 0.0)):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, [0.0, 1.0, 0.0])
    r /= np.linalg.norm(r)
    t = np.zeros((3, 4))
    t[:, 0], t[:, 1], t[:, 2], t[:, 3] = r, np.cross(f, r), f, eye
    return t


def _cameras(n, seed, radius=4.0, far=100.0):
    from turbonerf_b200.renderer import Camera
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        eye = rng.normal(size=3)
        eye = radius * eye / np.linalg.norm(eye)
        cams.append(Camera((W, H), 0.1, far, (0.8 * W, 0.8 * W), (W / 2, H / 2), (0.0, 0.0), look_at(eye)))
    return cams


def _odict(c):
    return dict(width=c.resolution[0], height=c.resolution[1], near=c.near, far=c.far, focal=c.focal_length,
                principal=c.principal_point, shift=c.shift, transform=c.transform)


def _images(n, seed):
    rng = np.random.default_rng(seed)
    im = rng.integers(0, 256, (n, H, W, 4), dtype=np.uint8)
    im[..., 3] = np.where(rng.random((n, H, W)) < 0.4, rng.integers(0, 40, (n, H, W)), 255)  # transparent patches
    return im


def _compare(out, ref, n, what):
    alive = out["alive"]
    assert_bitwise(alive, ref["alive"], f"{what} alive")
    m = alive.astype(bool)
    assert m.any()
    for key, comps in (("ori", 3), ("dir", 3), ("pix_rgba", 4)):
        for c in range(comps):
            assert_bitwise(out[key][c * n:(c + 1) * n][m], ref[key][c * n:(c + 1) * n][m], f"{what} {key}[{c}]")
    for key in ("t", "t_max", "img_id"):
        assert_bitwise(out[key][m], ref[key][m], f"{what} {key}")


@pytest.mark.parametrize("threshold,probability", [(1.0, 1.0), (0.5, 0.3)])
def test_dataset_rays_match_oracle(threshold, probability):
    import torch

    from turbonerf_b200.native import Bbox, CameraC, call
    n_img, n = 5, 4099
    cams = _cameras(n_img, seed=11)
    imgs = _images(n_img, seed=12)
    bbox = (-1.5, -1.5, -1.5, 1.5, 1.5, 1.5)
    r = np.random.default_rng(13).random((2, n)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    cam_arr = (CameraC * n_img)(*[c.c_struct() for c in cams])
    cam_dev = torch.frombuffer(bytearray(bytes(cam_arr)), dtype=torch.uint8).cuda()
    img_dev, rnd = dev(imgs), dev(r)
    out_t = dict(pix_rgba=torch.zeros(4 * n, device="cuda"), img_id=torch.zeros(n, dtype=torch.int32, device="cuda"),
                 ori=torch.zeros(3 * n, device="cuda"), dir=torch.zeros(3 * n, device="cuda"),
                 t=torch.zeros(n, device="cuda"), t_max=torch.zeros(n, device="cuda"),
                 alive=torch.zeros(n, dtype=torch.uint8, device="cuda"))
    b = Bbox(*bbox)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    call("tn_dataset_rays", None, n, n, n_img, W, H, p(cam_dev), p(img_dev), ctypes.byref(b), p(rnd), threshold,
         probability, p(out_t["pix_rgba"]), p(out_t["img_id"]), p(out_t["ori"]), p(out_t["dir"]), p(out_t["t"]),
         p(out_t["t_max"]), p(out_t["alive"]))
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in out_t.items()}
    out["img_id"] = out["img_id"].view(np.uint32)
    ref, live = oracle.dataset_rays(n, [_odict(c) for c in cams], imgs, bbox, r, threshold, probability)
    assert int(out["alive"].sum()) == live
    _compare(out, ref, n, f"rays ({threshold}, {probability})")


def _trainer(path="fused", cameras=None):
    from turbonerf_b200.trainer import Dataset, SyntheticNeRF, Trainer
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=5)
    nerf = SyntheticNeRF.from_scene(sc)
    nerf.dataset = Dataset(cameras or _cameras(6, seed=21, radius=5.0), _images(6, seed=22))
    tr = Trainer(nerf, path=path, n_rays_per_step=4096, occupancy_cells_per_step=0, n_grid_params=16 * (1 << 15) * 2)
    tr.setup_data(batch_size=1 << 16)
    return sc, nerf, tr


def _trainer_rays(tr, n):
    h = lambda i, dt=np.float32: tr.buffer(i, dt).cpu().numpy()  # noqa: E731
    out = dict(ori=h(17), dir=h(18), t=h(19), t_max=h(20), alive=h(21, np.uint8)[:n], pix_rgba=h(22))
    return out, h(26)


def _compare_trainer(out, ref, n, what):
    """The trainer's rays after a step: the march has since dropped the live rays that take no
    sample, so its live set lies inside the dataset kernel's; every ray live there matches."""
    m = ref["alive"].astype(bool)
    assert m.any() and not np.any(out["alive"].astype(bool) & ~m), what
    for key, comps in (("ori", 3), ("dir", 3), ("pix_rgba", 4)):
        for c in range(comps):
            assert_bitwise(out[key][c * n:(c + 1) * n][m], ref[key][c * n:(c + 1) * n][m], f"{what} {key}[{c}]")
    for key in ("t", "t_max"):
        assert_bitwise(out[key][m], ref[key][m], f"{what} {key}")


def test_trainer_steps_on_dataset_rays_and_alpha_selection():
    sc, nerf, tr = _trainer()
    n = tr.n_rays_per_step
    cams = [_odict(c) for c in nerf.dataset.cameras]
    for step in range(3):
        m = tr.train_step()
        assert m.step == step + 1 and m.n_rays > 0 and m.n_samples > 0
        out, draws = _trainer_rays(tr, n)
        ref, live = oracle.dataset_rays(n, cams, nerf.dataset.images, sc.bbox, draws.reshape(2, n))
        _compare_trainer(out, ref, n, f"trainer step {step}")
    # alpha selection on: transparent texels keep a quarter of their rays
    tr.alpha_selection_threshold, tr.alpha_selection_probability = 0.5, 0.25
    tr.train_step()
    out, draws = _trainer_rays(tr, n)
    ref, live_sel = oracle.dataset_rays(n, cams, nerf.dataset.images, sc.bbox, draws.reshape(2, n), 0.5, 0.25)
    _compare_trainer(out, ref, n, "trainer with alpha selection")
    _, live_all = oracle.dataset_rays(n, cams, nerf.dataset.images, sc.bbox, draws.reshape(2, n))
    assert live_sel < live_all
    tr.teardown()


def test_fused_and_plain_paths_march_the_same_dataset_batch():
    _, _, a = _trainer("fused")
    _, _, b = _trainer("plain")
    ma, mb = a.train_step(), b.train_step()
    assert (ma.n_rays, ma.n_samples) == (mb.n_rays, mb.n_samples) and ma.n_samples > 0
    assert_bitwise(a.buffer(17).cpu().numpy(), b.buffer(17).cpu().numpy(), "ray origins")
    a.teardown()
    b.teardown()
