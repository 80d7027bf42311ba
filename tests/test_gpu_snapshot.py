"""Snapshots of a training run on the GPU (tn_trainer_save / tn_trainer_load): the file carries
the reference's sections, a fresh trainer loaded from it holds bit for bit the same weights,
optimizer state, grid and step counters, and its next steps equal those of the trainer that
was saved."""
import numpy as np
import pytest

from tests.helpers import assert_bitwise
from turbonerf_b200 import native, scenes
from turbonerf_b200.trainer import FileManager, SyntheticNeRF, Trainer

pytestmark = pytest.mark.gpu

STATE = {0: np.float32, 2: np.float32, 3: np.float32, 4: np.uint32, 5: np.float32, 6: np.uint8}


def _trainer(path="fused", n_mlp=7168):
    sc = scenes.march_scene_cascaded(n_rays=8, n_levels=3)
    tr = Trainer(SyntheticNeRF.from_scene(sc), path=path, n_rays_per_step=4096, occupancy_cells_per_step=4096,
                 n_grid_params=16 * (1 << 15) * 2, n_mlp_params=n_mlp)
    tr.setup_data(batch_size=1 << 16)
    return tr


def _state(tr):
    tr.flush()
    return {k: tr.buffer(k, dt).cpu().numpy() for k, dt in STATE.items()}


@pytest.mark.parametrize("path", ["fused", "plain"])
def test_save_load_resumes_exactly(tmp_path, path):
    a = _trainer(path)
    for _ in range(3):
        a.train_step()
    f = str(tmp_path / "run.turbo")
    FileManager.save(a, f, "/data/synthetic")
    info = FileManager.info(f)
    assert info["has_resume"] and info["step_count"] == 3 and info["dataset_path"] == "/data/synthetic"
    assert info["n_params"] == a.n_grid_params + a.n_mlp_params
    # the reference's sections: header, fp32 parameters, bitfield
    raw = open(f, "rb").read()
    sa = _state(a)
    n = info["n_params"]
    assert_bitwise(np.frombuffer(raw[300:300 + 4 * n], np.float32), sa[0], "file parameters")
    assert_bitwise(np.frombuffer(raw[300 + 4 * n:300 + 4 * n + info["n_occ_grid_bits"]], np.uint8), sa[6], "file bits")

    b = _trainer(path)
    FileManager.load(b, f)
    sb = _state(b)
    for k in STATE:
        assert_bitwise(sb[k], sa[k], f"loaded buffer {k}")
    assert [b.stat(i) for i in (3, 4, 5)] == [a.stat(i) for i in (3, 4, 5)]
    for step in range(2):
        ma, mb = a.train_step(), b.train_step()
        assert (ma.step, ma.n_rays, ma.n_samples) == (mb.step, mb.n_rays, mb.n_samples) == (ma.step, ma.n_rays,
                                                                                              ma.n_samples)
        assert ma.step == 4 + step and mb.loss == pytest.approx(ma.loss, rel=1e-6)
    sa, sb = _state(a), _state(b)
    for k in STATE:
        assert_bitwise(sb[k], sa[k], f"buffer {k} after resumed steps")
    a.teardown()
    b.teardown()


def test_reference_sections_alone_set_weights_and_bits(tmp_path):
    a = _trainer()
    a.train_step()
    f = str(tmp_path / "run.turbo")
    FileManager.save(a, f)
    info = FileManager.info(f)
    ref_only = str(tmp_path / "ref.turbo")
    with open(f, "rb") as src, open(ref_only, "wb") as dst:
        dst.write(src.read(300 + 4 * info["n_params"] + info["n_occ_grid_bits"]))
    assert not FileManager.info(ref_only)["has_resume"]
    b = _trainer()
    fresh = _state(b)
    FileManager.load(b, ref_only)
    sa, sb = _state(a), _state(b)
    assert_bitwise(sb[0], sa[0], "weights")
    assert_bitwise(sb[6], sa[6], "bitfield")
    for k in (2, 3, 4, 5):
        assert_bitwise(sb[k], fresh[k], f"buffer {k} left as it was")
    assert b.stat(5) == 0
    b.train_step()
    a.teardown()
    b.teardown()


def test_load_rejects_another_layout(tmp_path):
    a = _trainer()
    f = str(tmp_path / "run.turbo")
    FileManager.save(a, f)
    b = _trainer(n_mlp=4096)
    with pytest.raises(native.TurboError, match="parameters"):
        FileManager.load(b, f)
    a.teardown()
    b.teardown()


def test_resumed_dataset_run_draws_the_same_rays(tmp_path):
    """The dataset rays of a step are drawn from the seed and the step index, so a trainer that
    resumes from a snapshot takes the same rays as the one that kept going."""
    from tests.test_gpu_dataset import _trainer as dataset_trainer
    _, _, a = dataset_trainer()
    for _ in range(2):
        a.train_step()
    f = str(tmp_path / "ds.turbo")
    FileManager.save(a, f)
    _, _, b = dataset_trainer()
    FileManager.load(b, f)
    ma, mb = a.train_step(), b.train_step()
    assert (ma.step, ma.n_rays, ma.n_samples) == (mb.step, mb.n_rays, mb.n_samples) and ma.step == 3
    for k, dt in ((17, np.float32), (18, np.float32), (22, np.float32), (26, np.float32), (21, np.uint8)):
        assert_bitwise(b.buffer(k, dt).cpu().numpy(), a.buffer(k, dt).cpu().numpy(), f"ray buffer {k}")
    sa, sb = _state(a), _state(b)
    for k in STATE:
        assert_bitwise(sb[k], sa[k], f"buffer {k} after the resumed step")
    a.teardown()
    b.teardown()


def test_loaded_trainer_renders_the_same_frame(tmp_path):
    from tests.test_gpu_render import _camera
    from turbonerf_b200.renderer import CPURenderBuffer, Renderer, RenderPattern, RenderRequest
    a = _trainer()
    for _ in range(2):
        a.train_step()
    f = str(tmp_path / "run.turbo")
    FileManager.save(a, f)
    b = _trainer()
    FileManager.load(b, f)
    cam = _camera(64, 48, (0.3, 0.8, 4.0))
    imgs = []
    for tr in (a, b):
        out = CPURenderBuffer()
        Renderer(RenderPattern.LinearChunks).submit(RenderRequest(cam, [tr], out))
        imgs.append(out.get_rgba())
    assert imgs[0][..., 3].max() > 0
    assert_bitwise(imgs[1], imgs[0], "rendered frame")
    a.teardown()
    b.teardown()


def test_save_and_load_report_bad_paths_and_truncated_resume_blocks(tmp_path):
    a = _trainer()
    a.train_step()
    with pytest.raises(native.TurboError, match="cannot create"):
        FileManager.save(a, str(tmp_path / "missing-dir" / "run.turbo"))
    with pytest.raises(native.TurboError, match="cannot open"):
        FileManager.load(a, str(tmp_path / "missing.turbo"))
    f = str(tmp_path / "run.turbo")
    FileManager.save(a, f)
    cut = str(tmp_path / "cut.turbo")
    with open(f, "rb") as src, open(cut, "wb") as dst:
        dst.write(src.read()[:-4])  # the densities end one float short
    before = _state(a)
    with pytest.raises(native.TurboError, match="truncated"):
        FileManager.load(a, cut)
    after = _state(a)
    for k in STATE:
        assert_bitwise(after[k], before[k], f"buffer {k} untouched by a rejected load")
    a.teardown()
