"""The CUDA library against the committed golden fixtures (tests/golden/*.npz, written by the
oracle): march outputs and occupancy update bit-exact, losses and gradients within the
parity tolerances. Runs without the oracle library."""
import os

import numpy as np
import pytest

from tests.helpers import RTOL_GRAD, assert_bitwise, assert_close, assert_norm_close, dev, host, i32, pick_branches

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return dict(np.load(os.path.join(HERE, name + ".npz")))


def test_march_matches_golden():
    from turbonerf_b200 import hotpath as hp
    fx = _load("march_small")
    n = fx["ori"].size // 3
    g = hp.GridSpec(int(fx["n_levels"]), int(fx["res"]), float(fx["base"]))
    m = hp.MarchSpec(float(fx["cone"]), float(fx["dt_min"]), float(fx["dt_max"]), 0)
    bbox = tuple(float(v) for v in fx["bbox"])
    batch = int(fx["batch"])
    ctx = hp.Context()
    alive = dev(fx["alive_in"].copy())
    ori, dr, t, tmax = dev(fx["ori"]), dev(fx["dir"]), dev(fx["t"]), dev(fx["t_max"])
    bits = dev(fx["bitfield"])
    n_steps, info = hp.march_count(ctx, g, bits, bbox, m, n, n, ori, dr, t, tmax, alive, batch)
    offsets, smp = hp.march_emit(ctx, g, bits, bbox, m, 0.25, n, n, batch + 1, info, ori, dr, t, alive, n_steps)
    ctx.check()
    info_h = host(info).view(np.uint32)
    ns = int(fx["n_samples"])
    assert (int(info_h[0]), int(info_h[1])) == (int(fx["n_rays"]), ns)
    assert_bitwise(host(n_steps).view(np.uint32), fx["n_steps"], "n_steps")
    assert_bitwise(host(alive), fx["alive"], "alive")
    assert_bitwise(host(offsets).view(np.uint32), fx["offsets"], "offsets")
    for k in ("t", "dt", "m_norm", "dt_norm"):
        assert_bitwise(host(smp[k])[:ns], fx["s_" + k], k)
    assert_bitwise(host(smp["pos"]).reshape(3, batch + 1)[:, :ns].ravel(), fx["s_pos"].ravel(), "pos")


def test_losses_match_golden():
    from turbonerf_b200 import hotpath as hp
    fx = _load("loss_small")
    n, ss = fx["counts"].size, fx["sigma"].size
    ctx = hp.Context()
    rb = hp.ray_batch(i32(fx["counts"]), i32(fx["offsets"]), n, n, ss)
    out = hp.recon_loss_fwd_bwd(ctx, rb, dev(fx["sigma"]), dev(fx["rgb"]), dev(fx["dt"]), dev(fx["target"]),
                                dev(fx["bg"]), inv_nrays=1.0 / n)
    # every ray against the fixture's branch closest to it (rays whose cut rounding decides carry
    # one branch per legitimate cut)
    gpu = {k: host(out[k]) for k in ("ray_rgba", "loss", "dL_ddensity", "dL_drgb")}
    branches = [{k: fx["br_" + k][b] for k in gpu} for b in range(fx["br_ray_rgba"].shape[0])]
    ref, _ = pick_branches(gpu, branches, fx["counts"], fx["offsets"], ray_keys=("ray_rgba", "loss"),
                           sample_keys=("dL_ddensity", "dL_drgb"), ray_stride=n, sample_stride=ss)
    for c in range(4):
        assert_close(gpu["ray_rgba"][c * n:(c + 1) * n], ref["ray_rgba"][c * n:(c + 1) * n], 1e-5, "rgba")
    assert_norm_close(gpu["dL_ddensity"], ref["dL_ddensity"], RTOL_GRAD, "dL/ddensity")
    assert_norm_close(gpu["dL_drgb"], ref["dL_drgb"], RTOL_GRAD, "dL/drgb")
    d = hp.distortion_fwd_bwd(ctx, rb, dev(fx["sigma"]), dev(fx["m_norm"]), dev(fx["dt_norm"]), 1e-3)
    assert_norm_close(host(d["ray_loss"]), fx["dist_loss"], 1e-4, "distortion loss")
    assert_norm_close(host(d["dL_ddensity"]), fx["dist_dd"], RTOL_GRAD, "distortion gradient")


def test_occupancy_matches_golden():
    from turbonerf_b200 import hotpath as hp
    fx = _load("occupancy_small")
    L, res = fx["density"].shape[0], 16
    ctx = hp.Context()
    d, b = dev(fx["density"].ravel().copy()), dev(fx["bitfield"].copy())
    nocc = hp.occupancy_update(ctx, hp.GridSpec(L, res, 1.0), d, b, dev(fx["levels"]), i32(fx["cells"]),
                               dev(fx["values"]), dev(fx["rsel"]))
    assert_bitwise(host(d), fx["out_density"].ravel(), "density")
    assert_bitwise(host(b), fx["out_bitfield"], "bitfield")
    assert int(host(nocc)[0]) == int(fx["n_occupied"])


def test_render_matches_golden():
    """Renderer.submit on the fixture's scene (2 cascades of 32^3, base 2, its blob field as the
    network) against the oracle's image, within the composite tolerance."""
    from tests.golden.make_golden import render_camera
    from turbonerf_b200.renderer import Camera, CPURenderBuffer, Renderer, RenderRequest
    from turbonerf_b200.trainer import BoundingBox, SyntheticNeRF, Trainer
    fx = _load("render_small")
    b = BoundingBox(4.0)
    nerf = SyntheticNeRF(b, int(fx["n_levels"]), fx["blobs"], fx["waves"], None, fx["bitfield"],
                         int(fx["res"]), float(fx["base"]))
    tr = Trainer(nerf, n_rays_per_step=4096, n_grid_params=16 * (1 << 15) * 2)
    tr.setup_data(batch_size=1 << 16)
    c = render_camera()
    cam = Camera((c["width"], c["height"]), c["near"], c["far"], c["focal"], c["principal"], c["shift"],
                 fx["transform"])
    buf = CPURenderBuffer()
    Renderer().submit(RenderRequest(cam, [tr], buf))
    img = buf.get_rgba()
    ref = fx["rgba"]
    for ch in range(4):
        assert_close(img[..., ch].ravel(), ref[..., ch].ravel(), 1e-5, f"rendered channel {ch}")
    assert np.all(img[ref[..., 3] == 0] == 0)
    tr.teardown()
