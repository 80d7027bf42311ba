"""CPU checks of .turbo files (tn_turbo_file_info, no GPU work): the reference's header layout
(NeRFFileData, src/services/file-manager.cuh:18-32) written here byte by byte, the resume block
after the bitfield, and the rejections of the reference's loader (file-manager.cuh:99-120):
a wrong project name, an unsupported version, a truncated body."""
import struct

import numpy as np
import pytest

from turbonerf_b200 import native
from turbonerf_b200.trainer import FileManager

N_COLOR, N_DENSITY, BITS = 24, 40, 64


def _header(project=b"TurboNeRF", dataset=b"/data/lego", version=0, aabb=4, n_color=N_COLOR, n_density=N_DENSITY):
    h = project.ljust(16, b"\0") + dataset.ljust(256, b"\0")
    h += struct.pack("<7I", version, n_color, n_density, 0, BITS, aabb, 1)
    assert len(h) == 300
    return h


def _body(n_params=N_COLOR + N_DENSITY):
    return np.arange(n_params, dtype=np.float32).tobytes() + bytes(range(BITS))


def _resume(version=1, step=7):
    r = b"TNRESUME" + struct.pack("<6I", version, 3, 4, N_DENSITY, N_COLOR, step) + struct.pack("<2Q", 100, 10)
    assert len(r) == 48
    return r


def _write(tmp_path, data, name="a.turbo"):
    p = tmp_path / name
    p.write_bytes(data)
    return str(p)


def test_reference_file_reads_without_resume_block(tmp_path):
    path = _write(tmp_path, _header() + _body())
    info = FileManager.info(path)
    assert info["n_params"] == N_COLOR + N_DENSITY and info["n_occ_grid_bits"] == BITS
    assert info["aabb_scale"] == 4 and info["dataset_path"] == "/data/lego"
    assert not info["has_resume"] and info["step_count"] == 0
    assert info["file_bytes"] == 300 + 4 * (N_COLOR + N_DENSITY) + BITS


def test_resume_block_is_found_after_the_bitfield(tmp_path):
    path = _write(tmp_path, _header() + _body() + _resume(step=7) + bytes(64))
    info = FileManager.info(path)
    assert info["has_resume"] and info["step_count"] == 7
    assert (info["n_levels"], info["resolution"]) == (3, 4)
    # bytes after the bitfield that are not a resume block are ignored, as the reference's loader does
    info = FileManager.info(_write(tmp_path, _header() + _body() + bytes(80), "b.turbo"))
    assert not info["has_resume"]


@pytest.mark.parametrize("data", [
    _header(project=b"NotTurbo") + _body(),
    _header(version=1) + _body(),
    _header() + _body()[:-1],
    _header()[:200],
    b"",
    _header() + _body() + _resume(version=2),
])
def test_bad_files_are_rejected(tmp_path, data):
    with pytest.raises(native.TurboError):
        FileManager.info(_write(tmp_path, data))


def test_missing_file_is_rejected(tmp_path):
    with pytest.raises(native.TurboError, match="cannot open"):
        FileManager.info(str(tmp_path / "missing.turbo"))
