"""CPU checks of the C ABI: the library loads, exports every entry point that
include/turbo_hot.h declares, the ctypes table matches the header, and argument checks
return status codes (no GPU work is launched)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    hdr = open(os.path.join(ROOT, "include", "turbo_hot.h")).read()
    return re.findall(r"^\s*(?:int|void|const char\*)\s+(tn_\w+)\(", hdr, re.M)


def test_library_exports_every_declared_symbol():
    from turbonerf_b200 import native
    L = native.lib()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(native.SIGNATURES), set(names) ^ set(native.SIGNATURES)


def test_struct_layouts_match_header():
    from turbonerf_b200 import native
    assert ctypes.sizeof(native.Bbox) == 24
    assert ctypes.sizeof(native.GridDesc) == 16
    assert ctypes.sizeof(native.MarchDesc) == 20
    assert ctypes.sizeof(native.RayBatchDesc) == 40
    assert native.lib().tn_version() == 1


def test_argument_errors_return_status_without_gpu():
    """Bad descriptors are rejected on the host with a TN_E_* status and a message."""
    from turbonerf_b200 import native
    L = native.lib()
    g = native.GridDesc(9, 128, 1.0, 0)  # more than 8 cascades
    st = L.tn_occupancy_sample_points(None, ctypes.byref(g), 0, None, None, None, 0, 1.0, None, 0)
    assert st == native.TN_E_LEVELS
    assert "n_levels" in native.last_error()
    g = native.GridDesc(2, 100, 1.0, 0)  # resolution not a power of two
    st = L.tn_occupancy_sample_points(None, ctypes.byref(g), 0, None, None, None, 0, 1.0, None, 0)
    assert st == native.TN_E_INVALID
    st = L.tn_adam_step(None, 10, 8, 4, 1.0, 1e-2, 0.9, 0.99, 1e-15, 1e-6, None, None, None, None, None, None)
    assert st == native.TN_E_NULL
    with pytest.raises(native.TurboError):
        native.check(native.TN_E_INVALID)
    with pytest.raises(native.NoRaysError):
        native.check(native.TN_E_NO_RAYS)


def test_tuning_defaults_and_validation_without_gpu():
    """The launch-shape table: defaults, and every field outside its listed values rejected on
    the host (tn_tuning_validate; tn_ctx_set_tuning runs the same check)."""
    from turbonerf_b200 import native
    L = native.lib()
    t = native.Tuning()
    L.tn_tuning_default(ctypes.byref(t))
    assert t.as_dict() == {"count_rays_per_block": 64, "emit_warps_per_block": 8, "emit_rays_per_warp": 1,
                           "loss_rays_per_block": 4, "compact_tile": 128, "multi_chunk_rays": 64, "side_sms": 0}
    assert L.tn_tuning_validate(ctypes.byref(t)) == native.TN_OK
    allowed = {"count_rays_per_block": [32, 64, 128, 256], "emit_warps_per_block": [1, 2, 4, 8, 16],
               "emit_rays_per_warp": [1, 2, 4], "loss_rays_per_block": [2, 4, 8],
               "compact_tile": [128, 256, 512, 1024, 2048], "multi_chunk_rays": [32, 64, 128, 256],
               "side_sms": list(range(1024))}
    for field, values in allowed.items():
        for v in range(0, 4097):
            u = native.Tuning(**t.as_dict())
            setattr(u, field, v)
            st = L.tn_tuning_validate(ctypes.byref(u))
            assert (st == native.TN_OK) == (v in values), (field, v, st)
            if st != native.TN_OK:
                assert st == native.TN_E_INVALID and field in L.tn_last_error().decode()
    assert L.tn_tuning_validate(None) == native.TN_E_NULL
