"""The allocation-free scan entry point, tn_scan_offsets_noalloc, called through the C ABI.

It serves callers that cannot allocate device memory and hold no tn_ctx, such as a plugin
whose host application owns every device allocation. Its scratch is a fixed array inside the
library, so it must give exactly what tn_scan_offsets gives, call after call, with no state
leaking from one call into the next. This file is collected last (tests run in file order)
so that a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_noalloc(counts_t, batch_size):
    import torch
    from turbonerf_b200 import native
    n = counts_t.numel()
    offsets = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(4, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = native.lib().tn_scan_offsets_noalloc(stream, n, ctypes.c_void_p(counts_t.data_ptr()),
                                             ctypes.c_void_p(offsets.data_ptr()), batch_size,
                                             ctypes.c_void_p(info.data_ptr()))
    native.check(st)
    torch.cuda.synchronize()
    return offsets.cpu().numpy().view(np.uint32), info.cpu().numpy().view(np.uint32)


def test_noalloc_scan_matches_context_scan_twice_in_a_row():
    import torch
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(42)
    ctx = hp.Context()
    # two different calls back to back: the second must not see anything left by the first
    for n, batch_size in ((300_001, 1 << 22), (70_000, 1 << 19)):
        counts = rng.integers(0, 60, n).astype(np.uint32)
        counts[rng.random(n) < 0.1] = 0
        c = torch.from_numpy(counts.view(np.int32)).cuda()
        off_ref, info_ref = hp.scan_offsets(ctx, c, batch_size)
        ctx.check()
        off, info = _run_noalloc(c, batch_size)
        assert np.array_equal(off, off_ref.cpu().numpy().view(np.uint32))
        assert np.array_equal(info[:3], info_ref.cpu().numpy().view(np.uint32)[:3])


def test_noalloc_scan_rejects_sizes_beyond_its_limit():
    import torch
    from turbonerf_b200 import native
    limit = 1 << 21
    c = torch.zeros(limit + 1, dtype=torch.int32, device="cuda")
    st = native.lib().tn_scan_offsets_noalloc(None, limit + 1, ctypes.c_void_p(c.data_ptr()),
                                             ctypes.c_void_p(c.data_ptr()), 10, ctypes.c_void_p(c.data_ptr()))
    assert st == native.TN_E_CAPACITY
    assert "limit" in native.last_error()
