"""The allocation-free scan entry point, tn_scan_offsets_noalloc, called through the C ABI.

It serves callers that cannot allocate device memory and hold no tn_ctx, such as a plugin
whose host application owns every device allocation, or a loop that must not pay the device
synchronisation of cudaMalloc. Its scratch is a fixed array inside the library, so it must
give exactly what tn_scan_offsets gives (and what the oracle's scan and batch cut give), call
after call, with no state leaking from one call into the next, up to its stated limit. With no
context to check, its device-side errors come back in a caller-owned error word.

This file is collected last (tests run in file order) so that a failure here leaves every
other test already run.
"""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

LIMIT = 1 << 21  # TN_SCAN_NOALLOC_MAX_COUNTS
FLAG_CAPACITY, FLAG_NO_RAYS, FLAG_NO_SAMPLES = 2, 4, 8


def _run_noalloc(counts_t, batch_size, error_word=True):
    import torch
    from turbonerf_b200 import native
    n = counts_t.numel()
    offsets = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(4, dtype=torch.int32, device="cuda")
    # the error word starts non-zero: the call must overwrite it
    err = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = native.lib().tn_scan_offsets_noalloc(stream, n, ctypes.c_void_p(counts_t.data_ptr()),
                                             ctypes.c_void_p(offsets.data_ptr()), batch_size,
                                             ctypes.c_void_p(info.data_ptr()),
                                             ctypes.c_void_p(err.data_ptr()) if error_word else None)
    native.check(st)
    torch.cuda.synchronize()
    return (offsets.cpu().numpy().view(np.uint32), info.cpu().numpy().view(np.uint32),
            int(err.cpu().numpy().view(np.uint32)[0]))


def test_noalloc_scan_matches_context_scan_twice_in_a_row():
    import torch
    from turbonerf_b200 import hotpath as hp
    rng = np.random.default_rng(42)
    ctx = hp.Context()
    # different calls back to back: none may see anything left by the one before. The last
    # one runs at exactly the limit, where the ticket and error words sit right after the
    # last block's prefix entry.
    for n, batch_size in ((300_001, 1 << 22), (70_000, 1 << 19), (LIMIT, 1 << 24), (LIMIT, 1 << 24)):
        counts = rng.integers(0, 60, n).astype(np.uint32)
        counts[rng.random(n) < 0.1] = 0
        c = torch.from_numpy(counts.view(np.int32)).cuda()
        off_ref, info_ref = hp.scan_offsets(ctx, c, batch_size)
        assert ctx.check() == 0
        off, info, err = _run_noalloc(c, batch_size)
        assert err == 0
        assert np.array_equal(off, off_ref.cpu().numpy().view(np.uint32))
        assert np.array_equal(info[:3], info_ref.cpu().numpy().view(np.uint32)[:3])
        # the oracle's restatement of the reference's scan and cut
        st, off_o, nr_o, ns_o = oracle.scan_cut(counts, batch_size)
        assert st == 0
        assert np.array_equal(off, off_o)
        assert (int(info[0]), int(info[1])) == (nr_o, ns_o)
        assert int(info[2]) == int(counts.sum())


def test_noalloc_scan_reports_errors_in_the_error_word():
    import torch
    # all counts zero: the cut keeps n - 1 rays and no sample (reference: "No samples")
    z = torch.zeros(5000, dtype=torch.int32, device="cuda")
    _, info, err = _run_noalloc(z, 1 << 18)
    assert err == FLAG_NO_SAMPLES and int(info[1]) == 0
    # one ray: the cut always drops the last ray below the batch size, so none is left
    one = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    _, info, err = _run_noalloc(one, 1 << 18)
    assert err == FLAG_NO_RAYS and int(info[0]) == 0
    # a count total past 2^32 at the limit: 2^21 counts of 4096 = 2^33
    big = torch.full((LIMIT,), 4096, dtype=torch.int32, device="cuda")
    _, info, err = _run_noalloc(big, 1 << 20)
    assert err & FLAG_CAPACITY
    assert int(info[2]) == 0xFFFFFFFF
    # a good call right after the failing ones reports no error
    ok = torch.full((10_000,), 3, dtype=torch.int32, device="cuda")
    off, info, err = _run_noalloc(ok, 1 << 18)
    assert err == 0 and int(info[0]) == 9_999 and int(info[1]) == 3 * 9_999
    # without an error word the call still succeeds
    off2, info2, _ = _run_noalloc(ok, 1 << 18, error_word=False)
    assert np.array_equal(off, off2) and np.array_equal(info, info2)


def test_noalloc_scan_allocates_no_device_memory():
    import torch
    n = LIMIT
    c = torch.randint(0, 50, (n,), dtype=torch.int32, device="cuda")
    offsets = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(4, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    from turbonerf_b200 import native
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (stream, n, ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(offsets.data_ptr()), 1 << 24,
            ctypes.c_void_p(info.data_ptr()), ctypes.c_void_p(err.data_ptr()))
    native.check(native.lib().tn_scan_offsets_noalloc(*args))  # warm: module and address set up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        native.check(native.lib().tn_scan_offsets_noalloc(*args))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert int(err.item()) == 0


def test_noalloc_scan_rejects_sizes_beyond_its_limit():
    import torch
    from turbonerf_b200 import native
    c = torch.zeros(LIMIT + 1, dtype=torch.int32, device="cuda")
    st = native.lib().tn_scan_offsets_noalloc(None, LIMIT + 1, ctypes.c_void_p(c.data_ptr()),
                                             ctypes.c_void_p(c.data_ptr()), 10, ctypes.c_void_p(c.data_ptr()),
                                             None)
    assert st == native.TN_E_CAPACITY
    assert "limit" in native.last_error()
