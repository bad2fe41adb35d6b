"""GPU test of bm_fft_noalloc, the allocation-free FFT entry point.

That entry point exists for callers that cannot allocate device memory when they need a
transform (a host that has already handed the GPU's memory to other work, or a solver in the
middle of an asynchronous step where a cudaMalloc/cudaFree would synchronise the device and
stall it). They pass their own device buffers; the only scratch, the twiddle table, lives in
a fixed device array inside the library (lines of at most 4096 points).

The test calls it through the C ABI twice in a row (different lengths and directions, so the
shared table is rewritten between calls) and compares with the allocating entry point
bm_debug_fft within the FP64 FFT tolerance used elsewhere (1e-13 relative to max |X|). This
file is named to be collected last, and it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_fft_noalloc_matches_allocating_entry_point(bm):
    import torch
    L = bm.lib()
    rng = np.random.default_rng(2024)
    # two calls in a row with different lengths and directions, then the longest line the scratch
    # table holds (4096, whose transform needs more than 48 KB of shared memory) and a 3 * 2^k one
    for n, howmany, inverse in [(1024, 7, 0), (384, 5, 1), (4096, 3, 0), (3072, 2, 1)]:
        x = rng.normal(size=(howmany, n)) + 1j * rng.normal(size=(howmany, n))
        ref = bm.debug_fft(x, precision=bm.FP64, inverse=bool(inverse))
        xin = torch.from_numpy(np.ascontiguousarray(x).view(np.float64).copy()).cuda()
        out = torch.empty_like(xin)
        torch.cuda.synchronize()
        rc = L.bm_fft_noalloc(0, n, howmany, inverse, ctypes.c_void_p(xin.data_ptr()),
                              ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.bm_last_error().decode()
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex128).reshape(howmany, n)
        assert _relmax(got, ref) < 1e-13
        # the input buffer is left untouched
        assert np.array_equal(xin.cpu().numpy().view(np.complex128).reshape(howmany, n), x)


def test_fft_noalloc_in_place_and_device_kept(bm):
    import torch
    L = bm.lib()
    rng = np.random.default_rng(77)
    for n, howmany, inverse in [(4096, 2, 1), (512, 9, 0)]:
        x = rng.normal(size=(howmany, n)) + 1j * rng.normal(size=(howmany, n))
        ref = bm.debug_fft(x, precision=bm.FP64, inverse=bool(inverse))
        buf = torch.from_numpy(np.ascontiguousarray(x).view(np.float64).copy()).cuda()
        torch.cuda.synchronize()
        rc = L.bm_fft_noalloc(0, n, howmany, inverse, ctypes.c_void_p(buf.data_ptr()),
                              ctypes.c_void_p(buf.data_ptr()), None)
        assert rc == 0, L.bm_last_error().decode()
        torch.cuda.synchronize()
        got = buf.cpu().numpy().view(np.complex128).reshape(howmany, n)
        assert _relmax(got, ref) < 1e-13
        assert torch.cuda.current_device() == 0


def test_fft_noalloc_rejects_lines_beyond_scratch(bm):
    import torch
    L = bm.lib()
    buf = torch.zeros(2 * 8192, dtype=torch.float64, device="cuda")
    rc = L.bm_fft_noalloc(0, 8192, 1, 0, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), None)
    assert rc != 0
    assert "4096" in L.bm_last_error().decode()
