"""ap_histogram_cdf_noalloc: the histogram -> CDF step for callers that cannot allocate.

Some callers of this library run where they may not call cudaMalloc (a host
callback, a render loop that must stay off the allocator, a plugin whose host
owns all device memory), so they cannot hand ap_histogram_cdf its scratch
histogram.  The no-allocation entry point uses an array built into the library
instead; this test checks, through the C ABI, that two calls in a row give the
same CDF as the allocating entry point (bit-exact, the tolerance of the other
colouring tests) and that oversized requests are refused.  It sits in a file of
its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from fractura_b200 import _lib, abi

pytestmark = pytest.mark.gpu


def _iter_maps():
    rng = np.random.default_rng(7)
    H, W, max_iter = 270, 480, 5000
    a = rng.gamma(2.0, 300.0, size=(H, W)).astype(np.float32)
    a[rng.random((H, W)) < 0.1] = -1.0          # interior pixels are not counted
    b = (a * 0.5 + 7.25).astype(np.float32)
    b[a < 0] = -1.0
    return [(a, max_iter), (b, max_iter)]


def test_noalloc_cdf_matches_allocating_entry_point():
    import torch
    L = _lib.load()
    num_bins = abi_bins = 65536
    hist = torch.empty(num_bins, dtype=torch.int32, device="cuda")
    for host_map, max_iter in _iter_maps():          # two calls in a row
        H, W = host_map.shape
        it = torch.from_numpy(host_map).cuda()
        want = torch.empty(abi_bins, dtype=torch.float32, device="cuda")
        got = torch.full((abi_bins,), -7.0, dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream()
        sh = C.c_void_p(st.cuda_stream)
        _lib.check(L.ap_histogram_cdf(C.c_void_p(it.data_ptr()), W, H, max_iter, num_bins,
                                      C.c_void_p(hist.data_ptr()), C.c_void_p(want.data_ptr()), sh),
                   "ap_histogram_cdf")
        _lib.check(L.ap_histogram_cdf_noalloc(C.c_void_p(it.data_ptr()), W, H, max_iter, num_bins,
                                              C.c_void_p(got.data_ptr()), sh),
                   "ap_histogram_cdf_noalloc")
        st.synchronize()
        assert torch.equal(got, want)
        assert float(want[-1]) == 1.0


def test_noalloc_rejects_oversized_histograms():
    L = _lib.load()
    rc = L.ap_histogram_cdf_noalloc(None, 4, 4, 100, 65537, None, None)
    assert rc == abi.AP_E_INVALID
    assert b"65536" in L.ap_last_error()
