"""Histogram -> CDF on the device (ap_histogram_cdf: histogram_kernel and the CDF scan)
against the oracle's apo_histogram_cdf (the float64 scan of
math_core/cuda_kernels.py:1922-2013): histogram and CDF bit for bit, for bin counts on
both sides of the chunked scan's limit (65536) and of its 4096-bin chunks, with and
without escaped pixels, on iteration maps of several shapes."""
import ctypes as C

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib

pytestmark = pytest.mark.gpu


def device_cdf(it, max_iter, num_bins):
    import torch
    H, W = it.shape
    d_it = torch.from_numpy(it).cuda()
    hist = torch.full((num_bins,), 7, dtype=torch.int32, device="cuda")   # stale contents are cleared
    cdf = torch.zeros(num_bins, dtype=torch.float32, device="cuda")
    L = _lib.load()
    _lib.check(L.ap_histogram_cdf(C.c_void_p(d_it.data_ptr()), W, H, max_iter, num_bins,
                                  C.c_void_p(hist.data_ptr()), C.c_void_p(cdf.data_ptr()), None),
               "ap_histogram_cdf")
    return hist.cpu().numpy(), cdf.cpu().numpy()


@pytest.mark.parametrize("num_bins", [2, 3, 1000, 4095, 4096, 4097, 65535, 65536, 65537, 200003])
@pytest.mark.parametrize("shape", [(360, 640), (37, 53)])
def test_histogram_cdf_matches_oracle(num_bins, shape):
    H, W = shape
    rng = np.random.default_rng(num_bins * 31 + H)
    max_iter = 1000
    # escaped values spread over [0, max_iter), a third interior (-1), some exactly max_iter
    it = (rng.random((H, W)) * max_iter).astype(np.float32)
    it[rng.random((H, W)) < 0.33] = -1.0
    it[rng.random((H, W)) < 0.01] = float(max_iter)
    hist, cdf = device_cdf(it, max_iter, num_bins)
    fr = oracle.Frame(W, H)
    fr.iter_map[...] = it
    oracle.histogram_cdf(fr, max_iter, num_bins)
    assert np.array_equal(hist, fr.hist)
    assert np.array_equal(cdf.view(np.uint32), fr.cdf.view(np.uint32))


@pytest.mark.parametrize("num_bins", [4096, 65536, 70000])
def test_histogram_cdf_of_an_interior_frame(num_bins):
    """No pixel escapes: the CDF is the bin ramp q / (num_bins - 1)."""
    it = np.full((54, 96), -1.0, np.float32)
    hist, cdf = device_cdf(it, 500, num_bins)
    assert not hist.any()
    want = (np.arange(num_bins, dtype=np.float64) / (num_bins - 1)).astype(np.float32)
    assert np.array_equal(cdf.view(np.uint32), want.view(np.uint32))
