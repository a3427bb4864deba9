"""A frame split by row bands on the device (fractura_b200.sharded.DeviceBackend,
ap_render_rows, ap_histogram, ap_cdf_from_histogram).

* Bands rendered one after another on this GPU, their histograms summed and turned into
  one CDF, then coloured, equal the unsplit frame of render_frame_ssaa bit for bit
  (iteration map and RGB), for several splits, with histogram and closed-form colouring.
* render_split over a one-rank NCCL group (orbit broadcast, histogram all-reduce and band
  all-gather on the device) gives the same frame.
"""
import ctypes as C
import os
import socket
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import _lib, engine, sharded
from fractura_b200 import high_precision as hp
from helpers import load_golden

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")
CFG3 = next(x for x in PMETA if x["name"] == "cfg3")


def view(scheme, W=192, H=108, width="1e-159", arith="fast"):
    return dict(W=W, H=H, max_iter=20000, cx=CFG3["cx"], cy=CFG3["cy"], width=width, scheme=scheme,
                num_bins=65536 if scheme == 11 else 2048, fractal_type=0, bbsa_order=32, bbsa_tol=1e-6,
                glitch_mode="One-Pass Rebasing", arith=arith, bla_form="accurate")


def whole_frame(v):
    import torch
    hp.clear_reference_orbit_cache()
    it = torch.zeros((v["H"], v["W"]), dtype=torch.float32, device="cuda")
    rgb = engine.render_frame_ssaa(v["W"], v["H"], v["max_iter"], Decimal(v["cx"]), Decimal(v["cy"]),
                                   Decimal(v["width"]), None, color_scheme_id=v["scheme"],
                                   precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                                   glitch_mode=v["glitch_mode"], arith=v["arith"], bla_form="accurate",
                                   d_iter_buf=it)
    return it.cpu().numpy(), (rgb.cpu().numpy() if hasattr(rgb, "cpu") else np.asarray(rgb))


@pytest.mark.parametrize("scheme", [11, 5])
@pytest.mark.parametrize("bands", [[(0, 108)], [(0, 40), (40, 41), (41, 108)], [(0, 17), (17, 64), (64, 108)]])
@pytest.mark.parametrize("arith", ["fast", "ref_cuda"])
def test_bands_assemble_the_whole_frame(scheme, bands, arith):
    import torch
    v = view(scheme, arith=arith)
    it_want, rgb_want = whole_frame(v)
    be = sharded.DeviceBackend()
    orbit = be.find_reference(v)
    its = [be.render_band(v, orbit, r0, r1).clone() for r0, r1 in bands]
    cdf = None
    if scheme == 11:
        hist = sum(be.band_histogram(v, it).to(torch.int64) for it in its).to(torch.int32)
        cdf = be.cdf_from_histogram(v, hist)
    rgb = torch.cat([be.colour_band(v, it, cdf) for it in its], dim=0).cpu().numpy()
    it = torch.cat(its, dim=0).cpu().numpy()
    assert np.array_equal(it.view(np.uint32), it_want.view(np.uint32))
    assert np.array_equal(rgb, rgb_want)


def test_render_rows_rejects_bad_bands_and_other_passes():
    import torch
    from fractura_b200 import abi
    L = _lib.load()
    it = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    orbit = torch.zeros(5, dtype=torch.float64, device="cuda")
    b = abi.ApFrameBuffers()
    b.iter_map = C.c_void_p(it.data_ptr())
    b.ref_re = b.ref_im = C.c_void_p(orbit.data_ptr())
    p = abi.new_params(width=8, height=8, max_iter=10, tier=abi.AP_TIER_PERTURB, ref_len=4,
                       flags=abi.AP_FLAG_NO_RGB)
    assert L.ap_render_rows(C.byref(p), C.byref(b), 4, 5, None) == abi.AP_E_INVALID   # rows past the frame
    assert L.ap_render_rows(C.byref(p), C.byref(b), -1, 2, None) == abi.AP_E_INVALID
    assert L.ap_render_rows(C.byref(p), C.byref(b), 0, 8, None) == abi.AP_E_UNSUPPORTED  # no packed orbit
    p.tier = abi.AP_TIER_FP64
    assert L.ap_render_rows(C.byref(p), C.byref(b), 0, 8, None) == abi.AP_E_UNSUPPORTED


def test_render_split_one_rank_nccl_group():
    import torch
    import torch.distributed as dist
    v = view(11)
    it_want, rgb_want = whole_frame(v)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    import datetime
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        for balance in (None, "probe"):
            rgb, it = sharded.render_split(v, sharded.DeviceBackend(), balance=balance)
            torch.cuda.synchronize()
            assert np.array_equal(it.cpu().numpy().view(np.uint32), it_want.view(np.uint32))
            assert np.array_equal(rgb.cpu().numpy(), rgb_want)
    finally:
        dist.destroy_process_group()


def test_device_probe_costs():
    """The device probe behind probe balancing: row weights of a view (one per frame row,
    every probe pixel costing at least one step) and per-tile costs of a batch."""
    from fractura_b200 import batch as fb
    v = view(0)
    be = sharded.DeviceBackend()
    w = sharded.probe_row_weights(v, be.probe_map, 64, 36)
    assert w.shape == (v["H"],) and np.all(w >= 64)
    bands = sharded.band_bounds(v["H"], 3, w)
    assert bands[0][0] == 0 and bands[-1][1] == v["H"]
    tiles = [fb.Tile(cx=Decimal(v["cx"]), cy=Decimal(v["cy"]), width=Decimal(v["width"]) * f, W=64, H=48,
                     max_iter=v["max_iter"]) for f in (1, 4)]
    cost = sharded.probe_tile_costs(tiles, be.probe_tile, 16, 16)
    assert len(cost) == 2 and all(c >= 64 * 48 for c in cost)
