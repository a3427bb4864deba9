"""Export pipelines on the device (fractura_b200.pipeline).

* render_mosaic, batch path (single-reference and one-pass rebasing tiles, both
  reference profiles, palette and histogram colouring): every tile of the stitched
  image equals render_frame_ssaa of the tile's view, byte for byte, and on_tile gets
  the same tiles in row-major order.
* render_mosaic, pipeline path (Pauldelbrot re-render passes, 2x SSAA, or
  use_batch=False), and a Burning Ship one-pass mosaic: the same equality.
* FramePipeline on a zoom sequence: every frame equals its own synchronous render and
  frames arrive in order.
"""
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import engine
from fractura_b200 import high_precision as hp
from fractura_b200.pipeline import FramePipeline, mosaic_views, render_mosaic
from helpers import load_golden

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")
CFG3 = next(x for x in PMETA if x["name"] == "cfg3")
SHIP = next(x for x in PMETA if x["name"] == "ship")

W, H = 64, 36


def _per_tile(views, max_iter, kw, cmap=None):
    out = {}
    for row, col, tcx, tcy, tw in views:
        hp.clear_reference_orbit_cache()
        out[(row, col)] = engine.render_frame_ssaa(W, H, max_iter, tcx, tcy, tw, cmap, **kw).copy()
    return out


def _check(img, tiles, views):
    for row, col, *_ in views:
        got = img[row * H:(row + 1) * H, col * W:(col + 1) * W]
        assert np.array_equal(got, tiles[(row, col)]), (row, col, int((got != tiles[(row, col)]).sum()))


@pytest.mark.parametrize("glitch_mode", ["Off (Single-Ref)", "One-Pass Rebasing"])
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
@pytest.mark.parametrize("scheme", [0, 11])
def test_mosaic_batch_path_equals_per_tile_frames(glitch_mode, arith, scheme):
    m = CFG3
    n, max_iter = 3, 20000
    width = Decimal(m["width"]) * 40
    kw = dict(color_scheme_id=scheme, precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
              glitch_mode=glitch_mode, arith=arith)
    got = []
    hp.clear_reference_orbit_cache()
    img = render_mosaic(n, W, H, max_iter, Decimal(m["cx"]), Decimal(m["cy"]), width,
                        on_tile=lambda r, c, t: got.append((r, c, t.copy())), **kw)
    views = mosaic_views(Decimal(m["cx"]), Decimal(m["cy"]), width, n, W, H)
    assert img.shape == (n * H, n * W, 3)
    tiles = _per_tile(views, max_iter, kw)
    _check(img, tiles, views)
    assert [(r, c) for r, c, _ in got] == [(r, c) for r, c, *_ in views]
    for r, c, t in got:
        assert np.array_equal(t, tiles[(r, c)])
    assert img.any()


@pytest.mark.parametrize("case", ["pauldelbrot", "ssaa2", "no_batch", "ship_one_pass", "fp32_batch",
                                  "ship_fp32_one_pass"])
def test_mosaic_pipeline_path_equals_per_tile_frames(case):
    m = SHIP if case.startswith("ship") else CFG3
    n, max_iter = 2, 5000
    width = Decimal(m["width"]) * 20
    kw = dict(precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
              glitch_mode="Off (Single-Ref)", fractal_type=m["fractal_type"])
    if case == "pauldelbrot":
        kw["glitch_mode"] = "Pauldelbrot"
    elif case == "ssaa2":
        kw["ssaa_factor"] = 2
    elif case == "ship_one_pass":
        kw["glitch_mode"] = "One-Pass Rebasing"
    elif case == "fp32_batch":
        kw["delta_form"] = "fp32"
    elif case == "ship_fp32_one_pass":
        kw["glitch_mode"], kw["delta_form"] = "One-Pass Rebasing", "fp32"
    hp.clear_reference_orbit_cache()
    img = render_mosaic(n, W, H, max_iter, Decimal(m["cx"]), Decimal(m["cy"]), width,
                        use_batch=(case != "no_batch"), **kw)
    views = mosaic_views(Decimal(m["cx"]), Decimal(m["cy"]), width, n, W, H)
    _check(img, _per_tile(views, max_iter, kw), views)


def test_frame_pipeline_zoom_sequence():
    m = CFG3
    frames = []
    for q in range(5):
        w = Decimal(m["width"]) * Decimal(2) ** (8 - 2 * q)
        frames.append(dict(max_iter=20000, center_x_dec=Decimal(m["cx"]), center_y_dec=Decimal(m["cy"]),
                           plot_width_dec=w, precision_mode="1e-300 (Perturbation)", bbsa_order=32,
                           bbsa_tol=1e-6, glitch_mode="One-Pass Rebasing", color_scheme_id=11 if q % 2 else 0,
                           arith="ref_cuda"))
    seen = []
    hp.clear_reference_orbit_cache()
    FramePipeline(W, H).render(frames, lambda i, rgb: seen.append((i, rgb.copy())))
    assert [i for i, _ in seen] == list(range(len(frames)))
    for i, rgb in seen:
        kw = dict(frames[i])
        hp.clear_reference_orbit_cache()
        want = engine.render_frame_ssaa(W, H, kw.pop("max_iter"), kw.pop("center_x_dec"), kw.pop("center_y_dec"),
                                        kw.pop("plot_width_dec"), None, **kw)
        assert np.array_equal(rgb, want), i
