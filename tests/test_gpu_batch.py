"""Batched tiles in one persistent kernel (fractura_b200.batch, ap_render_batch).

Every tile of a mixed batch (formulas, sizes, depths) equals the per-tile
coarse render of the engine, value for value; a captured CUDA graph replays
to the same values; every launch shape the autotuner may pick (patch shape,
blocks per SM, register budget, quantum) gives the same values, and so does a
quantum of one step, where every pixel is compacted after every step.
"""
import dataclasses
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import batch as fb
from fractura_b200 import engine
from fractura_b200 import high_precision as hp
from helpers import load_golden

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")


def _tiles(rebase=False):
    m = {x["name"]: x for x in PMETA}
    out = []
    sizes = [(160, 90), (37, 23), (64, 64), (200, 50), (16, 16), (96, 54)]
    for q, name in enumerate(["cfg3", "ship", "julia", "multibrot3", "multibrot4", "ship_julia"]):
        c = m[name]
        W, H = sizes[q]
        out.append(fb.Tile(cx=Decimal(c["cx"]), cy=Decimal(c["cy"]), width=Decimal(c["width"]), W=W, H=H,
                           max_iter=min(c["max_iter"], 20000), fractal_type=c["fractal_type"],
                           julia_cx=c["julia_cx"], julia_cy=c["julia_cy"], gen_n=c["gen_n"],
                           gen_kr=c["gen_kr"], gen_ki=c["gen_ki"], bla=(q % 2 == 0),
                           strict_glitch=False, rebase=rebase and c["fractal_type"] in (0, 1, 4)))
    return out


def _engine_tile(t, arith, bla_form):
    import torch
    kmap = torch.empty((t.H, t.W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((t.H, t.W), dtype=torch.float64, device="cuda")
    it = np.zeros((t.H, t.W), np.float32)
    engine.render_frame_ssaa(t.W, t.H, t.max_iter, t.cx, t.cy, t.width, None, color_scheme_id=0,
                             precision_mode="1e-300 (Perturbation)", fractal_type=t.fractal_type,
                             julia_cx=t.julia_cx, julia_cy=t.julia_cy, bbsa_tol=1e-6,
                             bbsa_order=32 if t.bla else 0,
                             glitch_mode="One-Pass Rebasing" if t.rebase else "Off (Single-Ref)",
                             gen_n=t.gen_n, gen_kr=t.gen_kr, gen_ki=t.gen_ki, h_iter_buf=it,
                             arith=arith, bla_form=bla_form, delta_form=t.delta_form, _extra_out=(kmap, s64))
    return it, kmap.cpu().numpy()


@pytest.mark.parametrize("arith,rebase", [("ref_cpu", False), ("ref_cuda", False), ("ref_cpu", True),
                                          ("ref_cuda", True), ("fast", True)])
@pytest.mark.parametrize("bla_form", ["reference", "accurate"])
def test_batch_matches_per_tile_frames(arith, bla_form, rebase):
    """Single-reference tiles, and one-pass rebasing tiles (Mandelbrot, Burning Ship,
    Multibrot) mixed with single-reference Julia tiles; in a 'fast' batch the one-pass
    tiles take the fused step and the Julia tiles the CUDA-source profile."""
    import torch
    hp.clear_reference_orbit_cache()
    tiles = _tiles(rebase)
    s = torch.cuda.Stream()
    b = fb.prepare_batch(tiles, arith=arith, bla_form=bla_form, stream=s)
    b.render(fb.BatchConfig())
    torch.cuda.synchronize()
    for t, out in zip(tiles, b.tiles_out):
        it, k = _engine_tile(t, "ref_cuda" if (arith == "fast" and not t.rebase) else arith, bla_form)
        got = out["iter"].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), it.view(np.uint32)), int((got != it).sum())
        assert np.array_equal(out["kmap"].cpu().numpy(), k)
    assert b.nominal_iterations() > 0


@pytest.mark.parametrize("rebase", [False, True])
def test_graph_replay_and_every_launch_shape_agree(rebase):
    import torch
    hp.clear_reference_orbit_cache()
    s = torch.cuda.Stream()
    b = fb.prepare_batch(_tiles(rebase), arith="fast" if rebase else "ref_cpu", stream=s)
    b.render(fb.BatchConfig())
    torch.cuda.synchronize()
    ref = [o["iter"].clone() for o in b.tiles_out]
    for cfg in fb.CANDIDATES:
        for o in b.tiles_out:
            o["iter"].fill_(-7.0)
        b.render(cfg)
        torch.cuda.synchronize()
        for o, r in zip(b.tiles_out, ref):
            assert torch.equal(o["iter"], r), cfg
    for cfg in (fb.BatchConfig(quantum=1), fb.BatchConfig(quantum=7, blocks_per_sm=1)):
        for o in b.tiles_out:
            o["iter"].fill_(-7.0)
        b.render(cfg)
        torch.cuda.synchronize()
        for o, r in zip(b.tiles_out, ref):
            assert torch.equal(o["iter"], r), cfg
    g = b.capture(fb.CANDIDATES[1])
    for _ in range(2):
        for o in b.tiles_out:
            o["iter"].fill_(-7.0)
        g.replay()
        torch.cuda.synchronize()
        for o, r in zip(b.tiles_out, ref):
            assert torch.equal(o["iter"], r)
    if not rebase:
        cfg = fb.tune(b)
        assert cfg in fb.CANDIDATES
        assert len(fb.tuned_timings(b)) == len(fb.CANDIDATES)
        assert fb.tune(b) is cfg   # cached


@pytest.mark.parametrize("arith,rebase", [("ref_cpu", False), ("fast", True)])
def test_streamed_batch_equals_the_whole_batch(arith, rebase):
    """render_streamed (launches while references still arrive, several parts) gives every
    tile the values of prepare_batch + render of the whole batch."""
    import torch
    tiles = _tiles(rebase)
    s = torch.cuda.Stream()
    hp.clear_reference_orbit_cache()
    b = fb.prepare_batch(tiles, arith=arith, bla_form="accurate", stream=s)
    b.render(fb.BatchConfig())
    torch.cuda.synchronize()
    hp.clear_reference_orbit_cache()
    sb = fb.render_streamed(tiles, arith=arith, bla_form="accurate", stream=s, workers=2)
    s.synchronize()
    assert len(sb.parts) >= 1 and sum(p.n for p in sb.parts) == len(tiles)
    for want, got in zip(b.tiles_out, sb.tiles_out):
        assert torch.equal(want["iter"], got["iter"]) and torch.equal(want["kmap"], got["kmap"])
    assert sb.nominal_iterations() == b.nominal_iterations()


@pytest.mark.parametrize("rebase", [False, True])
@pytest.mark.parametrize("bla_form", ["reference", "accurate"])
def test_fp32_tiles_match_per_tile_frames(rebase, bla_form):
    """Tiles in the FP32-mantissa form (delta_form='fp32', every formula) beside FP64 tiles
    in one batch: each equals the engine's coarse render of the tile in its own form, in
    the default launch shape, the widest candidate, and quanta of 1 and 7 steps (every
    pixel's state goes through the shared slots at every step)."""
    import torch
    hp.clear_reference_orbit_cache()
    tiles = [dataclasses.replace(t, delta_form="fp32") if q % 3 != 2 else t for q, t in enumerate(_tiles(rebase))]
    want = [_engine_tile(t, "ref_cuda", bla_form) for t in tiles]
    s = torch.cuda.Stream()
    hp.clear_reference_orbit_cache()
    b = fb.prepare_batch(tiles, arith="ref_cuda", bla_form=bla_form, stream=s)
    for cfg in (fb.BatchConfig(), fb.CANDIDATES[-1], fb.BatchConfig(quantum=1),
                fb.BatchConfig(quantum=7, blocks_per_sm=1)):
        for o in b.tiles_out:
            o["iter"].fill_(-7.0)
        b.render(cfg)
        torch.cuda.synchronize()
        for t, out, (it, k) in zip(tiles, b.tiles_out, want):
            got = out["iter"].cpu().numpy()
            assert np.array_equal(got.view(np.uint32), it.view(np.uint32)), (cfg, t.fractal_type, int((got != it).sum()))
            assert np.array_equal(out["kmap"].cpu().numpy(), k)
