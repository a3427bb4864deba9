"""Export-side consumers of the render path: mosaics and frame sequences.

render_mosaic renders a grid_n x grid_n mosaic of a canvas, as the reference's mosaic
exporter does (workers/image_workers.py:428-601): tile (row, col) is the view of width
w / n centred at x_min + (col + 1/2) w / n, y_max - (row + 1/2) h / n (h = w H / W), each
tile target_w x target_h, rendered with the canvas's parameters; with stitch=True the
tiles are placed in one (n H) x (n W) image on the device and copied to the host once.
Tiles in a form the persistent batch kernel serves (perturbation tiers, factor 1, glitch
mode "Off (Single-Ref)" or "One-Pass Rebasing", no series start, the reference
arithmetic profiles) are rendered by one batch launch and coloured tile by tile on the
device; every other mosaic goes tile by tile through FramePipeline.

FramePipeline renders a sequence of frames the way the reference's frame exporter does
(workers/base.py:443-542): frame i on stream i % 2 with that stream's device RGB buffer
and a pinned host buffer from a pool of four, render_frame_ssaa called with
sync_stream=False so that the host prepares frame i + 1 (orbit search, parameters) while
frame i computes, at most two frames in flight, each handed to the consumer in order
once its stream has finished.
"""
import ctypes as C
from collections import deque
from decimal import Decimal, localcontext

import numpy as np

from . import _lib, abi
from .config import decimal_context

BATCH_GLITCH_MODES = ("Off (Single-Ref)", "One-Pass Rebasing")


def mosaic_views(canvas_cx, canvas_cy, plot_width, grid_n, target_w, target_h):
    """[(row, col, tile_cx, tile_cy, tile_plot_w)] of a mosaic, row-major, in the
    reference's Decimal arithmetic (workers/image_workers.py:468-515)."""
    cx, cy, pw = (x if isinstance(x, Decimal) else Decimal(str(x)) for x in (canvas_cx, canvas_cy, plot_width))
    n = int(grid_n)
    if n < 1:
        raise ValueError("grid_n must be >= 1")
    out = []
    with localcontext(decimal_context(pw)):
        n_dec = Decimal(n)
        aspect = Decimal(int(target_h)) / Decimal(int(target_w))
        total_h = pw * aspect
        tile_w = pw / n_dec
        tile_h = total_h / n_dec
        x_min = cx - (pw / Decimal(2))
        y_max = cy + (total_h / Decimal(2))
        half = Decimal("0.5")
        for row in range(n):
            tcy = y_max - (Decimal(row) + half) * tile_h
            for col in range(n):
                tcx = x_min + (Decimal(col) + half) * tile_w
                out.append((row, col, tcx, tcy, tile_w))
    return out


class FramePipeline:
    """Frames on two CUDA streams with pinned host buffers (see the module docstring).

        pipe = FramePipeline(W, H)
        pipe.render(frames, consume)   # frames: dicts of render_frame_ssaa arguments
                                       # consume(i, host_rgb): called in frame order

    The host buffer passed to consume goes back to the pool when consume returns:
    copy what you keep."""

    def __init__(self, target_w, target_h, is_hdr=False, host_buffers=4):
        import torch
        self.W, self.H, self.is_hdr = int(target_w), int(target_h), bool(is_hdr)
        dt = torch.uint16 if self.is_hdr else torch.uint8
        self.streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        self.d_rgb = [torch.empty((self.H, self.W, 3), dtype=dt, device="cuda") for _ in range(2)]
        self.free = deque(torch.empty((self.H, self.W, 3), dtype=dt).pin_memory().numpy()
                          for _ in range(max(2, int(host_buffers))))

    def render(self, frames, consume):
        from . import engine
        pending = deque()

        def finish():
            i, h, st = pending.popleft()
            st.synchronize()
            consume(i, h)
            self.free.append(h)

        for i, kw in enumerate(frames):
            slot = i % 2
            st = self.streams[slot]
            if not self.free:
                finish()
            h = self.free.popleft()
            kw = dict(kw)
            max_iter = kw.pop("max_iter")
            cx, cy, w = kw.pop("center_x_dec"), kw.pop("center_y_dec"), kw.pop("plot_width_dec")
            cmap = kw.pop("cmap_name", None)
            engine.render_frame_ssaa(self.W, self.H, max_iter, cx, cy, w, cmap, d_rgb_buf=self.d_rgb[slot],
                                     h_rgb_buf=h, stream=st, stream_slot=slot + 1, is_hdr=self.is_hdr,
                                     sync_stream=False, **kw)
            pending.append((i, h, st))
            if len(pending) >= 2:
                finish()
        while pending:
            finish()


# ------------------------------------------------------------------ mosaics
RENDER_KEYS = ("ssaa_factor", "edge_threshold", "color_scheme_id", "precision_mode", "fractal_type", "julia_cx",
               "julia_cy", "bbsa_tol", "bbsa_order", "glitch_mode", "gen_n", "gen_kr", "gen_ki",
               "palette_offset", "color_density", "color_contrast", "arith", "bla_form", "delta_form")

_DEFAULTS = dict(ssaa_factor=1, edge_threshold=0.35, color_scheme_id=0, precision_mode="1e-300 (Perturbation)",
                 fractal_type=0, julia_cx=0.0, julia_cy=0.0, bbsa_tol=1e-4, bbsa_order=4,
                 glitch_mode="Off (Legacy Single-Ref)", gen_n=3, gen_kr=0.25, gen_ki=1.0, palette_offset=0.0,
                 color_density=1.0, color_contrast=1.0, arith=None, bla_form=None, delta_form=None)


def batch_serves(tile_w, kw):
    """Whether the persistent batch kernel renders a mosaic tile of width tile_w with the
    render arguments kw exactly as render_frame_ssaa does: the FP64-delta perturbation
    tier, factor 1, a glitch mode with no re-render pass and no Pauldelbrot flags, no
    series start (orders 4 and 8), the reference arithmetic profiles, FP64 or FP32
    deltas, and no one-pass rebasing of Julia tiles."""
    from . import engine
    if engine.select_tier(tile_w, kw["precision_mode"]) != abi.AP_TIER_PERTURB:
        return False
    gm = str(kw["glitch_mode"])
    if any(s in gm for s in ("Auto Rebasing", "Strict", "Pauldelbrot")):
        return False
    if max(1, int(kw["ssaa_factor"])) != 1 or int(kw["bbsa_order"]) in (4, 8):
        return False
    if (kw["arith"] or engine.DEFAULT_ARITH) not in ("ref_cpu", "ref_cuda"):
        return False
    if kw["delta_form"] not in (None, "fp64", "fp32"):
        return False
    return not ("One-Pass Rebasing" in gm and int(kw["fractal_type"]) in (2, 3))


def _colour_tile(L, torch, it, rgb, lut, kw, max_iter, is_hdr, arith_code, st):
    """ap_colour of one tile's iteration map (histogram scheme: ap_histogram_cdf first),
    with the parameters render_frame_ssaa colours a frame with."""
    H, W = it.shape
    scheme = int(kw["color_scheme_id"])
    num_bins = 65536 if scheme == 11 else 2048
    p = abi.new_params(width=W, height=H, factor=1, max_iter=int(max_iter), scheme_id=scheme, num_bins=num_bins,
                       arith=arith_code, palette_offset=float(kw["palette_offset"]),
                       color_density=float(kw["color_density"]), color_contrast=float(kw["color_contrast"]),
                       is_hdr=int(bool(is_hdr)))
    b = abi.ApFrameBuffers()
    b.iter_map, b.rgb, b.lut = C.c_void_p(it.data_ptr()), C.c_void_p(rgb.data_ptr()), C.c_void_p(lut.data_ptr())
    sh = C.c_void_p(st.cuda_stream)
    keep = None
    if scheme == 11:
        hist = torch.empty(num_bins, dtype=torch.int32, device="cuda")
        cdf = torch.empty(num_bins, dtype=torch.float32, device="cuda")
        _lib.launch(L.ap_histogram_cdf, C.c_void_p(it.data_ptr()), W, H, int(max_iter), num_bins,
                    C.c_void_p(hist.data_ptr()), C.c_void_p(cdf.data_ptr()), sh, what="ap_histogram_cdf")
        b.cdf = C.c_void_p(cdf.data_ptr())
        keep = (hist, cdf)
    _lib.launch(L.ap_colour, C.byref(p), C.byref(b), sh, what="ap_colour")
    return keep


def render_mosaic(grid_n, target_w, target_h, max_iter, canvas_cx, canvas_cy, plot_width, cmap_name=None,
                  stitch=True, on_tile=None, dynamic_iter_mode="Off", is_hdr=False, use_batch=True, stream=None,
                  **render_kwargs):
    """A grid_n x grid_n mosaic of the canvas (see the module docstring).

    Every tile is the frame render_frame_ssaa gives for its view and the render arguments
    (ssaa_factor, color_scheme_id, precision_mode, fractal_type, glitch_mode, bbsa_tol,
    bbsa_order, arith, bla_form, ...); max_iter per tile is compute_dynamic_max_iter of
    dynamic_iter_mode at the tile's view, as the reference's exporter does.  Returns the
    stitched (grid_n H, grid_n W, 3) image (stitch=True, else None); on_tile(row, col,
    rgb) receives each tile on the host, in row-major order (a view into a reused
    buffer: copy what you keep).  use_batch=False sends every tile through FramePipeline.
    """
    import torch
    from . import batch as fb
    from . import engine
    unknown = set(render_kwargs) - set(RENDER_KEYS)
    if unknown:
        raise TypeError(f"unknown render arguments {sorted(unknown)}")
    if not stitch and on_tile is None:
        raise ValueError("nothing to deliver: stitch=False needs on_tile")
    kw = dict(_DEFAULTS, **render_kwargs)
    W, H, n = int(target_w), int(target_h), int(grid_n)
    views = mosaic_views(canvas_cx, canvas_cy, plot_width, n, W, H)
    tile_w = views[0][4]
    iters = [engine.compute_dynamic_max_iter(max_iter, tile_w, dynamic_iter_mode, center_x_dec=tcx,
                                             center_y_dec=tcy, fractal_type=kw["fractal_type"],
                                             julia_cx=float(kw["julia_cx"]), julia_cy=float(kw["julia_cy"]),
                                             gen_n=kw["gen_n"], gen_kr=kw["gen_kr"], gen_ki=kw["gen_ki"],
                                             precision_mode=kw["precision_mode"], bbsa_tol=kw["bbsa_tol"],
                                             bbsa_order=kw["bbsa_order"])
             for (_, _, tcx, tcy, _) in views]
    dt = torch.uint16 if is_hdr else torch.uint8
    if use_batch and batch_serves(tile_w, kw):
        return _mosaic_batch(views, iters, W, H, n, kw, cmap_name, is_hdr, dt, stitch, on_tile, stream)
    master = np.zeros((n * H, n * W, 3), dtype=np.uint16 if is_hdr else np.uint8) if stitch else None

    def consume(i, rgb):
        row, col = views[i][0], views[i][1]
        if master is not None:
            master[row * H:(row + 1) * H, col * W:(col + 1) * W] = rgb
        if on_tile is not None:
            on_tile(row, col, rgb)

    frames = ({**{k: kw[k] for k in RENDER_KEYS}, "max_iter": it, "center_x_dec": tcx, "center_y_dec": tcy,
               "plot_width_dec": tw, "cmap_name": cmap_name}
              for (_, _, tcx, tcy, tw), it in zip(views, iters))
    FramePipeline(W, H, is_hdr=is_hdr).render(frames, consume)
    return master


def _mosaic_batch(views, iters, W, H, n, kw, cmap_name, is_hdr, dt, stitch, on_tile, stream):
    """The mosaic's tiles in one persistent batch launch, coloured tile by tile into a
    stitched device image, copied to the host once."""
    import torch
    from . import batch as fb
    from . import engine
    arith = kw["arith"] or engine.DEFAULT_ARITH
    cpu_sem = arith == "ref_cpu"
    scheme = int(kw["color_scheme_id"])
    bla = int(kw["bbsa_order"]) == 32 and not (cpu_sem and scheme == 11)
    rebase = "One-Pass Rebasing" in str(kw["glitch_mode"])
    tiles = [fb.Tile(cx=tcx, cy=tcy, width=tw, W=W, H=H, max_iter=int(it), fractal_type=int(kw["fractal_type"]),
                     julia_cx=float(kw["julia_cx"]), julia_cy=float(kw["julia_cy"]), gen_n=int(kw["gen_n"]),
                     gen_kr=float(kw["gen_kr"]), gen_ki=float(kw["gen_ki"]), bla=bla, strict_glitch=False,
                     rebase=rebase, bla_tol=float(kw["bbsa_tol"]), delta_form=kw["delta_form"] or "fp64")
             for (_, _, tcx, tcy, tw), it in zip(views, iters)]
    st = stream or torch.cuda.Stream()
    L = _lib.load()
    b = fb.prepare_batch(tiles, arith=arith, bla_form=kw["bla_form"] or "reference", stream=st)
    lut = engine.get_device_lut(cmap_name, is_hdr)
    with torch.cuda.stream(st):
        b.render(fb.BatchConfig())
        master = torch.empty((n * H, n * W, 3), dtype=dt, device="cuda")
        rgb = torch.empty((H, W, 3), dtype=dt, device="cuda")
        keep = []
        for (row, col, *_), t, out in zip(views, tiles, b.tiles_out):
            keep.append(_colour_tile(L, torch, out["iter"], rgb, lut, kw, t.max_iter, is_hdr,
                                     engine._arith_code(arith), st))
            master[row * H:(row + 1) * H, col * W:(col + 1) * W].copy_(rgb)
        host = torch.empty(master.shape, dtype=dt).pin_memory()
        host.copy_(master, non_blocking=True)
    st.synchronize()
    img = host.numpy()
    if on_tile is not None:
        for row, col, *_ in views:
            on_tile(row, col, img[row * H:(row + 1) * H, col * W:(col + 1) * W])
    return img if stitch else None
