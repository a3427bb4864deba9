"""One frame split across GPUs by row bands, and a batch of tiles split across GPUs.

The reference renders every frame on one GPU (math_core/cuda_kernels.py:15) and has no
multi-GPU code.  Here one process drives each GPU (torch.distributed; NCCL between GPUs,
gloo on the CPU) and a frame is shared out as contiguous bands of rows:

  1. rank 0 searches the reference orbit on the host and broadcasts it -- the orbit, its
     length, the reference position (u, v) and its c -- so every rank perturbs around
     the same reference;
  2. every rank uploads the orbit, builds its BLA table and packed records, and renders
     its own rows (ap_render_rows) with the pixels' global row indices, so every pixel
     gets the value the unsplit frame gives it;
  3. histogram colouring (scheme 11): every rank counts its rows (ap_histogram), the
     int32[num_bins] counts are all-reduced (sum), and every rank turns the sum into the
     CDF (ap_cdf_from_histogram) -- the CDF of the whole frame;
  4. every rank colours its rows; the bands are all-gathered, so every rank ends with
     the whole frame.

Split frames serve coarse passes (factor 1) in the glitch modes that need no re-render
pass ("One-Pass Rebasing", "Off (Single-Ref)"): a Pauldelbrot re-render would need the
whole frame's glitch map on one host.  Rows are balanced by a per-row cost estimate
(uniform unless given).

shard_tiles() shares a batch of tiles out by estimated cost (longest processing time
first), for ranks that each run the persistent batch kernel on their own tiles.  Costs
come from pixels x max_iter (tile_cost) or from a small probe of each tile
(probe_tile_costs); a frame's bands can follow a probe of the frame (balance="probe"):
the probe is the adaptive max-iter probe's pass (math_core/engine.py:1063-1281), and a
pixel's cost is its escape step (max_iter when it stays bounded).

The steps of a split frame go through a backend object -- find_reference, render_band,
band_histogram, cdf_from_histogram, colour_band -- so the same orchestration drives the
engine's device code (DeviceBackend) and, in the multi-process CPU tests, the oracle.
"""
import ctypes as C
from decimal import Decimal

import numpy as np


# ------------------------------------------------------------------ partitions
def band_bounds(H, world, weights=None):
    """Contiguous row bands [(r0, r1), ...] for `world` ranks covering rows 0..H-1.

    With per-row costs (weights[H], non-negative) each band takes about 1/world of the
    total; otherwise rows are shared evenly.  Every rank computes the same bounds."""
    H, world = int(H), int(world)
    if world < 1 or H < 0:
        raise ValueError("world >= 1 and H >= 0 required")
    if weights is None:
        cuts = [(H * q) // world for q in range(world + 1)]
    else:
        w = np.asarray(weights, np.float64)
        if w.shape != (H,) or np.any(w < 0) or not np.all(np.isfinite(w)):
            raise ValueError("weights must be H finite non-negative row costs")
        cum = np.concatenate([[0.0], np.cumsum(w)])
        total = cum[-1]
        cuts = [0]
        for q in range(1, world):
            target = total * q / world
            r = int(np.searchsorted(cum, target, side="left"))
            cuts.append(min(H, max(cuts[-1], r)))
        cuts.append(H)
    return [(cuts[q], cuts[q + 1]) for q in range(world)]


def shard_tiles(costs, world):
    """Tiles shared out over `world` ranks, longest processing time first: each tile (by
    decreasing cost) goes to the rank with the least cost so far (ties: lowest rank).
    Returns one list of tile indices per rank, each in the batch's order."""
    costs = [float(c) for c in costs]
    if any(c < 0 or not np.isfinite(c) for c in costs):
        raise ValueError("tile costs must be finite and non-negative")
    loads = [0.0] * int(world)
    owner = [0] * len(costs)
    for t in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        r = min(range(len(loads)), key=lambda q: (loads[q], q))
        owner[t] = r
        loads[r] += costs[t]
    return [[t for t in range(len(costs)) if owner[t] == r] for r in range(len(loads))]


def tile_cost(tile):
    """Estimated cost of a tile: pixels x max_iter (the batch kernel's worst case)."""
    return float(tile.W) * float(tile.H) * float(tile.max_iter)


# ------------------------------------------------------------------ probe-estimated costs
def costs_from_probe(iters, max_iter):
    """Per-pixel cost estimate from a probe's smooth values: the escape step, or
    max_iter for a pixel that stays bounded (value < 0)."""
    it = np.asarray(iters, np.float64)
    return np.where(it < 0.0, float(max_iter), np.maximum(it, 1.0))


def row_weights(probe_costs, H):
    """Per-row costs of an H-row frame from a probe's [h, w] cost map of the same view
    (probe row q samples frame row q (H - 1) / (h - 1)): each frame row takes the cost
    of the probe row nearest to it."""
    pc = np.asarray(probe_costs, np.float64)
    h = pc.shape[0]
    per_row = pc.sum(axis=1)
    if h == 1 or H == 1:
        return np.full(int(H), per_row.mean())
    q = np.rint(np.arange(int(H), dtype=np.float64) * (h - 1) / (H - 1)).astype(np.int64)
    return per_row[q]


def probe_row_weights(view, probe, probe_w=128, probe_h=72):
    """Row costs of a view for band_bounds, from probe(view, probe_w, probe_h) -> the
    probe's smooth values [probe_h, probe_w] (a DeviceBackend's probe_map: the adaptive
    max-iter probe's pass, math_core/engine.py:1063-1281, at the view's max_iter)."""
    return row_weights(costs_from_probe(probe(view, probe_w, probe_h), view["max_iter"]), view["H"])


def probe_tile_costs(tiles, probe, probe_w=32, probe_h=32):
    """Estimated cost of each tile: its probe's mean per-pixel cost x its pixels, with
    probe(tile, probe_w, probe_h) -> smooth values (a DeviceBackend's probe_tile)."""
    out = []
    for t in tiles:
        c = costs_from_probe(probe(t, probe_w, probe_h), t.max_iter)
        out.append(float(c.mean()) * float(t.W) * float(t.H))
    return out


# ------------------------------------------------------------------ collectives
def _group_info(group):
    import torch.distributed as dist
    return dist.get_rank(group), dist.get_world_size(group)


def broadcast_reference(orbit, group=None, src=0):
    """The reference (ref_cx, ref_cy, u, v, re, im, ref_len) of rank src on every rank."""
    import torch.distributed as dist
    box = [None]
    if _group_info(group)[0] == src:
        cx, cy, u, v, re, im, rl = orbit
        rl = int(rl)
        box = [(str(cx), str(cy), float(u), float(v), np.ascontiguousarray(re[:rl + 1], np.float64),
                np.ascontiguousarray(im[:rl + 1], np.float64), rl)]
    dist.broadcast_object_list(box, src=src, group=group)
    cx, cy, u, v, re, im, rl = box[0]
    return Decimal(cx), Decimal(cy), u, v, re, im, rl


def allreduce_histogram(hist, group=None):
    """Sum of every rank's band histogram (int32 tensor, in place)."""
    import torch.distributed as dist
    dist.all_reduce(hist, op=dist.ReduceOp.SUM, group=group)
    return hist


def gather_bands(band, bands, group=None):
    """The whole frame on every rank from each rank's rows (a tensor [r1 - r0, ...]):
    bands are padded to the tallest, all-gathered, and cut back."""
    import torch
    import torch.distributed as dist
    rank, world = _group_info(group)
    tall = max(r1 - r0 for r0, r1 in bands)
    pad = torch.zeros((tall,) + tuple(band.shape[1:]), dtype=band.dtype, device=band.device)
    pad[:band.shape[0]] = band
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[q][:bands[q][1] - bands[q][0]] for q in range(world)], dim=0)


def render_split(view, backend, group=None, weights=None, balance=None):
    """One frame (a view dict: W, H, max_iter, cx, cy, width, scheme, num_bins, ...) split
    over the ranks of `group` by row bands.  Returns (rgb, iteration map) of the whole
    frame on every rank, as tensors on the backend's device.  Bands are even, or follow
    the per-row `weights`, or with balance="probe" rank 0's probe of the view
    (backend.probe_map, broadcast with the reference)."""
    import torch.distributed as dist
    rank, world = _group_info(group)
    orbit = backend.find_reference(view) if rank == 0 else None
    if balance == "probe":
        box = [probe_row_weights(view, backend.probe_map) if rank == 0 else None]
        dist.broadcast_object_list(box, src=0, group=group)
        weights = box[0]
    elif balance is not None:
        raise ValueError("balance must be None or 'probe'")
    bands = band_bounds(view["H"], world, weights)
    orbit = broadcast_reference(orbit, group)
    r0, r1 = bands[rank]
    it_band = backend.render_band(view, orbit, r0, r1)
    cdf = None
    if view["scheme"] == 11:
        hist = backend.band_histogram(view, it_band)
        allreduce_histogram(hist, group)
        cdf = backend.cdf_from_histogram(view, hist)
    rgb_band = backend.colour_band(view, it_band, cdf)
    return gather_bands(rgb_band, bands, group), gather_bands(it_band, bands, group)


# ------------------------------------------------------------------ the engine's backend
class DeviceBackend:
    """The split frame's steps on this rank's GPU through the engine's C-ABI."""

    def __init__(self, stream=None):
        import torch
        self.stream = stream or torch.cuda.current_stream()

    @staticmethod
    def _ctx(view):
        from .config import decimal_context
        return decimal_context(Decimal(view["width"]))

    def find_reference(self, view):
        from decimal import localcontext
        from . import high_precision as hp
        pw = Decimal(view["width"])
        with localcontext(self._ctx(view)):
            ph = pw * (Decimal(view["H"]) / Decimal(view["W"]))
        return hp.find_optimal_reference_orbit(
            Decimal(view["cx"]), Decimal(view["cy"]), pw, ph, view["max_iter"], view["W"], view["H"],
            fractal_type=view.get("fractal_type", 0), gen_n=view.get("gen_n", 3),
            gen_kr=view.get("gen_kr", 0.25), gen_ki=view.get("gen_ki", 1.0), is_floatexp=pw < Decimal("1e-300"))

    def render_band(self, view, orbit, r0, r1):
        import torch
        from . import engine
        W, H = view["W"], view["H"]
        it = torch.full((H, W), -1.0, dtype=torch.float32, device="cuda")
        engine.render_frame_ssaa(
            W, H, view["max_iter"], Decimal(view["cx"]), Decimal(view["cy"]), Decimal(view["width"]), None,
            color_scheme_id=view["scheme"], precision_mode=view.get("precision_mode", "1e-300 (Perturbation)"),
            fractal_type=view.get("fractal_type", 0), bbsa_tol=view.get("bbsa_tol", 1e-6),
            bbsa_order=view.get("bbsa_order", 32), glitch_mode=view.get("glitch_mode", "One-Pass Rebasing"),
            gen_n=view.get("gen_n", 3), gen_kr=view.get("gen_kr", 0.25), gen_ki=view.get("gen_ki", 1.0),
            stream=self.stream, arith=view.get("arith"), bla_form=view.get("bla_form"), d_iter_buf=it,
            sync_stream=False, _rows=(r0, r1), _orbit=orbit)
        return it[r0:r1]

    def probe_map(self, view, probe_w, probe_h):
        """The view's probe (engine.probe_iter_map at the view's max_iter)."""
        from . import engine
        return engine.probe_iter_map(Decimal(view["cx"]), Decimal(view["cy"]), Decimal(view["width"]),
                                     int(view["max_iter"]), probe_w, probe_h,
                                     fractal_type=view.get("fractal_type", 0), gen_n=view.get("gen_n", 3),
                                     gen_kr=view.get("gen_kr", 0.25), gen_ki=view.get("gen_ki", 1.0),
                                     precision_mode=view.get("precision_mode", "1e-300 (Perturbation)"),
                                     bbsa_order=0, stream=self.stream)

    @staticmethod
    def probe_tile(tile, probe_w, probe_h):
        """A batch tile's probe (engine.probe_iter_map at the tile's max_iter)."""
        from . import engine
        return engine.probe_iter_map(Decimal(tile.cx), Decimal(tile.cy), Decimal(tile.width), int(tile.max_iter),
                                     probe_w, probe_h, fractal_type=tile.fractal_type, julia_cx=tile.julia_cx,
                                     julia_cy=tile.julia_cy, gen_n=tile.gen_n, gen_kr=tile.gen_kr,
                                     gen_ki=tile.gen_ki, bbsa_order=0)

    def band_histogram(self, view, it_band):
        import torch
        from . import _lib
        nb = int(view.get("num_bins", 65536))
        hist = torch.empty(nb, dtype=torch.int32, device=it_band.device)
        L = _lib.load()
        band = it_band.contiguous()
        with torch.cuda.stream(self.stream):
            _lib.launch(L.ap_histogram, C.c_void_p(band.data_ptr()), int(band.shape[1]), int(band.shape[0]),
                        int(view["max_iter"]), nb, C.c_void_p(hist.data_ptr()),
                        C.c_void_p(self.stream.cuda_stream), what="ap_histogram")
        self.stream.synchronize()
        return hist

    def cdf_from_histogram(self, view, hist):
        import torch
        from . import _lib
        cdf = torch.empty(hist.numel(), dtype=torch.float32, device=hist.device)
        L = _lib.load()
        with torch.cuda.stream(self.stream):
            _lib.launch(L.ap_cdf_from_histogram, C.c_void_p(hist.data_ptr()), int(hist.numel()),
                        C.c_void_p(cdf.data_ptr()), C.c_void_p(self.stream.cuda_stream),
                        what="ap_cdf_from_histogram")
        return cdf

    def colour_band(self, view, it_band, cdf):
        import torch
        from . import _lib, abi, engine
        band = it_band.contiguous()
        h, w = band.shape
        rgb = torch.empty((h, w, 3), dtype=torch.uint8, device=band.device)
        lut = engine.get_device_lut(view.get("cmap_name"))
        p = abi.new_params(width=w, height=h, max_iter=int(view["max_iter"]), scheme_id=int(view["scheme"]),
                           num_bins=int(view.get("num_bins", 65536 if view["scheme"] == 11 else 2048)),
                           arith=engine._arith_code(view.get("arith") or engine.DEFAULT_ARITH),
                           palette_offset=float(view.get("offset", 0.0)),
                           color_density=float(view.get("density", 1.0)),
                           color_contrast=float(view.get("contrast", 1.0)))
        b = abi.ApFrameBuffers()
        b.iter_map, b.rgb, b.lut = C.c_void_p(band.data_ptr()), C.c_void_p(rgb.data_ptr()), C.c_void_p(lut.data_ptr())
        b.cdf = None if cdf is None else C.c_void_p(cdf.data_ptr())
        L = _lib.load()
        with torch.cuda.stream(self.stream):
            _lib.launch(L.ap_colour, C.byref(p), C.byref(b), C.c_void_p(self.stream.cuda_stream), what="ap_colour")
        self.stream.synchronize()
        return rgb
