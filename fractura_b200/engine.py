"""Host side of the B200 escape-time engine: the reference's render entry points.

Drop-in counterparts of math_core/engine.py's public functions
(re-exported by math_core/__init__.py:1-41):

    render_frame(params)                          math_core/engine.py:1326
    render_frame_ssaa(target_w, ..., stream_slot) math_core/engine.py:1339
    recolor_frame(params, d_iter_buf, h_iter_buf) math_core/engine.py:2138
    compute_dynamic_max_iter(...)                 math_core/engine.py:1284
    probe_adaptive_max_iter(...)                  math_core/engine.py:1063
    get_scratch_device_array / clear_scratch_buffer_pool / get_stream_slot

Same names, argument meanings and return values.  Device buffers are torch
CUDA tensors (``d_rgb_buf`` / ``d_iter_buf``) instead of Numba device arrays;
``stream`` is a ``torch.cuda.Stream`` (or 0 / None for torch's current
stream).  Every pixel is computed by the CUDA library through its C ABI;
``compute_device="CPU"`` is rejected -- this engine has no CPU path.
"""
import ctypes as C
import math
import threading
from decimal import Decimal, localcontext

import numpy as np

from . import abi
from . import _lib
from .config import (
    ACCURATE_BLA_EPS, ARITH_PROFILES, GLOBAL_MAX_ITER, RenderParameters, compute_floatexp_scale,
    compute_required_prec_bits, decimal_context,
)
from .palette import LUT_SIZE, check_lut, synthetic_lut

_POOL = {}
_POOL_LOCK = threading.Lock()
_STREAM_SLOTS = {}
_STREAM_LOCK = threading.Lock()
_NEXT_SLOT = 1
_LUTS = {}
_LUT_LOCK = threading.Lock()

# Default arithmetic profile of every render (see include/apeiron_b200.h).
DEFAULT_ARITH = "ref_cpu"


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise _lib.EngineUnavailable("no CUDA device is visible to torch")
    return torch


# ----------------------------------------------------------------- plumbing
def get_stream_slot(stream, explicit_slot=None):
    """Distinct integer slot per stream for pooled scratch (math_core/engine.py:106-119)."""
    global _NEXT_SLOT
    if explicit_slot is not None and explicit_slot >= 0:
        return int(explicit_slot)
    if stream == 0 or stream is None:
        return 0
    with _STREAM_LOCK:
        slot = _STREAM_SLOTS.get(id(stream))
        if slot is None:
            slot = _NEXT_SLOT
            _NEXT_SLOT = (_NEXT_SLOT % 16) + 1
            _STREAM_SLOTS[id(stream)] = slot
        return slot


def get_scratch_device_array(shape, dtype, tag="scratch"):
    """Pooled device tensor keyed by (tag, shape, dtype) (math_core/engine.py:123-134)."""
    torch = _torch()
    shape = (shape,) if isinstance(shape, int) else tuple(int(s) for s in shape)
    tdt = _torch_dtype(dtype)
    key = (tag, shape, str(tdt))
    with _POOL_LOCK:
        buf = _POOL.get(key)
        if buf is None:
            buf = torch.empty(shape, dtype=tdt, device="cuda")
            _POOL[key] = buf
        return buf


def get_scratch_device_array_1d(min_size, dtype, tag="scratch_1d"):
    """Pooled 1-D tensor with capacity >= min_size (math_core/engine.py:137-148)."""
    torch = _torch()
    tdt = _torch_dtype(dtype)
    key = (tag, str(tdt))
    with _POOL_LOCK:
        buf = _POOL.get(key)
        if buf is None or buf.numel() < min_size:
            buf = torch.empty(max(int(min_size * 1.5), 65536), dtype=tdt, device="cuda")
            _POOL[key] = buf
        return buf


def clear_scratch_buffer_pool():
    """Free every pooled device buffer (math_core/engine.py:171-188)."""
    global _NEXT_SLOT
    with _POOL_LOCK:
        _POOL.clear()
    with _STREAM_LOCK:
        _STREAM_SLOTS.clear()
        _NEXT_SLOT = 1
    with _LUT_LOCK:
        _LUTS.clear()
    try:
        import torch
        if torch.cuda.is_available():
            torch.cuda.synchronize()
    except Exception:
        pass


def _torch_dtype(dtype):
    torch = _torch()
    m = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
         np.dtype(np.uint8): torch.uint8, np.dtype(np.uint16): torch.uint16,
         np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64}
    if isinstance(dtype, torch.dtype):
        return dtype
    return m[np.dtype(dtype)]


def register_lut(name, lut):
    """Register a float32[2048, 3] colour table under ``cmap_name``."""
    arr = check_lut(lut)
    with _LUT_LOCK:
        for key in [k for k in _LUTS if k[0] == name]:
            del _LUTS[key]
        _LUTS[(name, "host")] = arr


def get_device_lut(cmap_name, is_hdr=False):
    """Device copy of the LUT for ``cmap_name`` (an array, a registered name, or the synthetic table)."""
    torch = _torch()
    if isinstance(cmap_name, np.ndarray):
        return torch.from_numpy(check_lut(cmap_name)).cuda()
    key = (cmap_name, bool(is_hdr))
    with _LUT_LOCK:
        dev = _LUTS.get(key)
        if dev is None:
            host = _LUTS.get((cmap_name, "host"))
            if host is None:
                host = synthetic_lut(LUT_SIZE, is_hdr)
            elif is_hdr:
                host = (host / 255.0 * 65535.0).astype(np.float32)
            dev = torch.from_numpy(np.ascontiguousarray(host)).cuda()
            _LUTS[key] = dev
        return dev


def _stream_handle(stream):
    torch = _torch()
    if stream is None or (isinstance(stream, int) and stream == 0):
        s = torch.cuda.current_stream()
    elif isinstance(stream, torch.cuda.Stream):
        s = stream
    else:
        raise TypeError("stream must be a torch.cuda.Stream, 0 or None")
    return s, C.c_void_p(s.cuda_stream)


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


# ---------------------------------------------------------- view planning
def to_dd(dec_val, ctx=None):
    """Decimal -> (hi, lo) float64 pair (math_core/high_precision.py:17-21)."""
    with localcontext(ctx or decimal_context()):
        d = Decimal(dec_val)
        hi = float(d)
        return hi, float(d - Decimal(hi))


def select_tier(plot_width_dec, precision_mode):
    """Precision tier exactly as math_core/engine.py:1403-1408."""
    w = Decimal(str(plot_width_dec)) if not isinstance(plot_width_dec, Decimal) else plot_width_dec
    use_floatexp = w < Decimal("1e-300")
    use_fp64 = (w >= Decimal("1e-12")) and not use_floatexp
    use_dd = (w >= Decimal("1e-24") and "dd" in str(precision_mode).lower()) and not use_floatexp
    if use_dd:
        use_fp64 = False
    if use_floatexp:
        return abi.AP_TIER_FLOATEXP
    if use_fp64:
        return abi.AP_TIER_FP64
    if use_dd:
        return abi.AP_TIER_DD
    return abi.AP_TIER_PERTURB


def plan_direct_view(target_w, target_h, factor, center_x_dec, center_y_dec, plot_width_dec,
                     tier, julia_cx=0.0, julia_cy=0.0):
    """Mapping parameters of the FP64 / DD tiers (math_core/engine.py:1397-1400, :1643-1685)."""
    ctx = decimal_context(plot_width_dec)
    with localcontext(ctx):
        plot_height_dec = plot_width_dec * (Decimal(target_h) / Decimal(target_w))
        v = {}
        if tier == abi.AP_TIER_FP64:
            dx_f = float(plot_width_dec / Decimal(max(1, target_w - 1)))
            dy_f = float(plot_height_dec / Decimal(max(1, target_h - 1)))
            w_f, h_f = float(plot_width_dec), float(plot_height_dec)
            cx, cy = float(center_x_dec), float(center_y_dec)
            v.update(x_min_hi=cx - (w_f * 0.5), y_max_hi=cy + (h_f * 0.5),
                     dx_hi=dx_f / float(factor), dy_hi=dy_f / float(factor),
                     julia_cx_hi=float(julia_cx), julia_cy_hi=float(julia_cy))
        else:
            x_min = to_dd(center_x_dec - (plot_width_dec / Decimal(2)), ctx)
            y_max = to_dd(center_y_dec + (plot_height_dec / Decimal(2)), ctx)
            dx = to_dd((plot_width_dec / Decimal(max(1, target_w - 1))) / Decimal(factor), ctx)
            dy = to_dd((plot_height_dec / Decimal(max(1, target_h - 1))) / Decimal(factor), ctx)
            jx = to_dd(julia_cx, ctx)
            jy = to_dd(julia_cy, ctx)
            v.update(x_min_hi=x_min[0], x_min_lo=x_min[1], y_max_hi=y_max[0], y_max_lo=y_max[1],
                     dx_hi=dx[0], dx_lo=dx[1], dy_hi=dy[0], dy_lo=dy[1],
                     julia_cx_hi=jx[0], julia_cx_lo=jx[1], julia_cy_hi=jy[0], julia_cy_lo=jy[1])
        return v


def _arith_code(arith):
    if isinstance(arith, int):
        return arith
    return ARITH_PROFILES[arith]


# ------------------------------------------------------------------ frames
class _DeviceFrame:
    """Device buffers of one frame (pooled per stream slot)."""

    def __init__(self, W, H, is_hdr, slot, d_rgb_buf=None, d_iter_buf=None, need_glitch=False):
        torch = _torch()
        rgb_dt = np.uint16 if is_hdr else np.uint8
        self.rgb = d_rgb_buf if d_rgb_buf is not None else get_scratch_device_array(
            (H, W, 3), rgb_dt, f"out_rgb_{slot}")
        self.iter = d_iter_buf if d_iter_buf is not None else get_scratch_device_array(
            (H, W), np.float32, f"iter_map_{slot}")
        _check_dev(self.rgb, (H, W, 3), torch.uint16 if is_hdr else torch.uint8, "d_rgb_buf")
        _check_dev(self.iter, (H, W), torch.float32, "d_iter_buf")
        self.edge = None
        self.glitch_out = self.glitch_in = None
        if need_glitch:
            self.glitch_out = get_scratch_device_array((H, W), np.uint8, f"glitch_out_{slot}")
            self.glitch_in = get_scratch_device_array((H, W), np.uint8, f"glitch_in_{slot}")
        self.slot = slot
        self.W, self.H = W, H

    def edge_mask(self):
        if self.edge is None:
            self.edge = get_scratch_device_array((self.H, self.W), np.uint8, f"edge_mask_{self.slot}")
        return self.edge


def _check_dev(t, shape, dtype, name):
    if tuple(t.shape) != tuple(shape) or t.dtype != dtype or not t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA tensor of shape {shape} and dtype {dtype}")


def _buffers(fr, lut, cdf=None, orbit=None, bla=None, kmap=None, s64=None):
    b = abi.ApFrameBuffers()
    b.lut = _ptr(lut)
    b.cdf = _ptr(cdf)
    b.iter_map = _ptr(fr.iter)
    b.rgb = _ptr(fr.rgb)
    b.edge_mask = _ptr(fr.edge)
    b.glitch_out = _ptr(fr.glitch_out)
    b.glitch_in = _ptr(fr.glitch_in)
    if orbit is not None:
        b.ref_re, b.ref_im = _ptr(orbit[0]), _ptr(orbit[1])
    b.bla = _ptr(bla)
    b.kmap = _ptr(kmap)
    b.s64 = _ptr(s64)
    return b


def _render_direct(p, fr, lut, stream_h, scheme, factor, arith_code, num_bins, max_iter,
                   edge_threshold, slot, extra_out=None):
    """Coarse + edge passes of the FP64 / DD tiers (math_core/engine.py:1430-1717)."""
    L = _lib.load()
    kmap = s64 = None
    if extra_out is not None:
        kmap, s64 = extra_out
    cpu = arith_code == abi.AP_ARITH_REF_CPU
    if scheme == 11:
        hist = get_scratch_device_array((num_bins,), np.int32, f"hist_bins_{slot}")
        cdf = get_scratch_device_array((num_bins,), np.float32, f"cdf_lut_{slot}")
        p.mode = abi.AP_MODE_COARSE
        p.flags = abi.AP_FLAG_NO_RGB
        b = _buffers(fr, lut, cdf=cdf, kmap=kmap, s64=s64)
        _lib.launch(L.ap_render_pass, C.byref(p), C.byref(b), stream_h, what="ap_render_pass")
        _lib.launch(L.ap_histogram_cdf, _ptr(fr.iter), fr.W, fr.H, max_iter, num_bins, _ptr(hist),
                                      _ptr(cdf), stream_h, what="ap_histogram_cdf")
        _lib.launch(L.ap_colour, C.byref(p), C.byref(b), stream_h, what="ap_colour")
        if factor > 1:
            fr.edge_mask()
            b = _buffers(fr, lut, cdf=cdf)
            _lib.launch(L.ap_edge_detect, _ptr(fr.iter), _ptr(fr.edge), fr.W, fr.H,
                                        float(np.float32(edge_threshold)), stream_h, what="ap_edge_detect")
            p.flags = abi.AP_FLAG_MAP_FUSED if cpu else 0
            _lib.launch(L.ap_resolve_hist_pass, C.byref(p), C.byref(b), stream_h, what="ap_resolve_hist_pass")
        return cdf
    p.mode = abi.AP_MODE_COARSE
    p.flags = abi.AP_FLAG_MAP_FUSED if cpu else 0
    b = _buffers(fr, lut, kmap=kmap, s64=s64)
    _lib.launch(L.ap_render_pass, C.byref(p), C.byref(b), stream_h, what="ap_render_pass")
    if factor > 1:
        fr.edge_mask()
        b = _buffers(fr, lut)
        _lib.launch(L.ap_edge_detect, _ptr(fr.iter), _ptr(fr.edge), fr.W, fr.H,
                                    float(np.float32(edge_threshold)), stream_h, what="ap_edge_detect")
        p.mode = abi.AP_MODE_EDGE
        _lib.launch(L.ap_render_pass, C.byref(p), C.byref(b), stream_h, what="ap_render_pass")
    return None


def render_frame(params: RenderParameters):
    """Render one frame described by ``params`` (math_core/engine.py:1326)."""
    return render_frame_ssaa(params)


def render_frame_ssaa(target_w, target_h=None, max_iter=None, center_x_dec=None, center_y_dec=None,
                      plot_width_dec=None, cmap_name=None, ssaa_factor=1, edge_threshold=0.35,
                      color_scheme_id=0, precision_mode="1e-300 (Perturbation)", fractal_type=0,
                      julia_cx=0.0, julia_cy=0.0, bbsa_tol=1e-4, bbsa_order=4,
                      glitch_mode="Off (Legacy Single-Ref)", gen_n=3, gen_kr=0.25, gen_ki=1.0,
                      d_rgb_buf=None, h_rgb_buf=None, stream=0, is_hdr=False,
                      compute_device="GPU", cpu_threads=2, palette_offset=0.0,
                      color_density=1.0, color_contrast=1.0, sync_stream=True,
                      d_iter_buf=None, h_iter_buf=None, stream_slot=None, arith=None,
                      delta_form=None, bla_form=None, _extra_out=None, _rows=None, _orbit=None):
    """Render one frame and return its RGB image (math_core/engine.py:1339-2135).

    Same arguments as the reference; ``arith`` optionally selects the
    arithmetic profile ("ref_cpu" default, "ref_cuda", or "fast": the engine's own
    fused form, for glitch_mode "One-Pass Rebasing" only), ``delta_form``
    the perturbation delta arithmetic: "fp64" (default, the reference's) or
    "fp32" (FP32 mantissas with integer exponents on the coarse passes of
    perturbation frames, every formula), ``bla_form`` the chained-BLA table: "reference"
    (default: the reference's merge at ``bbsa_tol``) or "accurate" (the
    dc-aware merge at ``ACCURATE_BLA_EPS``).  The smooth iteration map is left in
    ``d_iter_buf`` (and copied to ``h_iter_buf`` when one is given).
    """
    if isinstance(target_w, RenderParameters):
        q = target_w
        return render_frame_ssaa(
            q.target_w, q.target_h, q.max_iter, q.center_x_dec, q.center_y_dec, q.plot_width_dec,
            q.cmap_name, ssaa_factor=q.ssaa_factor, edge_threshold=q.edge_threshold,
            color_scheme_id=q.color_scheme_id, precision_mode=q.precision_mode,
            fractal_type=q.fractal_type, julia_cx=q.julia_cx, julia_cy=q.julia_cy,
            bbsa_tol=q.bbsa_tol, bbsa_order=q.bbsa_order, glitch_mode=q.glitch_mode,
            gen_n=q.gen_n, gen_kr=q.gen_kr, gen_ki=q.gen_ki,
            d_rgb_buf=q.d_rgb_buf if d_rgb_buf is None else d_rgb_buf,
            h_rgb_buf=q.h_rgb_buf if h_rgb_buf is None else h_rgb_buf,
            stream=q.stream if q.stream is not None else stream, is_hdr=q.is_hdr,
            compute_device=q.compute_device, cpu_threads=q.cpu_threads,
            palette_offset=q.palette_offset, color_density=q.color_density,
            color_contrast=q.color_contrast, sync_stream=getattr(q, "sync_stream", sync_stream),
            d_iter_buf=getattr(q, "d_iter_buf", d_iter_buf),
            h_iter_buf=getattr(q, "h_iter_buf", h_iter_buf),
            stream_slot=getattr(q, "stream_slot", stream_slot),
            arith=getattr(q, "arith", arith), delta_form=getattr(q, "delta_form", delta_form),
            bla_form=getattr(q, "bla_form", bla_form), _extra_out=_extra_out)

    if compute_device == "CPU":
        raise NotImplementedError("this engine renders on the GPU only (compute_device='CPU')")
    torch = _torch()
    if stream is None:
        stream = 0
    slot = get_stream_slot(stream, explicit_slot=stream_slot)
    st, stream_h = _stream_handle(stream)
    W, H = int(target_w), int(target_h)
    max_iter = int(max_iter)
    if W < 1 or H < 1:
        raise ValueError("target_w and target_h must be positive")
    if max_iter < 0:
        raise ValueError("max_iter must be non-negative")
    factor = max(1, int(ssaa_factor))
    if not isinstance(plot_width_dec, Decimal):
        plot_width_dec = Decimal(str(plot_width_dec))
    if not isinstance(center_x_dec, Decimal):
        center_x_dec = Decimal(str(center_x_dec))
    if not isinstance(center_y_dec, Decimal):
        center_y_dec = Decimal(str(center_y_dec))
    arith_code = _arith_code(arith if arith is not None else DEFAULT_ARITH)
    if arith_code == abi.AP_ARITH_FAST and "One-Pass Rebasing" not in str(glitch_mode):
        raise ValueError("arith='fast' serves glitch_mode 'One-Pass Rebasing' only")
    if delta_form not in (None, "fp64", "fp32"):
        raise ValueError(f"delta_form must be 'fp64' or 'fp32', not {delta_form!r}")
    if bla_form not in (None, "reference", "accurate"):
        raise ValueError(f"bla_form must be 'reference' or 'accurate', not {bla_form!r}")
    tier = select_tier(plot_width_dec, precision_mode)
    lut = get_device_lut(cmap_name, is_hdr)
    scheme = int(color_scheme_id)
    num_bins = 65536 if scheme == 11 else 2048

    with torch.cuda.stream(st):
        fr = _DeviceFrame(W, H, is_hdr, slot, d_rgb_buf, d_iter_buf,
                          need_glitch=tier >= abi.AP_TIER_PERTURB)
        p = abi.new_params(width=W, height=H, factor=factor, max_iter=max_iter,
                           fractal_type=int(fractal_type), tier=tier, arith=arith_code,
                           gen_n=int(gen_n), gen_kr=float(gen_kr), gen_ki=float(gen_ki),
                           scheme_id=scheme, num_bins=num_bins,
                           palette_offset=float(palette_offset), color_density=float(color_density),
                           color_contrast=float(color_contrast),
                           edge_threshold=float(np.float32(edge_threshold)), is_hdr=int(bool(is_hdr)))
        if _rows is not None and tier < abi.AP_TIER_PERTURB:
            raise NotImplementedError("bands of a frame serve the perturbation tiers")
        if tier in (abi.AP_TIER_FP64, abi.AP_TIER_DD):
            for k, v in plan_direct_view(W, H, factor, center_x_dec, center_y_dec, plot_width_dec,
                                         tier, julia_cx, julia_cy).items():
                setattr(p, k, v)
            _render_direct(p, fr, lut, stream_h, scheme, factor, arith_code, num_bins, max_iter,
                           edge_threshold, slot, _extra_out)
        else:
            from . import perturbation
            perturbation.render_perturbation_frame(
                p, fr, lut, stream_h, st, W=W, H=H, factor=factor, max_iter=max_iter,
                center_x_dec=center_x_dec, center_y_dec=center_y_dec,
                plot_width_dec=plot_width_dec, tier=tier, scheme=scheme, num_bins=num_bins,
                fractal_type=int(fractal_type), julia_cx=julia_cx, julia_cy=julia_cy,
                bbsa_tol=bbsa_tol, bbsa_order=bbsa_order, glitch_mode=glitch_mode,
                gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki, edge_threshold=edge_threshold,
                slot=slot, arith_code=arith_code, extra_out=_extra_out,
                fp32_deltas=(delta_form == "fp32"),
                bla_eps=ACCURATE_BLA_EPS if bla_form == "accurate" else None, rows=_rows, orbit=_orbit)

        out = _copy_to_host(fr.rgb, h_rgb_buf, st, non_blocking=not sync_stream)
        if h_iter_buf is not None:
            _copy_to_host(fr.iter, h_iter_buf, st, non_blocking=not sync_stream)
    if sync_stream:
        st.synchronize()
    return out


def compute_bbsa_coeffs_cuda(d_ref_re, d_ref_im, ref_len, max_r, fractal_type, bbsa_tol=1e-4, bbsa_order=4,
                             gen_n=3, gen_kr=0.25, gen_ki=1.0, E_scale=0, stream=0, h_ref_re=None,
                             h_ref_im=None):
    """(skip, a1_re, a1_im, ..., a8_re, a8_im) of the series-approximation start of one
    reference orbit (math_core/engine.py:426-470): the reference's guards (types 0, 2, 4,
    positive tolerance, order and radius, ref_len >= 2; chained-BLA order 32 has no
    series), then the library's host recurrence (ap_bbsa_coeffs) on the host copy of the
    orbit (h_ref_re / h_ref_im, else a copy of the device arrays)."""
    from .perturbation import bbsa_coefficients
    zero = (0,) + (0.0,) * 16
    if fractal_type not in (0, 2, 4) or bbsa_tol <= 0.0 or bbsa_order <= 0 or ref_len < 2 or max_r <= 0.0:
        return zero
    if bbsa_order == 32:
        return zero

    def host(a):
        if a is None:
            return None
        if hasattr(a, "detach"):
            return a.detach().cpu().numpy()
        return np.asarray(a)
    re = host(h_ref_re) if h_ref_re is not None else host(d_ref_re)
    im = host(h_ref_im) if h_ref_im is not None else host(d_ref_im)
    out = bbsa_coefficients(_lib.load(), re, im, int(ref_len), float(max_r), int(fractal_type), float(bbsa_tol),
                            int(bbsa_order), int(gen_n), float(gen_kr), float(gen_ki), int(E_scale))
    return (int(out[0]),) + tuple(float(x) for x in out[1:17])


def eval_glitched_pixels_fallback_cuda(d_out_rgb, d_glitch_out, d_lut, glitched_indices, target_w, target_h,
                                       max_iter, center_x_dec, center_y_dec, plot_width_dec, plot_height_dec,
                                       color_scheme_id, fractal_type, julia_cx, julia_cy, gen_n=3, gen_kr=0.25,
                                       gen_ki=1.0, palette_offset=0.0, color_density=1.0, color_contrast=1.0,
                                       d_cdf_lut=None, num_bins=2048, cmap_name="inferno", is_hdr=False,
                                       stream=0, d_iter_map=None, stream_slot=0):
    """Re-evaluate the listed glitched pixels ((row, col) pairs) each on its own orbit and
    write their value, colour and cleared glitch flag (Strict Metric fallback of the CUDA
    path, math_core/engine.py:270-410).  Tiers as the reference picks them: FP64 at widths
    >= 1e-12, double-double >= 1e-30, 34-limb fixed point >= 1e-315 (Multibrot on the
    host), the host beyond.  With d_cdf_lut the colour is the histogram transfer.  The
    device arrays are torch CUDA tensors; d_lut None takes the registered LUT of cmap_name."""
    from .perturbation import strict_device_inputs, strict_device_tier, strict_values
    torch = _torch()
    coords = np.asarray(glitched_indices, dtype=np.int64).reshape(-1, 2).astype(np.int32)
    if len(coords) == 0:
        return
    st, stream_h = _stream_handle(stream)
    W, H = int(target_w), int(target_h)
    pw = plot_width_dec if isinstance(plot_width_dec, Decimal) else Decimal(str(plot_width_dec))
    ph = plot_height_dec if isinstance(plot_height_dec, Decimal) else Decimal(str(plot_height_dec))
    cx = center_x_dec if isinstance(center_x_dec, Decimal) else Decimal(str(center_x_dec))
    cy = center_y_dec if isinstance(center_y_dec, Decimal) else Decimal(str(center_y_dec))
    hist = d_cdf_lut is not None
    p = abi.new_params(width=W, height=H, max_iter=int(max_iter), fractal_type=int(fractal_type),
                       tier=abi.AP_TIER_FP64, arith=abi.AP_ARITH_REF_CUDA, gen_n=int(gen_n),
                       gen_kr=float(gen_kr), gen_ki=float(gen_ki), scheme_id=11 if hist else int(color_scheme_id),
                       num_bins=int(num_bins), palette_offset=float(palette_offset),
                       color_density=float(color_density), color_contrast=float(color_contrast),
                       is_hdr=int(bool(is_hdr)))
    lut = d_lut if d_lut is not None else get_device_lut(cmap_name, is_hdr)
    it = d_iter_map if d_iter_map is not None else get_scratch_device_array((H, W), np.float32,
                                                                            f"fallback_iter_{stream_slot}")
    b = abi.ApFrameBuffers()
    b.rgb, b.glitch_out, b.lut, b.iter_map = _ptr(d_out_rgb), _ptr(d_glitch_out), _ptr(lut), _ptr(it)
    b.cdf = _ptr(d_cdf_lut) if hist else None
    L = _lib.load()
    tier = strict_device_tier(pw, int(fractal_type))
    with torch.cuda.stream(st):
        dev = it.device

        def upload(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(dev, non_blocking=False)

        d_coords = upload(coords)
        if tier is None:
            values = strict_values(coords, W, H, int(max_iter), cx, cy, pw, ph, int(fractal_type), julia_cx,
                                   julia_cy, gen_n, gen_kr, gen_ki)
            d_vals = upload(values)
            q = abi.ApFrameParams.from_buffer_copy(p)
            q.arith = abi.AP_ARITH_REF_CPU  # the host evaluator colours with the CPU transfer functions
            _lib.launch(L.ap_set_pixels, C.byref(q), C.byref(b), _ptr(d_coords), _ptr(d_vals),
                        int(len(coords)), stream_h, what="ap_set_pixels")
        else:
            q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, cx, cy, pw, ph, julia_cx,
                                                         julia_cy)
            d_signs = upload(signs) if signs is not None else None
            d_limbs = upload(limbs.view(np.int32)) if limbs is not None else None
            _lib.launch(L.ap_strict_eval, C.byref(q), C.byref(b), C.byref(view), _ptr(d_coords),
                        _ptr(d_signs), _ptr(d_limbs), int(len(coords)), stream_h, what="ap_strict_eval")
        st.synchronize()


def _copy_to_host(dev, host, st, non_blocking=False):
    """Device -> host copy on stream ``st`` into ``host`` (or a new array).  With
    non_blocking and a pinned ``host`` the copy is only queued on ``st``; the caller
    synchronises the stream before reading it (sync_stream=False)."""
    torch = _torch()
    np_dt = {torch.uint8: np.uint8, torch.uint16: np.uint16, torch.float32: np.float32}[dev.dtype]
    if host is None or tuple(host.shape) != tuple(dev.shape) or host.dtype != np_dt:
        host = np.empty(tuple(dev.shape), np_dt)
    ht = torch.from_numpy(host) if host.flags.c_contiguous else None
    if ht is None:
        tmp = dev.cpu().numpy()
        host[...] = tmp
        return host
    with torch.cuda.stream(st):
        ht.copy_(dev, non_blocking=bool(non_blocking) and ht.is_pinned())
    return host


def recolor_frame(params: RenderParameters, d_iter_buf=None, h_iter_buf=None):
    """Recolour a cached iteration map without iterating (math_core/engine.py:2138-2222)."""
    torch = _torch()
    d_iter = d_iter_buf if d_iter_buf is not None else getattr(params, "d_iter_buf", None)
    h_iter = h_iter_buf if h_iter_buf is not None else getattr(params, "h_iter_buf", None)
    if params.compute_device == "CPU":
        raise NotImplementedError("this engine recolours on the GPU only (compute_device='CPU')")
    W, H = int(params.target_w), int(params.target_h)
    stream = params.stream if params.stream is not None else 0
    slot = get_stream_slot(stream, explicit_slot=getattr(params, "stream_slot", None))
    st, stream_h = _stream_handle(stream)
    with torch.cuda.stream(st):
        if d_iter is None:
            if h_iter is None:
                raise ValueError("recolor_frame needs d_iter_buf or h_iter_buf")
            d_iter = get_scratch_device_array((H, W), np.float32, f"iter_map_{slot}")
            d_iter.copy_(torch.from_numpy(np.ascontiguousarray(h_iter, np.float32)))
        fr = _DeviceFrame(W, H, params.is_hdr, slot, params.d_rgb_buf, d_iter)
        lut = get_device_lut(params.cmap_name, params.is_hdr)
        scheme = int(params.color_scheme_id)
        p = abi.new_params(width=W, height=H, max_iter=int(params.max_iter), scheme_id=scheme,
                           num_bins=65536, palette_offset=float(params.palette_offset),
                           color_density=float(params.color_density),
                           color_contrast=float(params.color_contrast),
                           is_hdr=int(bool(params.is_hdr)))
        L = _lib.load()
        cdf = None
        if scheme == 11:
            hist = get_scratch_device_array((65536,), np.int32, f"hist_bins_{slot}")
            cdf = get_scratch_device_array((65536,), np.float32, f"cdf_lut_{slot}")
            _lib.launch(L.ap_histogram_cdf, _ptr(d_iter), W, H, int(params.max_iter), 65536,
                                          _ptr(hist), _ptr(cdf), stream_h, what="ap_histogram_cdf")
        b = _buffers(fr, lut, cdf=cdf)
        _lib.launch(L.ap_colour, C.byref(p), C.byref(b), stream_h, what="ap_colour")
        out = _copy_to_host(fr.rgb, params.h_rgb_buf, st)
    if getattr(params, "sync_stream", True):
        st.synchronize()
    return out


# ---------------------------------------------------- iteration-depth helpers
def get_adaptive_max_iter_from_probe(iters_array, base_iter):
    """Depth from a probe map: max(1.35 * p98, 1.2 * max) (math_core/engine.py:1051-1060)."""
    escaped = iters_array[iters_array >= 0.0]
    if escaped.size == 0:
        return int(base_iter)
    max_escaped = float(np.max(escaped))
    p98 = float(np.percentile(escaped, 98))
    target = int(max(p98 * 1.35, max_escaped * 1.20))
    return min(GLOBAL_MAX_ITER, max(100, target))


def compute_dynamic_max_iter(base_max_iter, plot_width_dec, dynamic_mode,
                             center_x_dec=Decimal("0.0"), center_y_dec=Decimal("0.0"),
                             **probe_kwargs):
    """Dynamic iteration scaling (math_core/engine.py:1284-1323)."""
    clamped = min(GLOBAL_MAX_ITER, max(1, int(base_max_iter)))
    if dynamic_mode == "Off" or not dynamic_mode or base_max_iter <= 0:
        return clamped
    mode = str(dynamic_mode).lower()
    if "adaptive" in mode:
        try:
            return probe_adaptive_max_iter(center_x_dec=center_x_dec, center_y_dec=center_y_dec,
                                           plot_width_dec=plot_width_dec, base_iter=clamped,
                                           **probe_kwargs)
        except Exception:
            return clamped
    try:
        p = Decimal(str(plot_width_dec))
        if p <= 0 or p >= Decimal("4.0"):
            return clamped
        mantissa = float(p.scaleb(-p.adjusted()))
        depth = max(0.0, float(-p.adjusted()) + math.log10(4.0) - math.log10(max(1e-12, mantissa)))
        if "sqrt" in mode:
            mult = 1.0 + 0.85 * math.sqrt(depth)
        elif "linear" in mode or "log" in mode:
            mult = 1.0 + 0.35 * depth
        else:
            mult = 1.0
        return min(GLOBAL_MAX_ITER, max(clamped, int(round(clamped * mult))))
    except Exception:
        return clamped


def plan_probe(center_x_dec, center_y_dec, plot_width_dec, search_max, target_w=128, target_h=72,
               fractal_type=0, julia_cx=0.0, julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0,
               precision_mode="1e-300 (Perturbation)", bbsa_tol=1e-4, bbsa_order=4, arith=None):
    """Parameters of the adaptive max-iter probe's one coarse pass (host code):
    (ApFrameParams, (re, im, ref_len) of the reference orbit or None on the direct
    tiers).  math_core/engine.py:1069-1278, the probe kernels of
    math_core/cuda_kernels.py:1503-1584 and math_core/cpu_kernels.py:1024-1108.

    Pixel (i, j) samples x_min + i dx, y_max - j dy with dx = w / (W - 1): the
    view's corners are pixel centres, as on the render's grid at factor 1.  One
    sample per pixel at max_iter ``search_max``, no chained-BLA leaps, no glitch
    test, no colour; the tier is chosen as for a frame."""
    if not isinstance(plot_width_dec, Decimal):
        plot_width_dec = Decimal(str(plot_width_dec))
    if not isinstance(center_x_dec, Decimal):
        center_x_dec = Decimal(str(center_x_dec))
    if not isinstance(center_y_dec, Decimal):
        center_y_dec = Decimal(str(center_y_dec))
    W, H = int(target_w), int(target_h)
    if W < 1 or H < 1:
        raise ValueError("target_w and target_h must be positive")
    arith_code = _arith_code(arith if arith is not None else DEFAULT_ARITH)
    if arith_code == abi.AP_ARITH_FAST and "One-Pass Rebasing" not in str(glitch_mode):
        raise ValueError("arith='fast' serves glitch_mode 'One-Pass Rebasing' only")
    tier = select_tier(plot_width_dec, precision_mode)
    p = abi.new_params(width=W, height=H, factor=1, max_iter=int(search_max),
                       fractal_type=int(fractal_type), tier=tier, arith=arith_code,
                       gen_n=int(gen_n), gen_kr=float(gen_kr), gen_ki=float(gen_ki), scheme_id=0)
    if tier in (abi.AP_TIER_FP64, abi.AP_TIER_DD):
        for k, v in plan_direct_view(W, H, 1, center_x_dec, center_y_dec, plot_width_dec, tier,
                                     julia_cx, julia_cy).items():
            setattr(p, k, v)
        if tier == abi.AP_TIER_FP64:
            # the probe's FP64 spacing is a float division (math_core/engine.py:1188-1189),
            # the frame's a Decimal one rounded once: they can differ in the last bit
            with localcontext(decimal_context(plot_width_dec)):
                h_f = float(plot_width_dec * (Decimal(H) / Decimal(W)))
            p.dx_hi = float(plot_width_dec) / max(1, W - 1)
            p.dy_hi = h_f / max(1, H - 1)
        p.mode = abi.AP_MODE_COARSE
        p.flags = abi.AP_FLAG_NO_RGB | (abi.AP_FLAG_MAP_FUSED if arith_code == abi.AP_ARITH_REF_CPU else 0)
        return p, None
    from . import perturbation
    orbit = perturbation.probe_perturbation_params(
        p, W=W, H=H, search_max=int(search_max), center_x_dec=center_x_dec, center_y_dec=center_y_dec,
        plot_width_dec=plot_width_dec, tier=tier, fractal_type=int(fractal_type), julia_cx=julia_cx,
        julia_cy=julia_cy, bbsa_tol=bbsa_tol, bbsa_order=bbsa_order, gen_n=gen_n, gen_kr=gen_kr,
        gen_ki=gen_ki, arith_code=arith_code)
    return p, orbit


def probe_iter_map(center_x_dec, center_y_dec, plot_width_dec, search_max, target_w=128, target_h=72,
                   fractal_type=0, julia_cx=0.0, julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0,
                   precision_mode="1e-300 (Perturbation)", bbsa_tol=1e-4, bbsa_order=4, arith=None,
                   stream=0):
    """Smooth escape values of the adaptive max-iter probe (plan_probe's pass on the
    device), as a host float32 [target_h, target_w] array."""
    torch = _torch()
    L = _lib.load()
    p, orbit = plan_probe(center_x_dec, center_y_dec, plot_width_dec, search_max, target_w, target_h,
                          fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, precision_mode,
                          bbsa_tol, bbsa_order, arith)
    st, stream_h = _stream_handle(stream)
    b = abi.ApFrameBuffers()
    with torch.cuda.stream(st):
        d_iter = get_scratch_device_array((p.height, p.width), np.float32, "probe_iter")
        b.iter_map = _ptr(d_iter)
        if orbit is not None:
            from . import perturbation
            d_re, d_im = perturbation._upload_orbit(torch, orbit[0], orbit[1], orbit[2], 0, "probe")
            b.ref_re, b.ref_im = _ptr(d_re), _ptr(d_im)
        _lib.launch(L.ap_render_pass, C.byref(p), C.byref(b), stream_h, what="ap_render_pass")
        out = _copy_to_host(d_iter, None, st)
    st.synchronize()
    return out


def probe_adaptive_max_iter(center_x_dec, center_y_dec, plot_width_dec, base_iter,
                            target_w=128, target_h=72, fractal_type=0,
                            julia_cx=0.0, julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0,
                            precision_mode="1e-300 (Perturbation)", bbsa_tol=1e-4, bbsa_order=4,
                            compute_device="GPU", cpu_threads=2, arith=None, stream=0):
    """Iteration depth from a target_w x target_h probe (math_core/engine.py:1063-1281):
    probe_iter_map searched to max(1000, 2 base_iter), then
    get_adaptive_max_iter_from_probe.  ``arith`` selects the arithmetic profile
    ("ref_cpu" default: the values of the reference's CPU probe kernels; "ref_cuda":
    its device kernels)."""
    if compute_device == "CPU":
        raise NotImplementedError("this engine probes on the GPU only (compute_device='CPU')")
    search = min(GLOBAL_MAX_ITER, max(1000, int(base_iter * 2)))
    iters = probe_iter_map(center_x_dec, center_y_dec, plot_width_dec, search, target_w, target_h,
                           fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, precision_mode,
                           bbsa_tol, bbsa_order, arith=arith, stream=stream)
    return get_adaptive_max_iter_from_probe(iters, base_iter)
