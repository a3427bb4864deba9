"""Loader of the engine's CUDA library (fractura_b200/lib/libapeiron_b200.so).

The library is the only compute path.  If it is missing or cannot be loaded,
every entry point raises ``EngineUnavailable``; nothing falls back to the CPU.
"""
import ctypes as C
import os
import threading
from contextlib import contextmanager

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libapeiron_b200.so")

EXPORTS = (
    "ap_abi_version", "ap_last_error", "ap_render_pass", "ap_resolve_hist_pass",
    "ap_edge_detect", "ap_histogram_cdf", "ap_colour", "ap_build_bla", "ap_build_bla_dc", "ap_bbsa_coeffs", "ap_reference_orbit", "ap_reference_orbit_cert", "ap_decimal_escape", "ap_decimal_orbit", "ap_decimal_arith", "ap_decimal_to_double", "ap_glitch_bins", "ap_set_pixels", "ap_strict_eval", "ap_batch_plan", "ap_render_batch", "ap_smooth_forward", "ap_smooth_adjoint_blocks", "ap_smooth_adjoint", "ap_smooth_tangent", "ap_fma_peak_launch",
    "ap_histogram_cdf_noalloc", "ap_launch_counter", "ap_pack_orbit", "ap_pack_bla",
    "ap_pack_fe32", "ap_render_rows", "ap_histogram", "ap_cdf_from_histogram",
)


class EngineUnavailable(RuntimeError):
    """The CUDA engine library is not built or cannot be loaded."""


class EngineError(RuntimeError):
    """A C-ABI call returned an error code."""


_lib = None


def load():
    """Load and type the library (once)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineUnavailable(
            f"{LIB_PATH} is missing; build it with `python -m fractura_b200.build`")
    try:
        L = C.CDLL(LIB_PATH)
    except OSError as e:
        raise EngineUnavailable(f"cannot load {LIB_PATH}: {e}") from e
    P = C.POINTER(abi.ApFrameParams)
    B = C.POINTER(abi.ApFrameBuffers)
    vp, i32, f32, f64 = C.c_void_p, C.c_int32, C.c_float, C.c_double
    L.ap_abi_version.restype = C.c_int
    L.ap_last_error.restype = C.c_char_p
    L.ap_render_pass.argtypes = [P, B, vp]
    L.ap_resolve_hist_pass.argtypes = [P, B, vp]
    L.ap_render_rows.argtypes = [P, B, i32, i32, vp]
    L.ap_histogram.argtypes = [vp, i32, i32, i32, i32, vp, vp]
    L.ap_cdf_from_histogram.argtypes = [vp, i32, vp, vp]
    L.ap_colour.argtypes = [P, B, vp]
    L.ap_edge_detect.argtypes = [vp, vp, i32, i32, f32, vp]
    L.ap_histogram_cdf.argtypes = [vp, i32, i32, i32, i32, vp, vp, vp]
    L.ap_build_bla.argtypes = [vp, vp, i32, i32, f64, i32, i32, f64, f64, vp, vp]
    L.ap_build_bla_dc.argtypes = [vp, vp, i32, i32, f64, f64, i32, i32, f64, f64, vp, vp]
    L.ap_bbsa_coeffs.argtypes = [vp, vp, i32, f64, i32, f64, i32, i32, f64, f64, i32, vp]
    L.ap_reference_orbit.argtypes = [vp, i32, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp]
    L.ap_reference_orbit_cert.argtypes = [vp, i32, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp]
    L.ap_decimal_escape.argtypes = [vp, vp, i32, i32, i32, i32, i32, vp, vp, vp]
    L.ap_decimal_arith.argtypes = [i32, vp, vp, vp, vp, i32, vp, vp, vp]
    L.ap_decimal_orbit.argtypes = [vp, vp, i32, i32, i32, i32, i32, vp, vp, vp]
    L.ap_decimal_to_double.argtypes = [vp, vp, vp]
    L.ap_glitch_bins.argtypes = [vp, i32, i32, vp, vp]
    L.ap_set_pixels.argtypes = [P, B, vp, vp, i32, vp]
    L.ap_strict_eval.argtypes = [P, B, C.POINTER(abi.ApStrictView), vp, vp, vp, i32, vp]
    L.ap_batch_plan.argtypes = [vp, i32, i32, i32, vp]
    L.ap_smooth_forward.argtypes = [vp, vp, vp, vp, i32, vp]
    L.ap_smooth_adjoint_blocks.argtypes = [i32, i32]
    L.ap_smooth_adjoint_blocks.restype = i32
    L.ap_smooth_adjoint.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp]
    L.ap_smooth_tangent.argtypes = [vp, vp, vp]
    L.ap_render_batch.argtypes = [vp, vp, i32, i32, i32, i32, i32, i32, i32, vp, vp]
    L.ap_fma_peak_launch.argtypes = [i32, i32, i32, vp, C.POINTER(C.c_double), vp]
    L.ap_histogram_cdf_noalloc.argtypes = [vp, i32, i32, i32, i32, vp, vp]
    L.ap_launch_counter.restype = C.c_uint64
    L.ap_pack_orbit.argtypes = [vp, vp, i32, vp, vp]
    L.ap_pack_bla.argtypes = [vp, i32, i32, vp, vp, vp]
    L.ap_pack_fe32.argtypes = [vp, i32, vp, i32, vp, vp, vp]
    for name in EXPORTS:
        fn = getattr(L, name)
        if fn.restype is None:
            fn.restype = C.c_int
    if L.ap_abi_version() != abi.AP_ABI_VERSION:
        raise EngineUnavailable(
            f"library ABI {L.ap_abi_version()} != expected {abi.AP_ABI_VERSION}")
    _lib = L
    return L


def check(rc, what):
    if rc != 0:
        msg = load().ap_last_error().decode(errors="replace")
        raise EngineError(f"{what} failed ({rc}): {msg}")


def last_error():
    return load().ap_last_error().decode(errors="replace")


# ------------------------------------------------------------------ recording
# A frame's device work can be recorded while it is rendered and replayed
# later with identical arguments (bench.py times the replay: every input is
# then resident, and no host work sits between the launches).
_rec = threading.local()


class Recording:
    def __init__(self):
        self.ops = []  # (callable, args or None, what)


@contextmanager
def recording():
    rec = Recording()
    _rec.active = rec
    try:
        yield rec
    finally:
        _rec.active = None


def _snapshot(arg):
    obj = getattr(arg, "_obj", None)
    if isinstance(obj, C.Structure):
        copy = type(obj).from_buffer_copy(obj)
        return C.byref(copy)
    return arg


def launch(fn, *args, what):
    """Call a C-ABI entry point, raise on error, and record it if a recording is active."""
    check(fn(*args), what)
    rec = getattr(_rec, "active", None)
    if rec is not None:
        rec.ops.append((fn, tuple(_snapshot(a) for a in args), what))


def device_op(fn):
    """Run a device-side torch operation (copy, fill) and record it if a recording is active."""
    fn()
    rec = getattr(_rec, "active", None)
    if rec is not None:
        rec.ops.append((fn, None, "device_op"))


def replay(ops):
    for fn, args, what in ops:
        if args is None:
            fn()
        else:
            check(fn(*args), what)
