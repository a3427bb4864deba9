"""ctypes front end of the CPU oracle (test infrastructure only).

Loads oracle/_build/libap_oracle.so (built by ``make -C oracle``) and exposes
numpy-level helpers.  Only the tests, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py use this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from fractura_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libap_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _stale():
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(HERE, "ap_oracle.c"), os.path.join(HERE, "Makefile"),
            os.path.join(os.path.dirname(HERE), "include", "apeiron_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def lib():
    global _lib
    if _lib is None:
        if _stale():
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(abi.ApFrameParams)
        B = C.POINTER(abi.ApFrameBuffers)
        L.apo_render_pass.argtypes = [P, B]
        L.apo_resolve_hist_pass.argtypes = [P, B]
        L.apo_colour.argtypes = [P, B]
        L.apo_set_pixels.argtypes = [P, B, C.c_void_p, C.c_void_p, C.c_int]
        L.apo_strict_eval.argtypes = [P, B, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.apo_edge_detect.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float]
        L.apo_histogram_cdf.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p]
        L.apo_fp64_grid.argtypes = [P, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
        L.apo_set_threads.argtypes = [C.c_int]
        L.apo_sample_grid.argtypes = [P, B, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.c_void_p]
        L.apo_pert_grid.argtypes = [P, B, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_void_p]
        L.apo_build_bla.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                    C.c_int, C.c_double, C.c_double, C.c_void_p]
        L.apo_build_bla_dc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double,
                                       C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_void_p]
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with code {rc}")


def set_threads(n):
    lib().apo_set_threads(int(n))


def fp64_grid(params, xs, ys):
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    H, W = len(ys), len(xs)
    s32 = np.empty((H, W), np.float32)
    s64 = np.empty((H, W), np.float64)
    k = np.empty((H, W), np.int32)
    _check(lib().apo_fp64_grid(C.byref(params), ptr(xs), ptr(ys), W, H, ptr(s32), ptr(s64), ptr(k)),
           "fp64_grid")
    return s32, s64, k


def sample_grid(params, xs, ys):
    """Samples of the direct tiers (FP64, double-double) at sub-sample coordinates xs
    (columns) x ys (rows), mapped as the unified pass maps them.  Returns (s64, k)."""
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    H, W = len(ys), len(xs)
    s64 = np.empty((H, W), np.float64)
    k = np.empty((H, W), np.int32)
    b = abi.ApFrameBuffers()
    _check(lib().apo_sample_grid(C.byref(params), C.byref(b), ptr(xs), ptr(ys), W, H, ptr(s64), ptr(k)),
           "sample_grid")
    return s64, k


def pert_grid(params, ref_re, ref_im, bla, xs, ys, with_s64=False):
    """Perturbation samples at sub-sample coordinates xs (columns) x ys (rows).

    Returns (s float32, glitch, k) and, with ``with_s64``, the float64 smooth value too.
    """
    re = np.ascontiguousarray(ref_re, np.float64)
    im = np.ascontiguousarray(ref_im, np.float64)
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    b = abi.ApFrameBuffers()
    b.ref_re, b.ref_im = ptr(re), ptr(im)
    if bla is not None:
        bla = np.ascontiguousarray(bla, np.float64)
        b.bla = ptr(bla)
    H, W = len(ys), len(xs)
    s = np.empty((H, W), np.float32)
    g = np.empty((H, W), np.uint8)
    k = np.empty((H, W), np.int32)
    s64 = np.empty((H, W), np.float64)
    b.s64 = ptr(s64)
    _check(lib().apo_pert_grid(C.byref(params), C.byref(b), ptr(xs), ptr(ys), W, H, ptr(s), ptr(g),
                               ptr(k)), "pert_grid")
    if with_s64:
        return s, g, k, s64
    return s, g, k


def build_bla_dc(ref_re, ref_im, ref_len, fractal_type, eps, dc_max, levels, gen_n, gen_kr, gen_ki):
    T = np.zeros((levels, ref_len, 5), np.float64)
    _check(lib().apo_build_bla_dc(ptr(np.ascontiguousarray(ref_re, np.float64)),
                                  ptr(np.ascontiguousarray(ref_im, np.float64)), int(ref_len),
                                  int(fractal_type), float(eps), float(dc_max), int(levels), int(gen_n),
                                  float(gen_kr), float(gen_ki), ptr(T)), "build_bla_dc")
    return T


def build_bla(ref_re, ref_im, ref_len, fractal_type, tol, levels, gen_n, gen_kr, gen_ki):
    T = np.zeros((levels, ref_len, 5), np.float64)
    _check(lib().apo_build_bla(ptr(np.ascontiguousarray(ref_re, np.float64)),
                               ptr(np.ascontiguousarray(ref_im, np.float64)), int(ref_len),
                               int(fractal_type), float(tol), int(levels), int(gen_n), float(gen_kr),
                               float(gen_ki), ptr(T)), "build_bla")
    return T


class Frame:
    """Host buffers of one frame, laid out as ApFrameBuffers expects."""

    def __init__(self, W, H, is_hdr=False, lut=None):
        self.W, self.H = W, H
        self.iter_map = np.zeros((H, W), np.float32)
        self.rgb = np.zeros((H, W, 3), np.uint16 if is_hdr else np.uint8)
        self.glitch_out = np.zeros((H, W), np.uint8)
        self.glitch_in = np.zeros((H, W), np.uint8)
        self.edge = np.zeros((H, W), np.uint8)
        self.kmap = np.zeros((H, W), np.int32)
        self.s64 = np.zeros((H, W), np.float64)
        self.cdf = None
        self.hist = None
        self.lut = lut
        self.ref_re = self.ref_im = self.bla = None

    def buffers(self):
        b = abi.ApFrameBuffers()
        b.ref_re, b.ref_im, b.bla = ptr(self.ref_re), ptr(self.ref_im), ptr(self.bla)
        b.lut, b.cdf = ptr(self.lut), ptr(self.cdf)
        b.glitch_in, b.edge_mask = ptr(self.glitch_in), ptr(self.edge)
        b.iter_map, b.rgb, b.glitch_out = ptr(self.iter_map), ptr(self.rgb), ptr(self.glitch_out)
        b.kmap, b.s64 = ptr(self.kmap), ptr(self.s64)
        return b


def render_pass(params, fr):
    _check(lib().apo_render_pass(C.byref(params), C.byref(fr.buffers())), "render_pass")


def resolve_hist_pass(params, fr):
    _check(lib().apo_resolve_hist_pass(C.byref(params), C.byref(fr.buffers())), "resolve_hist_pass")


def colour(params, fr):
    _check(lib().apo_colour(C.byref(params), C.byref(fr.buffers())), "colour")


def strict_eval(params, fr, view, coords, signs=None, limbs=None):
    """Device-tier Strict Metric re-evaluation of the listed pixels (apo_strict_eval);
    ``view`` is an abi.ApStrictView."""
    coords = np.ascontiguousarray(coords, np.int32)
    signs = None if signs is None else np.ascontiguousarray(signs, np.int32)
    limbs = None if limbs is None else np.ascontiguousarray(limbs, np.uint32)
    _check(lib().apo_strict_eval(C.byref(params), C.byref(fr.buffers()), C.byref(view), ptr(coords),
                                 ptr(signs), ptr(limbs), int(len(coords))), "strict_eval")


def set_pixels(params, fr, coords, values):
    """Strict Metric write-back of the listed (row, col) pixels (apo_set_pixels)."""
    coords = np.ascontiguousarray(coords, np.int32)
    values = np.ascontiguousarray(values, np.float64)
    _check(lib().apo_set_pixels(C.byref(params), C.byref(fr.buffers()), ptr(coords), ptr(values),
                                int(len(values))), "set_pixels")


def edge_detect(fr, threshold):
    _check(lib().apo_edge_detect(ptr(fr.iter_map), ptr(fr.edge), fr.W, fr.H, float(threshold)),
           "edge_detect")


def histogram_cdf(fr, max_iter, num_bins=65536):
    fr.hist = np.zeros(num_bins, np.int32)
    fr.cdf = np.zeros(num_bins, np.float32)
    _check(lib().apo_histogram_cdf(ptr(fr.iter_map), fr.W, fr.H, int(max_iter), int(num_bins),
                                   ptr(fr.hist), ptr(fr.cdf)), "histogram_cdf")
