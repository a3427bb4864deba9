"""ctypes mirror of include/apeiron_b200.h (the engine's C ABI).

The field order and types must match the header exactly; ``check_layout``
compares the sizes against the library's own ``sizeof`` report.
"""
import ctypes as C

AP_ABI_VERSION = 7

AP_OK = 0
AP_E_INVALID = -1
AP_E_CUDA = -2
AP_E_UNSUPPORTED = -3

AP_TIER_FP64 = 0
AP_TIER_DD = 1
AP_TIER_PERTURB = 2
AP_TIER_FLOATEXP = 3
AP_TIER_FLOATEXP32 = 4

AP_ARITH_REF_CPU = 0
AP_ARITH_REF_CUDA = 1
AP_ARITH_FAST = 2

AP_MODE_COARSE = 0
AP_MODE_FULL = 1
AP_MODE_EDGE = 2

AP_FLAG_NO_RGB = 1
AP_FLAG_ESCAPE_GLITCH = 2
AP_FLAG_NAN_GUARD = 4
AP_FLAG_ITER_LAST_SUB = 8
AP_FLAG_MAP_FUSED = 16
AP_FLAG_HIST_COLOUR = 32
AP_FLAG_REBASE = 64


class ApFrameParams(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32),
        ("factor", C.c_int32), ("max_iter", C.c_int32),
        ("fractal_type", C.c_int32), ("tier", C.c_int32),
        ("arith", C.c_int32), ("mode", C.c_int32),
        ("flags", C.c_uint32), ("gen_n", C.c_int32),
        ("x_min_hi", C.c_double), ("x_min_lo", C.c_double),
        ("y_max_hi", C.c_double), ("y_max_lo", C.c_double),
        ("dx_hi", C.c_double), ("dx_lo", C.c_double),
        ("dy_hi", C.c_double), ("dy_lo", C.c_double),
        ("julia_cx_hi", C.c_double), ("julia_cx_lo", C.c_double),
        ("julia_cy_hi", C.c_double), ("julia_cy_lo", C.c_double),
        ("gen_kr", C.c_double), ("gen_ki", C.c_double),
        ("ref_px", C.c_double), ("ref_py", C.c_double),
        ("ref_cx", C.c_double), ("ref_cy", C.c_double),
        ("ref_len", C.c_int32), ("e_scale", C.c_int32),
        ("bla_levels", C.c_int32), ("strict_glitch", C.c_int32),
        ("rebase_pass", C.c_int32), ("bbsa_skip", C.c_int32),
        ("bbsa_inv_r", C.c_double),
        ("bbsa", C.c_double * 16),
        ("scheme_id", C.c_int32), ("num_bins", C.c_int32),
        ("palette_offset", C.c_double), ("color_density", C.c_double),
        ("color_contrast", C.c_double),
        ("edge_threshold", C.c_float), ("is_hdr", C.c_int32),
    ]


class ApFrameBuffers(C.Structure):
    _fields_ = [
        ("ref_re", C.c_void_p), ("ref_im", C.c_void_p),
        ("bla", C.c_void_p), ("lut", C.c_void_p), ("cdf", C.c_void_p),
        ("glitch_in", C.c_void_p), ("edge_mask", C.c_void_p),
        ("iter_map", C.c_void_p), ("rgb", C.c_void_p),
        ("glitch_out", C.c_void_p), ("kmap", C.c_void_p), ("s64", C.c_void_p),
        ("counters", C.c_void_p),
        ("orbit_packed", C.c_void_p), ("bla_packed", C.c_void_p),
    ]


class ApTileDesc(C.Structure):
    _fields_ = [
        ("p", ApFrameParams),
        ("orbit_packed", C.c_void_p), ("bla_packed", C.c_void_p),
        ("iter_map", C.c_void_p), ("kmap", C.c_void_p), ("s64", C.c_void_p),
        ("glitch_out", C.c_void_p), ("counters", C.c_void_p), ("reserved", C.c_int64),
    ]


class ApGradView(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("max_iter", C.c_int32),
        ("fractal_type", C.c_int32), ("gen_n", C.c_int32), ("ckpt_every", C.c_int32),
        ("cx", C.c_double), ("cy", C.c_double), ("w", C.c_double), ("pr", C.c_double),
        ("pi", C.c_double),
    ]


AP_STRICT_DD = 1
AP_STRICT_LIMBS = 2
AP_STRICT_FP64 = 3
AP_STRICT_NLIMBS = 34


class ApStrictView(C.Structure):
    _fields_ = [
        ("tier", C.c_int32), ("jx_sign", C.c_int32), ("jy_sign", C.c_int32),
        ("reserved", C.c_int32),
        ("jx_limbs", C.c_uint32 * AP_STRICT_NLIMBS), ("jy_limbs", C.c_uint32 * AP_STRICT_NLIMBS),
    ]


def new_params(**kw):
    """ApFrameParams with neutral defaults (factor 1, density/contrast 1)."""
    p = ApFrameParams()
    p.factor = 1
    p.color_density = 1.0
    p.color_contrast = 1.0
    p.num_bins = 65536
    p.gen_n = 3
    p.gen_kr = 0.25
    p.gen_ki = 1.0
    p.edge_threshold = 0.35
    for k, v in kw.items():
        if k == "bbsa":
            for q, x in enumerate(v):
                p.bbsa[q] = float(x)
        else:
            setattr(p, k, v)
    return p
