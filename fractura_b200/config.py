"""Render parameters and tier constants of the reference engine's boundary.

Mirrors the parts of the reference's config.py that sit on the escape-time
path: ``RenderParameters`` (config.py:196-243), the precision helpers
(config.py:36-74), the option tables (config.py:78-143) and the bailout
constants (config.py:25-26).  UI helpers of that module are not part of
this package.

Unlike the reference, importing this module does not change the process-wide
``decimal`` context; the engine computes in local contexts of at least the
reference's 500 digits.
"""
import decimal
from dataclasses import asdict, dataclass
from decimal import Decimal

GLOBAL_MAX_ITER = 500_000_000
DEFAULT_MAX_ITER = 500
DECIMAL_PREC = 500

INV_LN2_F32 = 1.4426950408889634     # 1 / ln 2
LN_BAILOUT_LOG = 1.7129177284488854  # ln(0.5 * ln 65536) = ln(8 ln 2)

FRACTAL_NAMES = [
    "Mandelbrot",
    "Burning Ship",
    "Julia Set (Mandelbrot)",
    "Julia Set (Burning Ship)",
    "General Mandelbrot",
]

COLOR_SCHEMES = {
    "Sqrt Fold": 0, "Logarithmic": 1, "Sigmoidal Tanh": 2, "Exponential Flare": 3,
    "High-Frequency Ripples": 4, "Golden Ratio Dual Sine": 5, "Cosine Smooth": 6,
    "Harmonic Cascade": 7, "Quintic S-Curve": 8, "Chirp Sweep": 9, "Soft Damping": 10,
    "Histogram Equalized": 11,
}

PRECISION_OPTIONS = {
    "1e-12 (FP64)": Decimal("1e-12"),
    "1e-24 (DD)": Decimal("1e-24"),
    "1e-300 (Perturbation)": Decimal("1e-300"),
    "1e-10000+ (Floatexp)": Decimal("1e-646000000"),
}

BBSA_OPTIONS = {
    "Off": {"order": 0, "tol": 0.0},
    "4th-order": {"order": 4, "tol": 1e-4},
    "8th-order": {"order": 8, "tol": 1e-4},
    "Chained BLA": {"order": 32, "tol": 1e-6},
}

GLITCH_CORRECTION_MODES = ["Off (Single-Ref)", "Pauldelbrot", "Strict Metric"]

DYNAMIC_ITER_MODES = ["Off", "On (Sqrt Scaling)", "On (Linear Scaling)", "On (Adaptive Preview)"]

# Per-step tolerance of the "accurate" chained-BLA form: the dropped quadratic term
# of a leap stays within ~1e-14 of the linear one, i.e. at FP64 rounding level, so
# leaps change smooth values no more than FP64 rounding of the skipped steps does.
ACCURATE_BLA_EPS = 1e-14

# Arithmetic profiles (see include/apeiron_b200.h): which multiply-adds are fused.
ARITH_PROFILES = {"ref_cpu": 0, "ref_cuda": 1, "fast": 2}


def decimal_context(plot_width_dec=None, extra_digits=150):
    """A local Decimal context with the precision the reference would be using.

    The reference raises the global precision to max(500, digits + 150) for
    deep views (config.py:63-74); the same rule applies here, locally.
    """
    prec = DECIMAL_PREC
    if plot_width_dec is not None:
        try:
            p = Decimal(str(plot_width_dec))
            if p > 0:
                prec = max(prec, -int(p.adjusted()) + extra_digits)
        except (decimal.InvalidOperation, ValueError):
            pass
    ctx = decimal.Context(prec=prec)
    return ctx


def compute_required_prec_bits(plot_width_dec):
    """Orbit precision in bits: floor(digits * log2(10)) + 128, at least 64 (config.py:36-48)."""
    try:
        p = Decimal(str(plot_width_dec))
        if p > 0:
            adj = -int(p.adjusted())
            return max(64, int(adj * 3.321928094887362) + 128)
        return 256
    except Exception:
        return 256


def compute_floatexp_scale(plot_width_dec):
    """Base-2 exponent E with delta_c * 2^E = O(1) (config.py:51-60)."""
    try:
        p = Decimal(str(plot_width_dec))
        if p <= 0:
            return 0
        return max(0, int(-p.adjusted() * 3.32192809488736235))
    except Exception:
        return 0


@dataclass
class RenderParameters:
    """Frame description accepted by render_frame (config.py:196-243)."""
    target_w: int = 1280
    target_h: int = 720
    max_iter: int = 1000
    center_x_dec: Decimal = Decimal("-0.75")
    center_y_dec: Decimal = Decimal("0.0")
    plot_width_dec: Decimal = Decimal("4.0")
    cmap_name: object = "inferno"
    ssaa_factor: int = 1
    edge_threshold: float = 0.35
    color_scheme_id: int = 0
    precision_mode: str = "1e-300 (Perturbation)"
    fractal_type: int = 0
    julia_cx: float = 0.0
    julia_cy: float = 0.0
    bbsa_tol: float = 1e-4
    bbsa_order: int = 4
    glitch_mode: str = "Off (Single-Ref)"
    gen_n: int = 3
    gen_kr: float = 0.25
    gen_ki: float = 1.0
    d_rgb_buf: object = None
    h_rgb_buf: object = None
    stream: object = 0
    is_hdr: bool = False
    compute_device: str = "GPU"
    cpu_threads: int = 2
    palette_offset: float = 0.0
    color_density: float = 1.0
    color_contrast: float = 1.0
    sync_stream: bool = True
    cancel_token: object = None
    d_iter_buf: object = None
    h_iter_buf: object = None
    stream_slot: int = 0
    # Engine options (no counterpart in the reference): arithmetic profile of the FP64
    # tiers ("ref_cpu" / "ref_cuda") and the perturbation delta form ("fp64" / "fp32").
    arith: str = "ref_cpu"
    delta_form: str = "fp64"
    # Chained-BLA table: "reference" (the reference's merge at bbsa_tol) or
    # "accurate" (dc-aware merge at ACCURATE_BLA_EPS).
    bla_form: str = "reference"

    def to_dict(self):
        return asdict(self)

    def as_dict(self):
        return asdict(self)

    def __getitem__(self, item):
        return getattr(self, item)

    def get(self, key, default=None):
        return getattr(self, key, default)
