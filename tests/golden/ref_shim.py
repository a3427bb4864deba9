"""Import shim for the reference implementation (fixture generation only).

The reference's ``color_engine`` needs matplotlib and PyQt5 at import time
(color_engine.py:3-6), which are absent; a stub module that serves the
package's synthetic LUT is placed in ``sys.modules`` first.  gmpy2 is absent
too, so the reference computes orbits with its in-tree Decimal fallback
(math_core/high_precision.py:802-873).  Only ``make_golden.py`` imports this.
"""
import os
import sys
import types

REF_ROOT = os.environ.get("APEIRON_REFERENCE_ROOT")
if not REF_ROOT:
    raise SystemExit("set APEIRON_REFERENCE_ROOT to the reference's source tree (the directory that holds "
                     "config.py and math_core/) to regenerate fixtures")
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fractura_b200.palette import synthetic_lut  # noqa: E402


def install():
    if REF_ROOT not in sys.path:
        sys.path.insert(0, REF_ROOT)
    stub = types.ModuleType("color_engine")
    stub.get_cpu_cmap_lut = lambda cmap_name=None, lut_size=2048, is_hdr=False: synthetic_lut(lut_size, is_hdr)
    stub.get_gpu_cmap_lut = stub.get_cpu_cmap_lut
    sys.modules["color_engine"] = stub
    import config  # noqa: F401
    from math_core import cpu_kernels, engine, high_precision
    return types.SimpleNamespace(config=config, ck=cpu_kernels, engine=engine, hp=high_precision)
