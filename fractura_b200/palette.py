"""Colour look-up tables consumed by the colouring kernels.

The reference harvests 2048-entry RGB tables from matplotlib/palettable
colormaps (color_engine.py:118-125: ``cmap(linspace(0, 1, 2048))[:, :3] * scale``
as float32, scale 255 or 65535).  Those libraries are not part of this
package; the kernels accept any float32[2048, 3] table.  ``synthetic_lut``
is the deterministic table used by the parity tests and the benchmark.
"""
import numpy as np

LUT_SIZE = 2048


def synthetic_lut(lut_size=LUT_SIZE, is_hdr=False):
    """Deterministic smooth float32[lut_size, 3] table in the reference's format."""
    t = np.arange(lut_size, dtype=np.float64) / (lut_size - 1)
    scale = 65535.0 if is_hdr else 255.0
    rgb = np.stack([
        0.5 + 0.5 * np.sin(2.0 * np.pi * (1.7 * t + 0.00)),
        0.5 + 0.5 * np.sin(2.0 * np.pi * (2.3 * t + 0.33)),
        0.5 + 0.5 * np.sin(2.0 * np.pi * (3.1 * t + 0.67)),
    ], axis=1) * scale
    return np.ascontiguousarray(rgb.astype(np.float32))


def check_lut(lut):
    """Validate a caller-supplied table: float32, C-contiguous, shape [2048, 3]."""
    lut = np.ascontiguousarray(lut, dtype=np.float32)
    if lut.shape != (LUT_SIZE, 3):
        raise ValueError(f"colour LUT must have shape ({LUT_SIZE}, 3), got {lut.shape}")
    return lut
