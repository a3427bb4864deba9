"""Host logic of the export pipelines: mosaic tile views and which mosaics the batch
kernel serves (workers/image_workers.py:468-515)."""
from decimal import Decimal, localcontext

import pytest

from fractura_b200.config import decimal_context
from fractura_b200.pipeline import batch_serves, mosaic_views, _DEFAULTS


def test_mosaic_views_tile_the_canvas():
    cx, cy, w = Decimal("-0.743643887037158704752191506114774"), Decimal("0.131825904205311970493132056385139"), \
        Decimal("3.2e-30")
    n, W, H = 3, 160, 90
    v = mosaic_views(cx, cy, w, n, W, H)
    assert [(r, c) for r, c, *_ in v] == [(r, c) for r in range(n) for c in range(n)]
    with localcontext(decimal_context(w)):
        tw = w / n
        th = (w * (Decimal(H) / Decimal(W))) / n
        assert all(t[4] == tw for t in v)
        eps = w * Decimal("1e-40")        # far below a pixel: the views agree to the context's precision

        def close(a, b):
            return abs(a - b) <= eps
        # the centre tile of an odd grid is the canvas centre; neighbours are one tile apart
        mid = v[n * (n // 2) + n // 2]
        assert close(mid[2], cx) and close(mid[3], cy)
        assert close(v[1][2] - v[0][2], tw)
        assert close(v[0][3] - v[n][3], th)
        # the tiles' union is the canvas: left edge of column 0, top edge of row 0
        assert close(v[0][2] - tw / 2, cx - w / 2)
        assert close(v[0][3] + th / 2, cy + w * Decimal(H) / Decimal(W) / 2)


def test_mosaic_views_reject_empty_grid():
    with pytest.raises(ValueError):
        mosaic_views(Decimal(0), Decimal(0), Decimal(1), 0, 16, 16)


@pytest.mark.parametrize("change,served", [
    ({}, False),                                                    # default: series start of order 4
    ({"bbsa_order": 32}, True),
    ({"bbsa_order": 0}, True),
    ({"bbsa_order": 32, "glitch_mode": "Off (Single-Ref)"}, True),
    ({"bbsa_order": 32, "glitch_mode": "One-Pass Rebasing"}, True),
    ({"bbsa_order": 32, "glitch_mode": "One-Pass Rebasing", "fractal_type": 2}, False),
    ({"bbsa_order": 32, "glitch_mode": "Pauldelbrot"}, False),
    ({"bbsa_order": 32, "ssaa_factor": 2}, False),
    ({"bbsa_order": 32, "arith": "ref_cuda"}, True),
    ({"bbsa_order": 32, "arith": "fast", "glitch_mode": "One-Pass Rebasing"}, False),
    ({"bbsa_order": 32, "delta_form": "fp32"}, True),
    ({"bbsa_order": 32, "delta_form": "fp32", "glitch_mode": "One-Pass Rebasing", "fractal_type": 1}, True),
    ({"bbsa_order": 32, "delta_form": "fp64x"}, False),
])
def test_batch_serves(change, served):
    kw = dict(_DEFAULTS, **change)
    assert batch_serves(Decimal("1e-20"), kw) is served
    assert batch_serves(Decimal("1e-10"), kw) is False        # FP64 tier
    assert batch_serves(Decimal("1e-310"), kw) is False       # FloatExp tier
