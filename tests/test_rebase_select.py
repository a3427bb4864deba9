"""Rebase-pixel choice from device cell counts equals the choice on the whole maps.

fractura_b200.perturbation.select_rebase_pixel_binned reads the 16 x 16 cell
counts and then only the cells it inspects; select_rebase_pixel
(math_core/engine.py:1923-1992 restated) reads the whole glitch and smooth maps.
Seeded maps with sparse and dense glitches, interior pixels, ties between
cells, visited pixels and frames whose every glitched pixel is visited.
"""
import numpy as np
import pytest

from fractura_b200.perturbation import select_rebase_pixel, select_rebase_pixel_binned


def _counts(g, W, H):
    gi = np.argwhere(g > 0)
    b = np.clip((gi[:, 0] * 16) // H, 0, 15) * 16 + np.clip((gi[:, 1] * 16) // W, 0, 15)
    return np.bincount(b, minlength=256)


def _fetchers(g, it, log):
    def cell(r0, r1, c0, c1):
        log.append((r0, r1, c0, c1))
        return g[r0:r1, c0:c1], it[r0:r1, c0:c1]

    def whole():
        log.append("all")
        return g, it
    return cell, whole


@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("shape", [(1080, 1920), (90, 160), (37, 53), (17, 16)])
def test_binned_choice_equals_full_map(seed, shape):
    H, W = shape
    rng = np.random.default_rng(seed * 100 + H)
    density = [0.994, 0.3, 0.01, 0.0005][seed % 4]
    g = (rng.random((H, W)) < density).astype(np.uint8)
    it = (8000 + 40 * rng.random((H, W))).astype(np.float32)
    it[rng.random((H, W)) < 0.05] = -1.0           # interior pixels
    it[rng.random((H, W)) < 0.01] = 200000.0       # at max_iter
    visited = set()
    for _ in range(5):                              # successive passes
        log = []
        cell, whole = _fetchers(g, it, log)
        a = select_rebase_pixel(g, it, 200000, visited, W, H)
        b = select_rebase_pixel_binned(_counts(g, W, H), cell, whole, 200000, visited, W, H)
        assert a == b
        if a is None:
            break
        if density > 0.1 and H * W > 10000:
            assert "all" not in log and len(log) == 1   # one cell fetched
        visited.add(a)


def test_every_glitched_pixel_visited():
    H, W = 20, 30
    g = np.zeros((H, W), np.uint8)
    g[3, 4] = g[15, 25] = 1
    it = np.full((H, W), 100.0, np.float32)
    visited = {(3, 4), (15, 25)}
    log = []
    cell, whole = _fetchers(g, it, log)
    assert select_rebase_pixel(g, it, 1000, visited, W, H) is None
    assert select_rebase_pixel_binned(_counts(g, W, H), cell, whole, 1000, visited, W, H) is None
    assert "all" in log
    assert select_rebase_pixel_binned(np.zeros(256, np.int64), cell, whole, 1000, set(), W, H) is None
