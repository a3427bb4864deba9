"""Multi-process plumbing on CPU (gloo, world size 2): the N > 1 path of bench.py.

* fractura_b200.dist: every rank sees the slowest rank's time and the summed
  work; the whole-job rate counts every rank's frames over the slowest time.
* bench.py --impl reference under torch.distributed.run: rank 0 alone runs the
  CPU reference arm and prints one JSON line; the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from fractura_b200 import dist as fd
        fd.barrier()
        slowest = fd.max_over_ranks(100.0 + 25.0 * rank)   # per-rank timed milliseconds
        total = fd.sum_over_ranks(1 + rank)
        rate = fd.whole_job_rate(1e9, 4, world, slowest)
        out.put((rank, slowest, total, rate, fd.active()))
        fd.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_world2_reductions():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_worker, args=(2, port, q), nprocs=2, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(2))
    for rank, slowest, total, rate, active in got:
        assert active
        assert slowest == 125.0          # both ranks see the slower rank
        assert total == 3.0
        assert rate == pytest.approx(1e9 * 4 * 2 / 0.125)


def test_whole_job_rate_single_process():
    from fractura_b200 import dist as fd
    assert not fd.active()
    assert fd.max_over_ranks(7.0) == 7.0
    assert fd.whole_job_rate(2.0, 3, 1, 1000.0) == pytest.approx(6.0)
    with pytest.raises(ValueError):
        fd.whole_job_rate(1.0, 1, 1, 0.0)


def test_reference_arm_under_torchrun_world2():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl",
           "reference", "--workload", "cfg1", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["value"] > 0


# ------------------------------------------------------------- split frames
def test_band_bounds_cover_and_balance():
    from fractura_b200.sharded import band_bounds
    for H in (1, 7, 54, 1080):
        for world in (1, 2, 3, 8):
            b = band_bounds(H, world)
            assert b[0][0] == 0 and b[-1][1] == H and len(b) == world
            assert all(b[q][1] == b[q + 1][0] for q in range(world - 1))
            sizes = [r1 - r0 for r0, r1 in b]
            assert max(sizes) - min(sizes) <= 1
    w = [10.0] * 100 + [1.0] * 900    # expensive top rows: the first band is short
    b = band_bounds(1000, 2, w)
    assert b[0][1] < 200 and b[1][0] == b[0][1]
    cost = [sum(w[r0:r1]) for r0, r1 in b]
    assert abs(cost[0] - cost[1]) <= 10.0


def test_shard_tiles_longest_first():
    from fractura_b200.sharded import shard_tiles
    costs = [5, 1, 9, 3, 3, 7, 2]
    parts = shard_tiles(costs, 3)
    assert sorted(t for p in parts for t in p) == list(range(len(costs)))
    loads = [sum(costs[t] for t in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert shard_tiles(costs, 1) == [list(range(len(costs)))]


SPLIT_VIEW = dict(W=96, H=54, factor=1, max_iter=20000, scheme=11, num_bins=65536, fractal_type=0, julia_cx=0.0,
                  julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0, bbsa_order=32, bbsa_tol=1e-6,
                  glitch_mode="One-Pass Rebasing", width="2e-159")


def _split_view():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import load_golden
    _, meta = load_golden("pert_samples.npz")
    m = next(x for x in meta if x["name"] == "cfg3")
    return dict(SPLIT_VIEW, cx=m["cx"], cy=m["cy"])


class OracleBackend:
    """The split frame's per-rank steps through the oracle (CPU): each rank evaluates
    only its own rows, at their global row indices (one-pass rebasing, dc-aware BLA)."""

    def __init__(self, arith=1, eps=1e-14):
        self.arith, self.eps = arith, eps

    def find_reference(self, view):
        from decimal import Decimal, localcontext
        import ref_orbit
        pw = Decimal(view["width"])
        with localcontext() as c:
            c.prec = ref_orbit.view_digits(pw)
            ph = pw * (Decimal(view["H"]) / Decimal(view["W"]))
        return ref_orbit.find_reference(Decimal(view["cx"]), Decimal(view["cy"]), pw, ph, view["max_iter"])

    def render_band(self, view, orbit, r0, r1):
        import numpy as np
        import torch
        from decimal import Decimal, localcontext
        import frames
        import oracle
        from fractura_b200 import abi
        W, H = view["W"], view["H"]
        bcx, bcy, u, v, re, im, rl = orbit
        pw = Decimal(view["width"])
        with localcontext() as c:
            c.prec = 500
            ph = pw * (Decimal(H) / Decimal(W))
            dx, dy = float(pw / Decimal(W - 1)), float(ph / Decimal(H - 1))
        px, py = float(W - 1) * float(u), float(H - 1) * float(v)
        T = oracle.build_bla_dc(re, im, rl, 0, self.eps, frames.max_delta_c(px, py, W, H, dx, dy), 16, 3, 0.25, 1.0)
        p = abi.new_params(width=W, height=H, max_iter=view["max_iter"], tier=abi.AP_TIER_PERTURB, arith=self.arith,
                           dx_hi=dx, dy_hi=dy, ref_px=px, ref_py=py, ref_cx=float(bcx), ref_cy=float(bcy),
                           ref_len=rl, bla_levels=16, flags=abi.AP_FLAG_REBASE | abi.AP_FLAG_NO_RGB)
        s, g, k = oracle.pert_grid(p, re[:rl + 1], im[:rl + 1], T, np.arange(W, dtype=np.float64),
                                   np.arange(r0, r1, dtype=np.float64))
        return torch.from_numpy(s)

    def probe_map(self, view, probe_w, probe_h):
        """A stand-in probe whose cost falls row by row (the upper rows four times dearer
        than the lower ones), so that probe balancing moves the band edge."""
        import numpy as np
        rows = np.linspace(4000.0, 1000.0, probe_h)[:, None]
        return np.repeat(rows, probe_w, axis=1).astype(np.float32)

    def band_histogram(self, view, it_band):
        import torch
        import oracle
        fr = oracle.Frame(it_band.shape[1], it_band.shape[0])
        fr.iter_map[...] = it_band.numpy()
        oracle.histogram_cdf(fr, view["max_iter"], view["num_bins"])
        return torch.from_numpy(fr.hist.copy())

    def cdf_from_histogram(self, view, hist):
        import numpy as np
        import torch
        h = hist.numpy().astype(np.float64)
        tot = h.sum()
        nb = len(h)
        if tot > 0:
            return torch.from_numpy((np.cumsum(h) / tot).astype(np.float32))
        return torch.from_numpy((np.arange(nb, dtype=np.float64) / (nb - 1)).astype(np.float32))

    def colour_band(self, view, it_band, cdf):
        import numpy as np
        import torch
        import oracle
        from fractura_b200 import abi
        from fractura_b200.palette import synthetic_lut
        h, w = it_band.shape
        fr = oracle.Frame(w, h, lut=synthetic_lut())
        fr.iter_map[...] = it_band.numpy()
        if cdf is not None:
            fr.cdf = np.ascontiguousarray(cdf.numpy())
        p = abi.new_params(width=w, height=h, max_iter=view["max_iter"], scheme_id=view["scheme"],
                           num_bins=view["num_bins"], arith=self.arith)
        oracle.colour(p, fr)
        return torch.from_numpy(fr.rgb.copy())


def _split_worker(rank, world, port, outdir, balance=None):
    import datetime

    import torch.distributed as dist
    for d in ("oracle", "tests"):
        sys.path.insert(0, os.path.join(ROOT, d))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import oracle
        from fractura_b200 import sharded
        oracle.set_threads(1)
        rgb, it = sharded.render_split(_split_view(), OracleBackend(), balance=balance)
        import numpy as np
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), rgb=rgb.numpy(), it=it.numpy())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("balance", [None, "probe"])
def test_split_frame_world2_equals_single_frame(tmp_path, balance):
    """One frame shared out over two gloo ranks by row bands (orbit broadcast from rank 0,
    band histograms all-reduced before the CDF, bands all-gathered; even bands or bands
    balanced by rank 0's probe) equals the frame the oracle renders in one process, bit
    for bit, on both ranks."""
    import numpy as np
    for d in ("oracle", "tests"):
        sys.path.insert(0, os.path.join(ROOT, d))
    import frames
    from fractura_b200 import abi
    port = _free_port()
    mp.start_processes(_split_worker, args=(2, port, str(tmp_path), balance), nprocs=2, join=True,
                       start_method="spawn")
    got = []
    for rank in range(2):
        d = np.load(tmp_path / f"rank{rank}.npz")
        got.append((rank, d["rgb"], d["it"]))
    # CUDA profile: its histogram frames leap (the CPU profile's do not, as the reference)
    fr, passes = frames.pert_frame(_split_view(), arith=abi.AP_ARITH_REF_CUDA, bla_eps=1e-14)
    assert passes == 0
    for rank, rgb, it in got:
        assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), rank
        assert np.array_equal(rgb, fr.rgb), rank


def test_probe_costs_and_row_weights():
    """Probe costs (escape step; max_iter when bounded) and their mapping to frame rows,
    and the bands and tile costs they give."""
    import numpy as np
    from fractura_b200 import sharded
    c = sharded.costs_from_probe(np.array([[-1.0, 0.0, 10.5]]), 100)
    assert np.array_equal(c, [[100.0, 1.0, 10.5]])
    pc = np.array([[1.0, 1.0], [2.0, 2.0], [3.0, 3.0]])
    w = sharded.row_weights(pc, 5)   # probe rows at frame rows 0, 2, 4
    assert np.array_equal(w, [2.0, 2.0, 4.0, 6.0, 6.0])
    assert np.array_equal(sharded.row_weights(pc, 1), [4.0])
    view = {"H": 90, "max_iter": 1000}
    wt = sharded.probe_row_weights(view, OracleBackend().probe_map)
    bands = sharded.band_bounds(90, 2, wt)
    assert bands[0][1] < 45 and bands[0][0] == 0 and bands[1][1] == 90   # the dear upper rows go to rank 0
    lo, hi = wt[:bands[0][1]].sum(), wt[bands[0][1]:].sum()
    assert abs(lo - hi) <= wt.max()

    class T:
        def __init__(self, W, H, mi):
            self.W, self.H, self.max_iter = W, H, mi
    tiles = [T(64, 64, 1000), T(32, 32, 1000), T(64, 64, 50)]
    probe = lambda t, w, h: np.full((h, w), -1.0 if t.max_iter == 50 else 10.0, np.float32)
    cost = sharded.probe_tile_costs(tiles, probe, 8, 8)
    assert cost == [10.0 * 64 * 64, 10.0 * 32 * 32, 50.0 * 64 * 64]
    assert sharded.shard_tiles(cost, 2) == [[2], [0, 1]]   # the bounded tile is the dearest
