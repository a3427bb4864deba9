"""GPU parity of the perturbation tier (FP64 deltas, chained BLA, Pauldelbrot rebasing)."""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, engine
from fractura_b200 import high_precision as hp
from helpers import load_golden, oracle_pert_frame, rgb_mismatch

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")
RS, RMETA = load_golden("render_pert.npz")


@pytest.mark.parametrize("name", [m["name"] for m in PMETA if m["bla_shape"][0] > 1])
def test_device_bla_table_matches_oracle(name):
    import torch
    m = next(x for x in PMETA if x["name"] == name)
    re, im = PS[name + "__re"], PS[name + "__im"]
    rl = m["ref_len"]
    d_re = torch.from_numpy(re).cuda()
    d_im = torch.from_numpy(im).cuda()
    out = torch.empty((16, rl, 5), dtype=torch.float64, device="cuda")
    L = _lib.load()
    _lib.check(L.ap_build_bla(C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr()), rl,
                              m["fractal_type"], 1e-6, 16, m["gen_n"], m["gen_kr"], m["gen_ki"],
                              C.c_void_p(out.data_ptr()), None), "ap_build_bla")
    T = oracle.build_bla(re, im, rl, m["fractal_type"], 1e-6, 16, m["gen_n"], m["gen_kr"], m["gen_ki"])
    got = out.cpu().numpy()
    if m["fractal_type"] == 4 and m["gen_n"] > 3:
        # x_max = tol_a^(1/(n-1)) goes through pow(); CUDA's and glibc's pow may differ by an ulp
        assert np.array_equal(got[..., :4], T[..., :4])
        assert np.allclose(got[..., 4], T[..., 4], rtol=1e-15, atol=0)
    else:
        assert got.tobytes() == T.tobytes()


@pytest.mark.parametrize("variant", ["plain", "bla"])
def test_config3_full_frame_matches_reference_samples(variant):
    """1920x1080 frame at the 1e-160 view (one pass, no rebase) against the reference's
    per-sample values (cpu_compute_perturbation_sample) on every 40th pixel."""
    m = next(x for x in PMETA if x["name"] == "cfg3")
    hp.clear_reference_orbit_cache()
    it = np.zeros((m["H"], m["W"]), np.float32)
    engine.render_frame_ssaa(m["W"], m["H"], m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]),
                             Decimal(m["width"]), None, color_scheme_id=0,
                             precision_mode="1e-300 (Perturbation)", fractal_type=0,
                             bbsa_tol=1e-6, bbsa_order=32 if variant == "bla" else 0,
                             glitch_mode="Off (Single-Ref)", h_iter_buf=it)
    st = m["stride"]
    ref = PS[f"cfg3__{variant}_s"]
    assert np.array_equal(it[::st, ::st].view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("name", [m["name"] for m in RMETA])
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
def test_pert_frame_with_rebasing(name, arith):
    import torch
    m = next(x for x in RMETA if x["name"] == name)
    W, H = m["W"], m["H"]
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        ssaa_factor=m["factor"], color_scheme_id=m["scheme"], precision_mode="1e-300 (Perturbation)",
        fractal_type=m["fractal_type"], julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        bbsa_tol=1e-6 if m["bbsa_order"] == 32 else 0.0, bbsa_order=m["bbsa_order"],
        glitch_mode=m["glitch_mode"], gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
        h_iter_buf=it, arith=arith, _extra_out=(kmap, s64))
    code = 0 if arith == "ref_cpu" else 1
    fr, _ = oracle_pert_frame(m, arith=code)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)
    if arith == "ref_cpu" and name != "cfg3_hist_ssaa2":
        assert np.array_equal(it.view(np.uint32), RS[name + "__iter"].view(np.uint32))


def test_packed_orbit_and_bla_layouts():
    """ap_pack_orbit / ap_pack_bla records hold exactly what the per-step code computes."""
    import torch
    m = next(x for x in PMETA if x["name"] == "cfg3")
    re, im, rl = PS["cfg3__re"], PS["cfg3__im"], m["ref_len"]
    L = _lib.load()
    d_re, d_im = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    po = torch.empty((rl + 1, 4), dtype=torch.float64, device="cuda")
    _lib.check(L.ap_pack_orbit(C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr()), rl,
                               C.c_void_p(po.data_ptr()), None), "ap_pack_orbit")
    got = po.cpu().numpy()
    r2 = re * re + im * im
    assert np.array_equal(got[:, 0], re) and np.array_equal(got[:, 1], im)
    assert not got[:, 3].any()  # level-0 radius: filled by ap_pack_bla
    # safe radius: inside it neither the bailout nor the Pauldelbrot threshold is reachable,
    safe2 = got[:, 2]
    s = np.sqrt(safe2)
    rz = np.sqrt(r2)
    assert np.all(safe2 >= 0.0)
    inside = safe2 > 0.0          # zero where |Z| >= 256 (no step is safe there)
    assert np.all((rz[inside] + s[inside]) ** 2 < 65536.0)
    assert np.all(safe2[rz >= 256.0] == 0.0)
    glitchable = inside & (r2 > 1e-8)
    assert np.all((rz[glitchable] - s[glitchable]) ** 2 > 1e-6 * r2[glitchable])
    # ... nor the one-pass rebase test |Z + dz| < |dz|: |Z| - s > s
    assert np.all(rz[inside] - s[inside] > s[inside])
    assert np.count_nonzero(safe2) > 0.9 * len(safe2)
    T = oracle.build_bla(re, im, rl, 0, 1e-6, 16, 3, 0.25, 1.0)
    d_T = torch.from_numpy(T).cuda()
    pb = torch.empty(80 * rl, dtype=torch.float64, device="cuda")
    _lib.check(L.ap_pack_bla(C.c_void_p(d_T.data_ptr()), 16, rl, C.c_void_p(pb.data_ptr()),
                             C.c_void_p(po.data_ptr()), None), "ap_pack_bla")
    pb = pb.cpu().numpy()
    R = pb[:16 * rl].reshape(rl, 16)
    rec = po.cpu().numpy()
    assert np.array_equal(rec[:rl, 3], R[:, 0]) and rec[rl, 3] == 0.0
    assert np.array_equal(rec[:, :3], got[:, :3])
    AB = pb[16 * rl:].reshape(rl, 16, 4)
    assert np.array_equal(R, T[:, :, 4].T)
    assert np.array_equal(AB, np.transpose(T[:, :, :4], (1, 0, 2)))
    # radii never increase with the level (the level search relies on it)
    assert np.all(np.diff(R, axis=1) <= 0)


BS, BSMETA = load_golden("render_bbsa.npz")


@pytest.mark.parametrize("name", [m["name"] for m in BSMETA])
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
def test_series_started_frame_matches_oracle(name, arith):
    """bbsa_order 4/8 frames through the engine equal the oracle's, value for value."""
    m = next(x for x in BSMETA if x["name"] == name)
    W, H = m["W"], m["H"]
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        color_scheme_id=0, precision_mode="1e-300 (Perturbation)", fractal_type=m["fractal_type"],
        julia_cx=m["julia_cx"], julia_cy=m["julia_cy"], bbsa_tol=m["bbsa_tol"],
        bbsa_order=m["bbsa_order"], glitch_mode=m["glitch_mode"], gen_n=m["gen_n"],
        gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], h_iter_buf=it, arith=arith)
    fr, _ = oracle_pert_frame(m, arith=0 if arith == "ref_cpu" else 1)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)


@pytest.mark.parametrize("shape", [(1080, 1920), (90, 160), (37, 53), (1, 1)])
def test_glitch_bins_match_numpy(shape):
    """ap_glitch_bins: glitched pixels per cell of the rebase loop's 16 x 16 grid."""
    import torch
    H, W = shape
    rng = np.random.default_rng(H * 7 + W)
    g = (rng.random((H, W)) < 0.4).astype(np.uint8)
    d_g = torch.from_numpy(g).cuda()
    counts = torch.full((256,), 7, dtype=torch.int32, device="cuda")   # stale contents are cleared
    L = _lib.load()
    for _ in range(2):
        _lib.check(L.ap_glitch_bins(C.c_void_p(d_g.data_ptr()), W, H, C.c_void_p(counts.data_ptr()), None),
                   "ap_glitch_bins")
        gi = np.argwhere(g > 0)
        b = np.clip((gi[:, 0] * 16) // H, 0, 15) * 16 + np.clip((gi[:, 1] * 16) // W, 0, 15)
        assert np.array_equal(counts.cpu().numpy(), np.bincount(b, minlength=256))
