"""Adjoint of the smooth escape value (fractura_b200.adjoint; config 5).

* The adjoint sweep (checkpoint segments recomputed, nothing stored) equals
  forward-mode tangents pixel by pixel and in sum, for Julia, Multibrot and
  Mandelbrot, and does not depend on the checkpoint spacing.
* Config 5: 512 x 512, Julia j = -0.8+0.156i and Multibrot n = 3, k = 0.1+0.2i,
  max_iter 2000, width 3.0; the target is rendered at theta + N(0, 1e-3) (seeded);
  loss = mean (s - s_target)^2 over pixels away from the boundary: the escape step
  is the same at every finite-difference point and the second difference is below
  1e-4 of the first.  The autograd gradient (the adjoint) matches central finite
  differences with h = 1e-7 to 1e-5 relative.
"""
import math

import numpy as np
import pytest

from fractura_b200 import adjoint as adj

pytestmark = pytest.mark.gpu

CASES = {
    "julia": dict(fractal_type=2, gen_n=3, theta=[0.0, 0.0, math.log(3.0), -0.8, 0.156]),
    "multibrot3": dict(fractal_type=4, gen_n=3, theta=[0.0, 0.0, math.log(3.0), 0.1, 0.2]),
    "mandelbrot": dict(fractal_type=0, gen_n=2, theta=[-0.65, 0.0, math.log(3.0), 0.0, 0.0]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_adjoint_equals_forward_mode(name):
    import torch
    c = CASES[name]
    W, H, mi = 192, 128, 2000
    s, k, ck = adj.forward(c["theta"], W, H, mi, c["fractal_type"], c["gen_n"])
    g = torch.from_numpy(np.random.default_rng(5).standard_normal((H, W))).cuda()
    total, pix = adj.adjoint(c["theta"], g, k, ck, W, H, mi, c["fractal_type"], c["gen_n"], per_pixel=True)
    ds = adj.forward_mode(c["theta"], W, H, mi, c["fractal_type"], c["gen_n"])
    want = g[..., None] * ds
    scale = want.abs().max().item()
    assert scale > 0
    assert torch.allclose(pix, want, rtol=1e-9, atol=1e-12 * scale)
    assert torch.allclose(total, want.sum(dim=(0, 1)), rtol=1e-9, atol=1e-12 * scale)
    if c["fractal_type"] == 0:
        assert total[3].item() == 0.0 and total[4].item() == 0.0


def test_checkpoint_spacing_does_not_change_the_gradient():
    import torch
    c = CASES["julia"]
    W, H, mi = 96, 64, 2000
    g = torch.from_numpy(np.random.default_rng(6).standard_normal((H, W))).cuda()
    out = []
    for every in (1024, 100, 7):
        s, k, ck = adj.forward(c["theta"], W, H, mi, c["fractal_type"], c["gen_n"], ckpt_every=every)
        out.append(adj.adjoint(c["theta"], g, k, ck, W, H, mi, c["fractal_type"], c["gen_n"],
                               ckpt_every=every))
    assert torch.equal(out[0], out[1]) and torch.equal(out[0], out[2])


@pytest.mark.parametrize("name", ["julia", "multibrot3"])
def test_config5_gradient_matches_central_differences(name):
    import torch
    c = CASES[name]
    W = H = 512
    mi, h = 2000, 1e-7
    theta0 = np.array(c["theta"])
    target_theta = theta0 + np.random.default_rng(20261203 + c["fractal_type"]).normal(0.0, 1e-3, 5)
    s_t, k_t, _ = adj.forward(target_theta, W, H, mi, c["fractal_type"], c["gen_n"], ckpt=False)
    # pixels whose escape step is the same at theta and at every FD point, and whose
    # second difference is negligible beside the first: away from the boundary, where
    # the central difference's third-order term dominates
    s0, k0, _ = adj.forward(theta0, W, H, mi, c["fractal_type"], c["gen_n"], ckpt=False)
    mask = (k0 > 0) & (k_t > 0)
    fd_points = []
    for q in range(5):
        pair = []
        for sign in (1.0, -1.0):
            th = theta0.copy()
            th[q] += sign * h
            s_q, k_q, _ = adj.forward(th, W, H, mi, c["fractal_type"], c["gen_n"], ckpt=False)
            mask &= k_q == k0
            pair.append(s_q)
        d1 = (pair[0] - pair[1]).abs()
        d2 = (pair[0] - 2.0 * s0 + pair[1]).abs()
        mask &= d2 <= 1e-4 * d1 + 1e-12
        fd_points.extend(pair)
    n = mask.sum().item()
    assert n > 0.5 * W * H
    m = mask.to(torch.float64)

    def loss(s):
        return (((s - s_t) ** 2) * m).sum() / n

    fd = np.array([(loss(fd_points[2 * q]).item() - loss(fd_points[2 * q + 1]).item()) / (2 * h)
                   for q in range(5)])
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    s = adj.smooth_escape(theta, W, H, mi, c["fractal_type"], c["gen_n"])
    loss(s).backward()
    got = theta.grad.numpy()
    norm = np.linalg.norm(fd)
    err = np.abs(got - fd) / np.maximum(np.abs(fd), 1e-3 * norm)
    assert np.all(err <= 1e-5), (got, fd, err, n / (W * H))


@pytest.mark.parametrize("name", sorted(CASES))
def test_forward_smooth_value_matches_oracle_fp64(name):
    """The adjoint's forward pass evaluates the same smooth value as the oracle's FP64
    direct sample (cpu_compute_fp64_sample restated, CUDA-source profile) at the same
    pixel c: the escape step is identical on >= 99.9 % of the pixels and, where it is,
    the smooth values agree to 1e-9 relative (the two differ only in which multiply-adds
    are fused, and for Multibrot in the reference's float32 1/ln n)."""
    import oracle
    from fractura_b200 import abi
    c = CASES[name]
    W, H, mi = 256, 192, 2000
    s, k, _ = adj.forward(c["theta"], W, H, mi, c["fractal_type"], c["gen_n"], ckpt=False)
    s, k = s.cpu().numpy(), k.cpu().numpy()
    th = c["theta"]
    w = math.exp(th[2])
    h = w * H / W
    xs = (th[0] - 0.5 * w) + np.arange(W, dtype=np.float64) * (w / (W - 1))
    ys = (th[1] + 0.5 * h) - np.arange(H, dtype=np.float64) * (h / (H - 1))
    p = abi.new_params(width=W, height=H, max_iter=mi, fractal_type=c["fractal_type"], gen_n=c["gen_n"],
                       gen_kr=th[3], gen_ki=th[4], julia_cx_hi=th[3], julia_cy_hi=th[4], tier=abi.AP_TIER_FP64,
                       arith=abi.AP_ARITH_REF_CUDA)
    _, s_o, k_o = oracle.fp64_grid(p, xs, ys)
    same = k == k_o
    assert same.mean() >= 0.999, same.mean()
    esc = same & (k >= 0)
    assert esc.sum() > 1000
    # Multibrot: the reference rounds 1/ln n to float32 in its smooth term (the oracle too);
    # the adjoint differentiates the smooth value with 1/ln n in float64, so the two differ
    # by up to |nu| 2^-24 (nu <= 2 here) on top of the 1e-9 of differently fused steps
    atol = 2.0 * 2.0 ** -24 if c["fractal_type"] == 4 else 0.0
    assert np.allclose(s[esc], s_o[esc], rtol=1e-9, atol=atol)
