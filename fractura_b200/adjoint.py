"""Gradients of the smooth escape value with respect to the view and the formula.

    s = smooth_escape(theta, W, H, max_iter, fractal_type=2, gen_n=3)
    loss = ((s - target)[mask] ** 2).mean()
    loss.backward()                      # theta.grad: d loss / d(cx, cy, ln w, Re P, Im P)

theta is a float64 tensor (cx, cy, ln w, Re P, Im P); P is the Julia parameter
(fractal_type 2, z0 = pixel) or the Multibrot coefficient K of z^n + K z + c
(fractal_type 4); Mandelbrot (0) has no P.  The forward pass is FP64 direct
iteration on the GPU (ap_smooth_forward), which also keeps the orbit every
CKPT_EVERY steps; the backward pass is the hand-written adjoint
(ap_smooth_adjoint), which recomputes each checkpoint segment instead of
storing orbits.  forward_mode() gives the same derivatives per pixel by
forward-mode tangents (ap_smooth_tangent), the independent check.
"""
import ctypes as C

import numpy as np

from . import _lib, abi

CKPT_EVERY = 1024


def _view(theta, W, H, max_iter, fractal_type, gen_n, ckpt_every=CKPT_EVERY):
    t = [float(x) for x in theta]
    return abi.ApGradView(width=int(W), height=int(H), max_iter=int(max_iter),
                          fractal_type=int(fractal_type), gen_n=int(gen_n), ckpt_every=int(ckpt_every),
                          cx=t[0], cy=t[1], w=float(np.exp(t[2])), pr=t[3], pi=t[4])


def _n_ckpt(max_iter, every):
    return (int(max_iter) + every - 1) // every + 1


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def forward(theta, W, H, max_iter, fractal_type=2, gen_n=3, ckpt=True, ckpt_every=CKPT_EVERY):
    """(s64 [H, W], kmap [H, W], checkpoints or None) on the current CUDA stream."""
    import torch
    v = _view(theta, W, H, max_iter, fractal_type, gen_n, ckpt_every)
    s = torch.empty((H, W), dtype=torch.float64, device="cuda")
    k = torch.empty((H, W), dtype=torch.int32, device="cuda")
    n_ck = _n_ckpt(max_iter, ckpt_every)
    ck = torch.empty((H, W, n_ck, 2), dtype=torch.float64, device="cuda") if ckpt else None
    L = _lib.load()
    _lib.check(L.ap_smooth_forward(C.byref(v), _ptr(s), _ptr(k), _ptr(ck), n_ck,
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "ap_smooth_forward")
    return s, k, ck


def adjoint(theta, grad_s, kmap, ckpt, W, H, max_iter, fractal_type=2, gen_n=3, per_pixel=False,
            ckpt_every=CKPT_EVERY):
    """dL/dtheta (float64 [5]) for dL/ds = grad_s; with per_pixel also each pixel's term."""
    import torch
    v = _view(theta, W, H, max_iter, fractal_type, gen_n, ckpt_every)
    L = _lib.load()
    nb = L.ap_smooth_adjoint_blocks(int(W), int(H))
    sums = torch.empty((nb, 5), dtype=torch.float64, device="cuda")
    pix = torch.empty((H, W, 5), dtype=torch.float64, device="cuda") if per_pixel else None
    g = grad_s.to(dtype=torch.float64, device="cuda").contiguous()
    _lib.check(L.ap_smooth_adjoint(C.byref(v), _ptr(g), _ptr(kmap), _ptr(ckpt),
                                   _n_ckpt(max_iter, ckpt_every), _ptr(pix), _ptr(sums),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "ap_smooth_adjoint")
    total = sums.sum(dim=0)
    return (total, pix) if per_pixel else total


def forward_mode(theta, W, H, max_iter, fractal_type=2, gen_n=3):
    """ds/dtheta per pixel ([H, W, 5]) by forward-mode tangents."""
    import torch
    v = _view(theta, W, H, max_iter, fractal_type, gen_n)
    ds = torch.empty((H, W, 5), dtype=torch.float64, device="cuda")
    L = _lib.load()
    _lib.check(L.ap_smooth_tangent(C.byref(v), _ptr(ds),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "ap_smooth_tangent")
    return ds


def _function():
    import torch

    class SmoothEscape(torch.autograd.Function):
        """s = smooth escape values of the view theta; backward by the adjoint sweep."""

        @staticmethod
        def forward(ctx, theta, W, H, max_iter, fractal_type, gen_n):
            th = theta.detach().cpu().tolist()
            s, k, ck = forward(th, W, H, max_iter, fractal_type, gen_n)
            ctx.save_for_backward(k, ck)
            ctx.meta = (th, W, H, max_iter, fractal_type, gen_n, theta.device, theta.dtype)
            return s

        @staticmethod
        def backward(ctx, grad_s):
            k, ck = ctx.saved_tensors
            th, W, H, max_iter, fractal_type, gen_n, dev, dt = ctx.meta
            g = adjoint(th, grad_s, k, ck, W, H, max_iter, fractal_type, gen_n)
            return g.to(device=dev, dtype=dt), None, None, None, None, None

    return SmoothEscape


_FN = None


def smooth_escape(theta, W, H, max_iter, fractal_type=2, gen_n=3):
    """Differentiable smooth escape values [H, W] (float64, -1 for interior pixels)."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(theta, int(W), int(H), int(max_iter), int(fractal_type), int(gen_n))
