"""FP64 forward restatements used as the finite-difference reference for the
adjoint tests (test infrastructure only).

Each function evaluates, in float64 numpy, the same mathematical operator as
the library's f32 forward pass on the inputs the gradient tests use:

* ``reduce_matrix``: the dense ReduceH/ReduceV weight matrix of one axis, built
  from the oracle's ReduceKernel tables and positions
  (resample/reduce_common.rs:137-316) with the clamp-to-edge source read
  folded in (sources/memory.rs:186-215);
* ``affine_bilinear``: Affine with a backward matrix and bilinear sampling
  (affine/core.rs:78-84, 496-513), Background/Black fill, and for 4-band images
  without ``premultiplied`` the alpha-premultiplying sampler
  (affine/core.rs:988-1019) -- valid where every sample lies inside the
  source (the tests pick such inputs, so the per-tile input-region check of
  the scheduler never applies);
* ``mapim_sample``: MapImOp's bilinear (floor) and renormalised separable
  samplers with Background fill (mapim.rs:1135-1274, affine/core.rs:648-696).
"""
import math

import numpy as np

from oracle import oracle as O


def reduce_matrix(n_in, factor, kernel):
    """(n_out, n_in) float64 matrix of one bound reduce axis."""
    from viprs_b200 import api
    n_out = api.reduce_output_len(factor, n_in)
    taps, _pad, _off, c64, _c16 = O.reduce_tables(factor, kernel, n_in, True)
    R = np.zeros((n_out, n_in), np.float64)
    for o in range(n_out):
        s, ph, _pos = O.reduce_plan(factor, kernel, n_in, True, float(o))
        for k in range(taps):
            R[o, min(max(s + k, 0), n_in - 1)] += c64[ph, k]
    return R


def reduce_h(x, R):
    return np.einsum("ow,hwb->hob", R, x)


def reduce_v(x, R):
    return np.einsum("oh,hwb->owb", R, x)


def affine_positions(bm, bt, out_w, out_h):
    Y, X = np.meshgrid(np.arange(out_h, dtype=np.float64), np.arange(out_w, dtype=np.float64), indexing="ij")
    return bm[0] * X + bm[1] * Y + bt[0], bm[2] * X + bm[3] * Y + bt[1]


def _bilinear(x, px, py, fill):
    """Bilinear samples of every band at (px, py); taps outside read `fill`."""
    H, W, B = x.shape
    x0 = np.trunc(px).astype(np.int64)
    y0 = np.trunc(py).astype(np.int64)
    fx = px - x0
    fy = py - y0

    def tap(dx, dy):
        ix, iy = x0 + dx, y0 + dy
        ok = (ix >= 0) & (ix < W) & (iy >= 0) & (iy < H)
        v = x[np.clip(iy, 0, H - 1), np.clip(ix, 0, W - 1)]
        return np.where(ok[..., None], v, fill)

    p00, p01, p10, p11 = tap(0, 0), tap(1, 0), tap(0, 1), tap(1, 1)
    fx = fx[..., None]
    fy = fy[..., None]
    top = p01 * fx + p00 * (1.0 - fx)
    bottom = p11 * fx + p10 * (1.0 - fx)
    return top * (1.0 - fy) + bottom * fy


def affine_bilinear(x, bm, bt, out_w, out_h, premultiplied=False, fill=0.0):
    px, py = affine_positions(bm, bt, out_w, out_h)
    B = x.shape[2]
    if B == 4 and not premultiplied:
        a = x[..., 3:4]
        pm = np.concatenate([x[..., :3] * a, a], axis=2)
        s = _bilinear(pm, px, py, fill)
        A = np.clip(s[..., 3:4], 0.0, 1.0)
        out = np.where(A > 0.0, s[..., :3] / np.where(A > 0.0, A, 1.0), 0.0)
        return np.concatenate([out, A], axis=2)
    return _bilinear(x, px, py, fill)


def _kernel_w(k, t):
    t = np.abs(t)
    if k == "bilinear":
        return np.where(t < 1.0, 1.0 - t, 0.0)
    if k in ("bicubic", "catmullrom"):
        return np.where(t < 1.0, 1.5 * t ** 3 - 2.5 * t ** 2 + 1.0,
                        np.where(t < 2.0, -0.5 * t ** 3 + 2.5 * t ** 2 - 4.0 * t + 2.0, 0.0))
    if k == "quadratic":
        return np.where(t < 0.5, 1.0 - 2.0 * t * t, np.where(t < 1.5, t * t - 2.5 * t + 1.5, 0.0))
    if k in ("lanczos2", "lanczos3"):
        L = 3.0 if k == "lanczos3" else 2.0
        p = math.pi * np.where(t < 1e-300, 1.0, t)
        v = L * np.sin(p) * np.sin(p / L) / (p * p)
        return np.where(t < 2.220446049250313e-16, 1.0, np.where(t < L, v, 0.0))
    raise ValueError(k)


def mapim_sample(src, idx, kernel, background=0.0):
    """MapImOp over float64 coordinates idx (h, w, 2); Background fill."""
    H, W, B = src.shape
    x = idx[..., 0]
    y = idx[..., 1]
    if kernel == "bilinear":
        x0 = np.floor(x).astype(np.int64)
        y0 = np.floor(y).astype(np.int64)
        fx = (x - x0)[..., None]
        fy = (y - y0)[..., None]

        def tap(dx, dy):
            ix, iy = x0 + dx, y0 + dy
            ok = (ix >= 0) & (ix < W) & (iy >= 0) & (iy < H)
            return np.where(ok[..., None], src[np.clip(iy, 0, H - 1), np.clip(ix, 0, W - 1)], background)

        top = tap(1, 0) * fx + tap(0, 0) * (1.0 - fx)
        bottom = tap(1, 1) * fx + tap(0, 1) * (1.0 - fx)
        return top * (1.0 - fy) + bottom * fy
    support = 3 if kernel == "lanczos3" else 2
    cx = np.floor(x).astype(np.int64)
    cy = np.floor(y).astype(np.int64)
    acc = np.zeros(x.shape + (B,), np.float64)
    wsum = np.zeros(x.shape, np.float64)
    for ky in range(-(support - 1), support + 1):
        iy = cy + ky
        wy = _kernel_w(kernel, iy - y)
        for kx in range(-(support - 1), support + 1):
            ix = cx + kx
            wx = _kernel_w(kernel, ix - x)
            w = wx * wy
            ok = (ix >= 0) & (ix < W) & (iy >= 0) & (iy < H)
            s = np.where(ok[..., None], src[np.clip(iy, 0, H - 1), np.clip(ix, 0, W - 1)], background)
            acc += s * w[..., None]
            wsum += w
    return np.where(wsum[..., None] > 0.0, acc / np.where(wsum > 0.0, wsum, 1.0)[..., None], background)
