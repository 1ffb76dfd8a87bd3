"""Adjoint (backward) kernels of reduce, affine and mapim on the GPU, through
the C ABI and the torch.autograd wrappers.

* Adjoint identity <A x, y> = <x, A^T y> for the linear operators (sums in
  f64 of the f32 results), relative error <= 1e-5.  Affine/mapim with a
  constant fill are affine maps, so the fill's contribution A(0) is removed
  first; 4-band images use the linear ``premultiplied`` form.
* FP64 central finite differences with h = 1e-3 (tests/fd_reference.py holds
  the float64 forwards) on a subset of pixels and on the matrix / coordinate
  parameters, relative error <= 1e-4.  Matrix entries are stepped by
  h / (output extent), so that every sample moves by at most h pixels, and the
  loss is restricted to the pixels whose samples stay inside one interpolation
  cell over the step (the interpolators are piecewise polynomials).
* The deterministic scatter is bit-identical from run to run and agrees with
  the f32-atomic scatter.
"""
import ctypes
import math
import zlib

import numpy as np
import pytest

import fd_reference as FR

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from viprs_b200 import _native as N  # noqa: E402
from viprs_b200 import api  # noqa: E402
from viprs_b200 import autograd as AG  # noqa: E402

RTOL_IDENTITY = 1e-5
RTOL_FD = 1e-4
H = 1e-3


def seed_of(*key):
    return zlib.crc32(repr(key).encode())


def dev(a, grad=False):
    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    return t.requires_grad_(grad)


def host(t):
    torch.cuda.synchronize()
    return t.detach().double().cpu().numpy()


def dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def identity_err(lhs, rhs, a, b):
    """|<A x, y> - <x, A^T y>| over sum |(A x)_i y_i|: f32 rounding of each
    product term scales with that sum, not with the (cancelling) dot product."""
    return abs(lhs - rhs) / max(float(np.sum(np.abs(np.asarray(a, np.float64) * np.asarray(b, np.float64)))), 1e-30)


def normwise(a, b):
    """max |a - b| over max |b| (gradients mix signs, so elements can be ~0)."""
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-30))


def floored(a, b, floor=1e-3):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def fd_check(g, fd, scale):
    """Per-entry FD error, floored at 1e-3 of the gradient's scale."""
    g = np.asarray(g, np.float64)
    fd = np.asarray(fd, np.float64)
    return float(np.max(np.abs(g - fd) / np.maximum(np.abs(fd), 1e-3 * scale)))


# ----------------------------------------------------------------------------- reduce

@pytest.mark.parametrize("horizontal", [1, 0])
@pytest.mark.parametrize("kernel", ["lanczos3", "lanczos2", "bicubic", "bilinear"])
@pytest.mark.parametrize("factor", [1.5, 2.0, 2.7027, 4.0, 9.3])
@pytest.mark.parametrize("n", [2, 5, 37, 300])
def test_reduce_adjoint_is_the_dense_transpose(horizontal, kernel, factor, n):
    n_out = api.reduce_output_len(factor, n)
    if n_out == 0:
        pytest.skip("empty output")
    rng = np.random.default_rng(n * 31 + int(factor * 10) + horizontal)
    shape = (7, n, 3) if horizontal else (n, 6, 2)
    x = rng.random(shape, dtype=np.float32)
    R = FR.reduce_matrix(n, factor, kernel)
    ref_y = FR.reduce_h(x.astype(np.float64), R) if horizontal else FR.reduce_v(x.astype(np.float64), R)
    xt = dev(x, True)
    y = AG.reduce_h(xt, factor, kernel) if horizontal else AG.reduce_v(xt, factor, kernel)
    assert floored(host(y), ref_y) <= 1e-5
    gy = rng.standard_normal(ref_y.shape).astype(np.float32)
    y.backward(dev(gy))
    gx = host(xt.grad)
    ref_gx = (np.einsum("ow,hob->hwb", R, gy.astype(np.float64)) if horizontal
              else np.einsum("oh,owb->hwb", R, gy.astype(np.float64)))
    assert normwise(gx, ref_gx) <= RTOL_IDENTITY
    assert identity_err(dot(host(y), gy), dot(x, gx), host(y), gy) <= RTOL_IDENTITY


@pytest.mark.parametrize("horizontal", [1, 0])
def test_reduce_fd_fp64(horizontal):
    rng = np.random.default_rng(7 + horizontal)
    factor, kernel = 2.7027, "lanczos3"
    shape = (9, 41, 3) if horizontal else (41, 8, 3)
    x = rng.random(shape, dtype=np.float32).astype(np.float64)
    R = FR.reduce_matrix(41, factor, kernel)
    fwd = (lambda v: FR.reduce_h(v, R)) if horizontal else (lambda v: FR.reduce_v(v, R))
    gy = rng.standard_normal(fwd(x).shape)
    xt = dev(x, True)
    y = AG.reduce_h(xt, factor, kernel) if horizontal else AG.reduce_v(xt, factor, kernel)
    y.backward(dev(gy))
    gx = host(xt.grad)
    gy = gy.astype(np.float32).astype(np.float64)
    flat = rng.choice(x.size, 16, replace=False)
    fd = []
    for f in flat:
        e = np.zeros(x.size)
        e[f] = H
        e = e.reshape(x.shape)
        fd.append((dot(gy, fwd(x + e)) - dot(gy, fwd(x - e))) / (2 * H))
    assert fd_check(gx.reshape(-1)[flat], fd, np.max(np.abs(gx))) <= RTOL_FD


@pytest.mark.parametrize("factors,kernel", [((2.0, 2.0), "lanczos3"), ((2.7027, 1.5), "lanczos3"),
                                            ((3.0, 2.0), "bicubic"), ((1.25, 4.5), "lanczos2")])
def test_reduce_hv_adjoint(factors, kernel):
    hf, vf = factors
    rng = np.random.default_rng(int(hf * 100 + vf))
    x = rng.random((37, 53, 3), dtype=np.float32)
    Rh = FR.reduce_matrix(53, hf, kernel)
    Rv = FR.reduce_matrix(37, vf, kernel)
    x64 = x.astype(np.float64)
    ref_y = FR.reduce_v(FR.reduce_h(x64, Rh), Rv)
    xt = dev(x, True)
    y = AG.reduce_hv(xt, hf, vf, kernel)
    assert floored(host(y), ref_y) <= 1e-5
    gy = rng.standard_normal(ref_y.shape).astype(np.float32)
    y.backward(dev(gy))
    gx = host(xt.grad)
    ref_gx = np.einsum("ow,hob->hwb", Rh, np.einsum("oh,owb->hwb", Rv, gy.astype(np.float64)))
    assert normwise(gx, ref_gx) <= RTOL_IDENTITY
    assert identity_err(dot(host(y), gy), dot(x, gx), host(y), gy) <= RTOL_IDENTITY
    # FP64 FD on a subset of pixels (edge pixels included: they carry the folded taps)
    picks = [(0, 0, 0), (36, 52, 2), (0, 27, 1), (18, 0, 0), (18, 26, 1), (36, 0, 2), (5, 51, 0)]
    for (py, px, pb) in picks:
        e = np.zeros_like(x64)
        e[py, px, pb] = H
        fd = (dot(gy, FR.reduce_v(FR.reduce_h(x64 + e, Rh), Rv)) -
              dot(gy, FR.reduce_v(FR.reduce_h(x64 - e, Rh), Rv))) / (2 * H)
        assert fd_check([gx[py, px, pb]], [fd], np.max(np.abs(gx))) <= RTOL_FD


# ----------------------------------------------------------------------------- affine

def _rot_backward(theta, s, in_w, in_h, out_w, out_h):
    """Backward matrix rotating by theta and scaling by s about the centres."""
    c, sn = math.cos(theta) * s, math.sin(theta) * s
    bm = [c, -sn, sn, c]
    bt = [in_w / 2 - (bm[0] * out_w / 2 + bm[1] * out_h / 2), in_h / 2 - (bm[2] * out_w / 2 + bm[3] * out_h / 2)]
    return bm, bt


def _affine_grad_raw(x, gy, bm, bt, extend, bg, premul, det, want_x=True):
    gx = torch.empty_like(x) if want_x else None
    g6 = torch.empty(6, dtype=torch.float64, device=x.device)
    mm = (ctypes.c_double * 4)(*bm)
    st = N.lib().viprs_affine_grad(api.image(x), api.image(gy), api.image(gx) if want_x else None, mm, bt[0],
                                   bt[1], 1, api.EXTEND[extend], bg, int(premul), 0, 0, int(det),
                                   ctypes.c_void_p(g6.data_ptr()), api._stream())
    N.check(st, "affine_grad")
    return gx, g6.cpu().tolist()


AFFINE_GEOMS = {
    # rotated + scaled about the centres: the general incremental walk, several tiles
    "rotated": lambda iw, ih, ow, oh: _rot_backward(0.43, 1.1, iw, ih, ow, oh),
    # axis-aligned scale: the bilinear fast path (constant fill) or the per-axis tables
    "axis": lambda iw, ih, ow, oh: ([0.83, 0.0, 0.0, 1.21], [3.3, -7.6]),
}


@pytest.mark.parametrize("geom", ["rotated", "axis"])
@pytest.mark.parametrize("extend", ["black", "background", "white", "copy", "repeat", "mirror"])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_affine_adjoint_identity(geom, extend, bands):
    rng = np.random.default_rng(seed_of(geom, extend, bands))
    in_h, in_w, out_h, out_w = 150, 180, 170, 210
    bm, bt = AFFINE_GEOMS[geom](in_w, in_h, out_w, out_h)
    premul = bands == 4  # the linear form of the 4-band sampler
    bg = 0.25
    x = rng.random((in_h, in_w, bands), dtype=np.float32)
    xt = dev(x)
    y = api.affine_backward_matrix(xt, bm, bt[0], bt[1], out_w, out_h, "bilinear", extend, bg, premul)
    y0 = api.affine_backward_matrix(torch.zeros_like(xt), bm, bt[0], bt[1], out_w, out_h, "bilinear", extend, bg,
                                    premul)
    gy = dev(rng.standard_normal((out_h, out_w, bands)))
    gx, _ = _affine_grad_raw(xt, gy, bm, bt, extend, bg, premul, det=False)
    lhs = dot(host(y) - host(y0), host(gy))
    assert identity_err(lhs, dot(x, host(gx)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    gd, _ = _affine_grad_raw(xt, gy, bm, bt, extend, bg, premul, det=True)
    gd2, _ = _affine_grad_raw(xt, gy, bm, bt, extend, bg, premul, det=True)
    assert torch.equal(gd, gd2), "deterministic scatter differs between runs"
    # the deterministic (2^-32 fixed-point) scatter satisfies the identity on its own
    assert identity_err(lhs, dot(x, host(gd)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    # f32 atomics add a pixel's (up to 16) contributions in a varying order:
    # agreement within a few f32 ulps of the largest gradient
    assert normwise(host(gd), host(gx)) <= 1e-5


def _affine_fd_case(bands, seed):
    rng = np.random.default_rng(seed)
    in_h, in_w, out_h, out_w = 48, 56, 26, 30
    bm, bt = _rot_backward(0.3, 0.85, in_w, in_h, out_w, out_h)
    x = rng.random((in_h, in_w, bands), dtype=np.float32)
    if bands == 4:
        x[..., 3] = 0.2 + 0.8 * x[..., 3]  # interpolated alpha stays inside (0, 1)
    gy = rng.standard_normal((out_h, out_w, bands)).astype(np.float32)
    px, py = FR.affine_positions(np.array(bm), np.array(bt), out_w, out_h)
    fx, fy = px - np.trunc(px), py - np.trunc(py)
    keep = (fx > 0.02) & (fx < 0.98) & (fy > 0.02) & (fy < 0.98)
    assert keep.mean() > 0.8
    return x, gy, gy * keep[..., None], np.array(bm), np.array(bt), out_w, out_h


@pytest.mark.parametrize("bands", [1, 3, 4])
def test_affine_fd_fp64(bands):
    x, gy, gy_cell, bm, bt, out_w, out_h = _affine_fd_case(bands, 100 + bands)
    x64 = x.astype(np.float64)

    def F(v, m, t):
        return FR.affine_bilinear(v, m, t, out_w, out_h, premultiplied=False, fill=0.0)

    xt = dev(x, True)
    bmt = torch.tensor(bm, dtype=torch.float64, requires_grad=True)
    btt = torch.tensor(bt, dtype=torch.float64, requires_grad=True)
    y = AG.affine_backward(xt, bmt, btt, out_w, out_h, "black")
    assert floored(host(y), F(x64, bm, bt)) <= 1e-5
    # matrix / translation: loss restricted to samples that stay in their cell
    (y * dev(gy_cell)).sum().backward()
    g6 = np.concatenate([bmt.grad.numpy(), btt.grad.numpy()])
    p = np.concatenate([bm, bt])
    steps = [H / out_w, H / out_h, H / out_w, H / out_h, H, H]
    gyc = gy_cell.astype(np.float64)
    fd = []
    for j in range(6):
        e = np.zeros(6)
        e[j] = steps[j]
        lp = dot(gyc, F(x64, (p + e)[:4], (p + e)[4:]))
        lm = dot(gyc, F(x64, (p - e)[:4], (p - e)[4:]))
        fd.append((lp - lm) / (2 * steps[j]))
    assert fd_check(g6, fd, np.max(np.abs(fd))) <= RTOL_FD
    # image: full loss, a subset of pixels inside the sampled area
    xt.grad = None
    y = AG.affine_backward(xt, bmt.detach(), btt.detach(), out_w, out_h, "black")
    y.backward(dev(gy))
    gx = host(xt.grad)
    gy64 = gy.astype(np.float64)
    rng = np.random.default_rng(5)
    fd, got = [], []
    for _ in range(16):
        py_, px_, pb = rng.integers(14, 34), rng.integers(16, 40), rng.integers(0, bands)
        e = np.zeros_like(x64)
        e[py_, px_, pb] = H
        fd.append((dot(gy64, F(x64 + e, bm, bt)) - dot(gy64, F(x64 - e, bm, bt))) / (2 * H))
        got.append(gx[py_, px_, pb])
    assert fd_check(got, fd, np.max(np.abs(gx))) <= RTOL_FD


@pytest.mark.parametrize("bands", [3, 4])
def test_affine_forward_matrix_autograd_fd(bands):
    """Gradients reach the FORWARD matrix and translation through the builder's inversion."""
    rng = np.random.default_rng(40 + bands)
    in_h, in_w, out_h, out_w = 48, 56, 26, 30
    x = rng.random((in_h, in_w, bands), dtype=np.float32)
    if bands == 4:
        x[..., 3] = 0.2 + 0.8 * x[..., 3]
    th, s = -0.35, 1.15
    M = np.array([s * math.cos(th), -s * math.sin(th), s * math.sin(th), s * math.cos(th)])
    # translation placing the output centre on the input centre
    c_in = np.array([in_w / 2, in_h / 2])
    c_out = np.array([out_w / 2, out_h / 2])
    t = c_out - np.array([M[0] * c_in[0] + M[1] * c_in[1], M[2] * c_in[0] + M[3] * c_in[1]])
    x64 = x.astype(np.float64)

    def back(m, tt):
        b = np.array([m[3], -m[1], -m[2], m[0]]) / (m[0] * m[3] - m[1] * m[2])
        return b, -np.array([b[0] * tt[0] + b[1] * tt[1], b[2] * tt[0] + b[3] * tt[1]])

    b, bt = back(M, t)
    px, py = FR.affine_positions(b, bt, out_w, out_h)
    fx, fy = px - np.trunc(px), py - np.trunc(py)
    keep = (fx > 0.02) & (fx < 0.98) & (fy > 0.02) & (fy < 0.98)
    gy = rng.standard_normal((out_h, out_w, bands)).astype(np.float32) * keep[..., None]
    Mt = torch.tensor(M, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(t, dtype=torch.float64, requires_grad=True)
    y = AG.affine(dev(x), Mt, tt, out_w, out_h)
    F = lambda m, tv: FR.affine_bilinear(x64, *back(m, tv), out_w, out_h)  # noqa: E731
    assert floored(host(y), F(M, t)) <= 1e-5
    (y * dev(gy)).sum().backward()
    got = np.concatenate([Mt.grad.numpy(), tt.grad.numpy()])
    gy64 = gy.astype(np.float64)
    p = np.concatenate([M, t])
    steps = [H / out_w] * 4 + [H, H]
    fd = []
    for j in range(6):
        e = np.zeros(6)
        e[j] = steps[j]
        fd.append((dot(gy64, F((p + e)[:4], (p + e)[4:])) - dot(gy64, F((p - e)[:4], (p - e)[4:]))) / (2 * steps[j]))
    assert fd_check(got, fd, np.max(np.abs(fd))) <= RTOL_FD


# ----------------------------------------------------------------------------- mapim

def _smooth(rng, h, w, b):
    yy, xx = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    out = np.zeros((h, w, b))
    for band in range(b):
        for _ in range(3):
            fx, fy, ph = rng.uniform(0.5, 3), rng.uniform(0.5, 3), rng.uniform(0, 2 * np.pi)
            out[..., band] += np.sin(2 * np.pi * (fx * xx / w + fy * yy / h) + ph)
    return (0.5 + 0.15 * out).astype(np.float32)


@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "quadratic", "lanczos2", "lanczos3"])
@pytest.mark.parametrize("extend_copy", [0, 1])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_mapim_adjoint_identity(kernel, extend_copy, bands):
    rng = np.random.default_rng(seed_of(kernel, extend_copy, bands))
    sh, sw, oh, ow = 60, 70, 50, 64
    src = rng.random((sh, sw, bands), dtype=np.float32)
    idx = np.stack([rng.uniform(-4, sw + 4, (oh, ow)), rng.uniform(-4, sh + 4, (oh, ow))], axis=2).astype(np.float32)
    idx[3, 5] = np.nan
    idx[7, 9, 1] = np.inf
    bg = 0.3
    premul = bands == 4
    st, it = dev(src), dev(idx)
    y = api.mapim(st, it, kernel, bool(extend_copy), bg, premul)
    y0 = api.mapim(torch.zeros_like(st), it, kernel, bool(extend_copy), bg, premul)
    gy = dev(rng.standard_normal((oh, ow, bands)))

    def grad(det):
        gs = torch.empty_like(st)
        N.check(N.lib().viprs_mapim_grad(api.image(st), api.image(it), api.image(gy), api.image(gs), None,
                                         api._kernel(kernel), extend_copy, bg, int(premul), int(det),
                                         api._stream()), "mapim_grad")
        return gs

    ga = grad(False)
    lhs = dot(host(y) - host(y0), host(gy))
    assert identity_err(lhs, dot(src, host(ga)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    gd, gd2 = grad(True), grad(True)
    assert torch.equal(gd, gd2), "deterministic scatter differs between runs"
    assert identity_err(lhs, dot(src, host(gd)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    assert normwise(host(gd), host(ga)) <= 1e-5


@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos3"])
@pytest.mark.parametrize("extend_copy", [0, 1])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_mapim_grad_smooth_field(kernel, extend_copy, bands):
    """Near-identity coordinate field (smooth displacement of a few pixels,
    reaching past the edges): each 16 x 16 block's taps span a small box, so
    the image gradient accumulates block-locally before the global adds."""
    rng = np.random.default_rng(seed_of(kernel, extend_copy, bands) + 17)
    sh, sw = 150, 230
    src = rng.random((sh, sw, bands), dtype=np.float32)
    d = _smooth(rng, sh, sw, 2).astype(np.float64) - 0.5
    yy, xx = np.meshgrid(np.arange(sh), np.arange(sw), indexing="ij")
    idx = np.stack([xx + 30 * d[..., 0] - 2.5, yy + 30 * d[..., 1] + 1.5], axis=2).astype(np.float32)
    bg = 0.25
    premul = bands == 4
    st, it = dev(src), dev(idx)
    y = api.mapim(st, it, kernel, bool(extend_copy), bg, premul)
    y0 = api.mapim(torch.zeros_like(st), it, kernel, bool(extend_copy), bg, premul)
    gy = dev(rng.standard_normal((sh, sw, bands)))

    def grad(det):
        gs = torch.empty_like(st)
        N.check(N.lib().viprs_mapim_grad(api.image(st), api.image(it), api.image(gy), api.image(gs), None,
                                         api._kernel(kernel), extend_copy, bg, int(premul), int(det),
                                         api._stream()), "mapim_grad")
        return gs

    ga = grad(False)
    lhs = dot(host(y) - host(y0), host(gy))
    assert identity_err(lhs, dot(src, host(ga)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    gd, gd2 = grad(True), grad(True)
    assert torch.equal(gd, gd2), "deterministic scatter differs between runs"
    assert identity_err(lhs, dot(src, host(gd)), host(y) - host(y0), host(gy)) <= RTOL_IDENTITY
    assert normwise(host(gd), host(ga)) <= 1e-5


@pytest.mark.parametrize("kernel", ["bilinear", "bicubic", "quadratic", "lanczos2", "lanczos3"])
@pytest.mark.parametrize("bands", [1, 3])
def test_mapim_fd_fp64(kernel, bands):
    rng = np.random.default_rng(len(kernel) * 10 + bands)
    sh, sw, oh, ow = 40, 48, 24, 28
    src = _smooth(rng, sh, sw, bands)
    # interior coordinates whose fractional parts keep the FD step inside one
    # polynomial piece of the kernel (integers, and half-integers for quadratic)
    base = np.stack([rng.integers(5, sw - 6, (oh, ow)), rng.integers(5, sh - 6, (oh, ow))], axis=2).astype(np.float64)
    frac = rng.choice([0.1, 0.2, 0.3, 0.4, 0.6, 0.7, 0.8, 0.9], (oh, ow, 2)) + rng.uniform(-0.05, 0.05, (oh, ow, 2))
    idx = (base + frac).astype(np.float32)
    gy = rng.standard_normal((oh, ow, bands)).astype(np.float32)
    s64, i64, gy64 = src.astype(np.float64), idx.astype(np.float64), gy.astype(np.float64)
    st, it = dev(src, True), dev(idx, True)
    y = AG.mapim(st, it, kernel)
    assert floored(host(y), FR.mapim_sample(s64, i64, kernel)) <= 1e-5
    y.backward(dev(gy))
    gi, gs = host(it.grad), host(st.grad)
    got, fd = [], []
    for _ in range(24):
        r, c, a = rng.integers(0, oh), rng.integers(0, ow), rng.integers(0, 2)
        e = np.zeros_like(i64)
        e[r, c, a] = H
        fd.append((dot(gy64, FR.mapim_sample(s64, i64 + e, kernel)) -
                   dot(gy64, FR.mapim_sample(s64, i64 - e, kernel))) / (2 * H))
        got.append(gi[r, c, a])
    assert fd_check(got, fd, np.max(np.abs(gi))) <= RTOL_FD
    got, fd = [], []
    for _ in range(12):
        r, c, b = rng.integers(8, sh - 8), rng.integers(8, sw - 8), rng.integers(0, bands)
        e = np.zeros_like(s64)
        e[r, c, b] = H
        fd.append((dot(gy64, FR.mapim_sample(s64 + e, i64, kernel)) -
                   dot(gy64, FR.mapim_sample(s64 - e, i64, kernel))) / (2 * H))
        got.append(gs[r, c, b])
    assert fd_check(got, fd, max(np.max(np.abs(gs)), 1e-6)) <= RTOL_FD


# ----------------------------------------------------------------------------- chain

def test_reduce_then_affine_chain_fd_fp64():
    """reduce_h(2) + reduce_v(2) (Lanczos3) -> affine(M, t) bilinear on a 4-band
    image (alpha-premultiplying sampler), end to end through autograd."""
    rng = np.random.default_rng(2024)
    in_h, in_w = 64, 72
    x = rng.random((in_h, in_w, 4), dtype=np.float32)
    x[..., 3] = 0.3 + 0.7 * x[..., 3]
    Rh = FR.reduce_matrix(in_w, 2.0, "lanczos3")
    Rv = FR.reduce_matrix(in_h, 2.0, "lanczos3")
    zh, zw = Rv.shape[0], Rh.shape[0]
    out_h, out_w = 20, 24
    th, s = 0.2, 1.1
    M = np.array([s * math.cos(th), -s * math.sin(th), s * math.sin(th), s * math.cos(th)])
    c_in, c_out = np.array([zw / 2, zh / 2]), np.array([out_w / 2, out_h / 2])
    t = c_out - np.array([M[0] * c_in[0] + M[1] * c_in[1], M[2] * c_in[0] + M[3] * c_in[1]])
    b = np.array([M[3], -M[1], -M[2], M[0]]) / (M[0] * M[3] - M[1] * M[2])
    bt = -np.array([b[0] * t[0] + b[1] * t[1], b[2] * t[0] + b[3] * t[1]])
    x64 = x.astype(np.float64)

    def F(v):
        return FR.affine_bilinear(FR.reduce_v(FR.reduce_h(v, Rh), Rv), b, bt, out_w, out_h)

    xt = dev(x, True)
    Mt = torch.tensor(M, dtype=torch.float64, requires_grad=True)
    tt = torch.tensor(t, dtype=torch.float64, requires_grad=True)
    y = AG.affine(AG.reduce_hv(xt, 2.0, 2.0, "lanczos3"), Mt, tt, out_w, out_h)
    assert floored(host(y), F(x64)) <= 1e-5
    gy = rng.standard_normal((out_h, out_w, 4)).astype(np.float32)
    y.backward(dev(gy))
    gx = host(xt.grad)
    gy64 = gy.astype(np.float64)
    got, fd = [], []
    for _ in range(16):
        r, c, bb = rng.integers(16, 48), rng.integers(18, 54), rng.integers(0, 4)
        e = np.zeros_like(x64)
        e[r, c, bb] = H
        fd.append((dot(gy64, F(x64 + e)) - dot(gy64, F(x64 - e))) / (2 * H))
        got.append(gx[r, c, bb])
    assert fd_check(got, fd, np.max(np.abs(gx))) <= RTOL_FD


def test_adjoint_errors_are_statuses():
    L = N.lib()
    x = torch.zeros((10, 12, 3), device="cuda")
    g_bad = torch.zeros((10, 5, 3), device="cuda")
    assert L.viprs_reduce_adjoint(api.image(g_bad), api.image(x), 2.0, 9, 1, api._stream()) == 10
    assert L.viprs_reduce_adjoint(api.image(g_bad), None, 2.0, 9, 1, api._stream()) == 9
    u8 = torch.zeros((10, 12, 3), device="cuda", dtype=torch.uint8)
    assert L.viprs_reduce_adjoint(api.image(u8), api.image(x), 2.0, 9, 1, api._stream()) == 2
    mm = (ctypes.c_double * 4)(1, 0, 0, 1)
    gy = torch.zeros((8, 8, 3), device="cuda")
    assert L.viprs_affine_grad(api.image(x), api.image(gy), api.image(x), mm, 0.0, 0.0, 2, 0, 0.0, 0, 0, 0, 0, None,
                               api._stream()) == 7
    src4 = torch.zeros((10, 12, 4), device="cuda")
    idx = torch.zeros((8, 8, 2), device="cuda")
    gy4 = torch.zeros((8, 8, 4), device="cuda")
    assert L.viprs_mapim_grad(api.image(src4), api.image(idx), api.image(gy4), None, None, 2, 0, 0.0, 0, 0,
                              api._stream()) == 2
