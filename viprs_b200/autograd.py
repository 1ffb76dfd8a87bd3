"""torch.autograd wrappers of the resample ops over the library's adjoint kernels.

viprs's resample operators are forward only; the backward passes here are the
library's own sm_100a kernels (viprs_reduce_adjoint, viprs_reduce_hv_adjoint,
viprs_affine_grad, viprs_mapim_grad), each the exact transpose / derivative
of the forward entry point it pairs with:

* ``reduce_h`` / ``reduce_v``: ReduceH / ReduceV on f32 (resample/reduceh.rs,
  reducev.rs); backward = the transposed banded weight matrix, evaluated as a
  gather over each input sample's contributing output span.
* ``reduce_hv``: the ReduceH -> ReduceV chain of PipelineBuilder
  (``reduce_h(..).reduce_v(..)``, builder/resample.rs), one fused stage.
* ``affine``: PipelineBuilder::affine with a FORWARD matrix (bilinear).  The
  backward matrix is the builder's inversion (builder/resample.rs:25-60),
  computed exactly by the library for the forward values and by torch (f64)
  for the chain rule, so gradients reach the forward matrix and translation.
* ``affine_backward``: Affine with a backward matrix given directly.
* ``mapim``: MapImOp on f32 with gradients wrt the image and the coordinates.

Image gradients of affine/mapim are a scatter: f32 atomics by default, or with
``deterministic=True`` a fixed-point accumulator whose integer adds make the
result bit-identical from run to run.

Images are f32 CUDA tensors shaped (height, width, bands).
"""
import ctypes

import torch

from . import _native as N
from . import api


def _img(t):
    return api.image(t)


def _f32(t, what):
    t = api._as_hwc(t)
    if t.dtype != torch.float32:
        raise TypeError(f"{what}: the adjoints run on f32 images")
    return t.contiguous()


class _ReduceFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, factor, kernel, horizontal):
        x = _f32(x, "reduce")
        ctx.meta = (x.shape, float(factor), api._kernel(kernel), int(horizontal))
        return api.reduce_h(x, factor, kernel) if horizontal else api.reduce_v(x, factor, kernel)

    @staticmethod
    def backward(ctx, gy):
        shape, factor, kernel, horizontal = ctx.meta
        gy = gy.contiguous()
        gx = torch.empty(shape, dtype=torch.float32, device=gy.device)
        N.check(N.lib().viprs_reduce_adjoint(_img(gy), _img(gx), factor, kernel, horizontal, api._stream()),
                "reduce_adjoint")
        return gx, None, None, None


_HV_PLANS = {}


def _hv_plan(shape, hf, vf, kernel):
    key = (tuple(shape), hf, vf, kernel)
    p = _HV_PLANS.get(key)
    if p is None:
        h, w, b = shape
        p = api.PipelineBuilder(w, h, b, torch.float32).reduce_h(hf, kernel).reduce_v(vf, kernel).build()
        _HV_PLANS[key] = p
    return p


class _ReduceHVFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, hf, vf, kernel):
        x = _f32(x, "reduce_hv")
        k = api._kernel(kernel)
        ctx.meta = (x.shape, float(hf), float(vf), k)
        return _hv_plan(x.shape, float(hf), float(vf), k)(x)

    @staticmethod
    def backward(ctx, gy):
        shape, hf, vf, k = ctx.meta
        gy = gy.contiguous()
        gx = torch.empty(shape, dtype=torch.float32, device=gy.device)
        N.check(N.lib().viprs_reduce_hv_adjoint(_img(gy), _img(gx), hf, vf, k, api._stream()), "reduce_hv_adjoint")
        return gx, None, None, None


def _extend(e):
    return api.EXTEND[e] if isinstance(e, str) else int(e)


class _AffineBackwardFn(torch.autograd.Function):
    """Affine with backward matrix `bm` (4,) and translation `bt` (2,), both f64
    tensors (CPU or CUDA); gradients flow to x, bm and bt."""

    @staticmethod
    def forward(ctx, x, bm, bt, out_w, out_h, extend, background, premultiplied, deterministic):
        x = _f32(x, "affine")
        m = [float(v) for v in bm.detach().cpu().tolist()]
        t = [float(v) for v in bt.detach().cpu().tolist()]
        ctx.save_for_backward(x)
        ctx.meta = (m, t, _extend(extend), float(background), int(premultiplied), int(deterministic),
                    bm.dtype, bm.device)
        return api.affine_backward_matrix(x, m, t[0], t[1], out_w, out_h, "bilinear", _extend(extend),
                                          float(background), bool(premultiplied))

    @staticmethod
    def backward(ctx, gy):
        (x,) = ctx.saved_tensors
        m, t, extend, bg, premul, det, mdt, mdev = ctx.meta
        gy = gy.contiguous()
        need_x = ctx.needs_input_grad[0]
        need_m = ctx.needs_input_grad[1] or ctx.needs_input_grad[2]
        gx = torch.empty_like(x) if need_x else None
        gm = torch.empty(6, dtype=torch.float64, device=x.device) if need_m else None
        mm = (ctypes.c_double * 4)(*m)
        N.check(N.lib().viprs_affine_grad(_img(x), _img(gy), _img(gx) if need_x else None, mm, t[0], t[1],
                                          api.KERNELS["bilinear"], extend, bg, premul, 0, 0, det,
                                          ctypes.c_void_p(gm.data_ptr()) if need_m else None, api._stream()),
                "affine_grad")
        g6 = gm.to(device=mdev, dtype=mdt) if need_m else None
        return (gx, g6[:4] if need_m else None, g6[4:] if need_m else None, None, None, None, None, None, None)


def affine_backward(x, bm, bt, out_w, out_h, extend="background", background=0.0, premultiplied=False,
                    deterministic=False):
    """Affine::try_new(bm, bt) (backward matrix), bilinear, differentiable in x, bm and bt."""
    return _AffineBackwardFn.apply(x, bm, bt, int(out_w), int(out_h), extend, background, premultiplied,
                                   deterministic)


def invert_forward(matrix, t):
    """The builder's inversion (builder/resample.rs:25-60) as f64 torch ops:
    backward matrix inv(M) and translation -inv(M) t.  Values are replaced by
    the library's exact inversion; gradients follow the torch expression."""
    a, b, c, d = matrix[0], matrix[1], matrix[2], matrix[3]
    det = a * d - b * c
    bm = torch.stack([d / det, -b / det, -c / det, a / det])
    bt = torch.stack([-(bm[0] * t[0] + bm[1] * t[1]), -(bm[2] * t[0] + bm[3] * t[1])])
    tv = t.detach().cpu().tolist()
    exact_m, etx, ety = api.forward_affine_to_backward([float(v) for v in matrix.detach().cpu().tolist()],
                                                       float(tv[0]), float(tv[1]))
    em = torch.tensor(exact_m, dtype=bm.dtype, device=bm.device)
    et = torch.tensor([etx, ety], dtype=bt.dtype, device=bt.device)
    return bm + (em - bm).detach(), bt + (et - bt).detach()


def affine(x, matrix, t, out_w, out_h, deterministic=False):
    """PipelineBuilder::affine(matrix, tx, ty, out_w, out_h, Bilinear) (Background 0),
    differentiable in x, the forward matrix (4,) and the translation (2,)."""
    bm, bt = invert_forward(matrix, t)
    return affine_backward(x, bm, bt, out_w, out_h, "background", 0.0, False, deterministic)


class _MapimFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, src, index, kernel, extend_copy, background, premultiplied, deterministic):
        src = _f32(src, "mapim")
        index = _f32(index, "mapim index")
        ctx.save_for_backward(src, index)
        ctx.meta = (api._kernel(kernel), int(extend_copy), float(background), int(premultiplied), int(deterministic))
        return api.mapim(src, index, kernel, bool(extend_copy), float(background), bool(premultiplied))

    @staticmethod
    def backward(ctx, gy):
        src, index = ctx.saved_tensors
        k, ec, bg, premul, det = ctx.meta
        gy = gy.contiguous()
        gs = torch.empty_like(src) if ctx.needs_input_grad[0] else None
        gi = torch.empty_like(index) if ctx.needs_input_grad[1] else None
        N.check(N.lib().viprs_mapim_grad(_img(src), _img(index), _img(gy), _img(gs) if gs is not None else None,
                                         _img(gi) if gi is not None else None, k, ec, bg, premul, det,
                                         api._stream()), "mapim_grad")
        return gs, gi, None, None, None, None, None


def reduce_h(x, factor, kernel="lanczos3"):
    return _ReduceFn.apply(x, factor, kernel, 1)


def reduce_v(x, factor, kernel="lanczos3"):
    return _ReduceFn.apply(x, factor, kernel, 0)


def reduce_hv(x, hfactor, vfactor, kernel="lanczos3"):
    """PipelineBuilder reduce_h(hfactor) then reduce_v(vfactor), one fused stage."""
    return _ReduceHVFn.apply(x, hfactor, vfactor, kernel)


def mapim(src, index, kernel="bicubic", extend_copy=False, background=0.0, premultiplied=False,
          deterministic=False):
    return _MapimFn.apply(src, index, kernel, extend_copy, background, premultiplied, deterministic)
