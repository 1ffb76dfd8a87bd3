"""ctypes front-end of the CPU restatement of viprs's resample path.

TEST INFRASTRUCTURE ONLY.  The parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this module as the checker or as
the timed CPU baseline.  The product package never imports it.

Images are numpy arrays shaped (height, width, bands), row-major and
band-interleaved like viprs's tiles (crates/viprs-core/src/image/region.rs).
"""
import ctypes
import math
import os

import numpy as np

from . import build_oracle

KERNELS = {
    "nearest": 0, "bilinear": 1, "linear": 1, "bicubic": 2, "cubic": 2, "quadratic": 3,
    "nohalo": 4, "lbb": 5, "vsqbs": 6, "catmullrom": 7, "lanczos2": 8, "lanczos3": 9,
}
FORMATS = {np.dtype(np.uint8): 0, np.dtype(np.uint16): 1, np.dtype(np.float32): 2}
TARGETS = {"fitbox": 0, "force": 1, "width": 2, "height": 3}
OP = {"shrinkh": 1, "shrinkv": 2, "reduceh": 3, "reducev": 4, "reduce": 5,
      "premultiply": 6, "unpremultiply": 7, "affine": 8, "shrink": 9, "extract": 10, "zoom": 11}
DEMAND = {"any": 0, "thin": 1, "fat": 2, "smalltile": 3, "full": 4, "oneline": 5}
EXTEND = {"black": 0, "white": 1, "background": 2, "copy": 3, "repeat": 4, "mirror": 5}
PLAN_KINDS = {1: "premultiply", 2: "shrinkh", 3: "shrinkv", 4: "reduceh", 5: "reducev",
              6: "affine", 7: "extract", 8: "unpremultiply", 9: "zoom"}


class OrNode(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("ufactor", ctypes.c_uint32), ("ceil_mode", ctypes.c_int32),
                ("factor", ctypes.c_double), ("vfactor", ctypes.c_double), ("kernel", ctypes.c_int32),
                ("demand_hint", ctypes.c_int32), ("m", ctypes.c_double * 4), ("tx", ctypes.c_double),
                ("ty", ctypes.c_double), ("out_w", ctypes.c_uint32), ("out_h", ctypes.c_uint32),
                ("extend", ctypes.c_int32), ("background", ctypes.c_double),
                ("premultiplied", ctypes.c_int32), ("ex", ctypes.c_uint32), ("ey", ctypes.c_uint32),
                ("ew", ctypes.c_uint32), ("eh", ctypes.c_uint32)]


class OrPlanNode(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("ufactor", ctypes.c_uint32), ("factor", ctypes.c_double),
                ("kernel", ctypes.c_int32), ("m", ctypes.c_double * 4), ("tx", ctypes.c_double),
                ("ty", ctypes.c_double), ("out_w", ctypes.c_uint32), ("out_h", ctypes.c_uint32),
                ("ex", ctypes.c_uint32), ("ey", ctypes.c_uint32), ("ew", ctypes.c_uint32),
                ("eh", ctypes.c_uint32), ("zx", ctypes.c_uint32), ("zy", ctypes.c_uint32)]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = build_oracle.LIB
        if not os.path.exists(path):
            path = build_oracle.build()
        _LIB = ctypes.CDLL(path)
        _LIB.or_kernel_weight.restype = ctypes.c_double
        _LIB.or_kernel_weight.argtypes = [ctypes.c_int32, ctypes.c_double]
    return _LIB


def _kernel(k):
    return KERNELS[k] if isinstance(k, str) else int(k)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def kernel_weight(kernel, x):
    return lib().or_kernel_weight(_kernel(kernel), float(x))


def reduce_tables(factor, kernel, input_len=0, bind=True):
    """taps, pad_before, offset and the 65-phase f64 / i16 tables (reduce_common.rs:137-316)."""
    L = lib()
    taps = ctypes.c_int32()
    pad = ctypes.c_int64()
    off = ctypes.c_double()
    st = L.or_reduce_tables(ctypes.c_double(factor), _kernel(kernel), ctypes.c_uint32(input_len),
                            int(bind), ctypes.byref(taps), ctypes.byref(pad), ctypes.byref(off),
                            None, None)
    if st:
        raise ValueError(f"reduce tables rejected: status {st}")
    c64 = np.zeros((65, taps.value), np.float64)
    c16 = np.zeros((65, taps.value), np.int16)
    L.or_reduce_tables(ctypes.c_double(factor), _kernel(kernel), ctypes.c_uint32(input_len),
                       int(bind), None, None, None, _ptr(c64), _ptr(c16))
    return taps.value, pad.value, off.value, c64, c16


def reduce_plan(factor, kernel, input_len, bind, index):
    s = ctypes.c_int64()
    p = ctypes.c_int32()
    pos = ctypes.c_double()
    lib().or_reduce_plan(ctypes.c_double(factor), _kernel(kernel), ctypes.c_uint32(input_len),
                         int(bind), ctypes.c_double(index), ctypes.byref(s), ctypes.byref(p),
                         ctypes.byref(pos))
    return s.value, p.value, pos.value


def make_node(kind, **kw):
    n = OrNode()
    n.kind = OP[kind]
    n.demand_hint = DEMAND[kw.pop("demand", "thin")]
    if "kernel" in kw:
        n.kernel = _kernel(kw.pop("kernel"))
    if "extend" in kw:
        n.extend = EXTEND[kw.pop("extend")]
    if "m" in kw:
        for i, v in enumerate(kw.pop("m")):
            n.m[i] = float(v)
    for k, v in kw.items():
        setattr(n, k, v)
    return n


def _as_image(img):
    a = np.ascontiguousarray(img)
    if a.ndim == 2:
        a = a[:, :, None]
    if a.dtype not in FORMATS:
        raise TypeError(f"unsupported sample type {a.dtype}")
    return a


def pipeline(img, nodes, demand_override=None, threads=1):
    """Run a node chain tile by tile, as RayonScheduler over MemorySource -> MemorySink."""
    a = _as_image(img)
    h, w, b = a.shape
    L = lib()
    arr = (OrNode * max(1, len(nodes)))(*nodes)
    ow = ctypes.c_uint32()
    oh = ctypes.c_uint32()
    st = L.or_pipeline_dims(arr, len(nodes), w, h, ctypes.byref(ow), ctypes.byref(oh))
    if st:
        raise ValueError(f"pipeline rejected: status {st}")
    out = np.zeros((oh.value, ow.value, b), a.dtype)
    dh = -1 if demand_override is None else DEMAND[demand_override]
    st = L.or_pipeline_run(_ptr(a), w, h, b, FORMATS[a.dtype], arr, len(nodes), dh, int(threads),
                           _ptr(out), ow.value, oh.value)
    if st:
        raise ValueError(f"pipeline failed: status {st}")
    return out


def thumbnail_plan(w, h, bands, target, tw, th, kernel="lanczos3", crop=False, allow_shrink_hint=True):
    nodes = (OrPlanNode * 16)()
    n = ctypes.c_int32()
    ow = ctypes.c_uint32()
    oh = ctypes.c_uint32()
    sol = ctypes.c_uint32()
    st = lib().or_thumbnail_plan(TARGETS[target], tw, th, _kernel(kernel), int(crop), w, h, bands,
                                 int(allow_shrink_hint), nodes, 16, ctypes.byref(n), ctypes.byref(ow),
                                 ctypes.byref(oh), ctypes.byref(sol))
    if st:
        raise ValueError(f"thumbnail plan rejected: status {st}")
    out = []
    for i in range(n.value):
        p = nodes[i]
        kind = PLAN_KINDS[p.kind]
        d = {"kind": kind}
        if kind in ("shrinkh", "shrinkv"):
            d["factor"] = p.ufactor
        elif kind in ("reduceh", "reducev"):
            d["factor"] = p.factor
            d["kernel"] = p.kernel
        elif kind == "affine":
            d.update(m=list(p.m), tx=p.tx, ty=p.ty, out_w=p.out_w, out_h=p.out_h, kernel=p.kernel)
        elif kind == "extract":
            d.update(x=p.ex, y=p.ey, w=p.ew, h=p.eh)
        out.append(d)
    return out, (ow.value, oh.value), sol.value


def resize_plan(w, h, hscale, vscale, kernel="lanczos3", gap=2.0):
    nodes = (OrPlanNode * 16)()
    n = ctypes.c_int32()
    ow = ctypes.c_uint32()
    oh = ctypes.c_uint32()
    st = lib().or_resize_plan(ctypes.c_double(hscale), ctypes.c_double(vscale), _kernel(kernel),
                              ctypes.c_double(gap), w, h, nodes, 16, ctypes.byref(n),
                              ctypes.byref(ow), ctypes.byref(oh))
    if st:
        raise ValueError(f"resize plan rejected: status {st}")
    out = []
    for i in range(n.value):
        p = nodes[i]
        kind = PLAN_KINDS[p.kind]
        d = {"kind": kind}
        if kind in ("shrinkh", "shrinkv"):
            d["factor"] = p.ufactor
        elif kind in ("reduceh", "reducev"):
            d["factor"] = p.factor
        elif kind == "affine":
            d.update(m=list(p.m), tx=p.tx, ty=p.ty, out_w=p.out_w, out_h=p.out_h)
        elif kind == "zoom":
            d.update(x=p.zx, y=p.zy)
        out.append(d)
    return out, (ow.value, oh.value)


def thumbnail(img, target="width", tw=0, th=0, kernel="lanczos3", crop=False, threads=1):
    """PipelineBuilder::thumbnail over a MemorySource (builder/resample.rs:871-979)."""
    a = _as_image(img)
    h, w, b = a.shape
    L = lib()
    ow = ctypes.c_uint32()
    oh = ctypes.c_uint32()
    st = L.or_thumbnail_dims(w, h, b, TARGETS[target], tw, th, _kernel(kernel), int(crop),
                             ctypes.byref(ow), ctypes.byref(oh))
    if st:
        raise ValueError(f"thumbnail rejected: status {st}")
    out = np.zeros((oh.value, ow.value, b), a.dtype)
    st = L.or_thumbnail_run(_ptr(a), w, h, b, FORMATS[a.dtype], TARGETS[target], tw, th,
                            _kernel(kernel), int(crop), int(threads), _ptr(out),
                            ctypes.byref(ow), ctypes.byref(oh))
    if st:
        raise ValueError(f"thumbnail failed: status {st}")
    return out


def resize(img, hscale, vscale=None, kernel="lanczos3", threads=1):
    """PipelineBuilder::resize (builder/resample.rs:637-711), the Zoom upscale included."""
    a = _as_image(img)
    h, w, b = a.shape
    vscale = hscale if vscale is None else vscale
    plan, (ow, oh) = resize_plan(w, h, hscale, vscale, kernel)
    out = np.zeros((oh, ow, b), a.dtype)
    owc = ctypes.c_uint32()
    ohc = ctypes.c_uint32()
    st = lib().or_resize_run(_ptr(a), w, h, b, FORMATS[a.dtype], ctypes.c_double(hscale),
                             ctypes.c_double(vscale), _kernel(kernel), int(threads), _ptr(out),
                             ctypes.byref(owc), ctypes.byref(ohc))
    if st:
        raise ValueError(f"resize failed: status {st}")
    return out


def zoom(img, xfac, yfac, threads=1):
    """PipelineBuilder::zoom (builder/geometry.rs:618-643, structural/zoom.rs)."""
    return pipeline(img, [make_node("zoom", demand="fat", ufactor=xfac, ceil_mode=yfac)], threads=threads)


def reduce_h(img, factor, kernel="lanczos3", threads=1):
    return pipeline(img, [make_node("reduceh", factor=factor, kernel=kernel)], threads=threads)


def reduce_v(img, factor, kernel="lanczos3", threads=1):
    return pipeline(img, [make_node("reducev", factor=factor, kernel=kernel)], threads=threads)


def shrink_h(img, factor, ceil=False, threads=1):
    return pipeline(img, [make_node("shrinkh", ufactor=factor, ceil_mode=int(ceil))], threads=threads)


def shrink_v(img, factor, ceil=False, threads=1):
    return pipeline(img, [make_node("shrinkv", ufactor=factor, ceil_mode=int(ceil))], threads=threads)


def reduce(img, hfactor, vfactor, kernel="lanczos3", threads=1):
    return pipeline(img, [make_node("reduce", factor=hfactor, vfactor=vfactor, kernel=kernel)],
                    threads=threads)


def affine_backward(img, m, tx, ty, out_w, out_h, kernel="bilinear", extend="background",
                    background=0.0, premultiplied=False, demand="smalltile", threads=1):
    """Affine with a BACKWARD matrix (output -> input), bounds = the input image."""
    n = make_node("affine", m=m, tx=float(tx), ty=float(ty), out_w=out_w, out_h=out_h,
                  kernel=kernel, extend=extend, background=float(background),
                  premultiplied=int(premultiplied), demand=demand)
    return pipeline(img, [n], threads=threads)


def _round_vips(v):
    """round_vips (resample/similarity.rs:223-230): half away from zero, truncated."""
    return int(v + 0.5) if v > 0.0 else int(v - 0.5)


def similarity_node(w, h, scale, angle):
    """SimilarityOp::new_auto_canvas (resample/similarity.rs:47-81, 178-221): the
    backward matrix, the canvas translation and the canvas size."""
    s = scale if math.isfinite(scale) and scale > 0.0 else 1.0
    rad = angle * (math.pi / 180.0)
    c, sn = math.cos(rad), math.sin(rad)
    a, b, cc, d = s * c, s * -sn, s * sn, s * c
    left = top = cw = ch = 0
    if w and h:
        W, H = float(w), float(h)
        x2, y2, x3, y3 = a * W, cc * W, b * H, d * H
        x4, y4 = _fma(b, H, a * W), _fma(d, H, cc * W)
        lo_x, hi_x = min(0.0, x2, x3, x4), max(0.0, x2, x3, x4)
        lo_y, hi_y = min(0.0, y2, y3, y4), max(0.0, y2, y3, y4)
        left, top = _round_vips(lo_x), _round_vips(lo_y)
        cw, ch = max(_round_vips(hi_x - lo_x), 0), max(_round_vips(hi_y - lo_y), 0)
    m = [c / s, sn / s, -sn / s, c / s]
    tx = _fma(m[1], float(top), m[0] * float(left))
    ty = _fma(m[3], float(top), m[2] * float(left))
    return m, tx, ty, cw, ch


def similarity(img, scale, angle, kernel="bilinear", threads=1):
    """PipelineBuilder::similarity (builder/resample.rs:595-626): the affine of
    similarity_node with Background(0) on SmallTile tiles."""
    a = _as_image(img)
    m, tx, ty, cw, ch = similarity_node(a.shape[1], a.shape[0], scale, angle)
    return affine_backward(a, m, tx, ty, cw, ch, kernel, "background", 0.0, demand="smalltile", threads=threads)


def forward_affine_to_backward(matrix, tx, ty):
    """PipelineBuilder::forward_affine_to_backward (builder/resample.rs:25-60)."""
    a, b, c, d = [float(v) for v in matrix]
    det = _fma(a, d, -b * c)
    if abs(det) <= np.finfo(np.float64).eps:
        raise ValueError("matrix determinant is singular")
    inv = 1.0 / det
    bm = [d * inv, -b * inv, -c * inv, a * inv]
    btx = -_fma(bm[1], ty, bm[0] * tx)
    bty = -_fma(bm[3], ty, bm[2] * tx)
    return bm, btx, bty


def _fma(a, b, c):
    """Single-rounding a*b+c (Rust f64::mul_add), exact through rationals."""
    from fractions import Fraction
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def affine(img, matrix, tx, ty, out_w, out_h, kernel="bilinear", threads=1):
    """PipelineBuilder::affine: forward matrix, Background(0), SmallTile demand."""
    bm, btx, bty = forward_affine_to_backward(matrix, tx, ty)
    return affine_backward(img, bm, btx, bty, out_w, out_h, kernel=kernel, threads=threads)


def mapim(img, index, kernel="bilinear", extend_copy=False, background=0.0, premultiplied=False,
          threads=1):
    """MapImOp over whole images: `index` is (h, w, 2) of uint8, uint16 or
    float32 source coordinates (read as f64).  2/4-band sources take the
    alpha-premultiplying sampler unless `premultiplied` (mapim.rs:993-1040)."""
    a = _as_image(img)
    sh, sw, b = a.shape
    idx = np.ascontiguousarray(index)
    if idx.dtype not in FORMATS:
        idx = idx.astype(np.float32)
    ih, iw = idx.shape[:2]
    out = np.zeros((ih, iw, b), a.dtype)
    st = lib().or_mapim_run(_ptr(a), sw, sh, b, FORMATS[a.dtype], _ptr(idx), FORMATS[idx.dtype], iw, ih,
                            _kernel(kernel), int(extend_copy), ctypes.c_double(background),
                            int(premultiplied), int(threads), _ptr(out))
    if st:
        raise ValueError(f"mapim failed: status {st}")
    return out
