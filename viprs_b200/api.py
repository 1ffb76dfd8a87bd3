"""Torch-facing mirror of viprs's resample API over the C ABI.

Tensors are CUDA tensors shaped (height, width, bands), row-major and
band-interleaved like viprs tiles.  Every call enqueues the library's sm_100a
kernels on torch's current stream; nothing runs on the CPU.

The names follow viprs: ``reduce_h``/``reduce_v``/``reduce``/``shrink_h``/
``shrink_v``/``shrink``/``affine``/``resize``/``thumbnail`` are the
PipelineBuilder methods (crates/viprs-runtime/src/pipeline/builder/resample.rs)
and ``PipelineBuilder`` chains them into one plan.
"""
import ctypes
import math

import torch

from . import _native as N

KERNELS = {
    "nearest": 0, "bilinear": 1, "linear": 1, "bicubic": 2, "cubic": 2, "quadratic": 3,
    "nohalo": 4, "lbb": 5, "vsqbs": 6, "catmullrom": 7, "lanczos2": 8, "lanczos3": 9,
}
EXTEND = {"black": 0, "white": 1, "background": 2, "copy": 3, "repeat": 4, "mirror": 5}
TARGETS = {"fitbox": 0, "force": 1, "force_exact": 1, "width": 2, "height": 3}
DEMAND = {"any": 0, "thin": 1, "thin_strip": 1, "fat": 2, "smalltile": 3, "small_tile": 3, "full": 4, "oneline": 5}
NODE = {"premultiply": 1, "shrink_h": 2, "shrink_v": 3, "reduce_h": 4, "reduce_v": 5, "affine": 6,
        "extract_area": 7, "unpremultiply": 8, "zoom": 9, "reduce": 10, "shrink": 11}


def _dtype_format(dtype):
    if dtype == torch.uint8:
        return 0
    if dtype == torch.uint16:
        return 1
    if dtype == torch.float32:
        return 2
    raise TypeError(f"unsupported sample type {dtype} (u8, u16 and f32 are on this path)")


def _kernel(k):
    return KERNELS[k] if isinstance(k, str) else int(k)


def _as_hwc(t):
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if t.dim() == 2:
        t = t.unsqueeze(-1)
    if t.dim() != 3:
        raise ValueError("expected a (height, width, bands) tensor")
    if not t.is_contiguous():
        t = t.contiguous()
    return t


def image(t):
    """viprs_image descriptor of a contiguous HWC CUDA tensor."""
    h, w, b = t.shape
    return N.Image(t.data_ptr(), w, h, b, _dtype_format(t.dtype), 0)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _empty(h, w, b, like):
    return torch.empty((h, w, b), dtype=like.dtype, device=like.device)


def reduce_output_len(factor, n):
    """ReduceConfig::output_len (viprs-core/src/resample.rs:92-98)."""
    return int(N.lib().viprs_reduce_output_len(float(factor), int(n)))


def reduce_h(t, factor, kernel="lanczos3"):
    t = _as_hwc(t)
    h, w, b = t.shape
    out = _empty(h, reduce_output_len(factor, w), b, t)
    N.check(N.lib().viprs_reduceh(image(t), image(out), float(factor), _kernel(kernel), _stream()), "reduce_h")
    return out


def reduce_v(t, factor, kernel="lanczos3"):
    t = _as_hwc(t)
    h, w, b = t.shape
    out = _empty(reduce_output_len(factor, h), w, b, t)
    N.check(N.lib().viprs_reducev(image(t), image(out), float(factor), _kernel(kernel), _stream()), "reduce_v")
    return out


def reduce(t, hfactor, vfactor, kernel="lanczos3"):
    t = _as_hwc(t)
    h, w, b = t.shape
    out = _empty(reduce_output_len(vfactor, h), reduce_output_len(hfactor, w), b, t)
    N.check(N.lib().viprs_reduce(image(t), image(out), float(hfactor), float(vfactor), _kernel(kernel),
                                 _stream()), "reduce")
    return out


def shrink_h(t, factor, ceil=False):
    t = _as_hwc(t)
    h, w, b = t.shape
    # factor 0 is rejected by the library (InvalidShrinkParameters), not here
    ow = 0 if factor <= 0 else (-(-w // factor) if ceil else w // factor)
    out = _empty(h, ow, b, t)
    N.check(N.lib().viprs_shrinkh(image(t), image(out), int(factor), int(ceil), _stream()), "shrink_h")
    return out


def shrink_v(t, factor, ceil=False):
    t = _as_hwc(t)
    h, w, b = t.shape
    oh = 0 if factor <= 0 else (-(-h // factor) if ceil else h // factor)
    out = _empty(oh, w, b, t)
    N.check(N.lib().viprs_shrinkv(image(t), image(out), int(factor), int(ceil), _stream()), "shrink_v")
    return out


def shrink(t, hfactor, vfactor):
    t = _as_hwc(t)
    h, w, b = t.shape
    out = _empty(h // vfactor if vfactor > 0 else 0, w // hfactor if hfactor > 0 else 0, b, t)
    N.check(N.lib().viprs_shrink(image(t), image(out), int(hfactor), int(vfactor), _stream()), "shrink")
    return out


def similarity_node(width, height, scale, angle, kernel="bilinear"):
    """The Affine node PipelineBuilder::similarity runs (resample/similarity.rs:47-81)."""
    n = N.Node()
    N.check(N.lib().viprs_similarity_node(float(scale), float(angle), _kernel(kernel), int(width), int(height),
                                          ctypes.byref(n)), "similarity")
    return n


def similarity(t, scale, angle, kernel="bilinear"):
    """PipelineBuilder::similarity: scale and rotate by `angle` degrees onto the
    transformed bounding box, Background(0) (resample/similarity.rs)."""
    t = _as_hwc(t)
    h, w, b = t.shape
    n = similarity_node(w, h, scale, angle, kernel)
    out = _empty(n.out_height, n.out_width, b, t)
    N.check(N.lib().viprs_similarity(image(t), image(out), float(scale), float(angle), _kernel(kernel), _stream()),
            "similarity")
    return out


def zoom(t, xfac, yfac):
    """PipelineBuilder::zoom: integer nearest-neighbour upscale (structural/zoom.rs)."""
    t = _as_hwc(t)
    h, w, b = t.shape
    # a zero factor is rejected by the library (builder/geometry.rs:618-624), not here
    out = _empty(h * max(int(yfac), 0), w * max(int(xfac), 0), b, t)
    N.check(N.lib().viprs_zoom(image(t), image(out), int(xfac), int(yfac), _stream()), "zoom")
    return out


def premultiply(t):
    t = _as_hwc(t)
    out = torch.empty_like(t)
    N.check(N.lib().viprs_premultiply(image(t), image(out), _stream()), "premultiply")
    return out


def unpremultiply(t):
    t = _as_hwc(t)
    out = torch.empty_like(t)
    N.check(N.lib().viprs_unpremultiply(image(t), image(out), _stream()), "unpremultiply")
    return out


def affine(t, matrix, tx, ty, out_w, out_h, kernel="bilinear"):
    """PipelineBuilder::affine: forward matrix, Background(0) extend."""
    t = _as_hwc(t)
    out = _empty(out_h, out_w, t.shape[2], t)
    m = (ctypes.c_double * 4)(*[float(v) for v in matrix])
    N.check(N.lib().viprs_affine(image(t), image(out), m, float(tx), float(ty), _kernel(kernel), _stream()),
            "affine")
    return out


def affine_backward_matrix(t, m, tx, ty, out_w, out_h, kernel="bilinear", extend="background",
                           background=0.0, premultiplied=False, tile_w=0, tile_h=0):
    """Affine with a backward matrix (output -> input), as Affine::try_new takes it."""
    t = _as_hwc(t)
    out = _empty(out_h, out_w, t.shape[2], t)
    mm = (ctypes.c_double * 4)(*[float(v) for v in m])
    N.check(N.lib().viprs_affine_backward_matrix(image(t), image(out), mm, float(tx), float(ty), _kernel(kernel),
                                                 EXTEND[extend] if isinstance(extend, str) else int(extend),
                                                 float(background), int(premultiplied), int(tile_w), int(tile_h),
                                                 _stream()), "affine")
    return out


def forward_affine_to_backward(matrix, tx, ty):
    f = (ctypes.c_double * 4)(*[float(v) for v in matrix])
    b = (ctypes.c_double * 4)()
    btx = ctypes.c_double()
    bty = ctypes.c_double()
    N.check(N.lib().viprs_forward_affine_to_backward(f, float(tx), float(ty), b, ctypes.byref(btx),
                                                     ctypes.byref(bty)), "forward_affine_to_backward")
    return list(b), btx.value, bty.value


def mapim(src, index, kernel="bilinear", extend_copy=False, background=0.0, premultiplied=False):
    """MapImOp (resample/mapim.rs): index is a (h, w, 2) uint8, uint16 or
    float32 tensor of source coordinates, read as f64.  2- and 4-band sources
    are alpha-premultiplied inside the sampler unless `premultiplied` says
    they already are (MapImOp::with_premultiplied, viprs's default false)."""
    src = _as_hwc(src)
    index = _as_hwc(index)
    if index.shape[2] != 2:
        raise ValueError("index must be a (h, w, 2) tensor")
    _dtype_format(index.dtype)
    out = _empty(index.shape[0], index.shape[1], src.shape[2], src)
    N.check(N.lib().viprs_mapim(image(src), image(index), image(out), _kernel(kernel), int(extend_copy),
                                float(background), int(premultiplied), _stream()), "mapim")
    return out


class Plan:
    """A device-resident, allocation-free execution of a builder chain."""

    def __init__(self, handle, in_shape, dtype):
        self._h = handle
        self.in_shape = in_shape
        self.dtype = dtype
        L = N.lib()
        w = ctypes.c_uint32()
        h = ctypes.c_uint32()
        N.check(L.viprs_plan_output_size(self._h, ctypes.byref(w), ctypes.byref(h)), "plan_output_size")
        self.out_shape = (h.value, w.value, in_shape[2])
        n = ctypes.c_int32()
        N.check(L.viprs_plan_launch_count(self._h, ctypes.byref(n)), "plan_launch_count")
        self.launches = n.value
        ws = ctypes.c_uint64()
        N.check(L.viprs_plan_workspace_bytes(self._h, ctypes.byref(ws)), "plan_workspace_bytes")
        self.workspace_bytes = ws.value

    def __call__(self, src, out=None):
        src = _as_hwc(src)
        if tuple(src.shape) != tuple(self.in_shape) or src.dtype != self.dtype:
            raise ValueError(f"plan expects {self.in_shape} {self.dtype}, got {tuple(src.shape)} {src.dtype}")
        if out is None:
            out = torch.empty(self.out_shape, dtype=self.dtype, device=src.device)
        N.check(N.lib().viprs_plan_execute(self._h, ctypes.c_void_p(src.data_ptr()),
                                           ctypes.c_void_p(out.data_ptr()), _stream()), "plan_execute")
        return out

    def run_stages(self, src, out, first, count):
        """Enqueue stages [first, first + count) only (per-kernel timing)."""
        N.check(N.lib().viprs_plan_execute_stages(self._h, int(first), int(count), ctypes.c_void_p(src.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr()), _stream()), "plan_execute_stages")
        return out

    def execute_host(self, host_src, host_dst):
        """Copy a host (pinned) buffer in, run, copy the result out, synchronise."""
        N.check(N.lib().viprs_plan_execute_host(self._h, ctypes.c_void_p(host_src.data_ptr()),
                                                ctypes.c_void_p(host_dst.data_ptr()), _stream()),
                "plan_execute_host")
        return host_dst

    def status(self):
        """Synchronise the current stream; raise ViprsError if a kernel of an
        earlier execution gave up a bounded wait (its output is incomplete)."""
        N.check(N.lib().viprs_plan_status(self._h, _stream()), "plan_status")

    def close(self):
        if self._h:
            N.lib().viprs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _plan_from(status_fn, in_shape, dtype, what):
    handle = ctypes.c_void_p()
    N.check(status_fn(ctypes.byref(handle)), what)
    return Plan(handle, in_shape, dtype)


def thumbnail_plan(width, height, bands, dtype=torch.uint8, target="width", target_width=0,
                   target_height=0, kernel="lanczos3", crop=False):
    """PipelineBuilder::thumbnail(Thumbnail::new(target, kernel)) for an in-memory image."""
    t = TARGETS[target] if isinstance(target, str) else int(target)
    return _plan_from(lambda p: N.lib().viprs_thumbnail_plan_create(width, height, bands, _dtype_format(dtype), t,
                                                                   target_width, target_height, _kernel(kernel),
                                                                   int(crop), p),
                      (height, width, bands), dtype, "thumbnail_plan")


def resize_plan(width, height, bands, dtype, hscale, vscale=None, kernel="lanczos3"):
    vscale = hscale if vscale is None else vscale
    return _plan_from(lambda p: N.lib().viprs_resize_plan_create(width, height, bands, _dtype_format(dtype),
                                                                float(hscale), float(vscale), _kernel(kernel), p),
                      (height, width, bands), dtype, "resize_plan")


def thumbnail(t, target="width", target_width=0, target_height=0, kernel="lanczos3", crop=False):
    t = _as_hwc(t)
    h, w, b = t.shape
    return thumbnail_plan(w, h, b, t.dtype, target, target_width, target_height, kernel, crop)(t)


def resize(t, hscale, vscale=None, kernel="lanczos3"):
    t = _as_hwc(t)
    h, w, b = t.shape
    return resize_plan(w, h, b, t.dtype, hscale, vscale, kernel)(t)


class PipelineBuilder:
    """Fluent chain of resample nodes, executed as one plan (PipelineBuilder mirror).

    >>> out = PipelineBuilder.from_tensor(img).reduce_v(2.0, "bilinear").reduce_h(2.0, "bilinear").run()
    """

    def __init__(self, width, height, bands, dtype, source=None):
        self.width, self.height, self.bands, self.dtype = width, height, bands, dtype
        self.source = source
        self.nodes = []
        self.demand_override = -1
        self._composite = None

    @classmethod
    def from_tensor(cls, t):
        t = _as_hwc(t)
        h, w, b = t.shape
        return cls(w, h, b, t.dtype, t)

    def _node(self, kind, demand="thin", **kw):
        if self._composite is not None:
            raise ValueError("thumbnail/resize must be the only op of this builder")
        n = N.Node()
        n.kind = NODE[kind]
        n.demand_hint = DEMAND[demand]
        n.kernel = 1
        n.extend = 2
        for k, v in kw.items():
            if k == "matrix":
                for i, x in enumerate(v):
                    n.matrix[i] = float(x)
            else:
                setattr(n, k, v)
        self.nodes.append(n)
        return self

    def reduce_h(self, factor, kernel="lanczos3"):
        return self._node("reduce_h", factor=float(factor), kernel=_kernel(kernel))

    def reduce_v(self, factor, kernel="lanczos3"):
        return self._node("reduce_v", factor=float(factor), kernel=_kernel(kernel))

    def reduce(self, hfactor, vfactor, kernel="lanczos3"):
        return self._node("reduce", factor=float(hfactor), vfactor=float(vfactor), kernel=_kernel(kernel))

    def shrink_h(self, factor, ceil=False):
        return self._node("shrink_h", factor_u=int(factor), ceil_mode=int(ceil))

    def shrink_v(self, factor, ceil=False):
        return self._node("shrink_v", factor_u=int(factor), ceil_mode=int(ceil))

    def shrink(self, hfactor, vfactor):
        return self._node("shrink", factor_u=int(hfactor), vfactor_u=int(vfactor))

    def premultiply(self):
        return self._node("premultiply")

    def unpremultiply(self):
        return self._node("unpremultiply")

    def affine(self, matrix, tx, ty, out_w, out_h, kernel="bilinear"):
        bm, btx, bty = forward_affine_to_backward(matrix, tx, ty)
        return self._node("affine", demand="smalltile", matrix=bm, tx=btx, ty=bty, out_width=int(out_w),
                          out_height=int(out_h), kernel=_kernel(kernel), extend=EXTEND["background"],
                          background=0.0)

    def extract_area(self, x, y, w, h):
        return self._node("extract_area", area_x=x, area_y=y, area_width=w, area_height=h)

    def zoom(self, xfac, yfac):
        return self._node("zoom", demand="fat", factor_u=xfac, vfactor_u=yfac)

    def similarity(self, scale, angle, kernel="bilinear"):
        if self._composite is not None:
            raise ValueError("thumbnail/resize must be the only op of this builder")
        w, h = self.output_size()
        self.nodes.append(similarity_node(w, h, scale, angle, kernel))
        return self

    def thumbnail(self, target="width", target_width=0, target_height=0, kernel="lanczos3", crop=False):
        if self.nodes:
            raise ValueError("thumbnail is planned on the source image: call it first")
        self._composite = thumbnail_plan(self.width, self.height, self.bands, self.dtype, target, target_width,
                                         target_height, kernel, crop)
        return self

    def resize(self, hscale, vscale=None, kernel="lanczos3"):
        if self.nodes:
            raise ValueError("resize is planned on the source image: call it first")
        self._composite = resize_plan(self.width, self.height, self.bands, self.dtype, hscale, vscale, kernel)
        return self

    def output_size(self):
        """(width, height) after the nodes so far (PipelineBuilder::current_dimensions)."""
        if self._composite is not None:
            h, w, _ = self._composite.out_shape
            return w, h
        arr = (N.Node * max(1, len(self.nodes)))(*self.nodes)
        ow, oh = ctypes.c_uint32(), ctypes.c_uint32()
        N.check(N.lib().viprs_chain_output_size(self.width, self.height, arr, len(self.nodes), ctypes.byref(ow),
                                                ctypes.byref(oh)), "chain_output_size")
        return ow.value, oh.value

    def build(self):
        if self._composite is not None:
            return self._composite
        arr = (N.Node * max(1, len(self.nodes)))(*self.nodes)
        return _plan_from(lambda p: N.lib().viprs_chain_plan_create(self.width, self.height, self.bands,
                                                                   _dtype_format(self.dtype), arr,
                                                                   len(self.nodes), self.demand_override, p),
                          (self.height, self.width, self.bands), self.dtype, "chain_plan")

    def run(self, src=None):
        src = self.source if src is None else src
        return self.build()(src)


def partition_batch(shapes, parts):
    """Split a batch of (h, w, bands) images over `parts` GPUs by byte
    weight: largest image first, each to the part with the fewest bytes so far
    (ties to the lowest part).  Returns one ascending index list per part.
    Every rank computes the same split from the same shapes, so no exchange
    is needed: each GPU copies its own images in and its thumbnails out."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(shapes)), key=lambda i: (-shapes[i][0] * shapes[i][1] * shapes[i][2], i))
    load = [0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda k: (load[k], k))
        h, w, b = shapes[i]
        load[p] += h * w * b
        out[p].append(i)
    return [sorted(o) for o in out]


def sm_count():
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count





class ThumbnailBatch:
    """Thumbnails of many u8 images of uneven size (FitBox etc.), run either as
    one persistent launch over a device work list (optionally through a CUDA
    graph) or image by image through per-image plans."""

    def __init__(self, shapes, target="fitbox", target_width=256, target_height=256, kernel="lanczos3",
                 crop=False):
        L = N.lib()
        n = len(shapes)
        hs = (ctypes.c_uint32 * n)(*[int(s[0]) for s in shapes])
        ws = (ctypes.c_uint32 * n)(*[int(s[1]) for s in shapes])
        bs = (ctypes.c_uint32 * n)(*[int(s[2]) for s in shapes])
        t = TARGETS[target] if isinstance(target, str) else int(target)
        h = ctypes.c_void_p()
        N.check(L.viprs_thumbnail_batch_create(n, ws, hs, bs, t, target_width, target_height, _kernel(kernel),
                                               int(crop), ctypes.byref(h)), "thumbnail_batch_create")
        self._init(h, shapes)

    def _init(self, h, shapes):
        L = N.lib()
        n = len(shapes)
        self._h = h
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        self.out_shapes = []
        for i in range(n):
            w = ctypes.c_uint32()
            hh = ctypes.c_uint32()
            N.check(L.viprs_batch_output_size(self._h, i, ctypes.byref(w), ctypes.byref(hh)), "batch_output_size")
            self.out_shapes.append((hh.value, w.value, self.shapes[i][2]))
        self._ptr_cache = None

    def work(self):
        items = ctypes.c_int32()
        stages = ctypes.c_int32()
        grid = ctypes.c_int32()
        N.check(N.lib().viprs_batch_work_items(self._h, ctypes.byref(items), ctypes.byref(stages),
                                               ctypes.byref(grid)), "batch_work_items")
        return items.value, stages.value, grid.value

    def launches(self):
        b = ctypes.c_int32()
        p = ctypes.c_int32()
        N.check(N.lib().viprs_batch_launch_count(self._h, ctypes.byref(b), ctypes.byref(p)), "batch_launch_count")
        return b.value, p.value

    def alloc_outputs(self, device="cuda"):
        return [torch.empty(s, dtype=torch.uint8, device=device) for s in self.out_shapes]

    def pointer_arrays(self, srcs, dsts):
        """Device arrays of the buffers' addresses (cached for the same buffers)."""
        key = (tuple(t.data_ptr() for t in srcs), tuple(t.data_ptr() for t in dsts))
        if self._ptr_cache is None or self._ptr_cache[0] != key:
            dev = srcs[0].device
            ps = torch.tensor([t.data_ptr() for t in srcs], dtype=torch.int64, device=dev)
            pd = torch.tensor([t.data_ptr() for t in dsts], dtype=torch.int64, device=dev)
            self._ptr_cache = (key, ps, pd)
        return self._ptr_cache[1], self._ptr_cache[2]

    def run(self, srcs, dsts=None, graph=False):
        dsts = self.alloc_outputs(srcs[0].device) if dsts is None else dsts
        ps, pd = self.pointer_arrays(srcs, dsts)
        fn = N.lib().viprs_batch_execute_graph if graph else N.lib().viprs_batch_execute
        N.check(fn(self._h, ctypes.c_void_p(ps.data_ptr()), ctypes.c_void_p(pd.data_ptr()), _stream()),
                "batch_execute")
        return dsts

    def run_host(self, host_srcs, host_dsts, dev_srcs, dev_dsts, graph=True):
        """Host buffers in and out: copy every (pinned) host image to its device
        buffer, run the batch, copy the thumbnails back, all on the current
        stream, then synchronise."""
        for h, d in zip(host_srcs, dev_srcs):
            d.copy_(h, non_blocking=True)
        self.run(dev_srcs, dev_dsts, graph=graph)
        for d, h in zip(dev_dsts, host_dsts):
            h.copy_(d, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return host_dsts

    def run_per_image(self, srcs, dsts=None):
        dsts = self.alloc_outputs(srcs[0].device) if dsts is None else dsts
        hs = (ctypes.c_uint64 * len(srcs))(*[t.data_ptr() for t in srcs])
        hd = (ctypes.c_uint64 * len(dsts))(*[t.data_ptr() for t in dsts])
        N.check(N.lib().viprs_batch_execute_per_image(self._h, hs, hd, _stream()), "batch_execute_per_image")
        return dsts

    def status(self):
        return int(N.lib().viprs_batch_status(self._h, _stream()))

    def autotune(self, srcs, dsts, repeats=3):
        ps, pd = self.pointer_arrays(srcs, dsts)
        best = ctypes.c_float()
        N.check(N.lib().viprs_batch_autotune(self._h, ctypes.c_void_p(ps.data_ptr()), ctypes.c_void_p(pd.data_ptr()),
                                             _stream(), int(repeats), ctypes.byref(best)), "batch_autotune")
        return self.config(), best.value

    def config(self):
        r = ctypes.c_uint32()
        lag = ctypes.c_int32()
        cap = ctypes.c_int32()
        N.check(N.lib().viprs_batch_get_config(self._h, ctypes.byref(r), ctypes.byref(lag), ctypes.byref(cap)),
                "batch_get_config")
        return {"ring_bytes": r.value, "ring_slots": lag.value, "blocks_per_sm": cap.value}

    def set_config(self, ring_bytes, ring_slots, blocks_per_sm):
        N.check(N.lib().viprs_batch_set_config(self._h, int(ring_bytes), int(ring_slots), int(blocks_per_sm)),
                "batch_set_config")

    def close(self):
        if self._h:
            N.lib().viprs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ChainBatch(ThumbnailBatch):
    """One builder chain (a PipelineBuilder's nodes, e.g. reduce_h + reduce_v)
    on every u8 image of a batch of uneven size, with ThumbnailBatch's
    execution paths."""

    def __init__(self, shapes, builder):
        if builder._composite is not None:
            raise ValueError("thumbnail/resize batches are ThumbnailBatch")
        n = len(shapes)
        hs = (ctypes.c_uint32 * n)(*[int(s[0]) for s in shapes])
        ws = (ctypes.c_uint32 * n)(*[int(s[1]) for s in shapes])
        bs = (ctypes.c_uint32 * n)(*[int(s[2]) for s in shapes])
        arr = (N.Node * max(1, len(builder.nodes)))(*builder.nodes)
        h = ctypes.c_void_p()
        N.check(N.lib().viprs_chain_batch_create(n, ws, hs, bs, arr, len(builder.nodes), builder.demand_override,
                                                 ctypes.byref(h)), "chain_batch_create")
        self._init(h, shapes)
