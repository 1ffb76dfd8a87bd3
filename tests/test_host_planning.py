"""Host planning of the product library (no GPU): tables and planners agree
with the CPU restatement, and integer shortcuts equal viprs's f64 formulas."""
import ctypes

import numpy as np
import pytest


KERNELS = ["nearest", "bilinear", "bicubic", "catmullrom", "lanczos2", "lanczos3"]


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("factor", [1.0, 1.0778947368421052, 1.5, 2.0, 2.7027027027027026, 4.0, 7.3, 19.0])
def test_reduce_kernel_table_matches_oracle(oracle, kernel, factor):
    from viprs_b200 import _native
    lib = _native.lib()
    k = oracle.KERNELS[kernel]
    taps = ctypes.c_int32()
    assert lib.viprs_reduce_kernel_table(factor, k, ctypes.byref(taps), None) == 0
    table = np.zeros((65, taps.value), np.int16)
    assert lib.viprs_reduce_kernel_table(factor, k, ctypes.byref(taps), table.ctypes.data_as(ctypes.c_void_p)) == 0
    otaps, _, _, _, c16 = oracle.reduce_tables(factor, kernel, 0, False)
    assert otaps == taps.value
    assert np.array_equal(table, c16)


def test_reduce_rejections():
    from viprs_b200 import _native
    lib = _native.lib()
    t = ctypes.c_int32()
    assert lib.viprs_reduce_kernel_table(400.0, 9, ctypes.byref(t), None) == 3   # too many taps
    assert lib.viprs_reduce_kernel_table(0.5, 9, ctypes.byref(t), None) == 1     # factor < 1
    assert lib.viprs_reduce_kernel_table(2.0, 5, ctypes.byref(t), None) == 7     # LBB is not separable


@pytest.mark.parametrize("n", [1, 2, 7, 431, 1000, 4000, 6000, 8192])
@pytest.mark.parametrize("factor", [1.0778947368421052, 2.0, 2.7027027027027026, 4.0])
def test_reduce_output_len(n, factor):
    from viprs_b200 import _native
    assert _native.lib().viprs_reduce_output_len(factor, n) == int(np.floor(n / factor + 0.5))


def test_forward_affine_to_backward_matches_oracle(oracle):
    from viprs_b200 import api
    rng = np.random.default_rng(5)
    for _ in range(50):
        th = rng.uniform(-0.5, 0.5)
        s = rng.uniform(0.8, 1.4)
        m = [s * np.cos(th), -s * np.sin(th), s * np.sin(th), s * np.cos(th)]
        tx, ty = rng.uniform(-20, 20, 2)
        assert api.forward_affine_to_backward(m, tx, ty) == oracle.forward_affine_to_backward(m, tx, ty)


def test_premultiply_integer_formula_equals_f64_formula():
    # structural/premultiply.rs:103-112 in f64 versus the kernel's integer form
    c, a = np.meshgrid(np.arange(256, dtype=np.float64), np.arange(256, dtype=np.float64), indexing="ij")
    na = np.clip(a, 0, 255) / 255.0
    prod = c * na
    ref = np.clip(np.where(prod >= 0, np.floor(prod + 0.5), np.ceil(prod - 0.5)), 0, 255)  # half away from zero
    ci, ai = c.astype(np.int64), a.astype(np.int64)
    got = (2 * ci * ai + 255) // 510
    assert np.array_equal(ref.astype(np.int64), got)


def test_unpremultiply_integer_formula_equals_f64_formula():
    # structural/unpremultiply.rs:97-108 in f64 versus the kernel's integer form
    c, a = np.meshgrid(np.arange(256, dtype=np.float64), np.arange(256, dtype=np.float64), indexing="ij")
    with np.errstate(divide="ignore", invalid="ignore"):
        q = (c * 255.0) / a
    ref = np.where(a == 0, 0, np.clip(np.floor(q + 0.5), 0, 255))
    ci, ai = c.astype(np.int64), a.astype(np.int64)
    got = np.where(ai == 0, 0, np.minimum(255, (510 * ci + ai) // np.maximum(2 * ai, 1)))
    assert np.array_equal(ref.astype(np.int64), got)


# ---------------------------------------------------------------- thumbnail planner
# The product planner (plan.cpp) pinned directly to the reference's own planner
# tests (thumbnail.rs:531-683), through viprs_thumbnail_plan_nodes (host only),
# and to the same tests' properties on the CPU restatement.

K_PREMUL, K_SHRINKH, K_SHRINKV, K_REDUCEH, K_REDUCEV, K_AFFINE, K_EXTRACT, K_UNPREMUL = 1, 2, 3, 4, 5, 6, 7, 8


def product_plan(w, h, bands, target, tw, th, kernel="lanczos3", crop=False, hint=True):
    from viprs_b200 import _native as N
    from viprs_b200 import api
    nodes = (N.Node * 32)()
    n, ow, oh, sf = ctypes.c_int32(), ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    st = N.lib().viprs_thumbnail_plan_nodes(api.TARGETS[target], tw, th, api.KERNELS[kernel], int(crop), w, h,
                                            bands, int(hint), nodes, 32, ctypes.byref(n), ctypes.byref(ow),
                                            ctypes.byref(oh), ctypes.byref(sf))
    assert st == 0
    return [nodes[i] for i in range(n.value)], (ow.value, oh.value), sf.value


def test_product_plan_4000x3000_width99():
    # thumbnail.rs:531-550
    nodes, size, sf = product_plan(4000, 3000, 3, "width", 99, 0, hint=True)
    assert sf == 16 and size == (99, 74)
    assert [n.kind for n in nodes] == [K_SHRINKH, K_SHRINKV, K_REDUCEH, K_REDUCEV]
    assert nodes[0].factor_u == 2 and nodes[1].factor_u == 2


def test_product_plan_crop_adds_centre_extract():
    # thumbnail.rs:552-575
    nodes, size, sf = product_plan(400, 200, 3, "fitbox", 120, 120, crop=True, hint=True)
    assert sf == 0 and size == (120, 120)
    assert any(n.kind == K_EXTRACT and n.area_width == 120 and n.area_height == 120 for n in nodes)


def test_product_plan_2048_to_400_integer_shrink_no_affine():
    # thumbnail.rs:587-603
    nodes, _, _ = product_plan(2048, 2048, 3, "width", 400, 0, hint=False)
    assert nodes[0].kind == K_SHRINKH and nodes[0].factor_u == 4
    assert nodes[1].kind == K_SHRINKV and nodes[1].factor_u == 4
    assert not any(n.kind == K_AFFINE for n in nodes)


def _after_reduce(nodes, w):
    """Width after the integer shrink and the reduce of a planned chain, as
    thumbnail.rs:605-626 computes it: round(after_shrink / residual), >= 1."""
    f = next((n.factor_u for n in nodes if n.kind == K_SHRINKH), 1)
    after_shrink = w // f
    r = next((n.factor for n in nodes if n.kind == K_REDUCEH), 1.0)
    return max(1, int(np.floor(after_shrink / r + 0.5))) if r > 1.0 + 1e-9 else after_shrink


def test_product_plan_never_undershoots_requested_width():
    # thumbnail.rs:605-626, over every target width 1 .. 2048 of a 2048 image
    for tw in range(1, 2049):
        nodes, _, _ = product_plan(2048, 2048, 3, "width", tw, 0, hint=False)
        assert _after_reduce(nodes, 2048) >= tw, tw


def test_product_plan_rgba_wraps_alpha():
    # thumbnail.rs:628-645
    nodes, _, _ = product_plan(37, 19, 4, "width", 11, 0, hint=False)
    assert nodes[0].kind == K_PREMUL and nodes[-1].kind == K_UNPREMUL


def test_product_plan_lanczos_affine_tail_is_bicubic():
    # thumbnail.rs:647-661
    from viprs_b200 import api
    nodes, _, _ = product_plan(1, 2048, 3, "height", 0, 400, hint=False)
    assert any(n.kind == K_AFFINE and n.kernel == api.KERNELS["bicubic"] and n.out_width == 1 and n.out_height == 400
               for n in nodes)


def test_product_plan_force_exact_same_size_keeps_dimensions():
    # thumbnail.rs:663-683 (property): ForceExact to the input size
    rng = np.random.default_rng(7)
    for _ in range(300):
        w, h = (int(v) for v in rng.integers(1, 1025, 2))
        bands = int(rng.choice([1, 3, 4]))
        _, size, sf = product_plan(w, h, bands, "force_exact", w, h, hint=True)
        assert sf == 0 and size == (w, h)


@pytest.mark.parametrize("case", [(4000, 3000, 3, "width", 99, 0, True), (400, 200, 3, "fitbox", 120, 120, False),
                                  (2048, 2048, 3, "width", 400, 0, False), (37, 19, 4, "width", 11, 0, False),
                                  (1, 2048, 3, "height", 0, 400, False), (6000, 4000, 4, "fitbox", 256, 256, False),
                                  (8192, 8192, 3, "width", 400, 0, False), (777, 1333, 1, "height", 0, 97, False)])
def test_product_plan_equals_oracle_plan(oracle, case):
    w, h, b, target, tw, th, hint = case
    nodes, size, sf = product_plan(w, h, b, target, tw, th, hint=hint)
    onodes, osize, osf = oracle.thumbnail_plan(w, h, b, target, tw, th, allow_shrink_hint=hint)
    assert size == tuple(osize) and sf == (osf or 0)
    assert [n.kind for n in nodes] == [ORACLE_KIND[n["kind"]] for n in onodes]
    for n, o in zip(nodes, onodes):
        if n.kind in (K_SHRINKH, K_SHRINKV):
            assert n.factor_u == o["factor"]
        elif n.kind in (K_REDUCEH, K_REDUCEV):
            assert n.factor == o["factor"] and n.kernel == o["kernel"]
        elif n.kind == K_AFFINE:
            assert (n.out_width, n.out_height, n.kernel) == (o["out_w"], o["out_h"], o["kernel"])
            assert list(n.matrix) == o["m"] and (n.tx, n.ty) == (o["tx"], o["ty"])
        elif n.kind == K_EXTRACT:
            assert (n.area_x, n.area_y, n.area_width, n.area_height) == (o["x"], o["y"], o["w"], o["h"])


ORACLE_KIND = {"premultiply": K_PREMUL, "shrinkh": K_SHRINKH, "shrinkv": K_SHRINKV, "reduceh": K_REDUCEH,
               "reducev": K_REDUCEV, "affine": K_AFFINE, "extract": K_EXTRACT, "unpremultiply": K_UNPREMUL}


def test_oracle_plan_never_undershoots_requested_width(oracle):
    # thumbnail.rs:605-626 on the CPU restatement's planner
    class _N:
        def __init__(self, n):
            self.kind = ORACLE_KIND[n["kind"]]
            self.factor_u = int(n.get("factor", 1)) if self.kind in (K_SHRINKH, K_SHRINKV) else 1
            self.factor = float(n.get("factor", 1.0))
    for tw in range(1, 2049, 7):
        onodes, _, _ = oracle.thumbnail_plan(2048, 2048, 3, "width", tw, 0, allow_shrink_hint=False)
        assert _after_reduce([_N(n) for n in onodes], 2048) >= tw, tw


def test_oracle_plan_reference_cases(oracle):
    # thumbnail.rs:628-661 on the CPU restatement's planner
    nodes, _, _ = oracle.thumbnail_plan(37, 19, 4, "width", 11, 0, allow_shrink_hint=False)
    assert nodes[0]["kind"] == "premultiply" and nodes[-1]["kind"] == "unpremultiply"
    nodes, _, _ = oracle.thumbnail_plan(1, 2048, 3, "height", 0, 400, allow_shrink_hint=False)
    assert any(n["kind"] == "affine" and n["kernel"] == 2 and (n["out_w"], n["out_h"]) == (1, 400) for n in nodes)


# ---------------------------------------------------------------- resize planner
# The product's resize planner (plan.cpp) pinned to the reference's own resize
# tests (resize.rs:392-535) through viprs_resize_plan_nodes (host only).

K_ZOOM = 9


def product_resize(w, h, hscale, vscale, kernel="lanczos3", gap=2.0):
    from viprs_b200 import _native as N
    from viprs_b200 import api
    nodes = (N.Node * 16)()
    n, ow, oh = ctypes.c_int32(), ctypes.c_uint32(), ctypes.c_uint32()
    st = N.lib().viprs_resize_plan_nodes(float(hscale), float(vscale), api.KERNELS[kernel], float(gap), w, h, nodes,
                                         16, ctypes.byref(n), ctypes.byref(ow), ctypes.byref(oh))
    assert st == 0
    return [nodes[i] for i in range(n.value)], (ow.value, oh.value)


def simulated_dimensions(w, h, nodes):
    from viprs_b200 import _native as N
    L = N.lib()
    for n in nodes:
        if n.kind == K_SHRINKH:
            w //= n.factor_u
        elif n.kind == K_SHRINKV:
            h //= n.factor_u
        elif n.kind == K_REDUCEH:
            w = L.viprs_reduce_output_len(n.factor, w)
        elif n.kind == K_REDUCEV:
            h = L.viprs_reduce_output_len(n.factor, h)
        elif n.kind == K_ZOOM:
            w, h = w * n.factor_u, h * n.vfactor_u
        elif n.kind == K_AFFINE:
            w, h = n.out_width, n.out_height
    return w, h


def test_resize_downscale_4x_shrink2_reduce2_default_gap():
    # resize.rs:399-412
    nodes, _ = product_resize(128, 128, 0.25, 0.25)
    assert [n.kind for n in nodes] == [K_SHRINKV, K_SHRINKH, K_REDUCEV, K_REDUCEH]
    assert nodes[0].factor_u == 2 and nodes[1].factor_u == 2
    assert abs(nodes[2].factor - 2.0) < 1e-9 and abs(nodes[3].factor - 2.0) < 1e-9


def test_resize_downscale_4x_gap1_full_integer_shrink():
    # resize.rs:414-426
    nodes, _ = product_resize(128, 128, 0.25, 0.25, gap=1.0)
    assert [(n.kind, n.factor_u) for n in nodes] == [(K_SHRINKV, 4), (K_SHRINKH, 4)]


def test_resize_nearest_downscale_skips_prefilter_shrink():
    # resize.rs:428-439
    from viprs_b200 import api
    nodes, _ = product_resize(128, 128, 0.25, 0.25, kernel="nearest")
    assert [n.kind for n in nodes] == [K_REDUCEV, K_REDUCEH]
    assert all(abs(n.factor - 4.0) < 1e-9 and n.kernel == api.KERNELS["nearest"] for n in nodes)


def test_resize_mixed_down_and_up():
    # resize.rs:441-458
    from viprs_b200 import api
    nodes, _ = product_resize(100, 100, 0.5, 2.5, kernel="bilinear")
    assert nodes[0].kind == K_REDUCEH and abs(nodes[0].factor - 2.0) < 1e-9
    assert nodes[0].kernel == api.KERNELS["bilinear"]
    assert nodes[1].kind == K_ZOOM and (nodes[1].factor_u, nodes[1].vfactor_u) == (1, 2)
    assert nodes[2].kind == K_AFFINE
    assert simulated_dimensions(100, 100, nodes) == (50, 250)


def test_resize_lbb_downscale_is_one_affine():
    # resize.rs:460-470
    from viprs_b200 import api
    nodes, _ = product_resize(100, 100, 0.6, 0.6, kernel="lbb")
    assert len(nodes) == 1 and nodes[0].kind == K_AFFINE and nodes[0].kernel == api.KERNELS["lbb"]
    assert simulated_dimensions(100, 100, nodes) == (60, 60)


def test_resize_lbb_2x_is_affine():
    # resize.rs:472-486
    nodes, _ = product_resize(25, 25, 2.0, 2.0, kernel="lbb")
    assert len(nodes) == 1 and nodes[0].kind == K_AFFINE
    assert list(nodes[0].matrix) == [0.5, 0.0, 0.0, 0.5] and (nodes[0].out_width, nodes[0].out_height) == (50, 50)


def test_resize_nearest_affine_offset_is_zero():
    # resize.rs:488-499
    nodes, _ = product_resize(100, 100, 1.5, 1.5, kernel="nearest")
    assert len(nodes) == 1 and nodes[0].kind == K_AFFINE and (nodes[0].tx, nodes[0].ty) == (0.0, 0.0)


def test_resize_vsqbs_2x_affine_not_zoom():
    # resize.rs:501-516
    nodes, _ = product_resize(2, 2, 2.0, 2.0, kernel="vsqbs")
    assert len(nodes) == 1 and nodes[0].kind == K_AFFINE
    n = nodes[0]
    assert list(n.matrix) == [0.5, 0.0, 0.0, 0.5] and abs(n.tx - 0.25) < 1e-12 and abs(n.ty - 0.25) < 1e-12
    assert (n.out_width, n.out_height) == (4, 4)


def test_resize_plan_dimensions_match_requested_scales():
    # resize.rs:518-535 (property)
    rng = np.random.default_rng(11)
    for _ in range(400):
        w, h = (int(v) for v in rng.integers(1, 257, 2))
        hs, vs = (float(v) for v in rng.uniform(0.05, 4.0, 2))
        nodes, (ow, oh) = product_resize(w, h, hs, vs)
        assert ow == max(1, int(np.floor(w * hs + 0.5))) and oh == max(1, int(np.floor(h * vs + 0.5)))
        assert simulated_dimensions(w, h, nodes) == (ow, oh)


def _host_image(buf, w, h, bands, fmt, stride=0):
    from viprs_b200 import _native
    im = _native.Image()
    im.data = ctypes.cast(buf, ctypes.c_void_p)
    im.width, im.height, im.bands, im.format, im.row_stride = w, h, bands, fmt, stride
    return im


def test_zoom_parameter_errors_before_any_device_work():
    """PipelineBuilder::zoom rejects a zero factor (builder/geometry.rs:618-624):
    the status comes from the host checks, before any allocation or launch, so
    host buffers that are never touched stand in for the images."""
    from viprs_b200 import _native
    lib = _native.lib()
    buf = (ctypes.c_uint8 * 64)()
    src = _host_image(buf, 4, 4, 1, 0)
    dst = _host_image(buf, 8, 8, 1, 0)
    assert lib.viprs_zoom(ctypes.byref(src), ctypes.byref(dst), 0, 2, None) == 1
    assert lib.viprs_zoom(ctypes.byref(src), ctypes.byref(dst), 2, 0, None) == 1
    # output larger than 2^32 - 1 pixels along an axis
    assert lib.viprs_zoom(ctypes.byref(src), ctypes.byref(dst), 0x40000000, 1, None) == 1


@pytest.mark.parametrize("fmt,stride", [(1, 9), (2, 10), (0, 3), (2, 12)])
def test_row_stride_must_hold_whole_samples(fmt, stride):
    """A row stride that is not a multiple of the sample size, or shorter than
    a row, is INVALID_ARGUMENT before any device work."""
    from viprs_b200 import _native
    lib = _native.lib()
    buf = (ctypes.c_uint8 * 256)()
    src = _host_image(buf, 4, 4, 1, fmt, stride)
    dst = _host_image(buf, 8, 8, 1, fmt)
    assert lib.viprs_zoom(ctypes.byref(src), ctypes.byref(dst), 2, 2, None) == 1


@pytest.mark.parametrize("fmt", [1, 2])
def test_data_must_be_sample_aligned(fmt):
    """u16 / f32 data at an odd address is INVALID_ARGUMENT before any device work."""
    from viprs_b200 import _native
    lib = _native.lib()
    buf = (ctypes.c_uint8 * 256)()
    base = ctypes.addressof(buf)
    src = _host_image(base + 1, 4, 4, 1, fmt)
    dst = _host_image(base, 8, 8, 1, fmt)
    assert lib.viprs_zoom(ctypes.byref(src), ctypes.byref(dst), 2, 2, None) == 1


@pytest.mark.parametrize("scale", [1.0, 0.75, 1.25, 2.0, 0.3, -4.0])
@pytest.mark.parametrize("angle", [0.0, 12.0, 30.0, 45.0, 90.0, 137.5, 180.0, -60.0, 270.0])
@pytest.mark.parametrize("size", [(4, 3), (4, 2), (5, 3), (640, 480), (1, 1), (1023, 17)])
def test_similarity_node_matches_oracle(oracle, scale, angle, size):
    """The product's similarity planner (viprs_similarity_node) against the
    oracle's restatement of SimilarityOp::new_auto_canvas, field for field."""
    from viprs_b200 import _native
    n = _native.Node()
    assert _native.lib().viprs_similarity_node(scale, angle, 1, size[0], size[1], ctypes.byref(n)) == 0
    m, tx, ty, cw, ch = oracle.similarity_node(size[0], size[1], scale, angle)
    assert list(n.matrix) == m and (n.tx, n.ty) == (tx, ty)
    assert (n.out_width, n.out_height) == (cw, ch)
    assert n.kind == 6 and n.extend == 2 and n.background == 0.0 and n.demand_hint == 3


def test_chain_output_size_on_host():
    """viprs_chain_output_size follows the builder's current dimensions."""
    from viprs_b200 import api
    b = api.PipelineBuilder(1024, 768, 3, None).shrink_h(2).zoom(3, 2).reduce_v(2.0)
    assert b.output_size() == (1536, 768)
    b.similarity(1.0, 90.0)
    assert b.output_size() == (768, 1536)
