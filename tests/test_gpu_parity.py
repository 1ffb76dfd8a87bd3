"""Parity of the sm_100a path (through the C ABI) with the CPU restatement of
viprs and with viprs's golden fixtures.  u8/u16 must be bit-exact; f32 is
checked with the floored relative error max|a-b|/max(|b|, 1e-3) <= 1e-5."""
import numpy as np
import pytest

from golden_cases import CASES, expected
from gpu_helpers import assert_same, rand_image, smooth_image, to_dev, to_host
from kat_vectors import AFFINE as AFFINE_KAT
from kat_vectors import MAPIM as MAPIM_KAT
from oracle_chain import run_chain

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from viprs_b200 import api  # noqa: E402
from viprs_b200._native import ViprsError  # noqa: E402

FMTS = [np.uint8, np.uint16, np.float32]
KERNELS = ["nearest", "bilinear", "bicubic", "lanczos2", "lanczos3"]


def gpu_chain(img, chain):
    b = api.PipelineBuilder.from_tensor(to_dev(img))
    for op, kw in chain:
        if op == "reduce_h":
            b.reduce_h(kw["factor"], kw["kernel"])
        elif op == "reduce_v":
            b.reduce_v(kw["factor"], kw["kernel"])
        elif op == "reduce":
            b.reduce(kw["hfactor"], kw["vfactor"], kw["kernel"])
        elif op == "shrink_h":
            b.shrink_h(kw["factor"], kw.get("ceil", False))
        elif op == "shrink_v":
            b.shrink_v(kw["factor"], kw.get("ceil", False))
        elif op == "resize":
            b.resize(kw["hscale"], kw["vscale"], kw.get("kernel", "lanczos3"))
        elif op == "thumbnail":
            b.thumbnail(kw["target"], kw["tw"], kw["th"], kw.get("kernel", "lanczos3"), kw.get("crop", False))
        else:
            raise ValueError(op)
    return to_host(b.run())


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_fixture_on_gpu(name):
    build, chain, shape, tol = CASES[name]
    img = build()
    got = gpu_chain(img, chain)
    exp = expected(name, shape)
    assert got.shape == exp.shape
    assert np.abs(got.astype(int) - exp.astype(int)).max() <= tol
    # and bit-exact against the restatement
    assert np.array_equal(got, run_chain(img, chain))


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("factor", [1.0, 1.3, 2.0, 2.7027027027027026, 4.0])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_reduce_h_v(oracle, fmt, kernel, factor, bands):
    rng = np.random.default_rng(hash((str(fmt), kernel, factor, bands)) % 2**32)
    img = rand_image(rng, 23, 41, bands, fmt)
    assert_same(to_host(api.reduce_h(to_dev(img), factor, kernel)), oracle.reduce_h(img, factor, kernel), fmt)
    img = rand_image(rng, 41, 23, bands, fmt)
    assert_same(to_host(api.reduce_v(to_dev(img), factor, kernel)), oracle.reduce_v(img, factor, kernel), fmt)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("hv", [(2.0, 2.0), (1.5, 3.25), (4.0, 1.0)])
def test_reduce_op(oracle, fmt, hv):
    rng = np.random.default_rng(7)
    img = rand_image(rng, 33, 29, 3, fmt)
    got = to_host(api.reduce(to_dev(img), hv[0], hv[1], "lanczos3"))
    assert_same(got, oracle.reduce(img, hv[0], hv[1], "lanczos3"), fmt)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("factor", [1, 2, 3, 5, 7, 19])
@pytest.mark.parametrize("bands", [1, 2, 3, 4, 5])
def test_shrink_h_v(oracle, fmt, factor, bands):
    rng = np.random.default_rng(factor * 10 + bands)
    img = rand_image(rng, 45, 61, bands, fmt)
    for ceil in (False, True):
        assert_same(to_host(api.shrink_h(to_dev(img), factor, ceil)), oracle.shrink_h(img, factor, ceil), fmt)
        assert_same(to_host(api.shrink_v(to_dev(img), factor, ceil)), oracle.shrink_v(img, factor, ceil), fmt)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("fhv", [(2, 2), (3, 5), (19, 19), (1, 4), (6, 1)])
def test_shrink_chains_both_orders(oracle, fmt, fhv):
    rng = np.random.default_rng(fhv[0] * 100 + fhv[1])
    img = rand_image(rng, 77, 83, 3, fmt)
    fh, fv = fhv
    hv = [("shrink_h", dict(factor=fh)), ("shrink_v", dict(factor=fv))]
    vh = [("shrink_v", dict(factor=fv)), ("shrink_h", dict(factor=fh))]
    for chain in (hv, vh):
        assert_same(gpu_chain(img, chain), run_chain(img, chain), fmt)
    assert_same(to_host(api.shrink(to_dev(img), fh, fv)), oracle.pipeline(img, [oracle.make_node("shrink", ufactor=fh, ceil_mode=fv)]), fmt)


@pytest.mark.parametrize("fmt", FMTS)
def test_virtual_plane_chain(oracle, fmt):
    # shrink -> reduce chain: reduce taps beyond the shrunk image read the shrink
    # of edge-replicated source pixels, not clamped shrunk pixels
    rng = np.random.default_rng(11)
    img = rand_image(rng, 190, 230, 3, fmt)
    chain = [("shrink_h", dict(factor=7)), ("shrink_v", dict(factor=6)),
             ("reduce_h", dict(factor=1.37, kernel="lanczos3")), ("reduce_v", dict(factor=1.21, kernel="lanczos3"))]
    assert_same(gpu_chain(img, chain), run_chain(img, chain), fmt)


def test_premultiply_unpremultiply(oracle):
    rng = np.random.default_rng(3)
    img = rand_image(rng, 31, 17, 4, np.uint8)
    pm = oracle.pipeline(img, [oracle.make_node("premultiply")])
    assert np.array_equal(to_host(api.premultiply(to_dev(img))), pm)
    up = oracle.pipeline(img, [oracle.make_node("unpremultiply")])
    assert np.array_equal(to_host(api.unpremultiply(to_dev(img))), up)


THUMB_CASES = [
    (640, 480, 3, "width", 100, 0), (1000, 700, 4, "fitbox", 256, 256), (300, 900, 3, "fitbox", 256, 256),
    (257, 255, 4, "fitbox", 256, 256), (2049, 1537, 3, "width", 400, 0), (999, 1001, 4, "height", 0, 333),
    (500, 1, 3, "width", 100, 0), (1, 1, 4, "fitbox", 10, 10), (400, 200, 3, "fitbox", 120, 120),
    (731, 389, 4, "force", 97, 211), (1536, 1024, 3, "fitbox", 256, 256), (96, 64, 1, "fitbox", 40, 24),
]


@pytest.mark.parametrize("case", THUMB_CASES)
def test_thumbnail(oracle, case):
    w, h, b, target, tw, th = case
    rng = np.random.default_rng(w * 7 + h)
    img = smooth_image(rng, h, w, b)
    for crop in (False, True):
        got = to_host(api.thumbnail(to_dev(img), target, tw, th, "lanczos3", crop))
        exp = oracle.thumbnail(img, target, tw, th, "lanczos3", crop, threads=4)
        assert_same(got, exp, np.uint8)


AFFINE_TAIL_CASES = [(731, 389, 640, 480), (1200, 700, 1500, 100), (600, 900, 640, 480),
                     (300, 200, 97, 211), (50, 41, 97, 211), (300, 200, 640, 480)]


@pytest.mark.parametrize("case", AFFINE_TAIL_CASES)
@pytest.mark.parametrize("bands", [3, 4])
def test_thumbnail_with_affine_tail(oracle, case, bands):
    # ForceExact plans whose geometry needs the bicubic affine correction
    # (Copy extend; ThinStrip tiles above 512 px, SmallTile below)
    w, h, tw, th = case
    plan, _, _ = oracle.thumbnail_plan(w, h, bands, "force", tw, th, allow_shrink_hint=False)
    assert any(n["kind"] == "affine" for n in plan)
    img = smooth_image(np.random.default_rng(w + h + bands), h, w, bands)
    got = to_host(api.thumbnail(to_dev(img), "force", tw, th))
    assert_same(got, oracle.thumbnail(img, "force", tw, th, threads=4), np.uint8)


@pytest.mark.parametrize("fmt", [np.uint8, np.float32])
@pytest.mark.parametrize("scale", [0.75, 0.5, 0.37, 0.2, 0.13])
def test_resize(oracle, fmt, scale):
    rng = np.random.default_rng(int(scale * 100))
    img = rand_image(rng, 157, 211, 4, fmt)
    got = to_host(api.resize(to_dev(img), scale, scale, "lanczos3"))
    assert_same(got, oracle.resize(img, scale, scale, "lanczos3"), fmt)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("fac", [(1, 1), (2, 3), (3, 1), (1, 2), (5, 4)])
@pytest.mark.parametrize("bands", [1, 3, 4])
@pytest.mark.parametrize("width", [53, 64])
def test_zoom(oracle, fmt, fac, bands, width):
    """Zoom: integer nearest-neighbour upscale (structural/zoom.rs).  Width 53
    gives rows that start off 16-byte boundaries (the per-row kernel), width 64
    rows whose pitch is a multiple of 16 (output rows of a source row together)."""
    rng = np.random.default_rng(fac[0] * 7 + fac[1] + bands + width)
    img = rand_image(rng, 37, width, bands, fmt)
    got = to_host(api.zoom(to_dev(img), fac[0], fac[1]))
    exp = oracle.zoom(img, fac[0], fac[1])
    assert np.array_equal(exp, np.repeat(np.repeat(img, fac[1], 0), fac[0], 1))
    assert got.shape == exp.shape and np.array_equal(got, exp)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("area", [(5, 7, 48, 30), (4, 3, 37, 41), (0, 1, 64, 9)])
def test_zoom_then_extract(oracle, fmt, area):
    """Zoom into an intermediate plane whose region starts inside the image
    (the ExtractArea after it asks for an offset window), bit-exact."""
    rng = np.random.default_rng(area[0] * 31 + area[2])
    img = rand_image(rng, 29, 35, 2, fmt)
    b = api.PipelineBuilder.from_tensor(to_dev(img)).zoom(3, 2).extract_area(*area)
    got = to_host(b.run())
    exp = oracle.pipeline(img, [oracle.make_node("zoom", demand="fat", ufactor=3, ceil_mode=2),
                                oracle.make_node("extract", ex=area[0], ey=area[1], ew=area[2], eh=area[3])])
    assert np.array_equal(exp, np.repeat(np.repeat(img, 2, 0), 3, 1)[area[1]:area[1] + area[3],
                                                                       area[0]:area[0] + area[2]])
    assert got.shape == exp.shape and np.array_equal(got, exp)


@pytest.mark.parametrize("fmt", [np.uint8, np.uint16, np.float32])
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos3"])
@pytest.mark.parametrize("sa", [(1.0, 0.0), (0.75, 12.0), (1.25, 90.0), (2.0, 45.0), (0.6, -137.5)])
@pytest.mark.parametrize("bands", [1, 3])
def test_similarity(oracle, fmt, kernel, sa, bands):
    """PipelineBuilder::similarity (resample/similarity.rs): the auto-canvas
    affine, bit-exact (u8/u16) or within the f32 bar against the oracle."""
    rng = np.random.default_rng(int(sa[0] * 100) + abs(int(sa[1])) + bands)
    img = rand_image(rng, 47, 61, bands, fmt)
    got = to_host(api.similarity(to_dev(img), sa[0], sa[1], kernel))
    exp = oracle.similarity(img, sa[0], sa[1], kernel)
    assert got.shape == exp.shape
    assert_same(got, exp, fmt)


def test_similarity_in_a_chain(oracle):
    """similarity after a reduce, through the builder (canvas from the
    chain's current size)."""
    rng = np.random.default_rng(11)
    img = rand_image(rng, 90, 120, 3, np.uint8)
    b = api.PipelineBuilder.from_tensor(to_dev(img)).reduce_h(2.0, "lanczos3").similarity(1.5, 30.0, "bicubic")
    got = to_host(b.run())
    mid = oracle.reduce_h(img, 2.0, "lanczos3")
    m, tx, ty, cw, ch = oracle.similarity_node(mid.shape[1], mid.shape[0], 1.5, 30.0)
    exp = oracle.pipeline(img, [oracle.make_node("reduceh", factor=2.0, kernel="lanczos3"),
                                oracle.make_node("affine", m=m, tx=tx, ty=ty, out_w=cw, out_h=ch, kernel="bicubic",
                                                 extend="background", background=0.0, demand="smalltile")])
    assert got.shape == exp.shape and np.array_equal(got, exp)


def test_zoom_zero_factor_is_an_error():
    img = to_dev(np.zeros((4, 4, 1), np.uint8))
    with pytest.raises(ViprsError):
        api.zoom(img, 0, 2)


@pytest.mark.parametrize("fmt", FMTS)
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos3"])
@pytest.mark.parametrize("scales", [(2.0, 2.0), (2.5, 2.5), (3.7, 1.6), (0.6, 2.3), (2.2, 0.45)])
def test_resize_upscale(oracle, fmt, kernel, scales):
    """Resize plans with the Zoom upscale (resize.rs:240-277): Zoom alone,
    Zoom + Copy-extend affine tail, and mixed down/up plans."""
    rng = np.random.default_rng(int(scales[0] * 100 + scales[1] * 10) + len(kernel))
    img = rand_image(rng, 61, 83, 3, fmt)
    plan, _ = oracle.resize_plan(83, 61, scales[0], scales[1], kernel)
    assert any(n["kind"] == "zoom" for n in plan)
    got = to_host(api.resize(to_dev(img), scales[0], scales[1], kernel))
    assert_same(got, oracle.resize(img, scales[0], scales[1], kernel), fmt)


def _rot(theta, s):
    return [s * np.cos(theta), -s * np.sin(theta), s * np.sin(theta), s * np.cos(theta)]


@pytest.mark.parametrize("fmt", [np.uint8, np.float32])
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos2", "lanczos3"])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_affine_rotated(oracle, fmt, kernel, bands):
    rng = np.random.default_rng(bands * 13 + len(kernel))
    img = rand_image(rng, 150, 170, bands, fmt)
    m = _rot(0.3, 1.15)
    cx, cy = 85.0, 75.0
    tx = cx - (m[0] * cx + m[1] * cy) + 4.5
    ty = cy - (m[2] * cx + m[3] * cy) - 3.25
    got = to_host(api.affine(to_dev(img), m, tx, ty, 181, 143, kernel))
    exp = oracle.affine(img, m, tx, ty, 181, 143, kernel)
    assert_same(got, exp, fmt)


@pytest.mark.parametrize("fmt", [np.uint8, np.float32])
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic"])
@pytest.mark.parametrize("extend", ["background", "copy", "white", "mirror", "repeat"])
def test_affine_axis_aligned_and_extend(oracle, fmt, kernel, extend):
    rng = np.random.default_rng(17)
    img = rand_image(rng, 60, 70, 3, fmt)
    m = [0.61, 0.0, 0.0, 0.83]
    got = to_host(api.affine_backward_matrix(to_dev(img), m, -3.3, 2.1, 130, 90, kernel, extend, 7.0))
    exp = oracle.affine_backward(img, m, -3.3, 2.1, 130, 90, kernel, extend, 7.0)
    assert_same(got, exp, fmt)


@pytest.mark.parametrize("fmt", [np.uint8, np.float32])
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos2", "lanczos3"])
@pytest.mark.parametrize("bands", [1, 3])
def test_mapim(oracle, fmt, kernel, bands):
    rng = np.random.default_rng(bands + len(kernel))
    src = rand_image(rng, 64, 80, bands, fmt)
    yy, xx = np.mgrid[0:50, 0:70].astype(np.float32)
    idx = np.stack([xx * 1.13 - 3.7 + rng.normal(0, 2, xx.shape), yy * 1.21 - 2.2 + rng.normal(0, 2, yy.shape)],
                   -1).astype(np.float32)
    idx[3, 5, 0] = np.nan
    idx[7, 9, 1] = np.inf
    for extend_copy in (False, True):
        got = to_host(api.mapim(to_dev(src), to_dev(idx), kernel, extend_copy, 5.0))
        exp = oracle.mapim(src, idx, kernel, extend_copy, 5.0)
        assert_same(got, exp, fmt)


@pytest.mark.parametrize("fmt", [np.uint8, np.float32])
@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "lanczos3"])
@pytest.mark.parametrize("bands", [2, 4])
def test_mapim_alpha_sampler(oracle, fmt, kernel, bands):
    # MapImOp's default for 2/4-band sources: taps premultiplied by their own
    # alpha, the result divided by the interpolated alpha (mapim.rs:993-1040)
    rng = np.random.default_rng(bands * 31 + len(kernel))
    src = rand_image(rng, 48, 57, bands, fmt)
    if fmt == np.uint8:
        src[::5, ::3, -1] = 0    # transparent pixels keep their colour bytes
        src[1::4, ::2, -1] = 255
    yy, xx = np.mgrid[0:40, 0:52].astype(np.float32)
    idx = np.stack([xx * 1.09 - 2.6 + rng.normal(0, 1.5, xx.shape), yy * 1.17 - 1.9 + rng.normal(0, 1.5, yy.shape)],
                   -1).astype(np.float32)
    idx[2, 4, 0] = np.nan
    for extend_copy in (False, True):
        got = to_host(api.mapim(to_dev(src), to_dev(idx), kernel, extend_copy, 3.0))
        exp = oracle.mapim(src, idx, kernel, extend_copy, 3.0)
        assert_same(got, exp, fmt)


@pytest.mark.parametrize("ifmt", [np.uint8, np.uint16])
@pytest.mark.parametrize("bands", [1, 3, 4])
def test_mapim_integer_index(oracle, ifmt, bands):
    # any index format is read as f64 (mapim.rs:1135-1274)
    rng = np.random.default_rng(bands + 100)
    src = rand_image(rng, 70, 90, bands, np.uint8)
    idx = np.stack([rng.integers(0, 95, (33, 41)), rng.integers(0, 75, (33, 41))], -1).astype(ifmt)
    for kernel in ("nearest", "bilinear", "bicubic"):
        got = to_host(api.mapim(to_dev(src), to_dev(idx), kernel))
        assert_same(got, oracle.mapim(src, idx, kernel), np.uint8)


@pytest.mark.parametrize("case", MAPIM_KAT, ids=[c[0] for c in MAPIM_KAT])
def test_mapim_reference_vectors_on_gpu(case):
    name, src, idx, kernel, copy, bg, pm, expected = case
    got = to_host(api.mapim(to_dev(src), to_dev(idx), kernel, copy, bg, pm)).ravel()
    if src.dtype == np.float32:
        assert np.array_equal(got, expected.astype(np.float32))
    else:
        assert got.tolist() == expected.tolist()


@pytest.mark.parametrize("case", AFFINE_KAT, ids=[c[0] for c in AFFINE_KAT])
def test_affine_reference_vectors_on_gpu(case):
    name, src, m, tx, ty, ow, oh, kernel, extend, bg, pm, expected = case
    got = to_host(api.affine_backward_matrix(to_dev(src), m, tx, ty, ow, oh, kernel, extend, bg, pm)).ravel()
    assert got.tolist() == expected.tolist()


def test_errors_are_statuses():
    t = to_dev(np.zeros((8, 1000, 3), np.uint8))
    with pytest.raises(ViprsError) as e:
        api.reduce_h(t, 0.5)
    assert e.value.status == 1
    with pytest.raises(ViprsError) as e:
        api.reduce_h(t, 400.0, "lanczos3")
    assert e.value.status == 3
    with pytest.raises(ViprsError) as e:
        api.reduce_v(t, 2.0, "lbb")
    assert e.value.status == 7
    with pytest.raises(ViprsError) as e:
        api.affine(t, [1, 2, 2, 4], 0, 0, 8, 8)
    assert e.value.status == 8
    with pytest.raises(ViprsError) as e:
        api.reduce_v(t, float("nan"))
    assert e.value.status == 1
    with pytest.raises(ViprsError) as e:
        api.affine(t, [1, 0, 0, 1], float("inf"), 0, 8, 8)
    assert e.value.status == 1  # InvalidAffineMatrix: non-finite translation
    with pytest.raises(ViprsError):
        api.shrink_h(t, 0)


def test_plan_reuse_and_launch_count():
    rng = np.random.default_rng(1)
    img = smooth_image(rng, 1200, 1600, 3)
    plan = api.thumbnail_plan(1600, 1200, 3, torch.uint8, "width", 200)
    a = to_host(plan(to_dev(img)))
    b = to_host(plan(to_dev(img)))
    assert np.array_equal(a, b)
    assert 1 <= plan.launches <= 4
    plan.status()  # no bounded wait of the warp shrink gave up


def test_strip_plan_status_clean(oracle):
    # the f32 strip kernel's waits report into the plan's error word
    rng = np.random.default_rng(2)
    img = rng.random((900, 1300, 4), dtype=np.float32)
    plan = api.resize_plan(1300, 900, 4, torch.float32, 0.37)
    out = to_host(plan(to_dev(img)))
    plan.status()
    assert_same(out, oracle.resize(img, 0.37, 0.37, "lanczos3"), np.float32)
