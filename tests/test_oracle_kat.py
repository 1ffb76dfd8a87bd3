"""Known-answer tests from viprs's unit tests, run against the CPU restatement."""
import numpy as np
import pytest


def test_reduceh_gradient_factor2_bilinear(oracle):
    # reduceh.rs:595-603
    img = np.arange(8, dtype=np.uint8).reshape(1, 8, 1)
    assert oracle.reduce_h(img, 2.0, "bilinear").ravel().tolist() == [1, 3, 5, 6]


def test_reduceh_small_multiband_edge_copy(oracle):
    # reduceh.rs:605-610
    img = np.array([10, 20, 30, 40, 50, 60, 70, 80, 90, 100, 110, 120], np.uint8).reshape(2, 2, 3)
    assert oracle.reduce_h(img, 2.0, "bilinear").ravel().tolist() == [25, 35, 45, 85, 95, 105]


@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "catmullrom", "lanczos2", "lanczos3"])
def test_reduceh_single_pixel_edge_copy(oracle, kernel):
    # reduceh.rs:575-593
    img = np.array([[[173]]], np.uint8)
    assert oracle.reduce_h(img, 2.0, kernel).ravel().tolist() == [173]


def test_bound_offset_factor2(oracle):
    # reduce_common.rs:374-383
    taps, pad, off, _, _ = oracle.reduce_tables(2.0, "bilinear", 8, True)
    assert abs(off + 0.5) < 1e-12
    start, phase, pos = oracle.reduce_plan(2.0, "bilinear", 8, True, 0.0)
    assert abs(pos - 1.0) < 1e-12
    assert start == -1


@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic", "catmullrom", "lanczos2", "lanczos3"])
@pytest.mark.parametrize("factor", [1.0, 1.5, 2.0, 2.5, 4.0])
def test_fixed_point_coefficients_within_truncation_budget(oracle, kernel, factor):
    # reduce_common.rs:350-372
    taps, _, _, c64, c16 = oracle.reduce_tables(factor, kernel, 0, False)
    sums = c16.astype(np.int64).sum(axis=1)
    assert np.all(np.abs(sums - 4096) <= taps)
    if kernel in ("bilinear", "lanczos3") and factor in (2.0, 1.5):
        assert np.all(np.abs(c64.sum(axis=1) - 1.0) < 1e-12)


def test_tap_limit(oracle):
    # reduce_common.rs:412-432: factor 400 exceeds MAX_POINT, factor 4 does not
    with pytest.raises(ValueError):
        oracle.reduce_tables(400.0, "lanczos3")
    assert oracle.reduce_tables(4.0, "lanczos3")[0] == 25


def test_shrinkv_factor19_fixed_point_average(oracle):
    # shrinkv.rs:980-994 against the libvips fixed-point formula
    w, b, f = 6, 3, 19
    h = f * 2
    data = ((np.arange(w * h * b) * 37 + 11) & 0xFF).astype(np.uint8).reshape(h, w, b)
    out = oracle.shrink_v(data, f)
    mult = (1 << 32) // (256 * f)
    sums = data.astype(np.uint64).reshape(2, f, w, b).sum(axis=1) + f // 2
    ref = ((sums * mult) >> 24).astype(np.uint8)
    assert np.array_equal(out, ref)


def test_thumbnail_plan_4000x3000_width99(oracle):
    # thumbnail.rs:531-550
    nodes, (ow, oh), sol = oracle.thumbnail_plan(4000, 3000, 3, "width", 99, 0, allow_shrink_hint=True)
    assert sol == 16 and (ow, oh) == (99, 74)
    assert [n["kind"] for n in nodes] == ["shrinkh", "shrinkv", "reduceh", "reducev"]
    assert nodes[0]["factor"] == 2 and nodes[1]["factor"] == 2


def test_thumbnail_plan_crop_extract(oracle):
    # thumbnail.rs:552-575
    nodes, (ow, oh), sol = oracle.thumbnail_plan(400, 200, 3, "fitbox", 120, 120, crop=True)
    assert sol == 0 and (ow, oh) == (120, 120)
    assert any(n["kind"] == "extract" and n["w"] == 120 and n["h"] == 120 for n in nodes)


def test_thumbnail_plan_2048_to_400(oracle):
    # thumbnail.rs:587-600: integer shrink 4, no affine
    nodes, _, _ = oracle.thumbnail_plan(2048, 2048, 3, "width", 400, 0, allow_shrink_hint=False)
    assert nodes[0] == {"kind": "shrinkh", "factor": 4}
    assert nodes[1] == {"kind": "shrinkv", "factor": 4}
    assert all(n["kind"] != "affine" for n in nodes)


def test_thumbnail_plan_8192_to_400_is_shrink19(oracle):
    # the in-memory plan for the 8192^2 thumbnail-400 workload
    nodes, (ow, oh), _ = oracle.thumbnail_plan(8192, 8192, 3, "width", 400, 0, allow_shrink_hint=False)
    assert (ow, oh) == (400, 400)
    assert [n["kind"] for n in nodes] == ["shrinkh", "shrinkv", "reduceh", "reducev"]
    assert nodes[0]["factor"] == 19 and nodes[1]["factor"] == 19
    assert nodes[2]["factor"] == (8192 / 400) / 19


def test_thumbnail_alpha_wrapping(oracle):
    # thumbnail.rs:438-456: 4-band images are wrapped in premultiply ... unpremultiply
    nodes, _, _ = oracle.thumbnail_plan(1000, 700, 4, "fitbox", 256, 256, allow_shrink_hint=False)
    assert nodes[0]["kind"] == "premultiply" and nodes[-1]["kind"] == "unpremultiply"


def test_resize_plan_cfg2b(oracle):
    # resize.rs:216-238: ShrinkV, ShrinkH, ReduceV, ReduceH order; 6000x4000 x0.37
    nodes, (ow, oh) = oracle.resize_plan(6000, 4000, 0.37, 0.37, "lanczos3")
    assert (ow, oh) == (2220, 1480)
    assert [n["kind"] for n in nodes] == ["reducev", "reduceh"]


def test_uniform_input_stays_uniform(oracle):
    img = np.full((37, 53, 3), 77, np.uint8)
    for out in (oracle.reduce_h(img, 1.7), oracle.reduce_v(img, 2.3), oracle.shrink_h(img, 3),
                oracle.thumbnail(img, "width", 20, 0)):
        assert np.all(out == 77)


def test_factor_one_identity(oracle):
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, (9, 11, 3), dtype=np.uint8)
    assert np.array_equal(oracle.reduce_h(img, 1.0), img)
    assert np.array_equal(oracle.shrink_v(img, 1), img)


def test_affine_identity_nearest(oracle):
    rng = np.random.default_rng(2)
    img = rng.integers(0, 256, (20, 30, 3), dtype=np.uint8)
    out = oracle.affine(img, [1, 0, 0, 1], 0, 0, 30, 20, kernel="nearest")
    assert np.array_equal(out, img)


# ---- affine and mapim unit-test vectors of the reference (tests/kat_vectors.py)

from kat_vectors import AFFINE, AFFINE_WHITE_EDGES, MAPIM  # noqa: E402


@pytest.mark.parametrize("case", AFFINE, ids=[c[0] for c in AFFINE])
def test_affine_reference_vectors(oracle, case):
    name, src, m, tx, ty, ow, oh, kernel, extend, bg, pm, expected = case
    out = oracle.affine_backward(src, m, tx, ty, ow, oh, kernel=kernel, extend=extend, background=bg,
                                 premultiplied=pm)
    assert out.ravel().tolist() == expected.tolist()


def test_affine_reference_white_extend(oracle):
    name, src, m, tx, ty, ow, oh, kernel, extend, parts = AFFINE_WHITE_EDGES
    out = oracle.affine_backward(src, m, tx, ty, ow, oh, kernel=kernel, extend=extend).ravel()
    for sl, exp in parts.items():
        assert out[sl].tolist() == exp


@pytest.mark.parametrize("case", MAPIM, ids=[c[0] for c in MAPIM])
def test_mapim_reference_vectors(oracle, case):
    name, src, idx, kernel, copy, bg, pm, expected = case
    out = oracle.mapim(src, idx, kernel, copy, bg, pm)
    if src.dtype == np.float32:
        assert np.array_equal(out.ravel(), expected.astype(np.float32))
    else:
        assert out.ravel().tolist() == expected.tolist()


def test_mapim_alpha_opaque_matches_premultiplied(oracle):
    # mapim.rs:1949-1989: with alpha 255 everywhere the alpha-premultiplying
    # sampler and the linear one agree
    rng = np.random.default_rng(5)
    src = rng.integers(0, 256, (9, 11, 4), dtype=np.uint8)
    src[..., 3] = 255
    yy, xx = np.mgrid[0:7, 0:8].astype(np.float32)
    idx = np.stack([xx * 1.2 + 0.3, yy * 1.1 + 0.45], -1).astype(np.float32)
    for kernel in ("nearest", "bilinear"):
        assert np.array_equal(oracle.mapim(src, idx, kernel), oracle.mapim(src, idx, kernel, premultiplied=True))


def test_zoom_repeats_nearest_neighbour(oracle):
    """structural/zoom.rs process_region_repeats_nearest_neighbour: Zoom(2, 2)
    of [[1, 2], [3, 4]]."""
    src = np.array([[1, 2], [3, 4]], np.uint8)[:, :, None]
    out = oracle.zoom(src, 2, 2)[:, :, 0]
    assert out.reshape(-1).tolist() == [1, 1, 2, 2, 1, 1, 2, 2, 3, 3, 4, 4, 3, 3, 4, 4]


def test_zoom_output_dimensions_scale_by_factor(oracle):
    """structural/zoom.rs output_dimensions_scale_by_factor: ZoomBridge(3, 2)
    maps 4 x 5 to 12 x 10."""
    out = oracle.zoom(np.zeros((5, 4, 1), np.uint8), 3, 2)
    assert out.shape == (10, 12, 1)


@pytest.mark.parametrize("rows,cols", [(1, 1), (3, 5), (6, 6)])
def test_zoom_factor_1_is_identity(oracle, rows, cols):
    """structural/zoom.rs zoom_factor_1_is_identity (sizes 1..=6)."""
    src = np.arange(rows * cols, dtype=np.uint8).reshape(rows, cols, 1)
    assert np.array_equal(oracle.zoom(src, 1, 1), src)


def test_similarity_canvas_kats(oracle):
    """resample/similarity.rs unit tests: auto canvas of the identity (4 x 3),
    a right angle (4 x 2 -> 2 x 4), scale 1.25 (5 x 3 -> 6 x 4, libvips's
    transform-rect rounding), invalid scales fall back to 1, empty input."""
    assert oracle.similarity_node(4, 3, 1.0, 0.0)[3:] == (4, 3)
    assert oracle.similarity_node(4, 2, 1.0, 90.0)[3:] == (2, 4)
    assert oracle.similarity_node(5, 3, 1.25, 0.0)[3:] == (6, 4)
    assert oracle.similarity_node(0, 3, -4.0, 0.0)[3:] == (0, 0)
    assert oracle.similarity_node(7, 5, float("nan"), 30.0) == oracle.similarity_node(7, 5, 1.0, 30.0)
    assert oracle.similarity_node(7, 5, -4.0, 30.0) == oracle.similarity_node(7, 5, 1.0, 30.0)
    assert oracle._round_vips(-1.2) == -1 and oracle._round_vips(-1.8) == -2


@pytest.mark.parametrize("kernel", ["nearest", "bilinear", "bicubic"])
def test_similarity_identity(oracle, kernel):
    """scale 1, angle 0 is the identity (similarity.rs scale1_angle0_is_identity,
    identity_preserves_uniform_input)."""
    src = np.arange(16, dtype=np.uint8).reshape(4, 4, 1)
    assert np.array_equal(oracle.similarity(src, 1.0, 0.0, kernel), src)
    uni = np.full((5, 7, 1), 173, np.uint8)
    assert np.array_equal(oracle.similarity(uni, 1.0, 0.0, kernel), uni)
