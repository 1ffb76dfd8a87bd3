"""Known-answer vectors of viprs's affine and mapim unit tests.

Each vector restates one value-asserting unit test of the reference: the
input pixels, the operator's parameters and the asserted output.  The oracle
tests (test_oracle_kat.py) run them against the CPU restatement and the GPU
tests (test_gpu_parity.py) through the C ABI, so both are pinned to the values
viprs (and, where the test says so, libvips 8.18.2) produces.

Affine vectors use the BACKWARD matrix (output -> input) of `Affine::new`,
an output region at the image origin and the source bounds of the whole input
tile, which is how the reference's `run_affine_*` helpers call it.  Mapim
vectors use `MapImOp::new`'s defaults (bilinear, Background(0), premultiplied
false) unless a field overrides them.
"""
import numpy as np

NAN = float("nan")

# (name, source (h, w, b) array, backward matrix, tx, ty, out_w, out_h, kernel,
#  extend, background, premultiplied, expected flat output)
AFFINE = []


def _aff(name, src, m, tx, ty, ow, oh, kernel, expected, extend="background", background=0.0,
         premultiplied=False):
    AFFINE.append((name, src, m, tx, ty, ow, oh, kernel, extend, background, premultiplied,
                   np.asarray(expected)))


_I = [1.0, 0.0, 0.0, 1.0]
_ramp = np.arange(16, dtype=np.uint8).reshape(4, 4, 1)

# affine/tests.rs:157-170
_aff("output_tile_fully_outside_input_fills_background", np.array([10, 20, 30, 40], np.uint8).reshape(2, 2, 1),
     _I, 10.0, 10.0, 4, 4, "bilinear", [0] * 16)
# affine/tests.rs:224-255, 346-360: identity transforms keep every pixel
_aff("identity_nearest", _ramp, _I, 0.0, 0.0, 4, 4, "nearest", _ramp.ravel())
_aff("identity_bilinear", _ramp, _I, 0.0, 0.0, 4, 4, "bilinear", _ramp.ravel())
_aff("identity_bicubic", _ramp, _I, 0.0, 0.0, 4, 4, "bicubic", _ramp.ravel())
# affine/tests.rs:257-272: 2-band images are not alpha-premultiplied
_two = np.array([11, 64, 42, 95, 203, 0, 7, 255], np.uint8).reshape(2, 2, 2)
_aff("identity_nearest_two_band", _two, _I, 0.0, 0.0, 2, 2, "nearest", _two.ravel())
# affine/tests.rs:427-546: 4-band nearest with tx = -2 over a 3 x 1 source, 7 x 1 output
_ext = np.array([10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33], np.uint8).reshape(1, 3, 4)
_aff("extend_black", _ext, _I, -2.0, 0.0, 7, 1, "nearest",
     [0] * 8 + [10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33] + [0] * 8, extend="black")
_aff("extend_copy", _ext, _I, -2.0, 0.0, 7, 1, "nearest",
     [10, 11, 12, 13, 10, 11, 12, 13, 10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33, 30, 31, 32, 33, 30, 31, 32,
      33], extend="copy")
_aff("extend_repeat", _ext, _I, -2.0, 0.0, 7, 1, "nearest",
     [20, 21, 22, 23, 30, 31, 32, 33, 10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33, 10, 11, 12, 13, 20, 21, 22,
      23], extend="repeat")
_aff("extend_mirror", _ext, _I, -2.0, 0.0, 7, 1, "nearest",
     [20, 21, 22, 23, 10, 11, 12, 13, 10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33, 30, 31, 32, 33, 20, 21, 22,
      23], extend="mirror")
# affine/tests.rs:838-856: transparent edge premultiplied before interpolation
_aff("bilinear_rgba_premultiplies_transparent_edges",
     np.array([255, 0, 0, 0, 0, 0, 255, 255], np.uint8).reshape(1, 2, 4), _I, 0.5, 0.0, 1, 1, "bilinear",
     [0, 0, 255, 128])
# affine/tests.rs:858-877: explicit premultiplied input interpolates every band linearly
_aff("bilinear_rgba_explicit_premultiplied", np.array([0, 0, 0, 0, 0, 0, 255, 255], np.uint8).reshape(1, 2, 4),
     _I, 0.5, 0.0, 1, 1, "bilinear", [0, 0, 128, 128], premultiplied=True)

# The white extend of affine/tests.rs:516-517 asserts only the pixels outside
# the source: checked separately (AFFINE_WHITE_EDGES).
AFFINE_WHITE_EDGES = ("extend_white", _ext, _I, -2.0, 0.0, 7, 1, "nearest", "white",
                      {slice(0, 8): [255] * 8, slice(20, 28): [255] * 8})

# (name, source array, index array, kernel, extend_copy, background, premultiplied, expected flat)
MAPIM = []


def _map(name, src, idx, expected, kernel="bilinear", extend_copy=False, background=0.0, premultiplied=False):
    MAPIM.append((name, src, idx, kernel, extend_copy, background, premultiplied, np.asarray(expected)))


def _idx(pairs, w, h=1, dtype=np.float32):
    return np.asarray(pairs, dtype).reshape(h, w, 2)


_src2 = np.array([10, 20], np.uint8).reshape(1, 2, 1)
# mapim.rs:1991-2030 (libvips 8.18.2 goldens): half a pixel left of the edge
_map("near_edge_background", _src2, _idx([-0.5, 0, 0, 0], 2), [5, 10])
_map("near_edge_copy", _src2, _idx([-0.5, 0, 0, 0], 2), [10, 10], extend_copy=True)
# mapim.rs:2032-2061 (libvips golden): far outside, Copy still gives the background
_map("copy_far_outside", np.array([50, 100], np.uint8).reshape(1, 2, 1), _idx([99, 0], 1), [0], extend_copy=True)
# mapim.rs:2063-2086: non-finite coordinates give the background under Copy
_map("copy_nan_background", np.array([77], np.uint8).reshape(1, 1, 1), _idx([NAN, 0], 1), [13],
     extend_copy=True, background=13.0)
# mapim.rs:2088-2118
_map("background_custom_value", np.array([50, 80], np.uint8).reshape(1, 2, 1), _idx([-5, 0, 0, 0], 2), [42, 50],
     background=42.0)
# mapim.rs:2120-2149
_ident2x2 = _idx([0, 0, 1, 0, 0, 1, 1, 1], 2, 2)
_map("copy_identity", np.array([10, 20, 30, 40], np.uint8).reshape(2, 2, 1), _ident2x2, [10, 20, 30, 40],
     extend_copy=True)
# mapim.rs:2151-2185
_map("premultiplied_true_identity_two_band", np.array([100, 200, 50, 150], np.uint8).reshape(1, 2, 2),
     _idx([0, 0, 1, 0], 2), [100, 200, 50, 150], premultiplied=True)
# mapim.rs:2187-2219
_map("alpha_full_opaque", np.array([128, 255], np.uint8).reshape(1, 1, 2), _idx([0, 0], 1), [128, 255])
# mapim.rs:2221-2247
_map("alpha_half_pixel_no_colour_bleed", np.array([255, 0, 0, 0, 0, 0, 255, 255], np.uint8).reshape(1, 2, 4),
     _idx([0.5, 0], 1), [0, 0, 255, 128])
# mapim.rs:2249-2281
_map("alpha_non_constant_stencil", np.array([255, 0, 0, 128, 0, 255, 0, 64], np.uint8).reshape(1, 2, 4),
     _idx([0.5, 0], 1), [170, 85, 0, 96])
# mapim.rs:2283-2314
_map("alpha_low_alpha_detail", np.array([127, 0, 0, 1, 0, 0, 0, 0], np.uint8).reshape(1, 2, 4),
     _idx([0.5, 0], 1), [127, 0, 0, 1])
# mapim.rs:2316-2345: f32 alpha in [0, 1]
_map("alpha_float_unit_range", np.array([1, 0, 0, 0, 0, 0, 1, 1], np.float32).reshape(1, 2, 4),
     _idx([0.5, 0], 1), [0.0, 0.0, 1.0, 0.5])
# mapim.rs:2347-2376, 2586-2623
_map("alpha_zero_gives_zero_colour", np.array([200, 0], np.uint8).reshape(1, 1, 2), _idx([0, 0], 1), [0, 0])
# mapim.rs:2487-2521
_map("half_pixel_bilinear", np.array([0, 100], np.uint8).reshape(1, 2, 1), _idx([0.5, 0], 1), [50])
_map("half_pixel_nearest", np.array([0, 100], np.uint8).reshape(1, 2, 1), _idx([0.5, 0], 1), [0], kernel="nearest")
# mapim.rs:2523-2544
_map("rgb_no_alpha_premultiply", np.array([100, 0, 10, 0, 100, 250], np.uint8).reshape(1, 2, 3),
     _idx([0.5, 0], 1), [50, 50, 130])
# mapim.rs:2625-2682 (libvips 8.18.2 golden): default RGBA sampling
_rgba = np.array([200, 100, 50, 0, 10, 20, 30, 255], np.uint8).reshape(1, 2, 4)
_map("rgba_default_golden", _rgba, _idx([0, 0, 1, 0], 2), [0, 0, 0, 0, 10, 20, 30, 255])
_map("rgba_premultiplied_true_passthrough", _rgba, _idx([0, 0, 1, 0], 2), _rgba.ravel(), premultiplied=True)
# mapim.rs:1660-1679: a u16 index image
_map("u16_index_identity", np.array([10, 20, 30, 40], np.uint8).reshape(2, 2, 1),
     _idx([0, 0, 1, 0, 0, 1, 1, 1], 2, 2, np.uint16), [10, 20, 30, 40])
# the same identity map as a u8 index image (the reference reads every index
# format through ToF64, mapim.rs:1135-1274)
_map("u8_index_identity", np.array([10, 20, 30, 40], np.uint8).reshape(2, 2, 1),
     _idx([0, 0, 1, 0, 0, 1, 1, 1], 2, 2, np.uint8), [10, 20, 30, 40])
