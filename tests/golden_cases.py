"""Golden cases shared by the oracle and GPU parity tests.

Each case restates an input formula and an op chain from viprs's own tests:
  tests/functional/golden/libvips/resample.rs, tests/functional/parity/resample.rs,
  tests/functional/parity/colour.rs:5-53, tests/functional/golden/legacy/resize.rs,
  tests/functional/golden/legacy/transforms.rs:228-255, tests/functional/golden/basic.rs:362-388.
The expected bytes live in tests/golden/fixtures (see tests/golden/make_golden.py).
"""
import os

import numpy as np

FIXTURES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fixtures")


def rgb_source(w, h):
    # golden/libvips/support_inputs.rs:26-36
    y, x = np.mgrid[0:h, 0:w]
    r = (x * 29 + y * 7 + 3) % 256
    g = (x * 11 + y * 23 + 17) % 256
    b = (x * 5 + y * 13 + 29) % 256
    return np.stack([r, g, b], -1).astype(np.uint8)


def grayscale_source(w, h):
    # golden/libvips/support_core.rs:37-45, parity/support.rs:94-102
    y, x = np.mgrid[0:h, 0:w]
    return ((x * 17 + y * 13 + 5) % 256).astype(np.uint8)[:, :, None]


def smooth_grayscale_source(w, h):
    # parity/support.rs:116-120
    y, x = np.mgrid[0:h, 0:w]
    return ((x * 4 + y * 3) % 256).astype(np.uint8)[:, :, None]


def structural_source(w=10, h=16):
    # golden/basic.rs:148-156
    y, x = np.mgrid[0:h, 0:w]
    return ((x * 17 + y * 13) % 256).astype(np.uint8)[:, :, None]


def golden_8x8_prefix(w, h):
    # grayscale_source() of the 8x8 golden support, first w*h bytes, reinterpreted as w x h
    return grayscale_source(8, 8).reshape(-1)[: w * h].reshape(h, w, 1)


# name -> (input builder, chain, expected shape (h, w, bands), tolerance)
# chain: list of (op, kwargs) applied in order through the builder API.
CASES = {
    "reduceh_libvips__rgb_factor2_linear.bin":
        (lambda: rgb_source(8, 6), [("reduce_h", dict(factor=2.0, kernel="bilinear"))], (6, 4, 3), 0),
    "reducev_libvips__rgb_factor2_linear.bin":
        (lambda: rgb_source(6, 8), [("reduce_v", dict(factor=2.0, kernel="bilinear"))], (4, 6, 3), 0),
    "reduceh_libvips__grayscale_factor1_5_lanczos3.bin":
        (lambda: golden_8x8_prefix(8, 6), [("reduce_h", dict(factor=1.5, kernel="lanczos3"))], (6, 5, 1), 0),
    "reducev_libvips__grayscale_factor1_5_lanczos3.bin":
        (lambda: golden_8x8_prefix(6, 8), [("reduce_v", dict(factor=1.5, kernel="lanczos3"))], (5, 6, 1), 0),
    "reduceh_libvips__grayscale_factor1_5_cubic.bin":
        (lambda: grayscale_source(8, 6), [("reduce_h", dict(factor=1.5, kernel="bicubic"))], (6, 5, 1), 0),
    "reducev_libvips__grayscale_factor1_5_cubic.bin":
        (lambda: grayscale_source(6, 8), [("reduce_v", dict(factor=1.5, kernel="bicubic"))], (5, 6, 1), 0),
    "reduce_libvips__edge_4x4_factor2_linear.bin":
        (lambda: np.arange(16, dtype=np.uint8).reshape(4, 4, 1),
         [("reduce_v", dict(factor=2.0, kernel="bilinear")), ("reduce_h", dict(factor=2.0, kernel="bilinear"))],
         (2, 2, 1), 0),
    "reduce_libvips__smooth_grayscale_factor2_lanczos3.bin":
        (lambda: smooth_grayscale_source(8, 8), [("reduce", dict(hfactor=2.0, vfactor=2.0, kernel="lanczos3"))],
         (4, 4, 1), 4),
    "shrink_libvips__rgb_factor4.bin":
        (lambda: rgb_source(16, 16), [("shrink_v", dict(factor=4)), ("shrink_h", dict(factor=4))], (4, 4, 3), 0),
    "libvips_parity_resample__test_reduceh_factor_1_5_lanczos3.bin":
        (lambda: smooth_grayscale_source(8, 6), [("reduce_h", dict(factor=1.5, kernel="lanczos3"))], (6, 5, 1), 0),
    "libvips_parity_resample__test_reducev_factor_1_5_lanczos3.bin":
        (lambda: smooth_grayscale_source(6, 8), [("reduce_v", dict(factor=1.5, kernel="lanczos3"))], (5, 6, 1), 0),
    "libvips_parity_resample__test_resize_half_bilinear_rgb.bin":
        (lambda: rgb_source(16, 12), [("resize", dict(hscale=0.5, vscale=0.5, kernel="bilinear"))], (6, 8, 3), 0),
    "libvips_parity_resample__test_resize_height_one_rounding.bin":
        (lambda: smooth_grayscale_source(100, 1), [("resize", dict(hscale=0.5, vscale=0.5, kernel="bilinear"))],
         (1, 50, 1), 0),
    "libvips_parity_resample__test_shrink_factor4_rgb.bin":
        (lambda: rgb_source(16, 16), [("shrink_v", dict(factor=4)), ("shrink_h", dict(factor=4))], (4, 4, 3), 0),
    "libvips_parity_resample__test_thumbnail_width_128_square.bin":
        (lambda: smooth_grayscale_source(512, 512), [("thumbnail", dict(target="width", tw=128, th=0))],
         (128, 128, 1), 16),
    "libvips_parity_resample__test_thumbnail_fit_box_40x24.bin":
        (lambda: grayscale_source(96, 64), [("thumbnail", dict(target="fitbox", tw=40, th=24))], (24, 36, 1), 20),
    "resize_libvips__smooth_gradient_linear_0_75x.bin":
        (lambda: smooth_grayscale_source(4, 4), [("resize", dict(hscale=0.75, vscale=0.75, kernel="bilinear"))],
         (3, 3, 1), 0),
    "resize_libvips__smooth_gradient_linear_0_75x_cache.bin":
        (lambda: smooth_grayscale_source(4, 4), [("resize", dict(hscale=0.75, vscale=0.75, kernel="bilinear"))],
         (3, 3, 1), 0),
    # 2x nearest: the resize plan is one Zoom(2, 2) node (resize.rs:240-263)
    "resize_libvips__smooth_gradient_nearest_2x.bin":
        (lambda: smooth_grayscale_source(4, 4), [("resize", dict(hscale=2.0, vscale=2.0, kernel="nearest"))],
         (8, 8, 1), 0),
    "resize_libvips__smooth_gradient_cubic_0_75x.bin":
        (lambda: smooth_grayscale_source(4, 4), [("resize", dict(hscale=0.75, vscale=0.75, kernel="bicubic"))],
         (3, 3, 1), 0),
    "shrinkh__grayscale_factor_2.bin":
        (lambda: structural_source(), [("shrink_h", dict(factor=2))], (16, 5, 1), 0),
    "shrinkv__grayscale_factor_2.bin":
        (lambda: structural_source(), [("shrink_v", dict(factor=2))], (8, 10, 1), 0),
}


def expected(name, shape):
    data = np.fromfile(os.path.join(FIXTURES, name), dtype=np.uint8)
    return data.reshape(shape)
