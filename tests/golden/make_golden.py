"""Regenerate the golden fixtures under tests/golden/ from the viprs source tree.

The fixtures are the raw u8 outputs that viprs's own tests compare against
(libvips outputs that viprs matches exactly, plus the two approximate
thumbnail fixtures).  Their inputs are regenerated from closed-form formulas
in tests/golden_cases.py, so only the expected outputs are stored.

Usage (needs a viprs checkout):
    python tests/golden/make_golden.py /path/to/viprs
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# (fixture path under tests/fixtures of the viprs tree, local name)
FIXTURES = [
    "reduceh_libvips/rgb_factor2_linear.bin",
    "reduceh_libvips/grayscale_factor1_5_lanczos3.bin",
    "reduceh_libvips/grayscale_factor1_5_cubic.bin",
    "reducev_libvips/rgb_factor2_linear.bin",
    "reducev_libvips/grayscale_factor1_5_lanczos3.bin",
    "reducev_libvips/grayscale_factor1_5_cubic.bin",
    "reduce_libvips/edge_4x4_factor2_linear.bin",
    "reduce_libvips/smooth_grayscale_factor2_lanczos3.bin",
    "shrink_libvips/rgb_factor4.bin",
    "libvips_parity_resample/test_reduceh_factor_1_5_lanczos3.bin",
    "libvips_parity_resample/test_reducev_factor_1_5_lanczos3.bin",
    "libvips_parity_resample/test_resize_half_bilinear_rgb.bin",
    "libvips_parity_resample/test_resize_height_one_rounding.bin",
    "libvips_parity_resample/test_shrink_factor4_rgb.bin",
    "libvips_parity_resample/test_thumbnail_width_128_square.bin",
    "libvips_parity_resample/test_thumbnail_fit_box_40x24.bin",
    "resize_libvips/smooth_gradient_linear_0_75x.bin",
    "resize_libvips/smooth_gradient_linear_0_75x_cache.bin",
    "resize_libvips/smooth_gradient_cubic_0_75x.bin",
    "resize_libvips/smooth_gradient_nearest_2x.bin",
    "shrinkh/grayscale_factor_2.bin",
    "shrinkv/grayscale_factor_2.bin",
]


def main(ref_root):
    out_dir = os.path.join(HERE, "fixtures")
    os.makedirs(out_dir, exist_ok=True)
    manifest = {}
    for rel in FIXTURES:
        src = os.path.join(ref_root, "tests", "fixtures", rel)
        name = rel.replace("/", "__")
        shutil.copyfile(src, os.path.join(out_dir, name))
        manifest[name] = {"source": "tests/fixtures/" + rel, "bytes": os.path.getsize(src)}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print(f"wrote {len(manifest)} fixtures")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/viprs")
    main(sys.argv[1])
