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
