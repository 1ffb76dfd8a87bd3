"""Parity at the full sizes of the benchmark configurations.

The small-shape parity tests do not reach every tiling of the kernels: the
fused reduce fits its tile to the image, the shrink ring chunks columns by the
ring slot size and the batch splits items by image size.  These tests run the
exact workloads the benchmark times -- the same seeded generators, shapes and
parameters -- through the C ABI and compare with the CPU restatement of viprs:
u8 bit-exact, f32 within a floored relative error of 1e-5.  The gradient
workloads are checked at full size by the adjoint identity
<A x, y> = <x, A^T y> with f64 dot products taken on the device.
"""
import ctypes
import os

import numpy as np
import pytest

from gpu_helpers import assert_same, max_rel_err
from oracle_chain import run_chain

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from viprs_b200 import _native as N  # noqa: E402
from viprs_b200 import api, synth  # noqa: E402

THREADS = os.cpu_count() or 1
BATCH_SEED = 0x5EED0003


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_chain_batch_reduce_uneven(oracle):
    """ChainBatch: one reduce_h(4)+reduce_v(4) chain on u8 images of uneven
    size and band count in one persistent launch, bit-exact per image."""
    rng = np.random.default_rng(0x5EED0008)
    shapes = [(768, 1024, 3), (501, 777, 1), (1200, 333, 4), (64, 2048, 3), (97, 89, 1), (768, 1024, 3)]
    imgs = [torch.from_numpy(rng.integers(0, 256, s, dtype=np.uint8)).cuda() for s in shapes]
    builder = api.PipelineBuilder(1024, 768, 3, torch.uint8).reduce_h(4.0).reduce_v(4.0)
    batch = api.ChainBatch(shapes, builder)
    outs = batch.run(imgs, graph=False)
    outs_g = batch.run(imgs, graph=True)
    for img, out, og in zip(imgs, outs, outs_g):
        exp = run_chain(host(img), [("reduce_h", dict(factor=4.0, kernel="lanczos3")),
                                    ("reduce_v", dict(factor=4.0, kernel="lanczos3"))], threads=THREADS)
        assert np.array_equal(host(out), exp)
        assert np.array_equal(host(og), exp)


def test_chain_batch_zoom(oracle):
    """ChainBatch with a Zoom node after a reduce: the generic persistent
    launch's pixel rows, bit-exact per image."""
    rng = np.random.default_rng(0x5EED0009)
    shapes = [(301, 457, 3), (64, 64, 4), (97, 89, 1)]
    imgs = [torch.from_numpy(rng.integers(0, 256, s, dtype=np.uint8)).cuda() for s in shapes]
    builder = api.PipelineBuilder(457, 301, 3, torch.uint8).reduce_h(2.0).zoom(3, 2)
    batch = api.ChainBatch(shapes, builder)
    outs = batch.run(imgs, graph=False)
    for img, out in zip(imgs, outs):
        exp = oracle.pipeline(host(img), [oracle.make_node("reduceh", factor=2.0, kernel="lanczos3"),
                                          oracle.make_node("zoom", demand="fat", ufactor=3, ceil_mode=2)])
        assert np.array_equal(host(out), exp)


def test_resize_1024x768x3_upscale_2_5(oracle):
    """Resize 2.5 of a 1024x768x3 u8 image: Zoom(2, 2) then the Copy-extend
    Lanczos3 affine tail at 1.25, against the oracle."""
    img = synth.smooth_u8(768, 1024, 3, 0x5EED000A)
    got = host(api.resize(img, 2.5, 2.5, "lanczos3"))
    exp = oracle.resize(host(img), 2.5, 2.5, "lanczos3", threads=THREADS)
    assert got.shape == (1920, 2560, 3)
    assert np.array_equal(got, exp)


def test_chain_batch_reduce_1024x768_x256(oracle):
    """The batched 1024x768x3 workload of the benchmark (256 images)."""
    n = 256
    imgs = [synth.smooth_u8(768, 1024, 3, 0x5EED0000 + i) for i in range(n)]
    builder = api.PipelineBuilder(1024, 768, 3, torch.uint8).reduce_h(4.0).reduce_v(4.0)
    batch = api.ChainBatch([(768, 1024, 3)] * n, builder)
    outs = batch.run(imgs, graph=True)
    for i in (0, 1, 137, 255):
        exp = run_chain(host(imgs[i]), [("reduce_h", dict(factor=4.0, kernel="lanczos3")),
                                        ("reduce_v", dict(factor=4.0, kernel="lanczos3"))], threads=THREADS)
        assert np.array_equal(host(outs[i]), exp)


def test_reduce_1024x768x3_quarter(oracle):
    img = synth.smooth_u8(768, 1024, 3, 0x5EED0000)
    plan = api.PipelineBuilder(1024, 768, 3, torch.uint8).reduce_h(4.0).reduce_v(4.0).build()
    got = host(plan(img))
    exp = run_chain(host(img), [("reduce_h", dict(factor=4.0, kernel="lanczos3")),
                                ("reduce_v", dict(factor=4.0, kernel="lanczos3"))], threads=THREADS)
    assert got.shape == (192, 256, 3)
    assert_same(got, exp, np.uint8)


def test_thumbnail_8192x8192x3_to_400(oracle):
    img = synth.smooth_u8(8192, 8192, 3, 0x5EED0001)
    plan = api.thumbnail_plan(8192, 8192, 3, torch.uint8, "width", 400)
    got = host(plan(img))
    exp = oracle.thumbnail(host(img), "width", 400, 0, "lanczos3", threads=THREADS)
    assert got.shape == (400, 400, 3)
    assert_same(got, exp, np.uint8)


def test_resize_6000x4000x4_f32(oracle):
    img = synth.uniform_f32(4000, 6000, 4, 0x5EED0002)
    plan = api.resize_plan(6000, 4000, 4, torch.float32, 0.37)
    got = host(plan(img))
    exp = oracle.resize(host(img), 0.37, 0.37, "lanczos3", threads=THREADS)
    assert got.shape == (1480, 2220, 4)
    assert max_rel_err(got, exp) <= 1e-5


def test_batch_512_uneven_thumbnails(oracle):
    """Every thumbnail of the 512-image batch, bit-exact against the oracle."""
    shapes = synth.uneven_batch_shapes(512, BATCH_SEED)
    srcs = [synth.smooth_u8(h, w, b, BATCH_SEED * 1000 + i) for i, (h, w, b) in enumerate(shapes)]
    batch = api.ThumbnailBatch(shapes, "fitbox", 256, 256)
    dsts = batch.run(srcs, graph=True)
    torch.cuda.synchronize()
    assert batch.status() == 0
    bad = []
    for i, (s, d) in enumerate(zip(srcs, dsts)):
        exp = oracle.thumbnail(host(s), "fitbox", 256, 256, "lanczos3", threads=THREADS)
        got = host(d)
        if got.shape != exp.shape or not np.array_equal(got, exp):
            bad.append((i, shapes[i]))
    assert not bad, f"{len(bad)} of 512 thumbnails differ: {bad[:8]}"


def _cfg4(n):
    plan = api.PipelineBuilder(1024, 1024, 4, torch.float32).reduce_h(2.0).reduce_v(2.0).build()
    mats = [api.forward_affine_to_backward(m, tx, ty) for m, tx, ty in synth.rotation_matrices(16, 0x5EED0004)]
    return plan, mats[:n]


def test_reduce_affine_forward_16x1024x1024x4(oracle):
    plan, mats = _cfg4(16)
    worst = 0.0
    for i, (bm, btx, bty) in enumerate(mats):
        x = synth.uniform_f32(1024, 1024, 4, 0x5EED0004 + i)
        z = plan(x)
        y = api.affine_backward_matrix(z, bm, btx, bty, 512, 512, "bilinear", "background", 0.0, False)
        zx = run_chain(host(x), [("reduce_h", dict(factor=2.0, kernel="lanczos3")),
                                 ("reduce_v", dict(factor=2.0, kernel="lanczos3"))], threads=THREADS)
        assert max_rel_err(host(z), zx) <= 1e-5
        ey = oracle.affine_backward(host(z), bm, btx, bty, 512, 512, kernel="bilinear", extend="background",
                                    background=0.0, premultiplied=False, threads=THREADS)
        worst = max(worst, max_rel_err(host(y), ey))
    assert worst <= 1e-5


def test_mapim_bicubic_4096_forward(oracle):
    src = synth.uniform_f32(4096, 4096, 1, 0x5EED0005)
    index = synth.displacement_index(4096, 0x5EED0005)
    out = api.mapim(src, index, "bicubic")
    exp = oracle.mapim(host(src), host(index), "bicubic", threads=THREADS)
    assert max_rel_err(host(out), exp) <= 1e-5


@pytest.mark.parametrize("kernel", ["lanczos2", "lanczos3"])
def test_affine_lanczos_u8_rotated_2048_bit_exact(oracle, kernel):
    """u8 Lanczos weights take their sines rounded to nearest on the device:
    a rotated 2048^2 x 4 image matches viprs's glibc-sin weights bit for bit."""
    rng = np.random.default_rng(0x5EED0006)
    img = rng.integers(0, 256, (2048, 2048, 4), dtype=np.uint8)
    img[::7, :, 3] = 0
    th, sc = 0.4137, 0.83
    m = [sc * np.cos(th), -sc * np.sin(th), sc * np.sin(th), sc * np.cos(th)]
    got = api.affine(torch.from_numpy(img).cuda(), m, 301.25, -417.5, 2048, 2048, kernel)
    exp = oracle.affine(img, m, 301.25, -417.5, 2048, 2048, kernel, threads=THREADS)
    assert np.array_equal(host(got), exp)


def test_mapim_lanczos3_u8_2048_bit_exact(oracle):
    rng = np.random.default_rng(0x5EED0007)
    src = rng.integers(0, 256, (2048, 2048, 3), dtype=np.uint8)
    index = synth.displacement_index(2048, 0x5EED0007)
    got = api.mapim(torch.from_numpy(src).cuda(), index, "lanczos3")
    exp = oracle.mapim(src, host(index), "lanczos3", threads=THREADS)
    assert np.array_equal(host(got), exp)


def _ddot(a, b):
    return float((a.double() * b.double()).sum())


def _identity_err(ax, y, x, aty):
    lhs, rhs = _ddot(ax, y), _ddot(x, aty)
    return abs(lhs - rhs) / max(float((ax.double() * y.double()).abs().sum()), 1e-30)


def test_reduce_affine_adjoint_identity_full_size():
    """<A x, y> = <x, A^T y> for reduce_h(2)+reduce_v(2) then the bilinear
    affine in its linear (premultiplied) form, 1024^2 x 4 -> 512^2 x 4."""
    L = N.lib()
    plan, mats = _cfg4(4)
    g = torch.Generator(device="cuda").manual_seed(11)
    for i, (bm, btx, bty) in enumerate(mats):
        x = synth.uniform_f32(1024, 1024, 4, 0x5EED0004 + i)
        z = plan(x)
        y = api.affine_backward_matrix(z, bm, btx, bty, 512, 512, "bilinear", "background", 0.0, True)
        gy = torch.randn((512, 512, 4), generator=g, device="cuda")
        gz = torch.empty_like(z)
        gx = torch.empty_like(x)
        g6 = torch.empty(6, dtype=torch.float64, device="cuda")
        mm = (ctypes.c_double * 4)(*bm)
        N.check(L.viprs_affine_grad(api.image(z), api.image(gy), api.image(gz), mm, btx, bty, 1, 2, 0.0, 1, 0, 0,
                                    0, ctypes.c_void_p(g6.data_ptr()), api._stream()), "affine_grad")
        N.check(L.viprs_reduce_hv_adjoint(api.image(gz), api.image(gx), 2.0, 2.0, 9, api._stream()),
                "reduce_hv_adjoint")
        torch.cuda.synchronize()
        assert _identity_err(y, gy, x, gx) <= 1e-5


@pytest.mark.parametrize("det", [0, 1])
def test_mapim_adjoint_identity_full_size(det):
    """<mapim(x), y> = <x, mapim^T y> for the 4096^2 bicubic workload
    (Background 0: mapim is linear in the source), atomic and deterministic
    scatter."""
    L = N.lib()
    src = synth.uniform_f32(4096, 4096, 1, 0x5EED0005)
    index = synth.displacement_index(4096, 0x5EED0005)
    out = api.mapim(src, index, "bicubic")
    gy = torch.randn((4096, 4096, 1), generator=torch.Generator(device="cuda").manual_seed(5), device="cuda")
    gs = torch.empty_like(src)
    N.check(L.viprs_mapim_grad(api.image(src), api.image(index), api.image(gy), api.image(gs), None, 2, 0, 0.0, 0,
                               det, api._stream()), "mapim_grad")
    torch.cuda.synchronize()
    assert _identity_err(out, gy, src, gs) <= 1e-5
