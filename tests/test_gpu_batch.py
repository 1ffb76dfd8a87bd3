"""Batched thumbnails: the persistent work-list kernel (plain and through a
CUDA graph) and the per-image path must give the same bytes as the CPU
restatement of viprs, image by image."""
import numpy as np
import pytest

from gpu_helpers import smooth_image, to_dev, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from viprs_b200 import api  # noqa: E402


def uneven_shapes(n, seed, wmin=40, wmax=1400):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w = int(round(np.exp(rng.uniform(np.log(wmin), np.log(wmax)))))
        h = max(1, int(round(w / rng.uniform(0.5, 2.0))))
        out.append((h, w, 3 if rng.random() < 0.5 else 4))
    return out


@pytest.mark.parametrize("target", [("fitbox", 256, 256), ("width", 100, 0), ("force", 97, 211)])
def test_batch_matches_oracle_and_per_image(oracle, target):
    shapes = uneven_shapes(24, 7)
    shapes += [(1, 300, 3), (1, 1, 4), (2000, 3, 3), (513, 511, 4)]
    rng = np.random.default_rng(3)
    imgs = [smooth_image(rng, h, w, b) for (h, w, b) in shapes]
    srcs = [to_dev(i) for i in imgs]
    tgt, tw, th = target
    batch = api.ThumbnailBatch(shapes, tgt, tw, th)
    persistent = batch.run(srcs)
    assert batch.status() == 0
    graphed = batch.run(srcs, graph=True)
    graphed2 = batch.run(srcs, dsts=graphed, graph=True)
    per_image = batch.run_per_image(srcs)
    torch.cuda.synchronize()
    for i, img in enumerate(imgs):
        exp = oracle.thumbnail(img, tgt, tw, th, threads=4)
        for got in (persistent[i], graphed2[i], per_image[i]):
            g = to_host(got)
            assert g.shape == exp.shape, (i, shapes[i], g.shape, exp.shape)
            assert np.array_equal(g, exp), f"image {i} {shapes[i]} differs"


def test_batch_config_and_autotune(oracle):
    shapes = uneven_shapes(16, 11, 200, 3000)
    rng = np.random.default_rng(5)
    imgs = [smooth_image(rng, h, w, b) for (h, w, b) in shapes]
    srcs = [to_dev(i) for i in imgs]
    batch = api.ThumbnailBatch(shapes, "fitbox", 256, 256)
    dsts = batch.alloc_outputs()
    cfg, best = batch.autotune(srcs, dsts, repeats=1)
    assert best > 0
    items, stages, grid = batch.work()
    assert items > 0 and stages >= len(shapes) and grid > 0
    for ring, slots, cap in [(4096, 0, 2), (16384, 4, 0), (24576, 3, 1)]:
        batch.set_config(ring, slots, cap)
        out = batch.run(srcs)
        assert batch.status() == 0
        for i, img in enumerate(imgs):
            assert np.array_equal(to_host(out[i]), oracle.thumbnail(img, "fitbox", 256, 256, threads=4))
    # one launch per stage level and kind (shrinks, then fused reduces here),
    # against one launch per stage per image on the plain path
    batched, per_image = batch.launches()
    assert 1 <= batched <= 4 and per_image >= len(shapes)
