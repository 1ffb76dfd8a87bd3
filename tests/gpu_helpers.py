"""Shared helpers of the GPU parity tests."""
import numpy as np
import torch


def to_dev(a):
    a = np.ascontiguousarray(a)
    if a.ndim == 2:
        a = a[:, :, None]
    if a.dtype == np.uint16:
        t = torch.from_numpy(a.view(np.int16)).cuda().view(torch.uint16)
    else:
        t = torch.from_numpy(a).cuda()
    return t


def to_host(t):
    torch.cuda.synchronize()
    if t.dtype == torch.uint16:
        return t.view(torch.int16).cpu().numpy().view(np.uint16)
    return t.cpu().numpy()


def rand_image(rng, h, w, b, dtype):
    if dtype == np.uint8:
        return rng.integers(0, 256, (h, w, b), dtype=np.uint8)
    if dtype == np.uint16:
        return rng.integers(0, 65536, (h, w, b), dtype=np.uint16)
    return rng.random((h, w, b), dtype=np.float32)


def smooth_image(rng, h, w, b, dtype=np.uint8):
    """Seeded smooth sum of 4 random-frequency sinusoids per band plus uniform
    noise of +-32 around 128, rounded and clamped to 0..255.  Each sinusoid
    sin(u(x) + v(y)) is evaluated as sin u cos v + cos u sin v (outer products),
    which keeps generation of 8192^2 images fast."""
    x = np.arange(w, dtype=np.float64)
    y = np.arange(h, dtype=np.float64)
    out = np.empty((h, w, b), np.float32)
    for c in range(b):
        acc = np.zeros((h, w), np.float64)
        for _ in range(4):
            fx, fy = rng.uniform(0.5, 8.0, 2)
            ph = rng.uniform(0, 2 * np.pi)
            u = 2 * np.pi * fx * x / w + ph
            v = 2 * np.pi * fy * y / h
            acc += 24.0 * (np.outer(np.cos(v), np.sin(u)) + np.outer(np.sin(v), np.cos(u)))
        out[:, :, c] = acc
    out += np.float32(128.0)
    out += rng.uniform(-32, 32, out.shape).astype(np.float32)
    return np.clip(np.rint(out), 0, 255).astype(dtype)


def max_rel_err(a, b, floor=1e-3):
    """Max of |a - b| / max(|b|, floor): the floored relative error used for f32."""
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def assert_same(got, exp, dtype, rel=1e-5):
    assert got.shape == exp.shape, (got.shape, exp.shape)
    if dtype == np.float32:
        err = max_rel_err(got, exp)
        assert err <= rel, f"f32 floored relative error {err} > {rel}"
    else:
        diff = np.abs(got.astype(np.int64) - exp.astype(np.int64))
        assert diff.max(initial=0) == 0, f"{int((diff > 0).sum())} samples differ (max {diff.max()})"
