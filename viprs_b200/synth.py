"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no public dataset is involved).

Pixels: per band, a smooth sum of 4 sinusoids A*sin(2*pi*(fx*x/W + fy*y/H) + phi)
with fx, fy ~ U(0.5, 8), phi ~ U(0, 2*pi), A = 24, plus 128 and uniform noise
U(-32, 32), rounded and clamped to 0..255.  Generated on the device with torch.
"""
import math

import torch


def smooth_u8(h, w, bands, seed, device="cuda"):
    g = torch.Generator().manual_seed(int(seed))
    x = torch.arange(w, dtype=torch.float32, device=device)
    y = torch.arange(h, dtype=torch.float32, device=device)
    out = torch.empty((h, w, bands), dtype=torch.uint8, device=device)
    dg = torch.Generator(device=device).manual_seed(int(seed) ^ 0x9E3779B9)
    for c in range(bands):
        acc = torch.zeros((h, w), dtype=torch.float32, device=device)
        for _ in range(4):
            fx, fy = (0.5 + 7.5 * torch.rand(2, generator=g)).tolist()
            ph = float(2 * math.pi * torch.rand(1, generator=g))
            u = 2 * math.pi * fx * x / w + ph
            v = 2 * math.pi * fy * y / h
            acc += 24.0 * (torch.outer(torch.cos(v), torch.sin(u)) + torch.outer(torch.sin(v), torch.cos(u)))
        acc += 128.0
        acc += torch.rand((h, w), generator=dg, device=device) * 64.0 - 32.0
        out[:, :, c] = acc.round_().clamp_(0, 255).to(torch.uint8)
    return out


def uniform_f32(h, w, bands, seed, device="cuda"):
    g = torch.Generator(device=device).manual_seed(int(seed))
    return torch.rand((h, w, bands), generator=g, device=device, dtype=torch.float32)


def uneven_batch_shapes(n, seed, wmin=256, wmax=6000):
    """Width log-uniform in [wmin, wmax], aspect w/h ~ U(0.5, 2), bands 3 or 4 (p = 0.5)."""
    g = torch.Generator().manual_seed(int(seed))
    shapes = []
    for _ in range(n):
        lw = math.log(wmin) + (math.log(wmax) - math.log(wmin)) * float(torch.rand(1, generator=g))
        w = int(round(math.exp(lw)))
        aspect = 0.5 + 1.5 * float(torch.rand(1, generator=g))
        h = max(1, int(round(w / aspect)))
        b = 3 if float(torch.rand(1, generator=g)) < 0.5 else 4
        shapes.append((h, w, b))
    return shapes


def rotation_matrices(n, seed, centre=256.0):
    """Per image a forward affine of the reduce+affine workload: rotation
    theta ~ U(-30, 30) degrees, scale s ~ U(0.8, 1.4) about the centre of a
    512 x 512 image, translation t ~ U(-20, 20)^2 px.  Returns (M, tx, ty)
    tuples, M = s R(theta) row-major, so that out = M in + (tx, ty)."""
    g = torch.Generator().manual_seed(int(seed))
    out = []
    for _ in range(n):
        th = math.radians(-30 + 60 * float(torch.rand(1, generator=g)))
        s = 0.8 + 0.6 * float(torch.rand(1, generator=g))
        t = (-20 + 40 * torch.rand(2, generator=g)).tolist()
        m = [s * math.cos(th), -s * math.sin(th), s * math.sin(th), s * math.cos(th)]
        tx = centre + t[0] - (m[0] * centre + m[1] * centre)
        ty = centre + t[1] - (m[2] * centre + m[3] * centre)
        out.append((m, tx, ty))
    return out


def displacement_index(size, seed, amplitude=8.0, sigma=32.0, device="cuda"):
    """2-band f32 coordinate image of the mapim workload: the identity grid
    plus a displacement made of N(0, 1) noise, Gaussian-filtered (sigma px,
    separable, zero padding) and scaled to `amplitude` px at its maximum."""
    import torch.nn.functional as F
    g = torch.Generator(device=device).manual_seed(int(seed))
    noise = torch.randn((2, 1, size, size), generator=g, device=device)
    r = int(3 * sigma)
    k = torch.exp(-0.5 * (torch.arange(-r, r + 1, device=device, dtype=torch.float32) / sigma) ** 2)
    k = (k / k.sum()).view(1, 1, 1, -1)
    d = F.conv2d(F.conv2d(noise, k, padding=(0, r)), k.view(1, 1, -1, 1), padding=(r, 0))[:, 0]
    d = d * (amplitude / d.abs().max())
    yy, xx = torch.meshgrid(torch.arange(size, device=device, dtype=torch.float32),
                            torch.arange(size, device=device, dtype=torch.float32), indexing="ij")
    return torch.stack([xx + d[0], yy + d[1]], dim=2).contiguous()
