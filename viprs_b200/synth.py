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
