"""Seeded synthetic float32 fields with the shapes, sizes and value
distributions of the benchmark configurations (no public dataset is named by
the reference; these generators stand in for real fields).

* ``sinusoid`` -- sum of ``waves`` random 3-D sinusoids ``a*sin(2*pi*(k.x)+phi)``
  on [0,1)^3 with ``a ~ U[0.1,1]``, each wavenumber component ``~ U[1,16]``,
  ``phi ~ U[0,2*pi)``, plus N(0, noise^2) noise and optional +-``outlier_mag``
  outliers at a seeded fraction of distinct positions.
* ``grf`` -- Gaussian random field with power spectrum ``P(k) ~ k^-slope``
  (FFT of seeded white noise), unit variance.
* ``white`` -- white noise ``U[-1,1]``.

Parameters are drawn with numpy's PCG64 so a seed fixes them everywhere; the
bulk arithmetic runs in torch on the requested device (float64, then rounded to
float32), so a field is reproducible on one device but may differ in the last
bit between CPU and GPU generation.  Tests always hand the same bytes to both
implementations they compare.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _params(seed: int, waves: int):
    rng = np.random.Generator(np.random.PCG64(seed))
    amp = rng.uniform(0.1, 1.0, waves)
    k = rng.uniform(1.0, 16.0, (waves, 3))
    phi = rng.uniform(0.0, 2.0 * math.pi, waves)
    return rng, amp, k, phi


def sinusoid(shape, seed: int, waves: int = 8, noise: float = 1e-3,
             outlier_frac: float = 0.0, outlier_mag: float = 1e6,
             device: str | torch.device = "cpu") -> torch.Tensor:
    """3-D (or 1-/2-D, padded with unit axes) sum-of-sinusoids field."""
    shape = tuple(int(s) for s in shape)
    dims = (shape + (1, 1, 1))[:3]
    rng, amp, k, phi = _params(seed, waves)
    dev = torch.device(device)
    axes = [torch.arange(n, dtype=torch.float64, device=dev) / n for n in dims]
    out = torch.empty(dims, dtype=torch.float32, device=dev)
    x = axes[0].view(-1, 1, 1)
    y = axes[1].view(1, -1, 1)
    z = axes[2].view(1, 1, -1)
    slab = max(1, (1 << 24) // max(1, dims[1] * dims[2]))
    for s0 in range(0, dims[0], slab):
        xs = x[s0:s0 + slab]
        acc = torch.zeros((xs.shape[0], dims[1], dims[2]), dtype=torch.float64, device=dev)
        for w in range(waves):
            ph = 2.0 * math.pi * (k[w, 0] * xs + k[w, 1] * y + k[w, 2] * z) + phi[w]
            acc += amp[w] * torch.sin(ph)
        out[s0:s0 + slab] = acc.to(torch.float32)
    flat = out.view(-1)
    n = flat.numel()
    if noise > 0:
        g = torch.Generator(device=dev).manual_seed(seed * 7919 + 1)
        for s0 in range(0, n, 1 << 24):
            s1 = min(n, s0 + (1 << 24))
            e = torch.randn(s1 - s0, generator=g, dtype=torch.float64, device=dev) * noise
            flat[s0:s1] = (flat[s0:s1].to(torch.float64) + e).to(torch.float32)
    if outlier_frac > 0:
        m = int(round(outlier_frac * n))
        pos = rng.choice(n, size=m, replace=False)
        sign = rng.choice(np.array([-1.0, 1.0]), size=m)
        flat[torch.from_numpy(pos).to(dev)] = torch.from_numpy(sign * outlier_mag).to(dev, torch.float32)
    return out.view(shape)


def grf(shape, seed: int, slope: float, device: str | torch.device = "cpu") -> torch.Tensor:
    """Gaussian random field with an isotropic power-law spectrum k^-slope."""
    shape = tuple(int(s) for s in shape)
    dev = torch.device(device)
    g = torch.Generator(device=dev).manual_seed(seed)
    white = torch.randn(shape, generator=g, dtype=torch.float32, device=dev)
    spec = torch.fft.rfftn(white)
    freqs = [torch.fft.fftfreq(n, device=dev) for n in shape[:-1]] + [torch.fft.rfftfreq(shape[-1], device=dev)]
    k2 = torch.zeros(spec.shape, dtype=torch.float32, device=dev)
    for ax, f in enumerate(freqs):
        view = [1] * len(shape)
        view[ax] = -1
        k2 = k2 + (f.view(view) * shape[ax]) ** 2
    k2[(0,) * len(shape)] = 1.0
    spec *= k2.pow(-slope / 4.0)
    spec[(0,) * len(shape)] = 0
    field = torch.fft.irfftn(spec, s=shape)
    field /= field.std()
    return field.to(torch.float32).contiguous()


def white(n: int, seed: int, device: str | torch.device = "cpu") -> torch.Tensor:
    g = torch.Generator(device=torch.device(device)).manual_seed(seed)
    return (torch.rand(int(n), generator=g, dtype=torch.float32, device=device) * 2.0 - 1.0).contiguous()


def mixed_field(n_floats: int, kind: str, seed: int, device="cpu") -> torch.Tensor:
    """A 1-D field of exactly n_floats values from one generator family
    (used by the many-fields configurations, whose sizes are not cubes)."""
    if kind == "white":
        return white(n_floats, seed, device)
    rows = max(1, -(-n_floats // (128 * 128)))
    if kind == "sinusoid":
        f = sinusoid((rows, 128, 128), seed, device=device)
    elif kind == "grf":
        f = grf((rows, 128, 128), seed, slope=3.0, device=device)
    else:
        raise ValueError(kind)
    return f.reshape(-1)[:n_floats].contiguous()


def field_set(n_fields: int, seed: int, min_bytes: int, max_bytes: int, rng=None):
    """Sizes, generators and seeds of a many-fields configuration: n_fields
    sizes log-uniform in [min_bytes, max_bytes] (rounded down to a multiple of
    4 bytes, so last chunks are partial), generators cycling sinusoid, GRF
    (k^-3), white noise.  Returns [(n_floats, kind, field_seed)]; build a field
    with mixed_field(*entry).  The sizes are drawn from `rng` when given (the
    caller keeps drawing from it), else from a fresh PCG64(seed)."""
    if rng is None:
        rng = np.random.Generator(np.random.PCG64(seed))
    kinds = ("sinusoid", "grf", "white")
    out = []
    for i in range(n_fields):
        nb = int(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes)))) & ~3
        out.append((nb // 4, kinds[i % 3], seed * 1000 + i))
    return out
