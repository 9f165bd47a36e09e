"""Seeded synthetic inputs for the benchmark workloads.

The reference's published numbers use datasets that are not available here
(``pressure_2000``, ``xx.f32``, ``acd-tst.bin.d64``); these generators stand in
for them with the shapes, sizes and value distributions of each workload:

* ``sinusoid_field``   1D f32, sum of 8 sinusoids + N(0, 1e-3) noise, 20% zeros
                       in runs of 256 (single-array 1D plain workload, N = 2^24).
* ``grf_field``        3D Gaussian random field with P(k) ~ k^-3, scaled to
                       [-50, 50] + N(0, 1e-4) noise (512^3 f32 outlier workload).
* ``uniform_sparse``   iid U[-1, 1] with Bernoulli(0.3) zeros (8192^2 f64 fixed
                       roofline stress workload).
* ``weight_like``      iid N(0, 0.02) values (batched workload, fixed mode).

All generators are torch-based so that large arrays can be made directly on the
device; ``device="cpu"`` gives the same recipe on the host.
"""
from __future__ import annotations

import math

import torch


def _gen(seed: int, device) -> torch.Generator:
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def sinusoid_field(n: int, seed: int = 0, device="cpu", dtype=torch.float32,
                   zero_frac: float = 0.2, run: int = 256, noise: float = 1e-3) -> torch.Tensor:
    """Sum of 8 sinusoids (freq U[1e-5,1e-2] cycles/sample, amp U[0.1,1],
    phase U[0,2pi)) plus iid N(0, sigma=noise); `zero_frac` of entries set to
    exactly 0.0 in contiguous runs of `run` at random offsets."""
    g = _gen(seed, "cpu")
    freq = torch.empty(8, dtype=torch.float64).uniform_(1e-5, 1e-2, generator=g)
    amp = torch.empty(8, dtype=torch.float64).uniform_(0.1, 1.0, generator=g)
    phase = torch.empty(8, dtype=torch.float64).uniform_(0.0, 2 * math.pi, generator=g)
    gd = _gen(seed + 1000, device)
    x = torch.zeros(n, dtype=torch.float64, device=device)
    chunk = 1 << 22
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        t = torch.arange(s, e, dtype=torch.float64, device=device)
        acc = torch.zeros(e - s, dtype=torch.float64, device=device)
        for k in range(8):
            acc += amp[k].item() * torch.sin(2 * math.pi * freq[k].item() * t + phase[k].item())
        x[s:e] = acc
    x += torch.randn(n, generator=gd, dtype=torch.float64, device=device) * noise
    if zero_frac > 0 and n >= run:
        nruns = int(round(zero_frac * n / run))
        starts = torch.randint(0, n - run + 1, (nruns,), generator=g)
        mask = torch.zeros(n, dtype=torch.bool)
        for s0 in starts.tolist():
            mask[s0:s0 + run] = True
        x[mask.to(device)] = 0.0
    return x.to(dtype)


def grf_field(shape, seed: int = 1, device="cpu", dtype=torch.float32, lo: float = -50.0,
              hi: float = 50.0, noise: float = 1e-4, slope: float = -3.0) -> torch.Tensor:
    """Gaussian random field with power spectrum P(k) ~ k^slope (FFT of seeded
    white noise), affinely scaled to [lo, hi], plus iid N(0, sigma=noise).
    `shape` is (z, y, x) with x fastest."""
    nz, ny, nx = shape
    gd = _gen(seed, device)
    w = torch.randn((nz, ny, nx), generator=gd, dtype=torch.float32, device=device)
    W = torch.fft.rfftn(w)
    del w
    kz = torch.fft.fftfreq(nz, device=device).view(nz, 1, 1)
    ky = torch.fft.fftfreq(ny, device=device).view(1, ny, 1)
    kx = torch.fft.rfftfreq(nx, device=device).view(1, 1, nx // 2 + 1)
    k2 = kz * kz + ky * ky + kx * kx
    amp = torch.where(k2 > 0, k2.clamp_min(1e-30) ** (slope / 4.0), torch.zeros_like(k2))
    W *= amp
    del k2, amp
    f = torch.fft.irfftn(W, s=(nz, ny, nx))
    del W
    fmin, fmax = f.min(), f.max()
    f = (f - fmin) * ((hi - lo) / (fmax - fmin)) + lo
    f += torch.randn(f.shape, generator=gd, dtype=torch.float32, device=device) * noise
    return f.to(dtype).contiguous()


def uniform_sparse(shape, seed: int = 2, device="cpu", dtype=torch.float64,
                   zero_prob: float = 0.3) -> torch.Tensor:
    """iid U[-1, 1] with Bernoulli(zero_prob) positions set to exactly 0.0."""
    gd = _gen(seed, device)
    x = torch.rand(shape, generator=gd, dtype=torch.float64, device=device) * 2.0 - 1.0
    z = torch.rand(shape, generator=gd, dtype=torch.float64, device=device) < zero_prob
    x[z] = 0.0
    return x.to(dtype).contiguous()


def weight_like(n: int, seed: int = 3, device="cpu", dtype=torch.float32, sigma: float = 0.02) -> torch.Tensor:
    gd = _gen(seed, device)
    return (torch.randn(n, generator=gd, dtype=torch.float32, device=device) * sigma).to(dtype)
