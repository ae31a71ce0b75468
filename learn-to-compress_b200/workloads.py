"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations.  The reference evaluates on public datasets (SOSD,
Kaggle, UCI) that are not available here; these generators stand in for them.

All generators are deterministic for a given (seed, device).  They use torch
only as an array library (they run on the CPU or on a GPU).
"""
from __future__ import annotations

import math

import numpy as np


def _torch():
    import torch
    return torch


def sorted_keys_u32(n: int = 1_000_000, seed: int = 1) -> np.ndarray:
    """x_i = 1000*i + U[0, 255] as uint32 (1,000,000 keys: the CPU-runnable case)."""
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.uint64)
    return (np.uint64(1000) * i + rng.integers(0, 256, n, dtype=np.uint64)).astype(np.uint32)


def piecewise_linear_u64(n: int, seed: int = 2, device="cpu", mean_seg: float = 50_000.0,
                         max_slope_log2: float = 20.0, sigma: float = 4096.0, noise_on: str = "cpu"):
    """Sorted uint64 keys: a piecewise-linear trend (segment lengths geometric
    with mean `mean_seg`, slopes log-uniform in [1, 2^max_slope_log2]) plus
    round(N(0, sigma)) noise, clipped at 0 and sorted.  Returns an int64 torch
    tensor holding the uint64 bit patterns (all values < 2^63).

    With noise_on="cpu" (default) the values do not depend on `device`: the
    noise comes from the CPU generator, and the trend of segment r at position
    i is C_r + slope_r * (i - start_r + 1), C_r summed in order on the host,
    so every device-side step is one IEEE-rounded elementwise operation.  A CPU
    run (the reference's timed arm) and a GPU run then see the same column.
    noise_on="device" draws the noise on `device` instead (faster for many
    columns; the values then depend on the device)."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    # segment lengths / slopes on the host (a few thousand segments)
    nseg = int(n / mean_seg * 1.5) + 16
    u = torch.rand(nseg, generator=g, dtype=torch.float64)
    lens = torch.clamp(torch.ceil(torch.log1p(-u) / math.log1p(-1.0 / mean_seg)), min=1).to(torch.int64)
    while int(lens.sum()) < n:
        lens = torch.cat([lens, lens])
    slopes = torch.exp(torch.rand(len(lens), generator=g, dtype=torch.float64) * (max_slope_log2 * math.log(2.0)))
    # segment bases: the trend's value just before each segment, accumulated in order
    lens_np, slopes_np = lens.numpy(), slopes.numpy()
    bases = np.zeros(len(lens_np), np.float64)
    acc = 0.0
    for r in range(len(lens_np)):
        bases[r] = acc
        acc = acc + float(slopes_np[r]) * float(lens_np[r])
    starts = np.concatenate([[0], np.cumsum(lens_np)[:-1]]).astype(np.int64)
    seg = torch.repeat_interleave(torch.arange(len(lens), device=device), lens.to(device))[:n]
    pos = (torch.arange(n, device=device, dtype=torch.int64) - torch.from_numpy(starts).to(device)[seg] + 1).to(torch.float64)
    trend = torch.from_numpy(bases).to(device)[seg] + torch.from_numpy(slopes_np).to(device)[seg] * pos
    del seg, pos
    if noise_on == "cpu":
        noise = torch.randn(n, generator=torch.Generator(device="cpu").manual_seed(seed + 1), dtype=torch.float64)
        noise = torch.round(noise * sigma).to(device)
    else:
        dev_g = torch.Generator(device=device).manual_seed(seed + 1)
        noise = torch.round(torch.randn(n, generator=dev_g, device=device, dtype=torch.float64) * sigma)
    x = torch.clamp(torch.round(trend) + noise, min=0).to(torch.int64)
    del trend, noise
    x, _ = torch.sort(x)
    return x


def regime_switching_u64(n: int, seed: int = 5, device="cpu", mean_regime: float = 200_000.0, sigma: float = 256.0):
    """Regimes of geometric length (mean `mean_regime`) that cycle linear,
    quadratic a*i^2 (a log-uniform in [1e-6, 1e-2], i relative to the regime
    start) and flat+noise; each regime continues from the previous level;
    noise round(N(0, sigma)) everywhere.  int64 tensor of uint64 patterns."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    nreg = int(n / mean_regime * 1.5) + 8
    u = torch.rand(nreg, generator=g, dtype=torch.float64)
    lens = torch.clamp(torch.ceil(torch.log1p(-u) / math.log1p(-1.0 / mean_regime)), min=1).to(torch.int64)
    while int(lens.sum()) < n:
        lens = torch.cat([lens, lens])
    out = torch.empty(n, dtype=torch.float64, device=device)
    level = 1e9
    pos = 0
    r = 0
    while pos < n:
        L = min(int(lens[r]), n - pos)
        i = torch.arange(L, dtype=torch.float64, device=device)
        kind = r % 3
        if kind == 0:
            slope = math.exp(float(torch.rand(1, generator=g, dtype=torch.float64)) * math.log(2.0 ** 16))
            seg = level + slope * i
        elif kind == 1:
            a = math.exp(math.log(1e-6) + float(torch.rand(1, generator=g, dtype=torch.float64)) * (math.log(1e-2) - math.log(1e-6)))
            seg = level + a * i * i
        else:
            seg = torch.full((L,), level, dtype=torch.float64, device=device)
        out[pos:pos + L] = seg
        level = float(seg[-1]) + 1.0
        pos += L
        r += 1
    dev_g = torch.Generator(device=device).manual_seed(seed + 1)
    noise = torch.round(torch.randn(n, generator=dev_g, device=device, dtype=torch.float64) * sigma)
    return torch.clamp(torch.round(out) + noise, min=0).to(torch.int64)


def families(n: int, family: str, dtype_bytes: int, rng: np.random.Generator) -> np.ndarray:
    """One column of the mixed batching workload.

    family: 'linear' (linear + N(0, sigma), sigma log-uniform in [1, 2^16]),
    'step' (steps of geometric length mean 500, jumps U[0, 2^20]), 'walk'
    (positive random walk, geometric increments mean 64), 'uniform'
    (U[0, 2^b), b in {8, 16, 32})."""
    top = 2.0 ** (32 if dtype_bytes == 4 else 62)
    if family == "linear":
        sigma = math.exp(rng.uniform(0, math.log(2.0 ** 16)))
        slope = math.exp(rng.uniform(0, math.log(2.0 ** 10)))
        x = slope * np.arange(n, dtype=np.float64) + rng.normal(0, sigma, n) + 4 * sigma + 1
    elif family == "step":
        steps = rng.geometric(1 / 500, size=n // 50 + 8)
        jumps = rng.integers(0, 2 ** 20, size=len(steps)).astype(np.float64)
        x = np.repeat(np.cumsum(jumps), steps)[:n]
        if len(x) < n:
            x = np.concatenate([x, np.full(n - len(x), x[-1] if len(x) else 0.0)])
    elif family == "walk":
        x = np.cumsum(rng.geometric(1 / 64, size=n).astype(np.float64))
    elif family == "uniform":
        b = int(rng.choice([8, 16, 32]))
        x = rng.integers(0, 2 ** b, size=n, dtype=np.uint64).astype(np.float64)
    else:
        raise ValueError(family)
    x = np.clip(np.round(x), 0, top - 1)
    return x.astype(np.uint64).astype(np.uint32 if dtype_bytes == 4 else np.uint64)


BATCH_FAMILIES = ("linear", "step", "walk", "uniform")


def batch_columns(ncols: int, seed: int, max_len: int | None = None):
    """The mixed batching workload: `ncols` columns with lengths log-uniform in
    [1K, 4M] (optionally capped at `max_len`), 50 % uint32 / 50 % uint64, each
    from one of the four `families`, each coded LeCo-fix (0), Delta-fix (2) or
    FOR (1).  Yields (values as a numpy array, codec, family) per column."""
    rng = np.random.default_rng(seed)
    for _ in range(ncols):
        n = int(math.exp(rng.uniform(math.log(1000), math.log(4_000_000))))
        if max_len is not None:
            n = min(n, max_len)
        s = 4 if rng.random() < 0.5 else 8
        fam = BATCH_FAMILIES[int(rng.integers(4))]
        codec = (0, 2, 1)[int(rng.integers(3))]
        yield families(n, fam, s, rng), codec, fam
