"""Seeded synthetic Brownian paths, the inputs of the benchmark workloads.

x[:, 0] = 0 and x[:, t] is the cumulative sum of N(0, 1/(L-1)) increments
per channel, generated in float64 with numpy's PCG64 (so every host builds the
same paths from the same seed) and stored in the requested dtype.
"""
from __future__ import annotations

import numpy as np


def brownian_np(n: int, length: int, dim: int, seed: int, scale=None) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    inc = rng.standard_normal((n, length - 1, dim)) / np.sqrt(max(length - 1, 1))
    x = np.zeros((n, length, dim))
    x[:, 1:, :] = np.cumsum(inc, axis=1)
    if scale is not None:
        x = x * np.asarray(scale, np.float64).reshape(n, 1, 1)
    return x


def brownian(n: int, length: int, dim: int, seed: int, scale=None, dtype=None, device=None):
    import torch

    dtype = torch.float32 if dtype is None else dtype
    return torch.tensor(brownian_np(n, length, dim, seed, scale), dtype=dtype, device=device)


def log_uniform(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n))
