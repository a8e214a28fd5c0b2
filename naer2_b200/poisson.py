"""Inverse-CDF tables of Poisson counts, shared bit for bit by the CUDA
kernels and every check: entry k is floor(2^32 * P(X <= k)) computed in
fp64 on the host; a uniform 32-bit word u draws the count
min{k : u < table[k]} (the last entry catches the far tail)."""

from __future__ import annotations

import math

import numpy as np

MAX_LEN = 256


def cdf_table(lam: float, tail: float = 2.0 ** -40) -> np.ndarray:
    """uint32 table of Poisson(lam); empty for lam <= 0. Its length covers all but `tail` of the mass
    (capped at MAX_LEN entries)."""
    if lam <= 0.0:
        return np.zeros(0, dtype=np.uint32)
    if lam > 150.0:
        raise ValueError(f"a Poisson mean of {lam} per step is beyond the table's range (150)")
    out = []
    p = math.exp(-lam)
    cdf = 0.0
    for k in range(MAX_LEN):
        cdf += p
        out.append(min(int(math.floor(cdf * 4294967296.0)), 0xFFFFFFFF))
        if 1.0 - cdf < tail and k >= lam:
            break
        p *= lam / (k + 1)
    out.append(0xFFFFFFFF)
    return np.asarray(out, dtype=np.uint32)


def count(table: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Counts for uniform words u (vectorised; the kernels' loop)."""
    if len(table) == 0:
        return np.zeros_like(u, dtype=np.int64)
    return np.minimum(np.searchsorted(table[:-1], u, side="right"), len(table) - 1).astype(np.int64)
