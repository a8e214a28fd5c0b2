"""Philox4x32-10 (Salmon et al., SC'11) vectorised in numpy: the host side's
copy of the generator the CUDA kernels use (csrc/n2b_device.cuh), for seeded
initial values and connectivity that do not depend on the machine."""

from __future__ import annotations

import numpy as np

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_LO = np.uint64(0xFFFFFFFF)


def philox4x32(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 of counters (arrays or scalars, broadcast) under key (k0, k1): four uint32 arrays."""
    c0, c1, c2, c3 = (np.asarray(c, dtype=np.uint32) for c in (c0, c1, c2, c3))
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    c0, c1, c2, c3 = (c.astype(np.uint32).copy() for c in (c0, c1, c2, c3))
    k0, k1 = np.uint32(k0), np.uint32(k1)
    with np.errstate(over="ignore"):
        for _ in range(10):
            p0 = _M0 * c0.astype(np.uint64)
            p1 = _M1 * c2.astype(np.uint64)
            n0 = (p1 >> np.uint64(32)).astype(np.uint32) ^ c1 ^ k0
            n1 = (p1 & _LO).astype(np.uint32)
            n2 = (p0 >> np.uint64(32)).astype(np.uint32) ^ c3 ^ k1
            n3 = (p0 & _LO).astype(np.uint32)
            c0, c1, c2, c3 = n0, n1, n2, n3
            k0 = np.uint32(k0 + _W0)
            k1 = np.uint32(k1 + _W1)
    return c0, c1, c2, c3


def _key(seed: int):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return seed & 0xFFFFFFFF, seed >> 32


def uniform(seed: int, n: int, stream: int = 0) -> np.ndarray:
    """n floats in [0, 1): the top 24 bits of word 0 of counter (i, 0, stream, 0x5EED) times 2^-24."""
    k0, k1 = _key(seed)
    w = philox4x32(np.arange(n, dtype=np.uint32), 0, stream, 0x5EED, k0, k1)[0]
    return (w >> np.uint32(8)).astype(np.float64) * (1.0 / (1 << 24))


def integers(seed: int, high: np.ndarray | int, shape, stream: int = 0) -> np.ndarray:
    """Uniform integers in [0, high) (high broadcast against shape), by the 64-bit product of two words
    (bias below 2^-32 * high)."""
    k0, k1 = _key(seed)
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.uint64)
    w = philox4x32((idx & _LO).astype(np.uint32), (idx >> np.uint64(32)).astype(np.uint32), stream, 0x1D7, k0, k1)
    r = (w[0].astype(np.uint64) << np.uint64(32)) | w[1].astype(np.uint64)
    high = np.broadcast_to(np.asarray(high, dtype=np.uint64), shape).reshape(-1)
    # floor(r * high / 2^64) without overflow: split r into 32-bit halves
    hi, lo = r >> np.uint64(32), r & _LO
    with np.errstate(over="ignore"):
        out = (hi * high + ((lo * high) >> np.uint64(32))) >> np.uint64(32)
    return out.astype(np.int64).reshape(shape)


def generator(seed: int) -> np.random.Generator:
    """numpy's Philox bit generator keyed by `seed` (C speed, stream-stable): bulk connectivity draws."""
    return np.random.Generator(np.random.Philox(key=int(seed) & 0xFFFFFFFFFFFFFFFF))


def normal(seed: int, n: int, mean: float = 0.0, std: float = 1.0, stream: int = 0) -> np.ndarray:
    """n normal draws (Box-Muller on two 24-bit uniforms of one counter)."""
    k0, k1 = _key(seed)
    w = philox4x32(np.arange(n, dtype=np.uint32), 0, stream, 0x6A55, k0, k1)
    u1 = ((w[0] >> np.uint32(8)).astype(np.float64) + 1.0) * (1.0 / (1 << 24))  # (0, 1]
    u2 = (w[1] >> np.uint32(8)).astype(np.float64) * (1.0 / (1 << 24))
    return mean + std * np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
