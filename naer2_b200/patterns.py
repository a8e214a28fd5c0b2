"""Built-in connectivity patterns. Each is an @n2.pattern callable class, usable
per source position like any pattern (reference naer2/decorators/pattern.py),
and also answers links(n_src, n_tgt, same) -> (offsets, targets): the whole
canonical CSR at once from a seeded Philox stream (numpy's Philox bit
generator), which Topology.build uses for flat populations. `same`: source and target are one population."""

from __future__ import annotations

import itertools
import math

import numpy as np
import torch

from . import philox
from .decorators import pattern
from .types import Points, Position, Region

_SEEDS = itertools.count(1000)


def _csr_by_source(src: np.ndarray, tgt: np.ndarray, n_src: int):
    """Links (src, tgt) grouped by source, stably (each row keeps the input order)."""
    order = np.argsort(src, kind="stable")
    offsets = np.zeros(n_src + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(np.bincount(src, minlength=n_src))
    return offsets, tgt[order]


class _Drawn:
    """Per-position calls served from the whole draw (made on the first call)."""

    def _rows(self, source_region, target_region):
        if getattr(self, "_cache", None) is None:
            n_src = len(source_region)
            n_tgt = len(target_region if target_region is not None else source_region)
            self._cache = self.links(n_src, n_tgt, same=target_region is None)
        return self._cache

    def __call__(self, position: Position, source_region: Region, target_region=None) -> Region:
        offsets, targets = self._rows(source_region, target_region)
        lo = int(source_region[0][0])
        s = int(position[0]) - lo
        return Points(torch.as_tensor(targets[offsets[s]:offsets[s + 1]], dtype=torch.int64).unsqueeze(1))


@pattern
class fixed_indegree(_Drawn):
    """Every target draws K sources uniformly, with replacement (multapses kept); autapses=False excludes a
    neuron drawing itself where source and target are one population (the reference's Brunel_indegree,
    test/networks/Brunel/connection.py:8-33, keeps autapses). Rows ordered by target."""

    def __init__(self, K: int, autapses: bool = True, seed: int | None = None, device=None):
        self.K = int(K)
        self.autapses = autapses
        self.seed = next(_SEEDS) if seed is None else int(seed)
        self.device = torch.device(device) if device is not None else None  # draw there (torch's Philox)
        self._cache = None

    def links(self, n_src: int, n_tgt: int, same: bool = False):
        exclude = same and not self.autapses
        if n_tgt == 0 or self.K == 0:
            return np.zeros(n_src + 1, dtype=np.int64), np.zeros(0, dtype=np.int64)
        if n_src - exclude <= 0:
            raise ValueError("no source to draw from")
        if self.device is not None and self.device.type == "cuda":
            dev = self.device
            g = torch.Generator(device=dev).manual_seed(self.seed)
            tgt_t = torch.arange(n_tgt, dtype=torch.int64, device=dev).repeat_interleave(self.K)
            src_t = torch.randint(0, n_src - (1 if exclude else 0), (n_tgt * self.K,), generator=g, device=dev)
            if exclude:
                src_t += (src_t >= tgt_t).to(torch.int64)
            order = torch.argsort(src_t, stable=True)
            off = torch.zeros(n_src + 1, dtype=torch.int64, device=dev)
            off[1:] = torch.cumsum(torch.bincount(src_t, minlength=n_src), 0)
            return off, tgt_t[order]
        tgt = np.repeat(np.arange(n_tgt, dtype=np.int64), self.K)
        src = philox.generator(self.seed).integers(0, n_src - (1 if exclude else 0), n_tgt * self.K, dtype=np.int64)
        if exclude:
            src += src >= tgt
        return _csr_by_source(src, tgt, n_src)


@pattern
class fixed_outdegree(_Drawn):
    """Every source draws k targets uniformly, with replacement -- the reference's PD14_connection
    (test/networks/PD14/connection.py:8-35): given a connection probability p, the total
    Q = ln(1 - p) / ln(1 - 1/(N_src N_tgt)) split as k = round(Q / N_src) per source; or k given."""

    def __init__(self, probability: float | None = None, k: int | None = None, seed: int | None = None,
                 device=None):
        if (probability is None) == (k is None):
            raise ValueError("give one of probability or k")
        self.probability = probability
        self.k = k
        self.seed = next(_SEEDS) if seed is None else int(seed)
        self.device = torch.device(device) if device is not None else None  # draw there (torch's Philox)
        self._cache = None

    def per_source(self, n_src: int, n_tgt: int) -> int:
        if self.k is not None:
            return int(self.k)
        if self.probability <= 0.0 or n_src == 0 or n_tgt == 0:
            return 0
        Q = math.log(1 - self.probability) / math.log(1 - 1 / (n_src * n_tgt))
        return round(Q / n_src)

    def links(self, n_src: int, n_tgt: int, same: bool = False):
        k = self.per_source(n_src, n_tgt)
        if self.device is not None and self.device.type == "cuda":
            offsets = torch.arange(n_src + 1, dtype=torch.int64, device=self.device) * k
            if k == 0:
                return offsets, torch.zeros(0, dtype=torch.int64, device=self.device)
            g = torch.Generator(device=self.device).manual_seed(self.seed)
            return offsets, torch.randint(0, n_tgt, (n_src * k,), generator=g, device=self.device)
        offsets = np.arange(n_src + 1, dtype=np.int64) * k
        if k == 0:
            return offsets, np.zeros(0, dtype=np.int64)
        return offsets, philox.generator(self.seed).integers(0, n_tgt, n_src * k, dtype=np.int64)


@pattern
class all_to_all(_Drawn):
    """Every source to every target (autapses=False: not to itself within one population)."""

    def __init__(self, autapses: bool = True):
        self.autapses = autapses
        self._cache = None

    def links(self, n_src: int, n_tgt: int, same: bool = False):
        tgt = np.tile(np.arange(n_tgt, dtype=np.int64), n_src)
        if same and not self.autapses:
            src = np.repeat(np.arange(n_src, dtype=np.int64), n_tgt)
            keep = src != tgt
            return _csr_by_source(src[keep], tgt[keep], n_src)
        return np.arange(n_src + 1, dtype=np.int64) * n_tgt, tgt


@pattern
class one_to_one(_Drawn):
    """Source i to target i."""

    def __init__(self):
        self._cache = None

    def links(self, n_src: int, n_tgt: int, same: bool = False):
        n = min(n_src, n_tgt)
        offsets = np.minimum(np.arange(n_src + 1, dtype=np.int64), n)
        return offsets, np.arange(n, dtype=np.int64)


__all__ = ["fixed_indegree", "fixed_outdegree", "all_to_all", "one_to_one"]
