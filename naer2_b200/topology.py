"""Connectivity: the canonical CSR a pattern builds (reference
naer2/topology.py:98-199), and the two device forms the hot path walks.

Canonical form (what a pattern gives, what per-link tensors are indexed by):
one row per source neuron, its links in the order the pattern returned them.

Device forms, one packed 32-bit word per link, `(delay_steps << 24) | index`:
  push  rows per SOURCE (the canonical order itself), index = target neuron;
        the source's block scatters its spikes along them;
  pull  rows per TARGET (a stable sort of the canonical links by target),
        index = source neuron; the target's block gathers them against the
        source's spike-bit ring.
Per-link weights (fp32) follow the same orders. The reference restructures
its canonical links into (source, target group, delay bucket) segments
(naer2/topology.py:291-438); at a fixed dt every delay is a whole number of
steps, so the delay rides in the link word instead and no bucket is needed.
"""

from __future__ import annotations

import inspect

import numpy as np
import torch

from .types import IndexBox, Region, _BaseBox, _BasePoints

MAX_INDEX = 1 << 24  # a link word's index field
MAX_DELAY_STEPS = 255  # its delay field


def _index_fn(target_region):
    """Coordinates [n, ndim] -> linear indices into target_region (row-major for a box, a lookup for points)."""
    if isinstance(target_region, _BaseBox):
        starts, steps, sizes = target_region.start.long(), target_region.step.long(), target_region.sizes
        strides = torch.ones(len(sizes), dtype=torch.int64)
        for d in range(len(sizes) - 2, -1, -1):
            strides[d] = strides[d + 1] * sizes[d + 1]

        def to_index(coords):
            if len(coords) == 0:
                return torch.zeros(0, dtype=torch.int64)
            return (((coords.long() - starts) // steps) * strides).sum(dim=1)

        return to_index
    if isinstance(target_region, _BasePoints):
        lookup = {tuple(c.tolist()): i for i, c in enumerate(target_region.coords)}
        return lambda coords: torch.tensor([lookup[tuple(c.tolist())] for c in coords], dtype=torch.int64)
    raise TypeError(f"Cannot index {type(target_region).__name__}")


def _coords(result) -> torch.Tensor:
    if isinstance(result, _BasePoints):
        return result.coords
    if isinstance(result, _BaseBox):
        return result.points
    return torch.zeros((0, 1), dtype=torch.int64)


def _flat_size(region) -> int | None:
    """n for a flat 0-based index box [[0, n, 1]], else None."""
    if isinstance(region, IndexBox) and region.coords.shape[0] == 1:
        start, _, step = region.coords[0].tolist()
        if start == 0 and step == 1:
            return len(region)
    return None


class Topology:
    """Canonical CSR: source_offsets [n_src + 1] int64, target_indices [n_links] int64.
    Multapses are kept as separate links."""

    def __init__(self, source_offsets: torch.Tensor, target_indices: torch.Tensor):
        self.source_offsets = source_offsets
        self.target_indices = target_indices

    @property
    def shape(self) -> tuple:
        return (len(self.target_indices),)

    def __len__(self) -> int:
        return len(self.target_indices)

    @property
    def n_sources(self) -> int:
        return len(self.source_offsets) - 1

    @staticmethod
    def build(pattern, source_region, target_region=None, same: bool = False):
        """Run the pattern for every source point (reference naer2/topology.py:130-199); a Topology, or
        (Topology, inferred target region) without target_region. A pattern exposing
        links(n_src, n_tgt) -> (offsets, targets) is asked for the whole CSR at once when both regions are
        flat index ranges (the built-in patterns; same links as the per-point calls). same: source and target
        are one population (a pattern may exclude autapses then)."""
        n_src, n_tgt = _flat_size(source_region), (_flat_size(target_region) if target_region is not None else None)
        if hasattr(pattern, "links") and n_src is not None and (target_region is None or n_tgt is not None):
            offsets, targets = pattern.links(n_src, n_tgt if n_tgt is not None else n_src,
                                             same=same or target_region is None)
            topo = Topology(torch.as_tensor(offsets, dtype=torch.int64), torch.as_tensor(targets, dtype=torch.int64))
            if topo.source_offsets.device != topo.target_indices.device:
                topo.source_offsets = topo.source_offsets.to(topo.target_indices.device)
            if target_region is None:
                size = int(topo.target_indices.max()) + 1 if len(topo) else 0
                return topo, Region(size)
            return topo
        takes_target = len(inspect.signature(pattern).parameters) > 2

        def call(pos):
            return pattern(pos, source_region, target_region) if takes_target else pattern(pos, source_region)

        rows = [_coords(call(pos)) for pos in source_region]
        if target_region is None:
            nonempty = [r for r in rows if len(r)]
            if nonempty:
                maxes = torch.cat(nonempty).max(dim=0).values.tolist()
                sizes = tuple(int(m) + 1 for m in maxes)
                inferred = Region(sizes[0] if len(sizes) == 1 else sizes)
            else:
                inferred = Region(0)
        else:
            inferred = target_region
        to_index = _index_fn(inferred)
        idx = [to_index(r) for r in rows]
        off = np.zeros(len(idx) + 1, dtype=np.int64)
        off[1:] = np.cumsum([len(r) for r in idx])
        targets = torch.cat(idx) if off[-1] else torch.zeros(0, dtype=torch.int64)
        topo = Topology(torch.from_numpy(off), targets)
        return (topo, inferred) if target_region is None else topo


def delay_steps(delay, n_links: int, dt: float, device=None) -> torch.Tensor:
    """Per-link delays in whole steps of dt (int64, on `device` or the delay tensor's): round(delay / dt) half
    to even, at least 1 (a spike is delivered from the next step on; the reference clamps delays to >= its
    0.1 ms resolution, test/networks/PD14/net.py:102)."""
    if isinstance(delay, torch.Tensor):
        d = delay.detach().reshape(-1)
        if device is not None:
            d = d.to(device)
        if d.numel() != n_links:
            raise ValueError(f"delay has {d.numel()} values for {n_links} links")
        steps = torch.round(d.to(torch.float64) / dt).to(torch.int64)
    else:
        value = 1 if delay is None else int(np.rint(float(delay) / dt))
        steps = torch.full((n_links,), value, dtype=torch.int64, device=device)
    steps = steps.clamp(min=1)
    if n_links and int(steps.max()) > MAX_DELAY_STEPS:
        raise ValueError(f"a delay of {int(steps.max())} steps exceeds {MAX_DELAY_STEPS}")
    return steps


def pack_links(index: torch.Tensor, steps: torch.Tensor) -> torch.Tensor:
    """(delay_steps << 24) | index as int32 holding the uint32 bit pattern."""
    if index.numel() and (int(index.min()) < 0 or int(index.max()) >= MAX_INDEX):
        raise ValueError("a link index outside [0, 2^24)")
    word = (steps.to(torch.int64) << 24) | index.to(torch.int64)
    return torch.where(word >= 2 ** 31, word - 2 ** 32, word).to(torch.int32)


def _rows(off: torch.Tensor) -> torch.Tensor:
    """The source row of every link of a CSR with offsets `off`."""
    return torch.repeat_interleave(torch.arange(len(off) - 1, device=off.device), off.diff())


def push_form(topo: Topology, steps: torch.Tensor, n_tgt: int):
    """(ptr int32 [n_src + 1], link int32 [n_links], perm int64 [n_links], split int32 [n_src]): rows per
    source, each row's delay-1 links first (stable: canonical order otherwise); perm[k] is the canonical link
    at position k; split[s] is row s's first link of delay >= 2 (the rest of the row is delivered one launch
    later). Computed on the topology's device."""
    tgt = topo.target_indices
    off = topo.source_offsets.to(tgt.device)
    if tgt.numel() and (int(tgt.min()) < 0 or int(tgt.max()) >= n_tgt):
        raise ValueError("a link targets a neuron outside the target population")
    steps = steps.to(tgt.device)
    far = steps >= 2
    n_src = len(off) - 1
    if not tgt.numel():
        perm = torch.zeros(0, dtype=torch.int64, device=tgt.device)
        split = off[:-1].to(torch.int32)
    else:
        row = _rows(off)
        near_per_row = torch.bincount(row, weights=(~far).to(torch.float64), minlength=n_src).to(torch.int64)
        split = (off[:-1] + near_per_row).to(torch.int32)
        perm = torch.arange(tgt.numel(), device=tgt.device) if bool(far.all()) else \
            torch.argsort(row * 2 + far.to(torch.int64), stable=True)
    return off.to(torch.int32), pack_links(tgt[perm], steps[perm]), perm, split


def pull_split_form(topo: Topology, steps: torch.Tensor, n_tgt: int):
    """(ptr int32 [n_tgt + 1], link int32 [n_links], perm int64 [n_links], fptr int32 [n_tgt + 1]): the pull
    form in two parts of one link array: first every target's delay-1 links (rows ptr[j]..ptr[j+1], pulled in
    the step itself), then every target's links of delay >= 2 (rows fptr[j]..fptr[j+1], fptr[0] = ptr[n_tgt],
    pulled one step ahead by any block); canonical order within a row; perm[k] is the canonical link at
    position k."""
    tgt = topo.target_indices
    off = topo.source_offsets.to(tgt.device)
    steps = steps.to(tgt.device)
    src = _rows(off)
    far = (steps >= 2).to(torch.int64)
    perm = torch.argsort(far * n_tgt + tgt, stable=True)
    if tgt.numel():
        near_counts = torch.bincount(tgt[far == 0], minlength=n_tgt)
        far_counts = torch.bincount(tgt[far == 1], minlength=n_tgt)
    else:
        near_counts = far_counts = torch.zeros(n_tgt, dtype=torch.int64, device=tgt.device)
    ptr = torch.zeros(n_tgt + 1, dtype=torch.int64, device=tgt.device)
    ptr[1:] = torch.cumsum(near_counts, 0)
    fptr = torch.zeros(n_tgt + 1, dtype=torch.int64, device=tgt.device)
    fptr[1:] = torch.cumsum(far_counts, 0)
    fptr += ptr[-1]
    return ptr.to(torch.int32), pack_links(src[perm], steps[perm]), perm, fptr.to(torch.int32)


def pull_form(topo: Topology, steps: torch.Tensor, n_tgt: int):
    """(ptr int32 [n_tgt + 1], link int32 [n_links], perm int64 [n_links]): the links sorted by target (stable:
    canonical order within a target); perm[k] is the canonical link at pull position k."""
    tgt = topo.target_indices
    off = topo.source_offsets.to(tgt.device)
    steps = steps.to(tgt.device)
    src = _rows(off)
    perm = torch.argsort(tgt, stable=True)
    counts = torch.bincount(tgt, minlength=n_tgt) if tgt.numel() else torch.zeros(n_tgt, dtype=torch.int64,
                                                                                  device=tgt.device)
    ptr = torch.zeros(n_tgt + 1, dtype=torch.int64, device=tgt.device)
    ptr[1:] = torch.cumsum(counts, 0)
    return ptr.to(torch.int32), pack_links(src[perm], steps[perm]), perm
