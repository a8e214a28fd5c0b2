"""Regions, points and positions of a population's node space -- the value
types of the reference's DSL (naer2/types/region.py, box.py, points.py,
position.py), restated for this package.

A Region is either a box (IndexBox / ContinuousBox: start, stop, step per
dimension; lattice points in row-major order) or an explicit point set
(IndexPoints / ContinuousPoints: [n, ndim]). A Position is one point, the
`position` a connectivity pattern is called with.
"""

from __future__ import annotations

import torch

_INT = (torch.int8, torch.int16, torch.int32, torch.int64)
_FLOAT = (torch.float16, torch.float32, torch.float64)


class Position:
    """One point of a node space: a rank-1 coordinate tensor (reference naer2/types/position.py:7-22)."""

    def __init__(self, coords: torch.Tensor):
        if coords.ndim != 1:
            raise ValueError(f"{type(self).__name__} must be rank-1 (vector)")
        self._check(coords)
        self.coords = coords

    @staticmethod
    def _check(coords):
        pass

    def __getitem__(self, idx):
        return self.coords[idx]

    def __getattr__(self, name):
        if name == "coords":
            raise AttributeError(name)
        return getattr(self.coords, name)

    def __eq__(self, other):
        return isinstance(other, type(self)) and bool(torch.equal(self.coords, other.coords))

    def __repr__(self):
        return f"{type(self).__name__}({self.coords})"


class IndexPosition(Position):
    @staticmethod
    def _check(coords):
        if coords.dtype not in _INT:
            raise TypeError("IndexPosition requires integer tensor")


class ContinuousPosition(Position):
    @staticmethod
    def _check(coords):
        if coords.dtype not in _FLOAT:
            raise TypeError("ContinuousPosition requires floating tensor")


class _BaseBox:
    """An axis-aligned box, [ndim, 3] rows of (start, stop, step); a missing step column defaults to 1
    (reference naer2/types/box.py:4-60)."""

    _position = Position

    def __init__(self, coords: torch.Tensor):
        if coords.ndim != 2 or coords.shape[1] not in (2, 3):
            raise ValueError(f"{type(self).__name__} coords must be shape [ndim, 2] or [ndim, 3], "
                             f"got {tuple(coords.shape)}")
        self._check(coords)
        if coords.shape[1] == 2:
            coords = torch.cat([coords, torch.ones(coords.shape[0], 1, dtype=coords.dtype)], dim=1)
        self.coords = coords

    @staticmethod
    def _check(coords):
        raise NotImplementedError

    start = property(lambda self: self.coords[:, 0])
    stop = property(lambda self: self.coords[:, 1])
    step = property(lambda self: self.coords[:, 2])

    @property
    def sizes(self) -> torch.Tensor:
        return torch.ceil((self.stop.double() - self.start.double()) / self.step.double()).clamp(min=0).long()

    def __len__(self) -> int:
        return int(self.sizes.prod().item())

    @property
    def points(self) -> torch.Tensor:
        """Every lattice point, [n, ndim], row-major (last dimension fastest)."""
        ranges = [torch.arange(self.coords[d, 0].item(), self.coords[d, 1].item(), self.coords[d, 2].item(),
                               dtype=self.coords.dtype) for d in range(self.coords.shape[0])]
        pts = torch.cartesian_prod(*ranges)
        return pts.unsqueeze(1) if pts.ndim == 1 else pts

    def position_at(self, i: int):
        sizes = self.sizes.tolist()
        out = []
        for d in range(len(sizes) - 1, -1, -1):
            out.append(self.coords[d, 0].item() + (i % sizes[d]) * self.coords[d, 2].item())
            i //= sizes[d]
        return self._position(torch.tensor(out[::-1], dtype=self.coords.dtype))

    def __iter__(self):
        for row in self.points:
            yield self._position(row)

    def __getitem__(self, idx):
        return self.coords[idx]

    def __repr__(self):
        return f"{type(self).__name__}({self.coords})"


class IndexBox(_BaseBox):
    _position = IndexPosition

    @staticmethod
    def _check(coords):
        if coords.dtype not in _INT:
            raise TypeError("IndexBox requires integer tensor")


class ContinuousBox(_BaseBox):
    _position = ContinuousPosition

    @staticmethod
    def _check(coords):
        if coords.dtype not in _FLOAT:
            raise TypeError("ContinuousBox requires floating tensor")


class _BasePoints:
    """An explicit point set, [n_points, ndim] (reference naer2/types/points.py:4-64)."""

    _position = Position

    def __init__(self, coords: torch.Tensor):
        if coords.ndim != 2:
            raise ValueError(f"{type(self).__name__} coords must be rank-2 [n_points, ndim], got ndim={coords.ndim}")
        self._check(coords)
        self.coords = coords

    @staticmethod
    def _check(coords):
        raise NotImplementedError

    @property
    def points(self) -> torch.Tensor:
        return self.coords

    def __len__(self) -> int:
        return int(self.coords.shape[0])

    def __iter__(self):
        for row in self.coords:
            yield self._position(row)

    def position_at(self, i: int):
        return self._position(self.coords[i])

    def __getitem__(self, idx):
        return self.coords[idx]

    def __repr__(self):
        return f"{type(self).__name__}({self.coords})"


class IndexPoints(_BasePoints):
    _position = IndexPosition

    @staticmethod
    def _check(coords):
        if coords.dtype not in _INT:
            raise TypeError("IndexPoints requires integer tensor")


class ContinuousPoints(_BasePoints):
    _position = ContinuousPosition

    @staticmethod
    def _check(coords):
        if coords.dtype not in _FLOAT:
            raise TypeError("ContinuousPoints requires floating tensor")


def Box(tensor: torch.Tensor):
    """IndexBox for an integer tensor, ContinuousBox for a floating one."""
    return IndexBox(tensor) if tensor.dtype in _INT else ContinuousBox(tensor)


def Points(tensor: torch.Tensor):
    """IndexPoints for an integer tensor, ContinuousPoints for a floating one."""
    return IndexPoints(tensor) if tensor.dtype in _INT else ContinuousPoints(tensor)


class _RegionMeta(type):
    """isinstance(x, Region) holds for every box and point set."""

    def __instancecheck__(cls, obj):
        return isinstance(obj, (_BaseBox, _BasePoints))


class Region(metaclass=_RegionMeta):
    """Factory of node-space regions (reference naer2/types/region.py:8-44):
    Region(1000) -> IndexBox [[0, 1000, 1]]; Region((H, W)) -> a 2-D grid;
    Region(tensor) -> Box, else Points; Region(region) -> itself."""

    def __new__(cls, *args):
        if len(args) == 1 and isinstance(args[0], (_BaseBox, _BasePoints)):
            return args[0]
        if len(args) == 1 and isinstance(args[0], int) and not isinstance(args[0], bool):
            return IndexBox(torch.tensor([[0, args[0]]], dtype=torch.int64))
        if len(args) == 1 and isinstance(args[0], tuple) and all(isinstance(d, int) for d in args[0]):
            return IndexBox(torch.tensor([[0, d] for d in args[0]], dtype=torch.int64))
        try:
            return Box(*args)
        except (ValueError, TypeError):
            return Points(*args)


__all__ = ["Region", "Box", "Points", "IndexBox", "ContinuousBox", "IndexPoints", "ContinuousPoints", "Position",
           "IndexPosition", "ContinuousPosition"]
