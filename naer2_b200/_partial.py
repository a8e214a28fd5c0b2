"""`edge @ ...` before the source is known (reference naer2/_partial.py:1-41):
accumulates, in any order, a pattern, a target port (str) and a fabric map
(dict), consumed by `>>` on a population."""


class _PartialConnection:
    def __init__(self, edge, pattern=None):
        self.edge = edge
        self.pattern = pattern
        self.port: str | None = None
        self.fabric_map: dict | None = None

    def __matmul__(self, other) -> "_PartialConnection":
        if isinstance(other, str):
            if self.port is not None:
                raise ValueError(f"target port already set to {self.port!r}")
            self.port = other
            return self
        if isinstance(other, dict):
            self.fabric_map = {**(self.fabric_map or {}), **other}
            return self
        if self.pattern is not None:
            raise ValueError(f"pattern already set to {self.pattern!r}")
        self.pattern = other
        return self
