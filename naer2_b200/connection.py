"""The connection chain `pop_a >> edge @ pattern >> pop_b` (reference
naer2/connection.py:1-309): ConnectionBuilder accumulates source, edge,
pattern, port and mappings; giving it the target builds the canonical
topology eagerly and returns the Connection. Per-link values are set on the
Connection: conn.delay (ms; a number or a per-link tensor) and any edge
attribute the target's receive hook reads as edge.<name> (e.g. conn.weight)."""

from __future__ import annotations

import itertools

import torch

from ._partial import _PartialConnection
from .fabric import Fabric
from .hook import used_members
from .registry import edge_types, node_types, pattern_types
from .topology import Topology


class ConnectionBuilder:
    def __init__(self, source):
        self._source = source
        self._target = None
        self._fabric: Fabric | None = None
        self._pattern = None
        self._target_port: str | None = None
        self._source_map: dict | None = None
        self._fabric_map: dict | None = None
        self._resolution: float | None = None

    @property
    def fabric(self) -> Fabric:
        return self._fabric

    @property
    def _topology(self):
        return self._fabric.topology if self._fabric is not None else None

    def _ensure_fabric(self) -> Fabric:
        if self._fabric is None:
            self._fabric = Fabric()
        return self._fabric

    def target(self, target):
        from .population import Population

        if not isinstance(target, Population):
            if target.__class__ not in node_types:
                raise ValueError(f"target {target!r} is not an instance of a node or a Population")
            if self._pattern is None:
                self._target = Population(target, 1)
            else:
                topology, region = Topology.build(self._pattern, self._source.shape)
                self._ensure_fabric().topology = topology
                self._target = Population(target, region)
        else:
            self._target = target
            if self._pattern is not None:
                self._ensure_fabric().topology = Topology.build(self._pattern, self._source.shape, target.shape,
                                                                same=self._source is target)
        if self._pattern is None:  # no pattern: one link from the (single) source neuron to each target neuron
            n_src, n_tgt = len(self._source.shape), len(self._target.shape)
            if n_src != 1:
                raise ValueError("a connection without a pattern needs a one-neuron source")
            self._ensure_fabric().topology = Topology(torch.tensor([0, n_tgt], dtype=torch.int64),
                                                      torch.arange(n_tgt, dtype=torch.int64))
        if self._target_port is not None and self._target_port not in self._target.ports:
            raise ValueError(f"target_port '{self._target_port}' not in {self._target!r}")
        self._source.network += self._target.network
        conn = Connection(self)
        self._source.network.connections.append(conn)
        self._target.incoming.append(conn)
        return conn

    def _set_fabric(self, fabric):
        if not isinstance(fabric, Fabric):
            if fabric.__class__ not in edge_types:
                raise ValueError(f"fabric {fabric!r} is not a Fabric")
            fabric = Fabric(fabric)
        self._fabric = fabric
        return self

    def pattern(self, pattern):
        if pattern not in pattern_types and not callable(pattern):
            raise ValueError(f"pattern {pattern!r} is not a registered Pattern")
        self._pattern = pattern
        return self

    def target_port(self, target_port: str):
        if not isinstance(target_port, str):
            raise ValueError("target port must be a string")
        if self._target is not None and target_port not in self._target.ports:
            raise ValueError(f"target_port '{target_port}' not in {self._target!r}")
        self._target_port = target_port
        return self

    def source_map(self, source_map: dict):
        if not isinstance(source_map, dict):
            raise ValueError("source_map must be a dict")
        self._source_map = {**(self._source_map or {}), **source_map}
        return self

    def fabric_map(self, fabric_map: dict):
        if not isinstance(fabric_map, dict):
            raise ValueError("fabric_map must be a dict")
        self._fabric_map = {**(self._fabric_map or {}), **fabric_map}
        return self

    def connect(self, to):
        from .population import Population

        if isinstance(to, _PartialConnection):
            self._fabric = Fabric(to.edge) if not isinstance(to.edge, Fabric) else to.edge
            self._pattern = to.pattern
            if to.port is not None:
                self.target_port(to.port)
            if to.fabric_map:
                self.fabric_map(to.fabric_map)
            return self
        if isinstance(to, Population) or to.__class__ in node_types:
            return self.target(to)
        if to.__class__ in edge_types:
            return self._set_fabric(Fabric(to))
        if isinstance(to, ConnectionBuilder) and to._target is None and to._source_map is not None:
            raise ValueError("a mapping after the target needs parentheses: write (A >> edge >> B) @ {...} -- "
                             "`>> B @ {...}` reads as `>> (B @ {...})`, a new connection from B with a source "
                             "mapping")
        if to in pattern_types or type(to) in pattern_types or callable(to):
            return self.pattern(to)
        raise ValueError(f"Cannot connect to {to!r}")

    def __rshift__(self, to):
        return self.connect(to)

    def at(self, place):
        if isinstance(place, str):
            return self.target_port(place)
        if not isinstance(place, dict):
            raise ValueError("at() expects a port name (str) or mapping (dict)")
        return self.source_map(place) if self._fabric is None else self.fabric_map(place)

    def __matmul__(self, mapping_or_port):
        return self.at(mapping_or_port)

    def delay(self, value):
        if type(value) not in (int, float):
            if not isinstance(value, torch.Tensor):
                raise ValueError("delay must be an int, float or tensor")
            if tuple(value.shape) != self.shape:
                raise ValueError(f"delay tensor must be shape {self.shape}")
        self._ensure_fabric().delay = value
        return self

    def __or__(self, value):
        return self.delay(value)

    @property
    def resolution(self):
        return self._resolution

    @property
    def shape(self) -> tuple:
        if self._topology is None:
            raise ValueError("shape is not available before the target is set")
        return self._topology.shape


_ORDER = itertools.count()


class Connection:
    """A fully specified connection between two populations."""

    def __init__(self, builder: ConnectionBuilder):
        object.__setattr__(self, "builder", builder)
        object.__setattr__(self, "_order", next(_ORDER))

    def __setattr__(self, name, value):
        if name == "resolution":
            if value is not None and not (isinstance(value, (int, float)) and value > 0):
                raise ValueError("resolution must be a positive number (or None: the network's)")
            self.builder._resolution = float(value) if value is not None else None
            return
        if name == "mode":  # how the hot path carries this connection: "push", "pull" or None (the tuner's)
            if value not in (None, "push", "pull"):
                raise ValueError("mode must be 'push', 'pull' or None")
            object.__setattr__(self, "_mode", value)
            return
        if name == "delay":
            self.builder.delay(value)
            return
        self._set_edge_attr(name, value)

    def _set_edge_attr(self, name, value) -> None:
        """conn.<name> = value, checked: the target's receive hook at this connection's port must read
        edge.<name> (after the fabric map), else nothing would ever read it (reference
        naer2/connection.py:246-276)."""
        builder = self.builder
        target = builder._target
        port = builder._target_port or "receive"
        hook = target.node.receive.get(port) if target is not None else None
        if hook is None:
            raise ValueError(f"cannot set '{name}': target has no receive hook at port '{port}'")
        rename = {hook_name: real for real, hook_name in (builder._fabric_map or {}).items()}
        used = {rename.get(n, n) for n in used_members(hook.ast, "edge")}
        if name not in used:
            raise ValueError(f"'{name}' is not used as edge.{name} by {target!r}'s receive hook (port '{port}') -- "
                             f"nothing would read this tensor")
        if isinstance(value, torch.Tensor) and value.numel() != 1 and tuple(value.shape) != builder.shape:
            raise ValueError(f"'{name}' must be a scalar or a tensor of shape {builder.shape}")
        setattr(builder._ensure_fabric(), name, value)

    @property
    def mode(self):
        return self.__dict__.get("_mode")

    def delay(self, value):
        self.builder.delay(value)
        return self

    def __or__(self, value):
        self.builder.delay(value)
        return self

    def __matmul__(self, other):
        self.builder.at(other)
        return self

    def __getattr__(self, name):
        return getattr(object.__getattribute__(self, "builder"), name)
