"""A connection's edge bundle: its edge instance (or none), canonical topology
and per-link values (reference naer2/fabric.py:12-170). `fabric.<name>`
reads and writes the per-link values (weight, delay, ...) in canonical link
order; a scalar stands for every link."""

from __future__ import annotations

from .registry import edge_types

_INTERNAL = frozenset({"instance", "edge", "dynamic_attrs", "static_attrs", "topology", "state"})


class Fabric:
    def __init__(self, instance=None):
        if instance is not None and instance.__class__ not in edge_types:
            raise ValueError("edge needs to be decorated by the @n2.edge decorator")
        object.__setattr__(self, "instance", instance)
        object.__setattr__(self, "edge", edge_types[instance.__class__] if instance is not None
                           else {"forward": None, "backward": None})
        object.__setattr__(self, "topology", None)
        object.__setattr__(self, "state", {})
        dynamic = {}
        if instance is not None:
            for member in self.edge["forward"].assigned_members | self.edge["backward"].assigned_members:
                if member not in instance.__dict__:
                    raise ValueError(f"Edge instance needs to have a member '{member}'")
                dynamic[member] = instance.__dict__[member].__class__
        object.__setattr__(self, "dynamic_attrs", dynamic)
        object.__setattr__(self, "static_attrs", {k: v for k, v in (instance.__dict__.items() if instance else ())
                                                  if k not in dynamic})

    def value(self, name: str, default=None):
        """A per-link value: set on the fabric, else the edge instance's attribute, else default."""
        if name in self.state:
            return self.state[name]
        if self.instance is not None and name in self.instance.__dict__:
            return getattr(self.instance, name)
        return default

    def __setattr__(self, name, value):
        if name in _INTERNAL:
            object.__setattr__(self, name, value)
        else:
            self.state[name] = value

    def __getattr__(self, name):
        state = object.__getattribute__(self, "state")
        if name in state:
            return state[name]
        raise AttributeError(f"'{type(self).__name__}' has no attribute '{name}'")
