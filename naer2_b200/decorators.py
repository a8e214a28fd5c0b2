"""@n2.node, @n2.edge and @n2.pattern (reference naer2/decorators/node.py:10-73,
edge.py:13-51, pattern.py:5-33): register a class's hooks, and give node
instances `* n` (a Population) and `>>` / `@` (a one-neuron source)."""

from __future__ import annotations

from .hook import Hook
from .receives import destination, edge as _edge, source, time
from .registry import Node, edge_types, node_types, pattern_types
from .types import Position, Region


def node(cls=None, *, send: str = "send", receive: str | dict | None = "receive", update: str = "update"):
    """Class decorator of a node (neuron) model with send / update / receive hooks. Both @n2.node and
    @n2.node(send=..., receive=...|{port: method}|None, update=...)."""
    if cls is not None:
        return _node(cls, send, receive, update)
    return lambda c: _node(c, send, receive, update)


def _node(cls, send_name, receive_name, update_name):
    if not isinstance(cls, type):
        raise ValueError(f"node decorator can only be applied to types (got {type(cls)})")
    if receive_name is None:
        receives = {}
    elif isinstance(receive_name, str):
        receives = {receive_name: Hook("receive", getattr(cls, receive_name)).verify({time, _edge, source})}
    elif isinstance(receive_name, dict):
        receives = {str(port): Hook("receive", getattr(cls, str(name))).verify({time, _edge, source})
                    for port, name in receive_name.items()}
    else:
        raise ValueError(f"'receive' must be a string, dict[str, str], or None (got {type(receive_name).__name__}) "
                         f"in decorator for {cls.__name__}")
    node_types[cls] = Node(send=Hook("send", getattr(cls, str(send_name))).verify({time}),
                           update=Hook("update", getattr(cls, str(update_name))).verify({time}),
                           receive=receives)
    from .connection import ConnectionBuilder
    from .population import Population

    cls.__mul__ = lambda self, amount: Population(self, amount)
    cls.__rshift__ = lambda self, right: ConnectionBuilder(Population(self, 1)) >> right
    cls.__matmul__ = lambda self, right: ConnectionBuilder(Population(self, 1)) @ right
    return cls


def edge(cls=None, *, forward: str = "forward", backward: str = "backward"):
    """Class decorator of an edge (synapse) model; its instances start `edge @ pattern` chains."""
    if cls is not None:
        return _edge_decorator(cls, forward, backward)
    return lambda c: _edge_decorator(c, forward, backward)


def _edge_decorator(cls, forward_name, backward_name):
    if not isinstance(cls, type):
        raise ValueError(f"edge decorator can only be applied to types (got {type(cls)})")
    allowed = {time, source, destination}
    edge_types[cls] = {"forward": Hook("forward", getattr(cls, str(forward_name))).verify(allowed),
                       "backward": Hook("backward", getattr(cls, str(backward_name))).verify(allowed)}
    from ._partial import _PartialConnection

    cls.__matmul__ = lambda self, other: _PartialConnection(self) @ other
    return cls


def pattern(cb):
    """Register a callable (or callable class) as a connectivity pattern:
    (position, source_region[, target_region]) -> Region of targets."""
    if not callable(cb):
        raise ValueError(f"pattern decorator can only be applied to callables (got {type(cb).__name__})")
    fn = cb.__call__ if isinstance(cb, type) else cb
    pattern_types[cb] = Hook("pattern", fn).verify({Position, Region})
    return cb


__all__ = ["node", "edge", "pattern"]
