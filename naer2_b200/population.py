"""Population: a node instance times a shape (reference naer2/population.py:22-662).

Its dynamic attributes (every self.<x> a hook assigns) are per-neuron state
tensors: set them as `pop.V = tensor` (or a scalar), read them back as the
live device tensors the kernel writes once the network has a runtime.
Scheduling is the network's fixed step dt (Network.resolution): every
population is updated every step; `timestep` may only restate that dt.
"""

from __future__ import annotations

import itertools

import numpy as np
import torch

from .registry import node_types
from .types import Region

_SEEDS = itertools.count(1)
_ORDER = itertools.count()  # creation order: the network lists its populations in it


class Population:
    def __init__(self, instance, shape, group_size: int = 256, timestep: float | None = None,
                 delay_resolution: float | None = None):
        object.__setattr__(self, "_state", {})
        object.__setattr__(self, "_net", None)
        self.shape = Region(shape)
        self.group_size = group_size  # neurons per block (the network's block uses the smallest)
        self.timestep = timestep
        self.delay_resolution = delay_resolution
        if instance.__class__ not in node_types:
            raise ValueError("node needs to be decorated by the @n2.node decorator")
        self.node = node_types[instance.__class__]
        assigned = self.node.send.assigned_members | self.node.update.assigned_members
        for hook in self.node.receive.values():
            assigned |= hook.assigned_members
        self.dynamic_attrs: dict = {}
        for member in sorted(assigned):
            if member not in instance.__dict__:
                raise ValueError(f"Node instance needs to have a member {member}")
            self.dynamic_attrs[member] = instance.__dict__[member].__class__
        self.instance = instance
        self.incoming: list = []
        self.seed = next(_SEEDS)  # the Philox key of this population's draws
        self._order = next(_ORDER)
        from .network import Network

        self.network = Network(self)

    # ------------------------------------------------------------------ state

    @property
    def ports(self):
        return self.node.receive.keys()

    def __len__(self) -> int:
        return len(self.shape)

    def state_tensor(self, attr: str, device=None) -> torch.Tensor:
        """The [n] tensor of a dynamic attribute (made from the instance's value on first use)."""
        st = self._state
        if attr not in st:
            default = getattr(self.instance, attr)
            py = self.dynamic_attrs.get(attr, type(default))
            dtype = torch.bool if py is bool else torch.int32 if py is int else torch.float32
            st[attr] = torch.full((len(self.shape),), default, dtype=dtype)
        if device is not None and st[attr].device != torch.device(device):
            st[attr] = st[attr].to(device)
        return st[attr]

    def __getattr__(self, name):
        st = object.__getattribute__(self, "_state")
        if name in st:
            return st[name]
        dyn = self.__dict__.get("dynamic_attrs", {})
        if name in dyn:
            return self.state_tensor(name)
        raise AttributeError(f"'{type(self).__name__}' has no attribute '{name}'")

    def __setattr__(self, name, value):
        dyn = self.__dict__.get("dynamic_attrs")
        if name[0] != "_" and dyn is not None and name in dyn:
            n = len(self.shape)
            cur = self._state.get(name)
            if cur is None:
                cur = self.state_tensor(name)
            v = torch.as_tensor(value)
            if v.numel() == 1:
                v = v.reshape(()).expand(n)
            if tuple(v.shape) != (n,):
                raise ValueError(f"'{name}' must be a scalar or a tensor of shape ({n},)")
            # in place: the runtime keeps the tensor's device pointer
            cur.copy_(v.to(device=cur.device, dtype=cur.dtype))
            return
        object.__setattr__(self, name, value)

    # ------------------------------------------------------------------ running

    def run(self, t_start: float, t_end: float) -> None:
        """Advance the population's network from t_start to t_end (the whole network moves together at a fixed
        dt; reference naer2/population.py:602-611 runs one population's kernel over [t_start, t_end))."""
        net = self.network
        if abs(net.t - t_start) > 1e-9 * max(1.0, abs(t_start)):
            raise ValueError(f"the network is at t={net.t}, not {t_start}")
        net.step(t_end - t_start)

    def check(self) -> None:
        """Raise on what the runs flagged (links out of range; reference naer2/population.py:613-616)."""
        self.network.check()

    def spikes(self) -> tuple[np.ndarray, np.ndarray]:
        """Recorded spikes (Network.record) as (steps, neuron indices), in step then index order."""
        return self.network.runtime.spikes(self)

    def emitted(self) -> list[tuple[float, int]]:
        """The last step's spikes as [(time, node)] (reference naer2/population.py:618-620); needs recording."""
        steps, ids = self.spikes()
        if len(steps) == 0:
            return []
        last = self.network.step_count - 1
        dt = self.network.resolution
        return [(last * dt, int(j)) for s, j in zip(steps, ids) if s == last]

    def __rshift__(self, right):
        from .connection import ConnectionBuilder

        return ConnectionBuilder(self).connect(right)

    def __matmul__(self, mapping):
        """A @ {real_name: hook_name}: a source map, before any edge is known."""
        from .connection import ConnectionBuilder

        if not isinstance(mapping, dict):
            raise ValueError("Population @ mapping expects a dict (source_map)")
        return ConnectionBuilder(self).source_map(mapping)

    def __repr__(self):
        return f"Population({type(self.instance).__name__} * {len(self.shape)})"
