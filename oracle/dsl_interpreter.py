"""CPU interpreter of the DSL's fixed-step semantics -- test infrastructure only: the tests check the
transpiled, run-time compiled step kernels (naer2_b200/transpiler) against it.

It runs the models' own hook functions, in Python, one neuron at a time, on float32 state (numpy scalars, so
that arithmetic rounds to single precision as the kernels' does), in the order the kernels define for one
step n at time t = (n + 1) dt (the semantics the reference's fused round implements per population,
naer2/transpiler/templates/fused_template.py:321-371: deliveries, then update and send):
  for every population, every neuron j: for every incoming connection (network order), every link of j's
  pull row (canonical order within the row) whose source spiked at step n - d: receive(self, time, edge,
  source); then update(self, time); then send(self, time); n2.spike() marks j as firing at step n.
random.random() draws Philox4x32-10 words keyed by the population's seed and counted by (neuron, step,
call site, arrival); call sites are numbered in the order their calls run, which matches the transpiler's
source-order numbering when a hook's calls are not conditional.
"""

from __future__ import annotations

import random as _random

import numpy as np
import torch

import naer2_b200 as n2
from naer2_b200 import receives
from naer2_b200.topology import delay_steps, pull_form

from . import philox


class _Self:
    """self of neuron j: dynamic attributes in float32 / int32 / bool arrays, static ones as float32."""

    def __init__(self, arrays: dict, static: dict):
        object.__setattr__(self, "_a", arrays)
        object.__setattr__(self, "_s", static)
        object.__setattr__(self, "_j", 0)

    def __getattr__(self, name):
        a = object.__getattribute__(self, "_a")
        if name in a:
            return a[name][object.__getattribute__(self, "_j")]
        s = object.__getattribute__(self, "_s")
        if name in s:
            return s[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        self._a[name][self._j] = value


class _Link:
    """A link's edge values: per-link float32 arrays (pull order) and static float32 values; `names` maps the
    names a hook uses to the edge's own names; the arrays are writable where `writable`."""

    def __init__(self, values: dict, names: dict | None = None, writable: bool = False):
        object.__setattr__(self, "_v", values)
        object.__setattr__(self, "_n", names)
        object.__setattr__(self, "_w", writable)
        object.__setattr__(self, "_l", 0)

    def _real(self, name):
        n = object.__getattribute__(self, "_n")
        return n.get(name, name) if n is not None else name

    def __getattr__(self, name):
        v = object.__getattribute__(self, "_v")[self._real(name)]
        return v[object.__getattribute__(self, "_l")] if isinstance(v, np.ndarray) else v

    def __setattr__(self, name, value):
        if not self._w:
            raise AttributeError("the link is read-only in a receive hook")
        self._v[self._real(name)][self._l] = value


def _f32(v):
    return np.float32(v) if isinstance(v, float) else v


def run(net, n_steps: int):
    """Run `net` (its populations' current state tensors, on the CPU) for n_steps from step 0; returns
    (rasters: [bool [n_steps, n]] per population, final state: [{attr: array}] per population, per-link edge
    values the edge hooks change: {(connection index, name): array in canonical order}).

    Edge hooks: at an arrival the link's forward hook runs before the receive hook; when a neuron fires, the
    backward hook of every incoming link runs after send (connection order, link order). Their `self` is the
    link, their destination the neuron."""
    dt = float(net.resolution)
    pops = list(net.populations)
    index = {id(p): k for k, p in enumerate(pops)}
    arrays, selves = [], []
    for p in pops:
        arr = {}
        for a, py in p.dynamic_attrs.items():
            t = p.state_tensor(a).detach().cpu()
            arr[a] = t.numpy().astype(np.bool_ if py is bool else np.int32 if py is int else np.float32).copy()
        arrays.append(arr)
        static = {k: _f32(v) for k, v in p.instance.__dict__.items()
                  if k not in p.dynamic_attrs and isinstance(v, (int, float, bool))}
        selves.append(_Self(arr, static))
    from naer2_b200.transpiler.runtime import EdgePlan

    incoming = [[] for _ in pops]
    edge_state = {}
    for ci, c in enumerate(net.connections):
        t = index[id(c._target)]
        topo = c.fabric.topology
        steps = delay_steps(c.fabric.value("delay"), len(topo), dt, device="cpu")
        ptr, link, perm = pull_form(topo, steps.cpu(), len(pops[t].shape))
        perm = perm.cpu()
        port = c._target_port or "receive"
        hook = pops[t].node.receive[port]
        plan = EdgePlan(c, hook)
        values = {n: plan.initial(c, n, len(topo))[perm].numpy().copy() for n in plan.per_link}
        values.update({n: np.float32(v) for n, v in plan.static.items()})
        for n in plan.written:
            edge_state[(ci, n)] = (values[n], perm.numpy())
        w = link.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
        incoming[t].append((index[id(c._source)], ptr.cpu().numpy(), w & 0xFFFFFF, w >> 24, hook,
                            _Link(values, plan.recv), plan, _Link(values, None, writable=True)))
    spikes = [np.zeros((n_steps, len(p.shape)), dtype=bool) for p in pops]
    offsets = [np.zeros((n_steps, len(p.shape)), dtype=np.float32) for p in pops]  # time within the step
    exact = bool(getattr(net, "exact", False))

    state = {"fired": False, "j": 0, "n": 0, "k": 0xFFFFFF, "site": 0, "seed": (0, 0), "t": np.float32(0),
             "spike_t": np.float32(0)}

    def spike(time=None):
        if not state["fired"]:
            state["fired"] = True
            state["spike_t"] = np.float32(time) if time is not None else state["t"]

    def uniform():
        c3 = ((state["site"] & 0xFF) << 24) | (state["k"] & 0xFFFFFF)
        state["site"] += 1
        n = state["n"]
        w = philox([state["j"], n & 0xFFFFFFFF, (n >> 32) & 0xFFFFFFFF, c3], state["seed"])[0]
        return np.float32((w >> 8) * 5.9604644775390625e-08)

    def call(hook, obj, t, edge=None, site_base=0, dst=None):
        kw = {}
        for ty, nm in hook.parameter_type_to_name.items():
            if ty is receives.time:
                kw[nm] = t
            elif ty is receives.edge:
                kw[nm] = edge
            elif ty is receives.source:
                kw[nm] = None
            elif ty is receives.destination:
                kw[nm] = dst
        state["site"] = site_base
        state["t"] = t
        hook.function(obj, **kw)

    saved = (n2.spike, _random.random)
    n2.spike, _random.random = spike, uniform
    try:
        for n in range(n_steps):
            t = np.float32((n + 1) * dt)
            t0 = np.float32(n * dt)
            state["n"] = n
            for k, p in enumerate(pops):
                obj = selves[k]
                state["seed"] = (int(p.seed) & 0xFFFFFFFF, (int(p.seed) >> 32) & 0xFFFFFFFF)
                node = p.node
                n_recv = len(incoming[k])
                for j in range(len(p.shape)):
                    object.__setattr__(obj, "_j", j)
                    state["j"], state["fired"], arrived = j, False, 0
                    state["spike_t"] = t
                    arrivals = []  # (time, connection, link) in collection order
                    for ci, (s, ptr, src, d, hook, edge, plan, link) in enumerate(incoming[k]):
                        for l in range(ptr[j], ptr[j + 1]):
                            m = n - int(d[l])
                            if m < 0 or not spikes[s][m, src[l]]:
                                continue
                            tau = np.float32(t0 + offsets[s][m, src[l]]) if exact else t
                            arrivals.append((tau, ci, l))
                    if exact:
                        arrivals.sort(key=lambda a: a[0])  # stable: equal times keep collection order
                    for idx, (tau, ci, l) in enumerate(arrivals):
                        s, ptr, src, d, hook, edge, plan, link = incoming[k][ci]
                        object.__setattr__(edge, "_l", l)
                        object.__setattr__(link, "_l", l)
                        state["k"] = arrived
                        arrived += 1
                        if plan.forward is not None:
                            call(plan.forward, link, tau, dst=obj)
                        call(hook, obj, tau, edge, site_base=32 * ci)
                        if exact and (idx + 1 == len(arrivals) or arrivals[idx + 1][0] != tau):
                            state["k"] = 0xFFFFFF  # send after each group of equal times
                            call(node.send, obj, tau, site_base=32 * n_recv + 32)
                    state["k"] = 0xFFFFFF
                    call(node.update, obj, t, site_base=32 * n_recv)
                    call(node.send, obj, t, site_base=32 * n_recv + 32)
                    spikes[k][n, j] = state["fired"]
                    if state["fired"]:
                        offsets[k][n, j] = np.float32(state["spike_t"] - t0)
                        for (s, ptr, src, d, hook, edge, plan, link) in incoming[k]:  # edge backward hooks
                            if plan.backward is None:
                                continue
                            for l in range(ptr[j], ptr[j + 1]):
                                object.__setattr__(link, "_l", l)
                                call(plan.backward, link, state["spike_t"], dst=obj)
    finally:
        n2.spike, _random.random = saved
    edges = {}
    for (ci, name), (v, perm) in edge_state.items():  # back to canonical link order
        out = np.empty_like(v)
        out[perm] = v
        edges[(ci, name)] = out
    if exact:
        return spikes, arrays, edges, offsets
    return spikes, arrays, edges
