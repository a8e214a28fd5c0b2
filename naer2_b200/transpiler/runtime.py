"""The run-time compiled path: a network whose populations' hooks are lowered to CUDA and compiled with
NVRTC (reference naer2/runtime.py:213-526, PopulationRuntime, which builds and launches the generated
Gluon kernels; here one generated step kernel per population, `n2b_jit_*` in the C ABI).

Built by Network.runtime when a population's model has no built-in kernel (models.params_of raises). Every
population of such a network runs its own transpiled hooks -- built-in models included, as their hooks
state them in Python. The interface Network uses is NetworkRuntime's: advance, start_recording, raster,
spikes, status, check, counters, reset_counters, close.
"""

from __future__ import annotations

import ast
import ctypes
import hashlib

import numpy as np
import torch

from .. import _lib
from ..topology import delay_steps, pull_form
from .template import NPB_C, build_source, ctype_of, edge_hook_context, hook_context, params_type, scan

BLOCK = 128  # exact-time intake: one thread per neuron
_CACHE: dict = {}  # (source hash, device) -> n2b_jit_kernel handle, for the process's lifetime


def compile_source(source: str, device: int) -> ctypes.c_void_p:
    key = (hashlib.sha256(source.encode()).hexdigest(), device)
    if key not in _CACHE:
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.n2b_jit_compile(source.encode(), b"n2b_user_step", None, 0, device, ctypes.byref(h)),
                   "n2b_jit_compile")
        _CACHE[key] = h
    return _CACHE[key]


def trivial(hook) -> bool:
    """A hook whose body does nothing (pass / a docstring)."""
    if hook is None:
        return True
    return all(isinstance(st, ast.Pass) or (isinstance(st, ast.Expr) and isinstance(st.value, ast.Constant))
               for st in hook.ast.body)


class EdgePlan:
    """What a connection's hooks read and write of its links. recv: {receive-facing name: edge name};
    per_link: edge names held per link (assigned by the edge hooks, or set as per-link tensors); written:
    those the edge hooks assign; static: {edge name: value} of the rest; forward / backward: the edge's
    non-trivial hooks (or None)."""

    def __init__(self, conn, receive_hook):
        from .. import receives
        from ..hook import used_members

        fabric = conn.fabric
        rename = {hook_name: real for real, hook_name in (conn._fabric_map or {}).items()}
        edge_param = receive_hook.parameter_type_to_name.get(receives.edge, "edge") if receive_hook else "edge"
        names = used_members(receive_hook.ast, edge_param) if receive_hook is not None else set()
        self.recv = {h: rename.get(h, h) for h in sorted(names)}
        has_edge = fabric.instance is not None
        self.forward = None if not has_edge or trivial(fabric.edge["forward"]) else fabric.edge["forward"]
        self.backward = None if not has_edge or trivial(fabric.edge["backward"]) else fabric.edge["backward"]
        used, written = set(self.recv.values()), set()
        for h in (self.forward, self.backward):
            if h is not None:
                used |= used_members(h.ast, "self")
                written |= h.assigned_members
        self.written = sorted(written)
        self.per_link, self.static = [], {}
        for name in sorted(used):
            v = fabric.value(name)
            if v is None:
                raise ValueError(f"{conn!r}: edge.{name} is read but the connection has no such attribute")
            if name in written or (isinstance(v, torch.Tensor) and v.numel() != 1):
                self.per_link.append(name)
            else:
                self.static[name] = float(v.item() if isinstance(v, torch.Tensor) else v)

    def initial(self, conn, name: str, n_links: int) -> torch.Tensor:
        """A per-link array's starting values, canonical order, float32 on the CPU."""
        v = conn.fabric.value(name)
        if isinstance(v, torch.Tensor) and v.numel() == n_links:
            return v.detach().reshape(-1).to("cpu", torch.float32)
        return torch.full((n_links,), float(v.item() if isinstance(v, torch.Tensor) else v), dtype=torch.float32)


def plan_of(net) -> dict:
    """The transpiled form of a network, everything its step kernels need and nothing of its Python model classes:
    per population its CUDA source, the Params fields with the values of the scalar ones, its state attributes
    (name -> "float" / "int" / "bool"), size, seed and spike-ring depth; per incoming connection (in order) its
    source population, pull CSR (int32 ptr, uint32 link words) and per-link edge arrays (pull order) with the
    pull permutation. JitRuntime builds from it; save_plan / load_plan keep it in a file, so that a network can
    be transpiled where its model classes are and stepped where only the plan is."""
    dev = net.device if net.device is not None else torch.device("cpu")
    dt = float(net.resolution)
    pops = list(net.populations)
    index = {id(p): k for k, p in enumerate(pops)}
    words = [(len(p.shape) + 31) // 32 for p in pops]
    # spike-bit ring depth of each population: above every delay of its outgoing connections
    steps_of, max_out = {}, [1] * len(pops)
    for c in net.connections:
        topo = c.fabric.topology
        steps = delay_steps(c.fabric.value("delay"), len(topo), dt, device=topo.target_indices.device)
        steps_of[id(c)] = steps
        if len(topo):
            s = index[id(c._source)]
            max_out[s] = max(max_out[s], int(steps.max()))
    depth = [max(2, 1 << int(np.ceil(np.log2(m + 1)))) for m in max_out]
    exact = bool(getattr(net, "exact", False))
    plan = {"dt": dt, "exact": exact, "pops": []}
    for k, p in enumerate(pops):
        node = p.node
        incoming = []
        conns = [c for c in net.connections if c._target is p]
        site = 0
        for c in conns:
            port = c._target_port or "receive"
            hook = node.receive.get(port)
            if hook is None:
                raise ValueError(f"{p!r} has no receive port {port!r}")
            ep = EdgePlan(c, hook)
            dyn = [h for h, real in ep.recv.items() if real in ep.per_link]
            stat = {h: ep.static[real] for h, real in ep.recv.items() if real not in ep.per_link}
            ctx = hook_context(p, hook, dyn, stat, site_base=site)
            site += 32
            inc = {"receive": (hook.ast, ctx), "edge_dynamic": ep.per_link, "edge_written": ep.written,
                   "alias": {h: real for h, real in ep.recv.items() if real in ep.per_link and h != real},
                   "forward": None, "backward": None, "conn": c, "plan": ep}
            for kind in ("forward", "backward"):
                eh = getattr(ep, kind)
                if eh is not None:
                    inc[kind] = (eh.ast, edge_hook_context(p, eh, ep.per_link, ep.static))
            incoming.append(inc)
        hooks = {"update": (node.update.ast, hook_context(p, node.update, site_base=site)),
                 "send": (node.send.ast, hook_context(p, node.send, site_base=site + 32))}
        src, fields = build_source(type(p.instance).__name__, dict(p.dynamic_attrs), hooks, incoming,
                                   exact=exact, n=len(p.shape))
        attrs = {a: ("bool" if py is bool else "int" if py is int else "float") for a, py in p.dynamic_attrs.items()}
        entry = {"name": type(p.instance).__name__, "n": len(p.shape), "words": words[k], "depth": depth[k],
                 "seed": int(p.seed) & 0xFFFFFFFFFFFFFFFF, "source": src,
                 "fields": [(name, ctype) for name, ctype, _ in fields], "attrs": attrs, "conns": []}
        for inc in incoming:
            c = inc["conn"]
            topo = c.fabric.topology
            ptr, link, perm = pull_form(topo, steps_of[id(c)], len(p.shape))
            ep = inc["plan"]
            per_link = {}
            for e in ep.per_link:
                v = ep.initial(c, e, len(topo))
                per_link[e] = (v[perm.cpu()] if v.numel() else torch.zeros(0)).to(torch.float32)
            entry["conns"].append({"src": index[id(c._source)], "ptr": ptr.to(torch.int32).cpu(),
                                   "link": link.to(torch.int32).cpu(), "perm": perm.cpu(), "per_link": per_link,
                                   "written": list(ep.written), "conn_id": id(c)})
        plan["pops"].append(entry)
    plan["device"] = dev
    return plan


def save_plan(plan: dict, path) -> None:
    """A plan in one .npz file: its structure as JSON, its arrays beside it."""
    import json

    arrays, meta = {}, {"dt": plan["dt"], "exact": plan["exact"], "pops": []}
    for k, p in enumerate(plan["pops"]):
        m = {key: p[key] for key in ("name", "n", "words", "depth", "seed", "source", "fields", "attrs")}
        m["conns"] = []
        for ci, c in enumerate(p["conns"]):
            for key in ("ptr", "link", "perm"):
                arrays[f"p{k}_c{ci}_{key}"] = c[key].numpy()
            for e, v in c["per_link"].items():
                arrays[f"p{k}_c{ci}_e_{e}"] = v.numpy()
            m["conns"].append({"src": c["src"], "per_link": list(c["per_link"]), "written": c["written"]})
        meta["pops"].append(m)
    arrays["plan_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrays)


def load_plan(path) -> dict:
    import json

    z = np.load(path)
    meta = json.loads(bytes(z["plan_json"]).decode())
    plan = {"dt": meta["dt"], "exact": meta["exact"], "pops": []}
    for k, m in enumerate(meta["pops"]):
        p = dict(m)
        p["fields"] = [tuple(f) for f in m["fields"]]
        p["conns"] = []
        for ci, c in enumerate(m["conns"]):
            p["conns"].append({"src": c["src"], "written": c["written"], "conn_id": None,
                               "ptr": torch.from_numpy(z[f"p{k}_c{ci}_ptr"]),
                               "link": torch.from_numpy(z[f"p{k}_c{ci}_link"]),
                               "perm": torch.from_numpy(z[f"p{k}_c{ci}_perm"]),
                               "per_link": {e: torch.from_numpy(z[f"p{k}_c{ci}_e_{e}"]) for e in c["per_link"]}})
        plan["pops"].append(p)
    return plan


_CTYPES = {"long long": ctypes.c_int64, "float": ctypes.c_float, "int": ctypes.c_int32, "u32": ctypes.c_uint32}


def _params_struct(fields: list):
    """The ctypes Params structure of a plan's fields (pointers as void *)."""
    return params_type([(name, ct, ctypes.c_void_p if ct.endswith("*") else _CTYPES[ct]) for name, ct in fields])


class JitRuntime:
    """The step kernels of a transpiled network: built from `net` (its plan made on the spot), or from a saved
    plan (`plan`; `net` then a PlannedNetwork holding the plan's state)."""

    def __init__(self, net, plan: dict | None = None):
        self.net = net
        dev = self.device = net.device
        dindex = dev.index if dev.index is not None else 0
        if plan is None:
            plan = plan_of(net)
        self.plan = plan
        dt = self.dt = float(plan["dt"])
        pops = self.pops = list(net.populations)
        self.keep = []
        words = self.words = [p["words"] for p in plan["pops"]]
        depth = self.depth = [p["depth"] for p in plan["pops"]]
        self.bits = [torch.zeros(d * w, dtype=torch.int32, device=dev) for d, w in zip(depth, words)]
        # each spike's time within its step (event-driven intake reads it; the clocked one ignores it)
        self.offs = [torch.zeros(d * max(1, p["n"]), dtype=torch.float32, device=dev)
                     for d, p in zip(depth, plan["pops"])]
        self.exact = bool(plan["exact"])
        self.err = torch.zeros(len(pops), dtype=torch.int32, device=dev)
        self.counters_t = torch.zeros(len(pops), 2, dtype=torch.int64, device=dev)
        self.record_rows = int(net.record_steps)
        self.rec_step0 = net.step_count
        self.rasters = [torch.zeros(max(1, self.record_rows) * w, dtype=torch.int32, device=dev) for w in words]
        self.raster_offs = [torch.zeros(max(1, self.record_rows) * max(1, p["n"]), dtype=torch.float32,
                                        device=dev) for p in plan["pops"]]
        self.kernels, self.params, self.sources = [], [], []
        self.edge_arrays = {}  # (connection id, edge name) -> (per-link values in pull order, pull permutation)
        tdtype = {"bool": torch.bool, "int": torch.int32, "float": torch.float32}
        for k, (p, pp) in enumerate(zip(pops, plan["pops"])):
            self.sources.append(pp["source"])
            self.kernels.append(compile_source(pp["source"], dindex))
            P = _params_struct(pp["fields"])()
            P.n, P.words, P.bit_mask = pp["n"], words[k], depth[k] - 1
            P.seed_lo, P.seed_hi = pp["seed"] & 0xFFFFFFFF, (pp["seed"] >> 32) & 0xFFFFFFFF
            for a, ty in pp["attrs"].items():
                t = p.state_tensor(a, dev)
                if t.dtype != tdtype[ty]:
                    t = t.to(tdtype[ty])
                if not t.is_contiguous():
                    t = t.contiguous()
                p._state[a] = t
                setattr(P, f"s_{a}", t.data_ptr())
            P.bits, P.raster = self.bits[k].data_ptr(), self.rasters[k].data_ptr()
            P.off, P.raster_off = self.offs[k].data_ptr(), self.raster_offs[k].data_ptr()
            P.raster_steps, P.rec0 = self.record_rows, self.rec_step0
            P.err = self.err[k:].data_ptr()
            P.counters = self.counters_t[k].data_ptr()
            for ci, c in enumerate(pp["conns"]):
                s = c["src"]
                ptr = self._dev(c["ptr"])
                link = self._dev(c["link"] if c["link"].numel() else torch.zeros(1, dtype=torch.int32))
                setattr(P, f"c{ci}_ptr", ptr.data_ptr())
                setattr(P, f"c{ci}_link", link.data_ptr())
                setattr(P, f"c{ci}_src_bits", self.bits[s].data_ptr())
                setattr(P, f"c{ci}_src_words", words[s])
                setattr(P, f"c{ci}_src_mask", depth[s] - 1)
                setattr(P, f"c{ci}_src_off", self.offs[s].data_ptr())
                setattr(P, f"c{ci}_src_n", plan["pops"][s]["n"])
                for e, v in c["per_link"].items():
                    v = self._dev(v if v.numel() else torch.zeros(1))
                    self.edge_arrays[(c["conn_id"], e)] = (v, c["perm"])
                    setattr(P, f"c{ci}_e_{e}", v.data_ptr())
            self.params.append(P)
        self.stream = torch.cuda.Stream(device=dev)
        self._s = ctypes.c_void_p(self.stream.cuda_stream)
        self.launches = 0

    def _dev(self, t):
        t = t.to(self.device).contiguous()
        self.keep.append(t)
        return t

    # ------------------------------------------------------------------ stepping

    def advance(self, n_steps: int) -> None:
        """Steps step_count .. step_count + n_steps - 1: per step one launch per population, in order, the whole
        window in one library call (n2b_jit_launch_window writes each launch's step and times)."""
        lib = _lib.load()
        n_steps = int(n_steps)
        if n_steps <= 0:
            return
        self.stream.wait_stream(torch.cuda.current_stream(self.device))
        step = self.net.step_count
        k = len(self.kernels)
        grids, blocks = (ctypes.c_uint32 * k)(), (ctypes.c_uint32 * k)()
        kerns, params, sizes = (ctypes.c_void_p * k)(), (ctypes.c_void_p * k)(), (ctypes.c_size_t * k)()
        for i, (kern, P, p) in enumerate(zip(self.kernels, self.params, self.pops)):
            per = BLOCK if self.exact else NPB_C  # neurons per block (clocked: SCAN threads each)
            size = len(p.shape)
            grids[i] = (size + per - 1) // per
            blocks[i] = BLOCK if self.exact else scan(size) * NPB_C
            kerns[i] = kern.value
            params[i] = ctypes.addressof(P)
            sizes[i] = ctypes.sizeof(P)
        _lib.check(lib.n2b_jit_launch_window(kerns, grids, blocks, params, sizes, k, step, n_steps, self.dt,
                                             self._s), "n2b_jit_launch_window")
        last = step + n_steps - 1
        for P in self.params:  # (the fields as the last launch had them)
            P.step, P.t, P.t0 = last, (last + 1) * self.dt, last * self.dt
        self.launches += n_steps * sum(1 for g in grids if g)
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def start_recording(self, steps: int) -> None:
        if self.record_rows == 0 or steps > self.record_rows:
            raise RuntimeError("recording needs Network.record(steps) before the first step "
                               f"(this runtime keeps {self.record_rows} rows)")
        self.rec_step0 = self.net.step_count
        for P in self.params:
            P.rec0 = self.rec_step0

    # ------------------------------------------------------------------ results

    def raster_words(self, pop) -> np.ndarray:
        k = self.pops.index(pop)
        words = self.words[k]
        rows = min(self.record_rows, self.net.step_count - self.rec_step0)
        if rows <= 0:
            return np.zeros((0, words), dtype=np.uint32)
        self.stream.synchronize()
        return self.rasters[k][: rows * words].cpu().numpy().view(np.uint32).reshape(rows, words)

    def raster(self, pop) -> np.ndarray:
        w = self.raster_words(pop)
        n = len(pop.shape)
        bits = np.unpackbits(w.view(np.uint8).reshape(len(w), -1, 4), axis=2, bitorder="little")
        return bits.reshape(len(w), -1)[:, :n].astype(bool)

    def spikes(self, pop):
        steps, ids = np.nonzero(self.raster(pop))
        return steps.astype(np.int64) + self.rec_step0, ids.astype(np.int64)

    def edge_state(self, conn, name: str) -> torch.Tensor:
        """A per-link edge value (a weight the edge hooks change, ...) in canonical link order."""
        if (id(conn), name) not in self.edge_arrays:
            raise KeyError(f"{name} is not held per link on this connection")
        self.stream.synchronize()
        v, perm = self.edge_arrays[(id(conn), name)]
        out = torch.empty_like(v)
        if perm.numel():
            out[perm.to(v.device)] = v[: perm.numel()]
        return out[: perm.numel()]

    def spike_times(self, pop) -> tuple:
        """(times ms float32, neuron ids) of the recorded spikes: each spike's step start plus its time within
        the step (the end of the step for a spike of the clocked send; its own time in the event-driven intake)."""
        raster = self.raster(pop)
        steps, ids = np.nonzero(raster)
        k = self.pops.index(pop)
        n = len(pop.shape)
        offs = self.raster_offs[k][: len(raster) * n].cpu().numpy()
        o = offs[steps * n + ids]
        t0 = ((steps + self.rec_step0) * self.dt).astype(np.float32)
        return (t0 + o).astype(np.float32), ids.astype(np.int64)

    def status(self) -> list:
        self.stream.synchronize()
        return self.err.cpu().tolist()

    def check(self) -> None:
        bad = sum(self.status())
        if bad:
            raise RuntimeError(f"{bad} links with a delay outside their source's spike ring")

    def counters(self) -> dict:
        self.stream.synchronize()
        c = self.counters_t.cpu().numpy()
        return {"events": int(c[:, 0].sum()), "spikes": int(c[:, 1].sum()),
                "per_population": [int(x) for x in c[:, 1]]}

    def reset_counters(self) -> None:
        self.stream.synchronize()
        self.counters_t.zero_()
        self.err.zero_()

    def close(self) -> None:
        self.stream.synchronize()
        self.kernels = []


class PlannedPopulation:
    """A population as a plan describes it: its size, seed and state tensors, no model class."""

    def __init__(self, entry: dict, state: dict):
        self.name = entry["name"]
        self.shape = range(entry["n"])
        self.seed = entry["seed"]
        self._state = dict(state)

    def state_tensor(self, attr: str, device=None) -> torch.Tensor:
        t = self._state[attr]
        if device is not None and t.device != torch.device(device):
            t = self._state[attr] = t.to(device)
        return t

    def __repr__(self):
        return f"PlannedPopulation({self.name} x {len(self.shape)})"


class PlannedNetwork:
    """Steps a saved plan (plan_of / save_plan / load_plan): the step kernels of a transpiled network, run where
    its Python model classes are not. states: per population {attribute: tensor [n]} (the initial state)."""

    def __init__(self, plan: dict, states: list, device, record_steps: int = 0):
        self.device = torch.device(device)
        self.resolution = float(plan["dt"])
        self.exact = bool(plan["exact"])
        self.step_count = 0
        self.record_steps = int(record_steps)
        self.populations = [PlannedPopulation(p, st) for p, st in zip(plan["pops"], states)]
        self.runtime = JitRuntime(self, plan)

    def run_steps(self, n_steps: int) -> None:
        self.runtime.advance(n_steps)
        self.step_count += int(n_steps)

    def close(self) -> None:
        self.runtime.close()
