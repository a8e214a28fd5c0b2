"""The GPU runtime of a network: its device buffers (PyTorch tensors) and the
libnaer2b handle that steps them (include/naer2b.h). Replaces the
reference's per-population PopulationRuntime (naer2/runtime.py:213-758) and
the fused-round launch (naer2/fusion.py:31-141): one handle per network, one
fused step kernel per step over every population, windows of steps replayed
from one CUDA graph.

Device layout (HBM), per population of n neurons:
  state        fp32 V [n] (and I [n] for PD14), int32 refractory counter [n]
  acc          int64 [D][n] arrival slots, D = pow2 > its largest incoming delay
  bits         uint32 [R][ceil(n/32)] spike-bit ring (sources of pull links only)
  raster       uint32 [rows][ceil(n/32)] recorded spikes (Network.record)
  ext_table    uint32 inverse-CDF table of its external Poisson count
per connection: int32 row offsets, uint32 link words (delay << 24 | index)
and fp32 weights (none for a single weight), push rows by source or pull
rows by target.

The input of a population is summed exactly in int64 fixed point with
`shift` = min(40, 61 - ceil(log2(max over neurons of the largest possible
step input))): no sum can overflow, and a weight w >= 2^(23 - shift) is
represented exactly.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from .models import params_of
from .topology import delay_steps, pack_links, pull_split_form, push_form

MAX_SHIFT = 40


def next_pow2(x: int) -> int:
    return 1 << max(0, math.ceil(math.log2(max(int(x), 1))))


def fixed_shift(max_input: float) -> int:
    if not max_input > 0.0:
        return MAX_SHIFT
    return int(max(0, min(MAX_SHIFT, 61 - math.ceil(math.log2(max_input)))))


def wfx(w: float, shift: int) -> int:
    """A weight in the fixed point of `shift`: fp32(w) * 2^shift rounded to nearest, ties to even."""
    return int(np.rint(np.ldexp(np.float32(w), shift)))


def weights_of(conn, n_links: int, device=None):
    """(scalar or None, per-link fp32 tensor or None): a connection's weights in canonical order (a tensor of
    one value counts as a scalar)."""
    w = conn.fabric.value("weight")
    if w is None:
        raise ValueError(f"connection {conn._source!r} -> {conn._target!r} has no weight")
    if isinstance(w, torch.Tensor):
        if w.numel() == 1:
            return float(np.float32(float(w.reshape(())))), None
        arr = w.detach().reshape(-1).to(torch.float32)
        if device is not None:
            arr = arr.to(device)
        if arr.numel() != n_links:
            raise ValueError(f"weight has {arr.numel()} values for {n_links} links")
        if arr.numel() == 0:
            return 0.0, None
        if bool((arr == arr[0]).all()):
            return float(arr[0]), None
        return None, arr.contiguous()
    return float(np.float32(w)), None


@dataclass
class PopDesc:
    """One population as the kernels see it (the n2b_population fields)."""
    model: int
    n: int
    acc_depth: int
    bit_depth: int
    shift: int
    ref_steps: int
    fire_threshold: int
    seed: int
    p: list
    ext_table: np.ndarray
    ext_weight: float
    ext_wfx: int
    state: dict  # kernel slot ("v", "i", "ref") -> attribute name


@dataclass
class ConnDesc:
    """One connection in its device form (push rows by source or pull rows by target), torch tensors on the
    device its topology was built on; `canonical()` gives the canonical rows (for the oracle)."""
    src: int
    tgt: int
    mode: str
    n_links: int
    ptr: torch.Tensor              # int32
    link: torch.Tensor             # int32 bit pattern of uint32: delay << 24 | index
    weight: float                  # when w is None
    w: torch.Tensor | None         # fp32 per link, in the form's order
    split: torch.Tensor | None     # push: per row its first link of delay >= 2
    topo: object = None            # the canonical Topology
    steps: torch.Tensor = None     # per-link delays in steps, canonical order
    warr: torch.Tensor | None = None  # per-link weights, canonical order

    def canonical(self):
        """(ptr int32, link uint32, w fp32 or None) as numpy arrays, rows per source in canonical order."""
        ptr = self.topo.source_offsets.cpu().numpy().astype(np.int32)
        link = pack_links(self.topo.target_indices, self.steps.to(self.topo.target_indices.device))
        w = self.warr.cpu().numpy() if self.warr is not None else None
        return ptr, link.cpu().numpy().view(np.uint32), w


@dataclass
class NetDesc:
    dt: float
    pops: list
    conns: list
    n_links: int


def describe(net, modes: dict | None = None, forms: bool = True) -> NetDesc:
    """The network as the kernels see it: per population its model constants, ring depths, fixed-point
    shift and external-drive table; per connection its CSR form, built where its topology lives (a pattern
    drawn on the GPU is restructured there). modes: connection id -> "push" / "pull" (default: the
    connection's own `mode`, else the network's tuned choice, else push). forms=False: the canonical rows only
    (ConnDesc.canonical), no device form (ptr, link, w and split None) -- a description for a host-side
    checker of a large network, without the form's sort."""
    dt = float(net.resolution)
    pops, conns = list(net.populations), list(net.connections)
    index = {id(p): k for k, p in enumerate(pops)}
    for p in pops:
        if p.timestep is not None and abs(p.timestep - dt) > 1e-12:
            raise ValueError(f"{p!r}: timestep {p.timestep} differs from the network's dt {dt} "
                             f"(this build steps every population at one dt)")
    kp = [params_of(p, dt) for p in pops]
    max_in_delay = [0] * len(pops)
    max_pull_delay = [0] * len(pops)
    in_max = [0.0] * len(pops)
    in_sum: list = [None] * len(pops)
    cinfo = []
    for c in conns:
        s, t = index[id(c._source)], index[id(c._target)]
        if kp[t]["port"] is None:
            raise ValueError(f"{pops[t]!r} takes no input (no receive hook)")
        port = c._target_port or "receive"
        if port not in pops[t].ports:
            raise ValueError(f"{pops[t]!r} has no receive port {port!r}")
        topo = c.fabric.topology
        dev = topo.target_indices.device
        n_links = len(topo)
        steps = delay_steps(c.fabric.value("delay"), n_links, dt, device=dev)
        wscalar, warr = weights_of(c, n_links, device=dev)
        mode = (modes or {}).get(id(c)) or c.mode or net.tuned.get(id(c), "push")
        if n_links:
            tgt = topo.target_indices
            absw = warr.abs().to(torch.float64) if warr is not None else None
            part = torch.bincount(tgt, weights=absw, minlength=len(pops[t].shape)).to(torch.float64)
            if warr is None:
                part = part * abs(wscalar)
            in_sum[t] = part.cpu() if in_sum[t] is None else in_sum[t] + part.cpu()
            max_in_delay[t] = max(max_in_delay[t], int(steps.max()))
            if mode == "pull":
                max_pull_delay[s] = max(max_pull_delay[s], int(steps.max()))
        cinfo.append((s, t, topo, steps, wscalar, warr, mode))
    for k in range(len(pops)):
        in_max[k] = float(in_sum[k].max()) if in_sum[k] is not None and len(in_sum[k]) else 0.0

    pdesc = []
    for k, (p, par) in enumerate(zip(pops, kp)):
        n = len(p.shape)
        table = par["ext_table"]
        max_input = in_max[k]
        if len(table):
            max_input += abs(par["ext_weight"]) * (len(table) - 1)
        sh = fixed_shift(max_input)
        pdesc.append(PopDesc(
            model=par["model"], n=n,
            acc_depth=next_pow2(max_in_delay[k] + 1) if par["port"] is not None else 0,
            bit_depth=next_pow2(max_pull_delay[k] + 1) if max_pull_delay[k] > 0 else 0,
            shift=sh, ref_steps=int(par["ref_steps"]), fire_threshold=int(par["fire_threshold"]),
            seed=int(p.seed) & 0xFFFFFFFFFFFFFFFF, p=[float(x) for x in par["p"]], ext_table=table,
            ext_weight=float(par["ext_weight"]), ext_wfx=wfx(par["ext_weight"], sh) if len(table) else 0,
            state=dict(par["state"])))

    cdesc = []
    for s, t, topo, steps, wscalar, warr, mode in cinfo:
        n_tgt = len(pops[t].shape)
        split = None
        if not forms:
            cdesc.append(ConnDesc(src=s, tgt=t, mode=mode, n_links=len(topo), ptr=None, link=None,
                                  weight=wscalar if wscalar is not None else 0.0, w=None, split=None, topo=topo,
                                  steps=steps, warr=warr))
            continue
        if mode == "pull":
            ptr, link, perm, split = pull_split_form(topo, steps, n_tgt)
        elif mode == "push":
            ptr, link, perm, split = push_form(topo, steps, n_tgt)
        else:
            raise ValueError(f"unknown connection mode {mode!r}")
        w = warr[perm].contiguous() if warr is not None else None
        cdesc.append(ConnDesc(src=s, tgt=t, mode=mode, n_links=len(topo), ptr=ptr, link=link,
                              weight=wscalar if wscalar is not None else 0.0, w=w, split=split,
                              topo=topo, steps=steps, warr=warr))
    return NetDesc(dt=dt, pops=pdesc, conns=cdesc, n_links=sum(c.n_links for c in cdesc))


class NetworkRuntime:
    """Device buffers + libnaer2b handle of one network (built by Network.runtime)."""

    def __init__(self, net, modes: dict | None = None):
        self.net = net
        self.device = net.device
        lib = _lib.load()
        self.desc = desc = describe(net, modes)
        self.dt = desc.dt
        pops = self.pops = list(net.populations)
        self.conns = list(net.connections)
        dev = self.device
        self.keep = []  # every device tensor the handle borrows

        def dev_tensor(a):
            t = torch.as_tensor(a).to(dev).contiguous()
            self.keep.append(t)
            return t

        self.cpop = (_lib.Population * max(len(pops), 1))()
        self.words, self.rasters = [], []
        self.record_rows = int(net.record_steps)
        self.rec_step0 = net.step_count
        for k, (p, d) in enumerate(zip(pops, desc.pops)):
            n, words = d.n, (d.n + 31) // 32
            self.words.append(words)
            cp = self.cpop[k]
            cp.model, cp.n, cp.acc_depth, cp.bit_depth = d.model, n, d.acc_depth, d.bit_depth
            cp.shift, cp.ref_steps, cp.fire_threshold = d.shift, d.ref_steps, d.fire_threshold
            cp.ext_len, cp.seed, cp.ext_wfx = len(d.ext_table), d.seed, d.ext_wfx
            for i, x in enumerate(d.p):
                cp.p[i] = x
            for slot, attr in d.state.items():
                tensor = p.state_tensor(attr, dev)
                want = torch.int32 if slot == "ref" else torch.float32
                if tensor.dtype != want:
                    raise TypeError(f"{p!r}.{attr} must be {want} (is {tensor.dtype})")
                if not tensor.is_contiguous():
                    p._state[attr] = tensor = tensor.contiguous()
                setattr(cp, slot, tensor.data_ptr())
            if d.acc_depth:
                cp.acc = dev_tensor(torch.zeros(d.acc_depth * n, dtype=torch.int64)).data_ptr()
            if d.bit_depth:
                cp.bits = dev_tensor(torch.zeros(d.bit_depth * words, dtype=torch.int32)).data_ptr()
            if len(d.ext_table):
                cp.ext_table = dev_tensor(torch.from_numpy(d.ext_table.view(np.int32).copy())).data_ptr()
            raster = None
            if self.record_rows > 0 and n:
                raster = dev_tensor(torch.zeros(self.record_rows * words, dtype=torch.int32))
                cp.raster, cp.raster_steps = raster.data_ptr(), self.record_rows
            self.rasters.append(raster)

        self.cconn = (_lib.Connection * max(len(desc.conns), 1))()
        for k, c in enumerate(desc.conns):
            cc = self.cconn[k]
            cc.src, cc.tgt, cc.n_links = c.src, c.tgt, c.n_links
            cc.mode = _lib.PULL if c.mode == "pull" else _lib.PUSH
            cc.ptr = dev_tensor(c.ptr).data_ptr()
            cc.link = dev_tensor(c.link if c.link.numel() else torch.zeros(1, dtype=torch.int32)).data_ptr()
            cc.weight = c.weight
            cc.w = dev_tensor(c.w).data_ptr() if c.w is not None else None
            cc.split = dev_tensor(c.split).data_ptr() if c.split is not None and c.split.numel() else None
        self.modes = [c.mode for c in desc.conns]
        self.n_links = desc.n_links

        block = net.block or min([p.group_size for p in pops] + [256])
        block = 64 if block <= 64 else 128 if block <= 128 else 256
        self.opt = _lib.Options(block=block, device=dev.index if dev.index is not None else 0, grid=int(net.grid or 0),
                                persistent=int(bool(net.persistent)),
                                barrier_limit_ns=int(getattr(net, "barrier_limit_ns", 0) or 0))
        nbytes = ctypes.c_size_t()
        _lib.check(lib.n2b_workspace_bytes(self.cpop, len(pops), self.cconn, len(desc.conns), ctypes.byref(self.opt),
                                           ctypes.byref(nbytes)), "n2b_workspace_bytes")
        self.workspace = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.Stream(device=dev)
        self._s = ctypes.c_void_p(self.stream.cuda_stream)
        self.handle = ctypes.c_void_p()
        self._enter()  # the state tensors' initial values are in place first
        _lib.check(lib.n2b_create(self.cpop, len(pops), self.cconn, len(desc.conns), ctypes.byref(self.opt),
                                  ctypes.c_void_p(self.workspace.data_ptr()), nbytes.value, self._s,
                                  ctypes.byref(self.handle)), "n2b_create")
        _lib.check(lib.n2b_set_step(self.handle, net.step_count, self._s), "n2b_set_step")
        _lib.check(lib.n2b_record(self.handle, self.rec_step0, self._s), "n2b_record")
        self._leave()
        self.window = 0
        self.launches = 0  # step kernels launched (one fused step each)

    # ------------------------------------------------------------------ stepping

    def _enter(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.device))

    def _leave(self):
        torch.cuda.current_stream(self.device).wait_stream(self.stream)

    def advance(self, n_steps: int) -> None:
        lib = _lib.load()
        window = max(1, int(self.net.window))
        full, rem = divmod(int(n_steps), window)
        self._enter()
        if full:
            if self.window != window:
                _lib.check(lib.n2b_capture(self.handle, window, self._s), "n2b_capture")
                self.window = window
            _lib.check(lib.n2b_replay(self.handle, full, self._s), "n2b_replay")
        if rem:
            _lib.check(lib.n2b_step(self.handle, rem, self._s), "n2b_step")
        self._leave()
        self.launches += n_steps

    def start_recording(self, steps: int) -> None:
        if self.record_rows == 0 or steps > self.record_rows:
            raise RuntimeError("recording needs Network.record(steps) before the first step "
                               f"(this runtime keeps {self.record_rows} rows)")
        self.rec_step0 = self.net.step_count
        self._enter()
        _lib.check(_lib.load().n2b_record(self.handle, self.rec_step0, self._s), "n2b_record")
        self._leave()

    # ------------------------------------------------------------------ results

    def raster_words(self, pop) -> np.ndarray:
        """The recorded rows as uint32 [rows, ceil(n/32)] (rows: the steps made since recording began)."""
        k = self.pops.index(pop)
        words = self.words[k]
        rows = min(self.record_rows, self.net.step_count - self.rec_step0)
        if self.rasters[k] is None or rows <= 0:
            return np.zeros((0, words), dtype=np.uint32)
        self.stream.synchronize()
        return self.rasters[k][: rows * words].cpu().numpy().view(np.uint32).reshape(rows, words)

    def raster(self, pop) -> np.ndarray:
        """The recorded rows as bool [rows, n]."""
        w = self.raster_words(pop)
        n = len(pop.shape)
        bits = np.unpackbits(w.view(np.uint8).reshape(len(w), -1, 4), axis=2, bitorder="little")
        return bits.reshape(len(w), -1)[:, :n].astype(bool)

    def spikes(self, pop):
        steps, ids = np.nonzero(self.raster(pop))
        return steps.astype(np.int64) + self.rec_step0, ids.astype(np.int64)

    def status(self) -> list:
        words = (ctypes.c_int32 * _lib.ERR_WORDS)()
        _lib.check(_lib.load().n2b_status(self.handle, words, _lib.ERR_WORDS, self._s), "n2b_status")
        return list(words)

    def check(self) -> None:
        words = self.status()
        if words[_lib.ERR_PUSH_LINK] or words[_lib.ERR_PULL_LINK]:
            raise RuntimeError(f"links out of range: {words[_lib.ERR_PUSH_LINK]} push, "
                               f"{words[_lib.ERR_PULL_LINK]} pull")
        if words[_lib.ERR_SPLIT] or words[_lib.ERR_ITEMS]:
            raise RuntimeError(f"deferred links dropped: {words[_lib.ERR_SPLIT]} below 2 steps past a row's split, "
                               f"{words[_lib.ERR_ITEMS]} past the work list's capacity")
        if words[_lib.ERR_BARRIER]:
            raise RuntimeError(f"a persistent window stopped: {words[_lib.ERR_BARRIER]} grid barrier wait(s) gave up "
                               "(the run is incomplete; reset_counters clears the stop)")

    def counters(self) -> dict:
        out = (ctypes.c_uint64 * (2 + len(self.pops)))()
        _lib.check(_lib.load().n2b_counters(self.handle, out, len(out), self._s), "n2b_counters")
        return {"events": int(out[0]), "spikes": int(out[1]),
                "per_population": [int(out[2 + k]) for k in range(len(self.pops))]}

    def reset_counters(self) -> None:
        self._enter()
        _lib.check(_lib.load().n2b_reset_counters(self.handle, self._s), "n2b_reset_counters")
        self._leave()

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.stream.synchronize()
            _lib.load().n2b_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
