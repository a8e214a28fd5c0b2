"""CPU oracle of the fixed-dt hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, and only as the checker (or the timed CPU baseline):
the product (naer2_b200) never imports, links or runs it.

A ctypes front end of oracle/liboracle.so (oracle.c: a sequential C
restatement of the reference's time-driven LIF loop and PD14 neuron hooks,
with Philox4x32-10 and the shared Poisson tables). `run` takes a network
description -- naer2_b200.runtime.describe(net), or one built by hand -- and
per-population initial state, and returns the state, spike rasters and
synaptic events after n steps.
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OrPop(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32), ("n", ctypes.c_int32), ("acc_depth", ctypes.c_int32), ("shift", ctypes.c_int32),
        ("ref_steps", ctypes.c_int32), ("fire_threshold", ctypes.c_uint32), ("seed", ctypes.c_uint64),
        ("p", ctypes.c_float * 8), ("ext_wfx", ctypes.c_int64), ("ext_table", ctypes.c_void_p),
        ("ext_len", ctypes.c_int32), ("ext_counts", ctypes.c_void_p), ("ext_step0", ctypes.c_int64),
        ("ext_steps", ctypes.c_int64), ("v", ctypes.c_void_p), ("i", ctypes.c_void_p), ("ref", ctypes.c_void_p),
        ("acc", ctypes.c_void_p), ("raster", ctypes.c_void_p), ("raster_step0", ctypes.c_int64),
        ("raster_steps", ctypes.c_int64),
    ]


class OrConn(ctypes.Structure):
    _fields_ = [("src", ctypes.c_int32), ("tgt", ctypes.c_int32), ("ptr", ctypes.c_void_p), ("link", ctypes.c_void_p),
                ("w", ctypes.c_void_p), ("weight", ctypes.c_float)]


_lib = None


def build() -> pathlib.Path:
    """Compile liboracle.so (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.or_philox4x32_10.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3
        lib.or_philox4x32_10.restype = None
        lib.or_wfx.argtypes = [ctypes.c_float, ctypes.c_int32]
        lib.or_wfx.restype = ctypes.c_int64
        lib.or_run.argtypes = [ctypes.POINTER(OrPop), ctypes.c_int32, ctypes.POINTER(OrConn), ctypes.c_int32,
                               ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]
        lib.or_run.restype = ctypes.c_int
        lib.or_poisson_counts.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int64,
                                          ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p]
        lib.or_poisson_counts.restype = None
        lib.or_set_threads.argtypes = [ctypes.c_int]
        lib.or_set_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def philox(counter, key) -> list:
    """Philox4x32-10 of a 4-word counter under a 2-word key."""
    c = (ctypes.c_uint32 * 4)(*[int(x) & 0xFFFFFFFF for x in counter])
    k = (ctypes.c_uint32 * 2)(*[int(x) & 0xFFFFFFFF for x in key])
    out = (ctypes.c_uint32 * 4)()
    load().or_philox4x32_10(c, k, out)
    return list(out)


def poisson_counts(table: np.ndarray, seed: int, step0: int, n_steps: int, n: int) -> np.ndarray:
    """int32 [n_steps, n]: the external counts a population keyed `seed` draws."""
    table = np.ascontiguousarray(table, dtype=np.uint32)
    out = np.zeros((n_steps, n), dtype=np.int32)
    load().or_poisson_counts(_ptr(table), len(table), int(seed) & 0xFFFFFFFFFFFFFFFF, step0, n_steps, n, _ptr(out))
    return out


def set_threads(n: int) -> int:
    """Threads of run(): 1 the sequential restatement, 0 every host thread (same results)."""
    return int(load().or_set_threads(int(n)))


def wfx(w: float, shift: int) -> int:
    return int(load().or_wfx(float(np.float32(w)), int(shift)))


class State:
    """A population's state as numpy arrays: v, i (fp32), ref (int32), acc (int64 [depth * n])."""

    def __init__(self, n: int, acc_depth: int, v=None, i=None, ref=None):
        self.v = np.ascontiguousarray(v if v is not None else np.zeros(n), dtype=np.float32).copy()
        self.i = np.ascontiguousarray(i if i is not None else np.zeros(n), dtype=np.float32).copy()
        self.ref = np.ascontiguousarray(ref if ref is not None else np.zeros(n), dtype=np.int32).copy()
        self.acc = np.zeros(max(acc_depth, 1) * n, dtype=np.int64)


def _ptr(a):
    return a.ctypes.data if a is not None else None


class Prepared:
    """A description with its connections' canonical rows converted to host arrays once (for networks whose
    rows are large, run in many chunks): pass it to run() in place of the description."""

    def __init__(self, desc):
        self.dt, self.pops = desc.dt, desc.pops
        self.rows = []
        for c in desc.conns:
            ptr, link, w = c.canonical()
            self.rows.append((c.src, c.tgt, c.weight, np.ascontiguousarray(ptr, dtype=np.int32),
                              np.ascontiguousarray(link, dtype=np.uint32),
                              None if w is None else np.ascontiguousarray(w, dtype=np.float32)))


def prepare(desc) -> Prepared:
    return Prepared(desc)


def run(desc, states: list, step0: int, n_steps: int, record: bool = True, ext_counts: dict | None = None,
        packed: bool = False):
    """Run the description's network (or a Prepared one) from step0 for n_steps in place on `states` (one State
    per population). Returns (rasters: list of bool [n_steps, n] -- packed: uint32 words [n_steps, ceil(n/32)],
    bit j of word w neuron 32 w + j -- or None, events). ext_counts: population index -> int32 [n_steps, n]
    external counts to use instead of the Philox draws."""
    lib = load()
    pops = (OrPop * max(len(desc.pops), 1))()
    keep = []
    rasters = []
    for k, (d, st) in enumerate(zip(desc.pops, states)):
        op = pops[k]
        op.model, op.n, op.acc_depth, op.shift = d.model, d.n, max(d.acc_depth, 1), d.shift
        op.ref_steps, op.fire_threshold, op.seed = d.ref_steps, d.fire_threshold, d.seed
        for i, x in enumerate(d.p):
            op.p[i] = x
        op.ext_wfx = d.ext_wfx
        table = np.ascontiguousarray(d.ext_table, dtype=np.uint32)
        keep.append(table)
        op.ext_table, op.ext_len = (_ptr(table), len(table)) if len(table) else (None, 0)
        if ext_counts is not None and k in ext_counts:
            cnt = np.ascontiguousarray(ext_counts[k], dtype=np.int32)
            keep.append(cnt)
            op.ext_counts, op.ext_step0, op.ext_steps = _ptr(cnt), step0, cnt.shape[0]
        op.v, op.i, op.ref = _ptr(st.v), _ptr(st.i), _ptr(st.ref)
        op.acc = _ptr(st.acc)
        words = (d.n + 31) // 32
        if record:
            r = np.zeros(n_steps * words, dtype=np.uint32)
            keep.append(r)
            op.raster, op.raster_step0, op.raster_steps = _ptr(r), step0, n_steps
            rasters.append((r, words))
        else:
            rasters.append(None)
    if isinstance(desc, Prepared):
        rows = desc.rows
    else:  # rows per source, canonical order
        rows = []
        for c in desc.conns:
            ptr, link, w = c.canonical()
            rows.append((c.src, c.tgt, c.weight, np.ascontiguousarray(ptr, dtype=np.int32),
                         np.ascontiguousarray(link, dtype=np.uint32),
                         None if w is None else np.ascontiguousarray(w, dtype=np.float32)))
    conns = (OrConn * max(len(rows), 1))()
    for k, (src, tgt, weight, ptr, link, w) in enumerate(rows):
        oc = conns[k]
        keep += [ptr, link]
        oc.src, oc.tgt, oc.ptr, oc.link = src, tgt, _ptr(ptr), _ptr(link)
        if w is not None:
            keep.append(w)
            oc.w = _ptr(w)
        oc.weight = weight
    events = ctypes.c_uint64(0)
    rc = lib.or_run(pops, len(desc.pops), conns, len(rows), step0, n_steps, ctypes.byref(events))
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
    out = []
    for d, rr in zip(desc.pops, rasters):
        if rr is None:
            out.append(None)
            continue
        r, words = rr
        if packed:
            out.append(r.reshape(n_steps, words))
            continue
        bits = np.unpackbits(r.view(np.uint8).reshape(n_steps, words, 4), axis=2, bitorder="little")
        out.append(bits.reshape(n_steps, words * 32)[:, :d.n].astype(bool))
    return out, int(events.value)


def states_of(net, desc) -> list:
    """Initial oracle states from a naer2_b200 network's population tensors (copied to the host)."""
    out = []
    for p, d in zip(net.populations, desc.pops):
        kw = {slot: p.state_tensor(attr).detach().cpu().numpy() for slot, attr in d.state.items()}
        out.append(State(d.n, d.acc_depth, **kw))
    return out
