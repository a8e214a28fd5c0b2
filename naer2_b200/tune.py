"""The autotuner: picks a network's launch configuration by measuring it.

Candidates differ in neurons per block (128 / 256), in how a window is launched (one persistent cooperative
launch, or one launch per step), in the grid (the library's default, or every co-resident block for a
persistent launch: RESIDENT), and in push or pull per connection. The push/pull split comes
from a cost model fitted on a short all-push run: per connection, push moves (spikes of its source per step)
x (its mean row length) link words, scattered into the target's arrival slots, while pull streams every one
of its links every step against the source's spike bits; pull is a candidate for the connections where its
bytes per step are below push's times `pull_factor`. Every candidate runs from the same initial state (the
population tensors are restored after each trial, and every trial builds its runtime anew, its rings empty),
for `steps` steps after `warmup`, timed with CUDA events; the fastest is kept (net.block, net.grid,
net.persistent, net.tuned) and the network is left at its initial state with no runtime.
"""

from __future__ import annotations

import itertools
import time

import torch


def _snapshot(net) -> dict:
    """Every state tensor the kernels use, created now if a trial would otherwise create it (and change it)."""
    from .models import params_of

    snap = {}
    for p in net.populations:
        for attr in params_of(p, net.resolution)["state"].values():
            snap[(id(p), attr)] = p.state_tensor(attr).detach().clone()
    return snap


def _restore(net, snap: dict) -> None:
    for p in net.populations:
        for attr in p.dynamic_attrs:
            t = p._state.get(attr)
            if t is not None and (id(p), attr) in snap:
                t.copy_(snap[(id(p), attr)])


def _trial(net, steps: int, warmup: int) -> tuple[float, dict]:
    net.close()
    net.step_count, net.t = 0, 0.0
    net.run_steps(warmup)
    rt = net.runtime
    c0 = rt.counters()
    s = rt.stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rt._enter()
    e0.record(s)
    net.run_steps(steps)
    e1.record(s)
    e1.synchronize()
    c1 = rt.counters()
    rt.check()
    ms = e0.elapsed_time(e1)
    spikes = [b - a for a, b in zip(c0["per_population"], c1["per_population"])]
    return ms * 1e3 / steps, {"events": c1["events"] - c0["events"], "spikes": spikes}


def pull_candidates(net, spikes_per_step: list, pull_factor: float = 4.0) -> dict:
    """Connection id -> "pull" where streaming all its links (5 B each) costs fewer bytes than push's scatter
    (9 B per event) x factor: a scattered event costs an L2 reduction, several times a streamed byte's share,
    so pull is worth measuring up to a few times push's bytes; the trials decide."""
    index = {id(p): k for k, p in enumerate(net.populations)}
    out = {}
    for c in net.connections:
        topo = c.fabric.topology
        n_src = topo.n_sources
        if n_src == 0 or len(topo) == 0:
            continue
        mean_row = len(topo) / n_src
        push_bytes = spikes_per_step[index[id(c._source)]] * mean_row * 9.0
        pull_bytes = len(topo) * 5.0 + n_src / 8.0
        if pull_bytes < push_bytes * pull_factor:
            out[id(c)] = "pull"
    return out


RESIDENT = 1 << 16  # a persistent launch's grid is capped at the co-resident blocks: this asks for all of them


def autotune(net, steps: int = 300, warmup: int = 100, blocks=(128, 256), persistent=(True, False),
             grids=(None, RESIDENT), pull_factor: float = 4.0, verbose: bool = False) -> dict:
    """Measure the candidates, keep the fastest; returns the report (every trial's us per step)."""
    if net.device is None or net.device.type != "cuda":
        raise RuntimeError("autotune needs the network on a CUDA device")
    snap = _snapshot(net)
    saved = (net.block, net.grid, net.persistent, dict(net.tuned), net.window, net.record_steps)
    net.record_steps = 0
    net.window = max(net.window, steps)
    report = {"trials": []}
    try:
        # the all-push baseline first: it also measures the rates the cost model needs
        net.tuned = {}
        net.block, net.grid, net.persistent = 256, None, True
        us, stats = _trial(net, steps, warmup)
        _restore(net, snap)
        spikes_per_step = [s / steps for s in stats["spikes"]]
        pulls = pull_candidates(net, spikes_per_step, pull_factor)
        report["trials"].append({"block": 256, "grid": None, "persistent": True, "pull": 0, "us_per_step": us})
        mode_sets = [{}] + ([pulls] if pulls else [])
        best = (us, 256, None, True, {})
        t0 = time.perf_counter()
        # pull sets also try 64-neuron tiles: a pulled row is walked by its tile's warps, so smaller tiles spread
        # the pulls over more SMs
        cands = [(b, g, p, m) for m in mode_sets for b in (tuple(blocks) + ((64,) if m and 64 not in blocks else ()))
                 for g in grids for p in persistent if p or g != RESIDENT]  # (per-step launches: not RESIDENT)
        for block, grid, pers, modes in cands:
            if (block, grid, pers, len(modes)) == (256, None, True, 0):
                continue
            net.block, net.grid, net.persistent, net.tuned = block, grid, pers, dict(modes)
            try:
                us, _ = _trial(net, steps, warmup)
            finally:
                _restore(net, snap)
            report["trials"].append({"block": block, "grid": grid, "persistent": pers, "pull": len(modes),
                                     "us_per_step": us})
            if verbose:
                print(report["trials"][-1], flush=True)
            if us < best[0]:
                best = (us, block, grid, pers, dict(modes))
        report["seconds"] = time.perf_counter() - t0
    except BaseException:
        net.block, net.grid, net.persistent, net.tuned, net.window, net.record_steps = saved
        raise
    finally:
        net.close()
        net.step_count, net.t = 0, 0.0
        _restore(net, snap)
    us, block, grid, pers, modes = best
    net.block, net.grid, net.persistent, net.tuned = block, grid, pers, modes
    net.window, net.record_steps = saved[4], saved[5]
    report["chosen"] = {"block": block, "grid": grid, "persistent": pers, "pull": len(modes), "us_per_step": us}
    net.tune_report = report
    return report
