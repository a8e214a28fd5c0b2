"""Benchmark: synaptic events/s of the fixed-dt hot path on one B200, headline workload the PD14 cortical
microcircuit at full size (77,169 neurons, ~3e8 synapses, per-link normal delays, dt 0.1 ms).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl naer2_b200|reference] [--config 1|2|3|4]

One bench step = 1,000 simulation steps (100 ms of network time) stepped by the persistent step kernel (one
cooperative launch per window of --window steps, replayed from a CUDA graph). Printed: one JSON line (rank 0).
  value     events delivered in the timed steps / device time (CUDA events on the runtime's stream, L2 flushed
            before every timed step), summed over ranks, time the max over ranks
  e2e       the same metric through the public API with host buffers: every step copies the network state in
            from pinned host memory, runs Network.step, and reads the spike raster and state back
  roofline  the step kernel's algorithmic bytes (9 B per synaptic event + 32 B per PD14 neuron per simulation
            step) per launch over its average launch time, against the measured HBM copy bandwidth; traffic:
            the DRAM bytes of one launch of the same window from the committed ncu capture
  cpu_baseline  the oracle (a C restatement of the reference's time-driven loop, all host threads) on a bounded
            sample of the same network
  workloads  at N=1 the other workloads, each measured the same way: Brunel's network at config 1's size,
            the 64 batched uneven instances against the same instances one network at a time (autotuned),
            and BPTT's training step against the plain forward
--impl reference times the CPU implementation (the oracle port, all host threads) on the same workload and the
same window of simulation steps (rank 0; other ranks exit). --config 1|3|4 prints one of the other workloads
as the line instead. Multi-GPU: independent replicas (one network per rank, its own seed).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import pathlib
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SIM_STEPS_PER_STEP = 1000
BYTES_PER_EVENT = 9  # int32 target + int8 delay + fp32 weight
NEURON_BYTES = {"brunel": 16, "pd14": 32}  # per neuron and step: V (and I, refractory) read + write, slot read + clear
METRIC = "synaptic events/s"
UNIT = "events/s"
KERNEL = "n2b::persistent_kernel<256>"


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


_RED_PEAK = {}


def l2_atomic_peak(dev) -> dict | None:
    """Reductions/s of the L2 atomic units for the delivery's own instruction (red.global.add.u64 at random
    slots of a 64 MiB array that stays in L2), measured here by naer2_b200/libn2b_peak.so: the best of 5 runs of
    148 x 8 blocks x 256 threads x 256 reductions. Measured once per process."""
    import ctypes

    import torch

    key = dev.index or 0
    if key in _RED_PEAK:
        return _RED_PEAK[key]
    path = ROOT / "naer2_b200" / "libn2b_peak.so"
    if not path.exists():
        return None
    lib = ctypes.CDLL(str(path))
    lib.n2b_red_peak.restype = ctypes.c_int
    lib.n2b_red_peak.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                 ctypes.c_void_p]
    n_slots = 1 << 23
    slots = torch.zeros(n_slots, dtype=torch.int64, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    grid, block, ops = sms * 8, 256, 256
    stream = torch.cuda.current_stream(dev)
    best = None
    for k in range(7):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if lib.n2b_red_peak(ctypes.c_void_p(slots.data_ptr()), n_slots, grid, block, ops,
                            ctypes.c_void_p(stream.cuda_stream)) != 0:
            return None
        e1.record(stream)
        e1.synchronize()
        if k >= 2:
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
    total = grid * block * ops
    assert int(slots.sum()) == 7 * total  # every reduction landed
    _RED_PEAK[key] = {"peak": total / (best / 1e3), "unit": "reductions/s",
                      "probe": f"red.global.add.u64, {grid}x{block} threads x {ops}, 64 MiB L2-resident array"}
    return _RED_PEAK[key]


def l2_atomics(events_per_s: float, dev) -> dict | None:
    """The step kernel's reduction rate (one red.global.add.u64 per synaptic event) against the measured peak."""
    pk = l2_atomic_peak(dev)
    if pk is None:
        return None
    return {"achieved": events_per_s, "peak": pk["peak"], "unit": pk["unit"], "frac": events_per_s / pk["peak"],
            "peak_probe": pk["probe"]}


class Clocks:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)  # the first sample lands inside the timed region
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def reduce_over_ranks(times, counts, world: int, device):
    """Times: the max over ranks; counts: the sum (the whole job's work). One collective each, every rank."""
    import torch

    if world <= 1:
        return [*map(float, times), *map(float, counts)]
    import torch.distributed as dist

    t = torch.tensor([float(x) for x in times], dtype=torch.float64, device=device)
    c = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [*t.tolist(), *c.tolist()]


# ---------------------------------------------------------------------------------------------------- workloads

SCALE = 1.0  # PD14's population sizes times this (--scale: smaller cases for profiling)


def build_workload(name: str, seed: int, device=None):
    """(network, populations list, neuron bytes per step, config dict) of a plain workload."""
    if name == "pd14_config2":
        from naer2_b200.networks import pd14

        net, pops = pd14.build(scale=SCALE, seed=seed, device=device)
        cfg = {"workload": name, "neurons": sum(len(p.shape) for p in pops), "populations": 8,
               "synapses_expected": pd14.expected_synapses(SCALE), "delays": "normal per link, >= dt, in steps",
               "dt_ms": 0.1, **({"scale": SCALE} if SCALE != 1.0 else {})}
        return net, pops, NEURON_BYTES["pd14"], cfg
    if name == "brunel_A_config1":
        from naer2_b200.networks import brunel

        net, pops = brunel.build(**brunel.CONFIG1, seed=seed, device=device)
        cfg = {"workload": name, "neurons": 12500, "synapses": 15_625_000, "delays_steps": "U{1..20}", "dt_ms": 0.1}
        return net, list(pops.values()), NEURON_BYTES["brunel"], cfg
    raise ValueError(name)


def workload_profile(name: str) -> dict | None:
    """The committed ncu capture of the workload's step kernel (DRAM bytes of one launch), if any."""
    p = ROOT / "profiles" / f"persistent_kernel_{name}.json"
    return json.loads(p.read_text()) if p.exists() else None


def state_tensors(net):
    """(population, attribute) of every state tensor the kernels step."""
    from naer2_b200.models import params_of

    out = []
    for p in net.populations:
        for attr in params_of(p, net.resolution)["state"].values():
            out.append((p, attr))
    return out


def measure(net, args, dev, world: int, sim: int, clocks: bool = True) -> dict:
    """Warm-up, the timed region (device time of K bench steps, L2 flushed before each) and the end-to-end pass
    through the public API with host buffers. Per rank; the caller reduces over ranks."""
    import torch
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    net.window = sim  # one persistent launch per bench step
    net.record(sim)
    rt = net.runtime
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        net.run_steps(sim)
    barrier()
    ev0 = rt.counters()["events"]
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clk = Clocks(dev.index or 0) if clocks else None
    if clk:
        clk.__enter__()
    try:
        barrier()
        for k in range(args.steps):
            flush.zero_()
            rt._enter()  # the runtime's stream after the flush
            starts[k].record(rt.stream)
            net.run_steps(sim)
            ends[k].record(rt.stream)
        barrier()
    finally:
        if clk:
            clk.__exit__(None, None, None)
    per_launch_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    dev_ms = sum(per_launch_ms)
    events = rt.counters()["events"] - ev0
    net.check()

    # end to end through the public API, host buffers
    hosts = []
    for p, attr in state_tensors(net):
        t = p.state_tensor(attr)
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t)
        hosts.append((p, attr, h))
    raster_host = [torch.empty(r.shape, dtype=r.dtype, pin_memory=True) for r in rt.rasters if r is not None]
    h2d = sum(h.numel() * h.element_size() for _, _, h in hosts)
    d2h = h2d + sum(r.numel() * r.element_size() for r in raster_host)
    barrier()
    ev1 = rt.counters()["events"]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for p, attr, h in hosts:  # inputs: the network state, from pinned host memory
            p.state_tensor(attr).copy_(h, non_blocking=True)
        net.record(sim)
        net.step(sim * net.resolution)
        for r, h in zip([r for r in rt.rasters if r is not None], raster_host):  # results: raster and state
            h.copy_(r, non_blocking=True)
        for p, attr, h in hosts:
            h.copy_(p.state_tensor(attr), non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_events = rt.counters()["events"] - ev1
    net.check()
    windows = args.steps * math.ceil(sim / max(net.window, 1))
    return {"dev_ms": dev_ms, "events": events, "e2e_s": e2e_s, "e2e_events": e2e_events, "h2d": h2d, "d2h": d2h,
            "clocks": clk.summary() if clk else None, "launches": 2 * windows, "windows": windows,
            "per_launch_ms": per_launch_ms, "n_links": rt.n_links, "grid": rt.opt.grid}


def roofline(events: float, steps: int, neurons: int, neuron_bytes: int, dev_ms: float, windows: int,
             profile: dict | None) -> dict:
    """Algorithmic bytes per launch (one window of simulation steps) over the average launch time."""
    ev_step = events / steps
    per_step = ev_step * BYTES_PER_EVENT + neurons * neuron_bytes
    steps_per_launch = steps / windows
    launch_bytes = per_step * steps_per_launch
    launch_s = dev_ms / 1e3 / windows
    achieved = launch_bytes / launch_s / 1e9
    peak, kind = measured_peaks()
    traffic = None
    if profile is not None and profile.get("steps_per_launch"):
        traffic = profile["dram_bytes_per_launch"] * steps_per_launch / profile["steps_per_launch"]
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": kind, "kernel": KERNEL, "bytes_per_launch": launch_bytes,
            "us_per_launch": launch_s * 1e6, "steps_per_launch": steps_per_launch,
            "us_per_sim_step": launch_s * 1e6 / steps_per_launch,
            "per_unit": f"{BYTES_PER_EVENT} B per synaptic event + {neuron_bytes} B per neuron per step",
            "traffic_source": profile.get("source") if profile else None}


def cpu_sample(prepared, states, dt: float, name: str, target_s: float = 12.0) -> dict:
    """The oracle on all host cores: a bounded sample of the same network, from its initial state."""
    import oracle

    used = oracle.set_threads(0)
    probe = 20
    t0 = time.perf_counter()
    _, ev = oracle.run(prepared, states, 0, probe, record=False)
    t_probe = time.perf_counter() - t0
    steps = max(20, min(400_000, int(probe * target_s / max(t_probe, 1e-3))))
    t0 = time.perf_counter()
    _, ev2 = oracle.run(prepared, states, probe, steps, record=False)
    el = time.perf_counter() - t0
    return {"value": ev2 / el, "unit": UNIT, "cores": used, "kind": "port",
            "sample": f"{name}: simulation steps {probe}-{probe + steps} ({steps * dt:.0f} ms of network time, "
                      f"{ev2} events) in {el:.1f} s, C oracle, {used} OpenMP threads, nproc {os.cpu_count()}",
            "realtime_factor": el / (steps * dt * 1e-3)}


def line_of(name: str, m: dict, args, world: int, sim: int, neurons: int, neuron_bytes: int, cfg: dict,
            dev=None) -> dict:
    steps = args.steps * sim
    value = m["events"] / (m["dev_ms"] / 1e3)
    rl = roofline(m["events_rank0"], steps, neurons, neuron_bytes, m["dev_ms_rank0"], m["windows"],
                  workload_profile(name))
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": m["dev_ms"] / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded draws: connectivity, weights, delays, initial state, Philox Poisson drive)",
           "config": {**cfg, "sim_steps_per_step": sim, "window_steps": sim,
                      "l2": "flushed before every timed step (256 MiB write)",
                      "parallelism": f"replicas x{world}" if world > 1 else "single GPU", "launch": "persistent"},
           "realtime_factor": (m["dev_ms"] / 1e3) / (steps * 1e-4),
           "e2e": {"value": m["e2e_events"] / m["e2e_s"], "unit": UNIT, "h2d_bytes_per_step": m["h2d"],
                   "d2h_bytes_per_step": m["d2h"]},
           "roofline": rl,
           "gpu_launches": m["launches"],
           "clocks": m["clocks"],
           "events_per_sim_step": m["events_rank0"] / steps,
           "synapses": m["n_links"], "grid": m["grid"]}
    if dev is not None:
        out["l2_atomics"] = l2_atomics(m["events_rank0"] / (m["dev_ms_rank0"] / 1e3), dev)
    return out


def run_plain(name: str, args, dev, rank: int, world: int, cpu: bool) -> dict:
    """A plain workload (PD14 or config 1) on every rank, reduced over ranks; rank 0 gets the line."""
    import torch

    from naer2_b200.runtime import describe
    from naer2_b200.stats import SpikeStats

    sim = SIM_STEPS_PER_STEP
    t0 = time.perf_counter()
    net, pops, nb, cfg = build_workload(name, 1 + rank, device=dev)
    neurons = sum(len(p.shape) for p in pops)
    prepared = states = None
    if cpu and rank == 0 and world == 1:
        import oracle

        desc = describe(net, forms=False)
        states = oracle.states_of(net, desc)
        prepared = oracle.prepare(desc)
        del desc
    build_s = time.perf_counter() - t0
    m = measure(net, args, dev, world, sim)
    stats = [SpikeStats(len(p.shape), net.resolution, t_skip_ms=0.0) for p in pops]
    for p, s in zip(pops, stats):  # the last end-to-end step's raster
        s.add_words(net.runtime.raster_words(p), 0)
    m["dev_ms_rank0"], m["events_rank0"] = m["dev_ms"], m["events"]
    m["dev_ms"], m["e2e_s"], m["events"], m["e2e_events"] = reduce_over_ranks(
        [m["dev_ms"], m["e2e_s"]], [m["events"], m["e2e_events"]], world, dev)
    line = line_of(name, m, args, world, sim, neurons, nb, cfg, dev)
    if name == "pd14_config2":
        from naer2_b200.networks import pd14

        names = pd14.NAMES
    else:
        names = ["E", "I"]
    line["rates_hz_last_step"] = {k: round(s.rate_hz(), 3) for k, s in zip(names, stats)}
    line["cv_isi_last_step"] = {k: round(s.cv_isi(), 3) for k, s in zip(names, stats)}
    line["build_s"] = build_s
    net.close()
    del net
    torch.cuda.empty_cache()
    if prepared is not None:
        line["cpu_baseline"] = cpu_sample(prepared, states, 0.1, name)
    return line


def run_batched(args, dev) -> dict:
    """Config 3: B uneven Brunel instances in one network (one persistent launch per window), tuned by the
    autotuner, against the same instances stepped one network at a time on the same GPU, each tuned by the
    same autotuner over the same candidates (same seeds: the same spikes). Aggregate synaptic events/s of both,
    and per-instance rates."""
    import torch

    from naer2_b200.networks import batched
    from naer2_b200.tune import autotune

    B = args.instances
    sim = SIM_STEPS_PER_STEP

    def timed(net, n_steps):
        rt = net.runtime
        c0 = rt.counters()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        rt._enter()
        e0.record(rt.stream)
        net.run_steps(n_steps)
        e1.record(rt.stream)
        e1.synchronize()
        c1 = rt.counters()
        net.check()
        return e0.elapsed_time(e1), c1["events"] - c0["events"], [b - a for a, b in zip(c0["per_population"],
                                                                                      c1["per_population"])]

    t0 = time.perf_counter()
    net, parts = batched.build(B, seed=1, device=dev)
    build_s = time.perf_counter() - t0
    report = autotune(net, steps=200, warmup=50) if args.tune else None
    net.window = sim
    net.run_steps(args.warmup * sim)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ms_b, ev_b, spk_b = 0.0, 0, None
    for _ in range(args.steps):
        flush.zero_()
        ms, ev, spk = timed(net, sim)
        ms_b, ev_b = ms_b + ms, ev_b + ev
        spk_b = spk if spk_b is None else [x + y for x, y in zip(spk_b, spk)]
    n_links = net.runtime.n_links
    neurons = sum(len(p.shape) for p in net.populations)
    chosen = dict(block=net.block, grid=net.grid, persistent=net.persistent, pull=len(net.tuned))
    net.close()
    del net, parts
    torch.cuda.empty_cache()
    # the same instances, one network at a time, each tuned the same way
    ms_p, ev_p, spk_p, plain_choice = 0.0, 0, [], []
    for b in range(B):
        inst, _ = batched.build_instance(b, seed=1, device=dev)
        if args.tune:
            r = autotune(inst, steps=200, warmup=50)
            plain_choice.append(r["chosen"])
        inst.window = sim
        inst.run_steps(args.warmup * sim)
        for _ in range(args.steps):
            flush.zero_()
            ms, ev, spk = timed(inst, sim)
            ms_p, ev_p = ms_p + ms, ev_p + ev
            if len(spk_p) < 2 * (b + 1):
                spk_p += spk
            else:
                spk_p[-2:] = [x + y for x, y in zip(spk_p[-2:], spk)]
        inst.close()
    steps = args.steps * sim
    rates_b, rates_p = [], []
    for b in range(B):
        n_e = batched.instance_params(b, 1)["NE"]
        n_i = batched.instance_params(b, 1)["NI"]
        rates_b.append([spk_b[2 * b] / n_e / (steps * 1e-4), spk_b[2 * b + 1] / n_i / (steps * 1e-4)])
        rates_p.append([spk_p[2 * b] / n_e / (steps * 1e-4), spk_p[2 * b + 1] / n_i / (steps * 1e-4)])
    value = ev_b / (ms_b / 1e3)
    plain = ev_p / (ms_p / 1e3)
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_b / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded draws on the GPU, 64 uneven Brunel instances)",
            "config": {"workload": "batched_config3", "instances": B, "neurons": neurons, "synapses": n_links,
                       "dt_ms": 0.1, "sim_steps_per_step": sim, "tuned": chosen,
                       "l2": "flushed before every timed step (256 MiB write)"},
            "l2_atomics": l2_atomics(value, dev),
            "plain_one_at_a_time": {"value": plain, "ms_per_step": ms_p / args.steps,
                                    "tuned": _summarise_choices(plain_choice)},
            "batched_over_plain": value / plain,
            "identical_spike_counts": spk_b == spk_p,
            "rates_hz_first4": [[round(x, 2) for x in r] for r in rates_b[:4]],
            "max_rate_difference_hz": max(abs(x - y) for rb, rp in zip(rates_b, rates_p) for x, y in zip(rb, rp)),
            "tune_trials": report["trials"] if report else None, "build_s": build_s}


def run_driven(args, dev) -> dict:
    """A densely driven LIF population (naer2_b200.networks.driven: 2,000 Poisson inputs at 5 spikes/ms, 5M input
    links into 10,000 neurons, a sparse recurrent part): events/s with the input connections pulled (the staged
    pull), with every connection pushed, and the autotuner's measured choice (unless --no-tune)."""
    import torch

    from naer2_b200.networks import driven
    from naer2_b200.tune import autotune

    sim = SIM_STEPS_PER_STEP
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(arm: str):
        net, pops = driven.build(**driven.CONFIG, seed=1, device=dev)
        chosen = None
        if arm == "tuned":
            chosen = autotune(net, steps=200, warmup=50)["chosen"]
        elif arm == "pull":
            net.tuned = {id(c): "pull" for c in net.connections if c._source is pops["in"]}
        net.window = sim
        net.run_steps(args.warmup * sim)
        rt = net.runtime
        ev0 = rt.counters()["events"]
        ms = 0.0
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            rt._enter()
            e0.record(rt.stream)
            net.run_steps(sim)
            e1.record(rt.stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        events = rt.counters()["events"] - ev0
        spikes = rt.counters()["per_population"]
        net.check()
        out = {"value": events / (ms / 1e3), "us_per_sim_step": ms * 1e3 / (args.steps * sim),
               "modes": list(rt.modes), "events_per_sim_step": events / (args.steps * sim),
               "block": rt.opt.block, "persistent": bool(rt.opt.persistent), "tuned": chosen,
               "pull_staged_error_words": rt.status()[5], "spikes": spikes}
        net.close()
        torch.cuda.empty_cache()
        return out

    arms = {a: timed(a) for a in (("pull", "push", "tuned") if args.tune else ("pull", "push"))}
    best = arms.get("tuned", max(arms.values(), key=lambda r: r["value"]))
    return {"metric": METRIC, "value": best["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded draws on the GPU)",
            "config": {"workload": "driven_dense_input", **driven.CONFIG, "sim_steps_per_step": sim,
                       "l2": "flushed before every timed step (256 MiB write)"},
            "arms": arms, "pull_over_push": arms["pull"]["value"] / arms["push"]["value"],
            "identical_spike_counts": arms["pull"]["spikes"] == arms["push"]["spikes"]}


def _summarise_choices(choices: list) -> dict | None:
    if not choices:
        return None
    out = {}
    for c in choices:
        grid = "default grid" if not c.get("grid") else "every co-resident block" if c["grid"] >= 1 << 16 else f"grid {c['grid']}"
        key = f"block {c['block']}, {'persistent' if c['persistent'] else 'per-step'}, {grid}, pull {c['pull']}"
        out[key] = out.get(key, 0) + 1
    return out


def run_bptt(args, dev) -> dict:
    """Config 4: surrogate-gradient BPTT of the recurrent LIF layer (B 128, T 500, 700 channels, 1024 hidden at
    10% density, delays 1-5 steps, 20 readouts, checkpoints every 50 steps). One bench step: the plain forward
    (input current + forward kernel, no tape), then one training step (taped forward + loss + backward through
    the adjoint kernels and the input projection's gradient), each timed with CUDA events after an L2 flush."""
    import torch

    from naer2_b200.bptt import SpikeEvents
    from naer2_b200.networks import bptt_task

    t0 = time.perf_counter()
    layer, x, y = bptt_task.build(seed=1, device=dev)
    T, B, C = x.shape
    xs = SpikeEvents.from_dense(x)  # the input as spike event lists, built once like a loader's output
    build_s = time.perf_counter() - t0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def train_step():
        layer.zero_grad(set_to_none=True)
        m = layer(xs, steps=T)
        loss = torch.nn.functional.cross_entropy(m, y)
        loss.backward()
        return loss

    U = layer.current(xs, steps=T).detach().contiguous()
    with torch.no_grad():
        m0, ts0 = layer.run_forward(U, tape=True)
        dm0 = torch.softmax(m0, 1) - torch.nn.functional.one_hot(y, m0.shape[1]).float()
    for _ in range(args.warmup):
        layer.infer(xs, steps=T)
        train_step()
    plain, train, fk, fk_tape, bk = [], [], [], [], []
    with Clocks(dev.index or 0) as clocks:
        for _ in range(args.steps):
            plain.append(timed(lambda: layer.infer(xs, steps=T))[0])
            train.append(timed(train_step)[0])
            fk.append(timed(lambda: layer.run_forward(U, tape=False))[0])
            fk_tape.append(timed(lambda: layer.run_forward(U, tape=True))[0])
            bk.append(timed(lambda: layer.run_backward(U, dm0, ts0))[0])
    assert layer.status(B, T) == [0, 0, 0, 0]
    with torch.no_grad():
        layer.run_forward(U, tape=True)
        spikes = layer.spikes(B, T)
        events = float((spikes.float().sum((0, 1)) * layer.wiring.out_degree.float()).sum())
    ms_plain, ms_train = sum(plain) / len(plain), sum(train) / len(train)
    ms_fk, ms_fkt, ms_bk = (sum(v) / len(v) for v in (fk, fk_tape, bk))
    return {"metric": METRIC, "value": events / (ms_plain / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_plain + ms_train, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Poisson class templates, 20 classes)",
            "config": {"workload": "bptt_config4", "batch": B, "steps_T": T, "channels": C, "hidden": layer.hidden,
                       "readouts": layer.readouts, "recurrent_links": layer.wiring.nnz, "checkpoint": layer.checkpoint,
                       "l2": "flushed before every timed call (256 MiB write)"},
            "plain_forward_ms": ms_plain, "train_step_ms": ms_train,
            "bptt_over_plain_forward": ms_train / ms_plain,
            "kernels_ms": {"forward_plain": ms_fk, "forward_taped": ms_fkt, "backward": ms_bk},
            "kernel_bptt_over_forward": (ms_fkt + ms_bk) / ms_fk,
            "recurrent_events_per_forward": events, "spike_rate": float(spikes.float().mean()),
            "realtime_factor": (ms_plain / 1e3) / (T * 1e-3), "build_s": build_s, "clocks": clocks.summary()}


def run_transpiled(args, dev) -> dict:
    """Config 1's network with TranspiledLIF neurons (the built-in LIF's dynamics, its Poisson drive drawn in its
    own hook): the run-time compiled step kernels, events/s over the timed steps."""
    import torch

    from naer2_b200.networks import brunel

    t0 = time.perf_counter()
    net, pops = brunel.build(**brunel.CONFIG1, seed=1, device=dev, transpiled=True)
    net.run_steps(1)  # builds the runtime: transpiles and compiles the hooks
    rt = net.runtime
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        net.run_steps(SIM_STEPS_PER_STEP)
    torch.cuda.synchronize(dev)
    ev0, l0 = rt.counters()["events"], rt.launches
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with Clocks(dev.index or 0) as clocks:
        for k in range(args.steps):
            flush.zero_()
            rt.stream.wait_stream(torch.cuda.current_stream(dev))
            starts[k].record(rt.stream)
            net.run_steps(SIM_STEPS_PER_STEP)
            ends[k].record(rt.stream)
        torch.cuda.synchronize(dev)
    dev_ms = sum(st.elapsed_time(e) for st, e in zip(starts, ends))
    events = rt.counters()["events"] - ev0
    net.check()
    return {"metric": METRIC, "value": events / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded draws on the GPU, Brunel model A at config 1's size)",
            "config": {"workload": "brunel_config1_transpiled", "neurons": sum(len(p.shape) for p in pops.values()),
                       "sim_steps_per_step": SIM_STEPS_PER_STEP, "launch": "one per population and step, from the host",
                       "l2": "flushed before every timed step (256 MiB write)"},
            "us_per_sim_step": dev_ms * 1e3 / (args.steps * SIM_STEPS_PER_STEP),
            "gpu_launches": rt.launches - l0, "build_s": build_s, "clocks": clocks.summary()}


def compact(line: dict) -> dict:
    """A workload's line without the keys the headline line already states."""
    drop = {"metric", "unit", "n_gpus", "higher_is_better", "scaling", "vs_baseline", "data", "warmup"}
    return {k: v for k, v in line.items() if k not in drop}


def run_reference(args) -> None:
    """The reference arm: the CPU implementation (the oracle port, all host threads) on the same workload -- the
    network built on the host from the same parameters -- over the same window of simulation steps (W bench
    steps of warm-up, then K timed), rank 0 only."""
    import oracle
    from naer2_b200.runtime import describe

    name = {1: "brunel_A_config1", 2: "pd14_config2"}.get(args.config, "pd14_config2")
    sim = SIM_STEPS_PER_STEP
    t0 = time.perf_counter()
    net, pops, nb, cfg = build_workload(name, 1, device=None)
    desc = describe(net, forms=False)
    states = oracle.states_of(net, desc)
    prepared = oracle.prepare(desc)
    del desc
    build_s = time.perf_counter() - t0
    used = oracle.set_threads(0)
    n = 0
    for _ in range(args.warmup):
        oracle.run(prepared, states, n, sim, record=False)
        n += sim
    t0 = time.perf_counter()
    events = 0
    for _ in range(args.steps):
        _, ev = oracle.run(prepared, states, n, sim, record=False)
        events += ev
        n += sim
    el = time.perf_counter() - t0
    value = events / el
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded draws: connectivity, weights, delays, initial state, Philox Poisson drive)",
            "config": {**cfg, "sim_steps_per_step": sim, "window_steps": sim,
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single GPU",
                       "launch": "persistent"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "port",
                             "sample": f"simulation steps {args.warmup * sim}-{n} of {name} (after {args.warmup} x "
                                       f"{sim} warm-up steps), C oracle, {used} OpenMP threads, nproc "
                                       f"{os.cpu_count()}; the network drawn on the host"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "realtime_factor": el / (args.steps * sim * 1e-4), "build_s": build_s}
    print(json.dumps(line))


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="naer2_b200", choices=["naer2_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true", help="the headline workload alone (no sub-objects)")
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="2: the PD14 microcircuit (the headline, default); 1: Brunel model A at config 1's size; "
                         "3: 64 uneven Brunel instances batched against one at a time; 4: BPTT of the recurrent "
                         "LIF layer (training step against the plain forward); 5: a densely driven population "
                         "(the autotuner's push/pull choice against all push)")
    ap.add_argument("--instances", type=int, default=64, help="config 3: instances")
    ap.add_argument("--no-tune", dest="tune", action="store_false", help="config 3: skip the autotuner")
    ap.add_argument("--transpiled", action="store_true",
                    help="config 1 with the neurons' hooks transpiled and compiled at run time (TranspiledLIF)")
    ap.add_argument("--scale", type=float, default=1.0, help="config 2: population sizes times this (profiling)")
    ap.add_argument("--sim-steps", type=int, default=1000,
                    help="simulation steps per bench step (default 1000; small values for profiling runs)")
    args = ap.parse_args()
    global SIM_STEPS_PER_STEP, SCALE
    SIM_STEPS_PER_STEP = args.sim_steps
    SCALE = args.scale
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.transpiled:
        if args.config != 1 or world > 1:
            raise SystemExit("--transpiled runs config 1 on one GPU")
        print(json.dumps(run_transpiled(args, dev)))
        return 0
    if args.config in (3, 4, 5):
        if world > 1:
            raise SystemExit(f"config {args.config} runs on one GPU")
        print(json.dumps({3: run_batched, 4: run_bptt, 5: run_driven}[args.config](args, dev)))
        return 0
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    name = "pd14_config2" if args.config == 2 else "brunel_A_config1"
    line = run_plain(name, args, dev, rank, world, cpu=not args.no_cpu_baseline)
    if world == 1 and args.config == 2 and not args.no_workloads:
        line["workloads"] = {
            "brunel_A_config1": compact(run_plain("brunel_A_config1", args, dev, 0, 1, cpu=False)),
            "batched_config3": compact(run_batched(args, dev)),
            "bptt_config4": compact(run_bptt(args, dev)),
            "driven_dense_input": compact(run_driven(args, dev)),
        }
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
