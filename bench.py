"""Benchmark: synaptic events/s of Brunel's model A at config 1's size
(N_E 10,000, N_I 2,500, C_E 1,000, C_I 250: 15.6M synapses, per-link delays
of 1-20 steps, dt 0.1 ms), stepped by the fused CUDA step kernel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl naer2_b200|reference]

One bench step = 1,000 simulation steps (100 ms of network time); the
config's 10,000 steps are 10 bench steps (the default K). Printed: one JSON
line (rank 0).
  value   events delivered in the timed steps / device time (CUDA events on
          the runtime's stream, L2 flushed before every timed step), summed
          over ranks, time the max over ranks
  e2e     the same metric through the public API with host buffers: every
          step copies the network state in from pinned host memory, runs
          Network.step, and reads the spike raster and state back
  roofline  the step kernel's algorithmic bytes (9 B per synaptic event +
          16 B per neuron per step) over its average launch time, against the
          measured HBM copy bandwidth
  cpu_baseline  the oracle (a C restatement of the reference's time-driven
          loop, all host threads) on a bounded sample of the same network
--impl reference times that CPU implementation alone (rank 0; others exit).
Multi-GPU: independent replicas (one network per rank, its own seed).
"""

from __future__ import annotations

import argparse
import json
import os
import pathlib
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SIM_STEPS_PER_STEP = 1000
BYTES_PER_EVENT = 9  # int32 target + int8 delay + fp32 weight
BYTES_PER_NEURON_STEP = 16  # V read + write, arrival slot read + clear
METRIC = "synaptic events/s"
UNIT = "events/s"
WORKLOAD = "brunel_A_config1"
MODE = "persistent"


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


def config(n_gpus: int) -> dict:
    return {"workload": WORKLOAD, "neurons": 12500, "synapses": 15_625_000, "delays_steps": "U{1..20}", "dt_ms": 0.1,
            "sim_steps_per_step": SIM_STEPS_PER_STEP, "l2": "flushed before every timed step (256 MiB write)",
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU", "launch": MODE}


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


def cpu_sample(desc, states, target_s: float = 12.0, threads: int = 0) -> dict:
    """The oracle on the host cores: a bounded sample of the same network (first steps from the same state)."""
    import oracle

    used = oracle.set_threads(threads)
    probe = 50
    t0 = time.perf_counter()
    _, ev = oracle.run(desc, states, 0, probe, record=False)
    t_probe = time.perf_counter() - t0
    steps = max(50, min(400_000, int(probe * target_s / max(t_probe, 1e-3))))
    t0 = time.perf_counter()
    _, ev2 = oracle.run(desc, states, probe, steps, record=False)
    el = time.perf_counter() - t0
    return {"value": ev2 / el, "unit": UNIT, "cores": used, "kind": "port",
            "sample": f"{WORKLOAD}: simulation steps {probe}-{probe + steps} ({steps * 0.1:.0f} ms of network time, "
                      f"{ev2} events) in {el:.1f} s, C oracle, {used} OpenMP threads, nproc {os.cpu_count()}",
            "realtime_factor": el / (steps * 1e-4)}


def run_reference(args) -> None:
    """The reference arm: the CPU implementation (the oracle port, all host threads) on the same workload."""
    import oracle
    from naer2_b200.networks import brunel
    from naer2_b200.runtime import describe

    net, _ = brunel.build(**brunel.CONFIG1, seed=1)
    desc = describe(net)
    states = oracle.states_of(net, desc)
    used = oracle.set_threads(0)
    per_step = 100  # simulation steps per bench step: a bounded sample of the 1,000 of ours
    n = 0
    for _ in range(args.warmup):
        oracle.run(desc, states, n, per_step, record=False)
        n += per_step
    t0 = time.perf_counter()
    events = 0
    for _ in range(args.steps):
        _, ev = oracle.run(desc, states, n, per_step, record=False)
        events += ev
        n += per_step
    el = time.perf_counter() - t0
    value = events / el
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox network)",
            "config": {**config(1), "sim_steps_per_step": per_step}, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "port",
                             "sample": f"{args.steps} x {per_step} simulation steps of {WORKLOAD} after "
                                       f"{args.warmup} x {per_step} warm-up, C oracle, {used} OpenMP threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "realtime_factor": el / (args.steps * per_step * 1e-4)}
    print(json.dumps(line))


def run_transpiled(args, dev) -> dict:
    """Config 1's network with TranspiledLIF neurons (the built-in LIF's dynamics, its Poisson drive drawn in its
    own hook): the run-time compiled step kernels, launched from the host once per population and step (no
    persistent window, no graph), events/s over the timed steps."""
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


def run_pd14(args, dev) -> dict:
    """Config 2: the full PD14 microcircuit (77,169 neurons, ~3e8 synapses) built on the GPU; events/s over the
    timed steps, population rates and CV-ISI over them."""
    import numpy as np
    import torch

    from naer2_b200.networks import pd14

    t0 = time.perf_counter()
    net, pops = pd14.build(scale=args.scale, seed=1, device=dev)
    net.persistent = args.mode == "persistent"
    net.record(args.steps * SIM_STEPS_PER_STEP)
    for p in pops:
        p.state_tensor("potential", dev)
    rt_build = time.perf_counter()
    net.run_steps(1)  # builds the runtime
    rt = net.runtime
    build_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        net.run_steps(SIM_STEPS_PER_STEP)
    net.record(args.steps * SIM_STEPS_PER_STEP)
    torch.cuda.synchronize(dev)
    ev0 = rt.counters()["events"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with Clocks(dev.index or 0) as clocks:
        for k in range(args.steps):
            flush.zero_()
            rt._enter()
            starts[k].record(rt.stream)
            net.run_steps(SIM_STEPS_PER_STEP)
            ends[k].record(rt.stream)
        torch.cuda.synchronize(dev)
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    events = rt.counters()["events"] - ev0
    net.check()
    steps = args.steps * SIM_STEPS_PER_STEP
    rates, cvs = [], []
    for p in pops:
        r = torch.from_numpy(rt.raster(p))  # [steps, n]
        n = r.shape[1]
        rates.append(float(r.sum()) / n / (steps * 1e-4))
        step_idx, nid = torch.nonzero(r, as_tuple=True)
        order = torch.argsort(nid * (steps + 1) + step_idx)
        nid, t = nid[order], step_idx[order].double()
        same = nid[1:] == nid[:-1]
        isi = (t[1:] - t[:-1])[same]
        owner = nid[1:][same]
        cnt = torch.bincount(owner, minlength=n).double()
        s1 = torch.bincount(owner, weights=isi, minlength=n)
        s2 = torch.bincount(owner, weights=isi * isi, minlength=n)
        ok = cnt >= 3
        mean = s1[ok] / cnt[ok]
        var = (s2[ok] - cnt[ok] * mean * mean) / (cnt[ok] - 1)
        cvs.append(float((var.clamp(min=0).sqrt() / mean).mean()) if int(ok.sum()) else float("nan"))
    ev_step = events / steps
    n_neurons = sum(len(p.shape) for p in pops)
    alg = ev_step * BYTES_PER_EVENT + n_neurons * (BYTES_PER_NEURON_STEP + 16)
    us = dev_ms * 1e3 / steps
    peak, kind = measured_peaks()
    return {"metric": METRIC, "value": events / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded draws on the GPU, PD14 microcircuit)",
            "config": {"workload": "pd14_config2", "scale": args.scale, "neurons": n_neurons,
                       "synapses": rt.n_links, "dt_ms": 0.1, "sim_steps_per_step": SIM_STEPS_PER_STEP,
                       "launch": MODE, "l2": "flushed before every timed step (256 MiB write)"},
            "realtime_factor": (dev_ms / 1e3) / (steps * 1e-4),
            "roofline": {"bound": "hbm", "achieved": alg / (us * 1e-6) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (us * 1e-6) / 1e9 / peak, "traffic": None, "peak_kind": kind,
                         "bytes_per_launch": alg, "us_per_launch": us},
            "l2_atomics": l2_atomics(events / (dev_ms / 1e3), dev),
            "rates_hz": dict(zip(pd14.NAMES, [round(x, 3) for x in rates])),
            "cv_isi": dict(zip(pd14.NAMES, [round(x, 3) for x in cvs])),
            "events_per_sim_step": ev_step, "build_s": build_s, "clocks": clocks.summary()}


def run_batched(args, dev) -> dict:
    """Config 3: B uneven Brunel instances in one network (one persistent launch per window), tuned by the
    autotuner, against the same instances stepped one network at a time on the same GPU (same seeds: the same
    spikes). Aggregate synaptic events/s of both, and per-instance rates."""
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
    chosen = dict(block=net.block, grid=net.grid, persistent=net.persistent, tuned=dict(net.tuned))
    net.close()
    del net, parts
    torch.cuda.empty_cache()
    # the same instances, one network at a time, the tuned configuration
    ms_p, ev_p, spk_p = 0.0, 0, []
    for b in range(B):
        inst, _ = batched.build_instance(b, seed=1, device=dev)
        # the single instances at two blocks per SM: measured faster for them than the persistent default
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        inst.block, inst.grid, inst.persistent = chosen["block"], 2 * sms, chosen["persistent"]
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
                       "dt_ms": 0.1, "sim_steps_per_step": sim, "tuned": {k: v for k, v in chosen.items()
                                                                             if k != "tuned"}},
            "l2_atomics": l2_atomics(value, dev),
            "plain_one_at_a_time": {"value": plain, "ms_per_step": ms_p / args.steps},
            "batched_over_plain": value / plain,
            "identical_spike_counts": spk_b == spk_p,
            "rates_hz_first4": [[round(x, 2) for x in r] for r in rates_b[:4]],
            "max_rate_difference_hz": max(abs(x - y) for rb, rp in zip(rates_b, rates_p) for x, y in zip(rb, rp)),
            "tune": report["trials"] if report else None, "build_s": build_s}


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


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="naer2_b200", choices=["naer2_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", type=int, default=1, choices=[1, 2, 3, 4],
                    help="1: Brunel model A at config 1's size (the default workload); 2: the PD14 microcircuit; "
                         "3: 64 uneven Brunel instances batched against one at a time; 4: BPTT of the "
                         "recurrent LIF layer (training step against the plain forward)")
    ap.add_argument("--instances", type=int, default=64, help="config 3: instances")
    ap.add_argument("--tune", action="store_true", help="config 3: run the autotuner first")
    ap.add_argument("--scale", type=float, default=1.0, help="config 2: population sizes times this")
    ap.add_argument("--mode", choices=["persistent", "per-step"], default="persistent",
                    help="a window of steps per cooperative launch, or one launch per step")
    ap.add_argument("--transpiled", action="store_true",
                    help="config 1 with the neurons' hooks transpiled and compiled at run time (TranspiledLIF)")
    ap.add_argument("--sim-steps", type=int, default=1000,
                    help="simulation steps per bench step (default 1000; small values for profiling runs)")
    args = ap.parse_args()
    global SIM_STEPS_PER_STEP, MODE
    SIM_STEPS_PER_STEP = args.sim_steps
    MODE = args.mode
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist

    from naer2_b200.networks import brunel
    from naer2_b200.runtime import describe

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.transpiled:
        if args.config != 1 or world > 1:
            raise SystemExit("--transpiled runs config 1 on one GPU")
        print(json.dumps(run_transpiled(args, dev)))
        return 0
    if args.config in (2, 3, 4):
        if world > 1:
            raise SystemExit(f"config {args.config} runs on one GPU")
        run = {2: run_pd14, 3: run_batched, 4: run_bptt}[args.config]
        print(json.dumps(run(args, dev)))
        return 0
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    net, pops = brunel.build(**brunel.CONFIG1, seed=1 + rank)
    net.persistent = args.mode == "persistent"
    desc = describe(net) if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    import oracle as _oracle_for_baseline_only  # noqa: F401  (the CPU baseline leg below)

    cpu_states = _oracle_for_baseline_only.states_of(net, desc) if desc is not None else None
    net.record(SIM_STEPS_PER_STEP)
    rt = net.runtime
    n_neurons = sum(len(p.shape) for p in net.populations)

    # ---- device-resident timing
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        net.run_steps(SIM_STEPS_PER_STEP)
    barrier()
    ev0 = rt.counters()["events"]
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with Clocks(local) as clocks:
        barrier()
        for k in range(args.steps):
            flush.zero_()
            rt._enter()  # the runtime's stream after the flush
            starts[k].record(rt.stream)
            net.run_steps(SIM_STEPS_PER_STEP)
            ends[k].record(rt.stream)
        barrier()
    dev_ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    events = rt.counters()["events"] - ev0
    launches = args.steps * SIM_STEPS_PER_STEP  # simulation steps (one step kernel each, or one window iteration)
    windows = args.steps * (SIM_STEPS_PER_STEP // max(net.window, 1) + (SIM_STEPS_PER_STEP % max(net.window, 1) > 0))
    # kernels launched: per-step mode one per step; persistent mode one per window; + one counter advance per window
    launches_all = (launches if MODE == "per-step" else windows) + windows
    net.check()

    # ---- end to end through the public API, host buffers
    hosts = []
    for p in net.populations:
        for attr in ("V", "ref"):
            t = p.state_tensor(attr)
            hosts.append((p, attr, torch.empty(t.shape, dtype=t.dtype, pin_memory=True)))
    for p, attr, h in hosts:
        h.copy_(p.state_tensor(attr))
    raster_host = [torch.empty(r.shape, dtype=r.dtype, pin_memory=True) for r in rt.rasters]
    h2d = sum(h.numel() * h.element_size() for _, _, h in hosts)
    d2h = h2d + sum(r.numel() * r.element_size() for r in raster_host)
    barrier()
    ev1 = rt.counters()["events"]
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for p, attr, h in hosts:  # inputs: the network state, from pinned host memory
            p.state_tensor(attr).copy_(h, non_blocking=True)
        net.record(SIM_STEPS_PER_STEP)
        net.step(SIM_STEPS_PER_STEP * net.resolution)
        for r, h in zip(rt.rasters, raster_host):  # results: the spike raster and the state
            h.copy_(r, non_blocking=True)
        for p, attr, h in hosts:
            h.copy_(p.state_tensor(attr), non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_events = rt.counters()["events"] - ev1

    # ---- max over ranks
    dev_ms, e2e_s, events_all, e2e_events_all = reduce_over_ranks([dev_ms, e2e_s], [events, e2e_events], world, dev)

    cpu = None
    if desc is not None:
        cpu = cpu_sample(desc, cpu_states)

    if rank == 0:
        value = events_all / (dev_ms / 1e3)
        ms_per_launch = dev_ms / launches
        ev_per_launch = events / launches
        alg_bytes = ev_per_launch * BYTES_PER_EVENT + n_neurons * BYTES_PER_NEURON_STEP
        achieved = alg_bytes / (ms_per_launch / 1e3) / 1e9
        peak, peak_kind = measured_peaks()
        traffic = None
        prof = ROOT / "profiles" / "persistent_kernel_brunel_config1.json"
        if prof.exists() and MODE == "persistent":  # one ncu capture, scaled to this run's events per step
            pr = json.loads(prof.read_text())
            traffic = pr["dram_bytes_per_step"] * ev_per_launch / pr["events_per_step"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox network, Brunel model A)",
            "config": config(world),
            "realtime_factor": (dev_ms / 1e3) / (args.steps * SIM_STEPS_PER_STEP * 1e-4),
            "e2e": {"value": e2e_events_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": ("n2b::persistent_kernel<256>" if MODE == "persistent" else "n2b::step_kernel<256>"),
                         "bytes_per_launch": alg_bytes, "us_per_launch": ms_per_launch * 1e3,
                         "note": "per simulation step: timed device time / steps (launch gaps and grid barriers "
                                 "included)"},
            "l2_atomics": l2_atomics(events / (dev_ms / 1e3), dev),
            "gpu_launches": launches_all,
            "clocks": clocks.summary(),
            "events_per_sim_step": ev_per_launch,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    net.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
