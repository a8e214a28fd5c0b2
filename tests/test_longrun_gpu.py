"""Long runs on the GPU against the oracle, at the workloads' full sizes: Brunel's network at config 1's size
for its whole 10,000 steps (1 s), and the PD14 microcircuit (77,169 neurons, ~3e8 synapses) for 10 s of
network time (100,000 steps).

Both sides sum every step's input exactly in integer fixed point and draw the same Philox Poisson counts, so
the runs do not diverge: every raster word of every step must be equal (and the final state bit for bit), not
just the statistics. The statistics are checked as well, by the reference's definitions (naer2_b200.stats:
rate after 50 ms, CV-ISI over neurons with at least 4 spikes): rates within 2% and mean CV-ISI within 0.05 per
population. Against the reference's own loop, whose rasters do diverge, the statistics are the check
(test_longrun_stats.py). Rasters are compared chunk by chunk as packed words (the whole PD14 raster would be
~1 GB)."""

import numpy as np
import pytest
import torch

import oracle
from naer2_b200.networks import brunel, pd14
from naer2_b200.runtime import describe
from naer2_b200.stats import SpikeStats

pytestmark = pytest.mark.gpu

RATE_REL_TOL = 0.02
CV_ABS_TOL = 0.05
PD14_STEPS = 100_000  # 10 s of network time at dt 0.1 ms


def run_long(net, steps: int, chunk: int):
    """Run `net` on the GPU and the oracle (all host threads) for `steps` steps from the same initial state,
    comparing every chunk's raster words; returns per population (GPU stats, oracle stats)."""
    desc = describe(net)
    states = oracle.states_of(net, desc)
    prepared = oracle.prepare(desc)
    oracle.set_threads(0)
    dt = desc.dt
    g_stats = [SpikeStats(d.n, dt) for d in desc.pops]
    o_stats = [SpikeStats(d.n, dt) for d in desc.pops]
    net.record(chunk)
    for k in range(steps // chunk):
        step0 = k * chunk
        net.record(chunk)
        net.run_steps(chunk)
        rt = net.runtime
        want, _ = oracle.run(prepared, states, step0, chunk, packed=True)
        for q, (p, w) in enumerate(zip(net.populations, want)):
            got = rt.raster_words(p)
            if not np.array_equal(got, w):
                bad = int(np.nonzero((got != w).any(1))[0][0])
                raise AssertionError(f"population {q}: rasters differ first at step {step0 + bad}")
            g_stats[q].add_words(got, step0)
            o_stats[q].add_words(w, step0)
    net.check()
    for p, d, st in zip(net.populations, desc.pops, states):
        for slot, attr in d.state.items():
            got = p.state_tensor(attr).cpu().numpy()
            want = getattr(st, slot)
            assert np.array_equal(got.view(np.uint32) if got.dtype == np.float32 else got,
                                  want.view(np.uint32) if want.dtype == np.float32 else want), (d, slot)
    return g_stats, o_stats


def assert_statistics_agree(g_stats, o_stats):
    for q, (g, o) in enumerate(zip(g_stats, o_stats)):
        gs, os_ = g.summary(), o.summary()
        assert abs(gs["rate_hz"] - os_["rate_hz"]) <= RATE_REL_TOL * os_["rate_hz"], (q, gs, os_)
        assert abs(gs["cv_isi"] - os_["cv_isi"]) <= CV_ABS_TOL, (q, gs, os_)


def test_config1_whole_run_matches_oracle(cuda):
    net, pops = brunel.build(**brunel.CONFIG1, seed=2)
    g_stats, o_stats = run_long(net, 10_000, chunk=2_000)
    assert_statistics_agree(g_stats, o_stats)
    for s in g_stats:  # Brunel's asynchronous irregular regime (the reference's own bounds,
        sm = s.summary()  # test/test_brunel_gpu.py:86-105: rate 30-46 Hz, CV > 0.3)
        assert 30.0 <= sm["rate_hz"] <= 46.0 and sm["cv_isi"] > 0.3, sm
    net.close()


def test_pd14_ten_seconds_match_oracle(cuda):
    net, pops = pd14.build(scale=1.0, seed=1, device=cuda)
    g_stats, o_stats = run_long(net, PD14_STEPS, chunk=10_000)
    assert_statistics_agree(g_stats, o_stats)
    rates = [s.summary()["rate_hz"] for s in g_stats]
    assert all(0.05 < r < 50.0 for r in rates), rates  # every population active, none saturated
    net.close()
    torch.cuda.empty_cache()
