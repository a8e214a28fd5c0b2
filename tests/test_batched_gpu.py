"""Batching and tuning on the GPU: instances stepped together give each instance exactly the spikes it has
alone, and the autotuner's choice changes timing only."""

import numpy as np
import pytest
import torch

import oracle
from naer2_b200.networks import batched, brunel
from naer2_b200.runtime import describe
from naer2_b200.tune import autotune

pytestmark = pytest.mark.gpu


def test_batched_instances_equal_the_instances_alone(cuda):
    B, steps = 3, 300
    net, parts = batched.build(B, seed=5, device=cuda)
    net.record(steps)
    net.run_steps(steps)
    net.check()
    together = [[net.runtime.raster(p["E"]), net.runtime.raster(p["I"])] for p in parts]
    for b in range(B):
        inst, pops = batched.build_instance(b, seed=5, device=cuda)
        inst.record(steps)
        inst.run_steps(steps)
        alone = [inst.runtime.raster(pops["E"]), inst.runtime.raster(pops["I"])]
        for x, y in zip(together[b], alone):
            assert np.array_equal(x, y)
        assert sum(int(x.sum()) for x in alone) > 0
        inst.close()


def test_batched_small_instance_matches_oracle(cuda):
    net, pops = brunel.build(**dict(batched.instance_params(0, 9), NE=1200, NI=300, CE=120, CI=30))
    desc = describe(net)
    st = oracle.states_of(net, desc)
    net.record(400)
    net.run_steps(400)
    want, events = oracle.run(desc, st, 0, 400)
    for p, w in zip(net.populations, want):
        assert np.array_equal(net.runtime.raster(p), w)
    assert net.counters()["events"] == events


def test_autotune_keeps_results_and_restores_state(cuda):
    net, pops = brunel.build(**brunel.CONFIG0, seed=13)
    v0 = pops["E"].V.clone()
    desc = describe(net)
    st = oracle.states_of(net, desc)
    report = autotune(net, steps=50, warmup=20, blocks=(128, 256), persistent=(True, False))
    assert len(report["trials"]) >= 4 and "chosen" in report
    assert torch.equal(pops["E"].V.cpu(), v0.cpu())  # the initial state back
    net.record(300)
    net.run_steps(300)
    want, _ = oracle.run(desc, st, 0, 300)
    for p, w in zip(net.populations, want):
        assert np.array_equal(net.runtime.raster(p), w)


def test_many_populations_use_the_global_tables(cuda):
    """More populations (40) and push connections (80) than the kernel parameters hold: the tables are read
    from the workspace; the results stay the oracle's."""
    from naer2_b200.models import LIF
    from naer2_b200.patterns import fixed_indegree

    rng = np.random.default_rng(3)
    pops = []
    for k in range(40):
        p = LIF(theta=5.0, V_r=0.0, t_ref=0.5, ext_rate=4.0, ext_weight=0.5) * int(rng.integers(20, 90))
        p.V = torch.from_numpy(rng.uniform(0, 5, len(p.shape)).astype(np.float32))
        p.seed = 500 + k
        pops.append(p)
    for k in range(80):
        s, t = int(rng.integers(40)), int(rng.integers(40))
        c = pops[s] >> fixed_indegree(int(rng.integers(1, 6)), seed=900 + k) >> pops[t]
        c.weight = torch.from_numpy(rng.normal(0.1, 0.3, c.shape[0]).astype(np.float32))
        c.delay = torch.from_numpy(rng.integers(1, 12, c.shape[0]).astype(np.float32) * 0.1)
    net = pops[0].network
    assert len(net.populations) == 40 and len(net.connections) == 80
    desc = describe(net)
    st = oracle.states_of(net, desc)
    net.record(300)
    net.run_steps(300)
    want, events = oracle.run(desc, st, 0, 300)
    assert sum(int(w.sum()) for w in want) > 100
    for p, w in zip(net.populations, want):
        assert np.array_equal(net.runtime.raster(p), w)
    assert net.counters()["events"] == events
    for p, d, o in zip(net.populations, desc.pops, st):
        assert np.array_equal(p.V.cpu().numpy().view(np.uint32), o.v.view(np.uint32))
