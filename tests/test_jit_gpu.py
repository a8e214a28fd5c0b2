"""Transpiled, NVRTC-compiled step kernels of user-defined models against the DSL interpreter
(oracle/dsl_interpreter.py), which runs the same hooks in Python on float32 state.

Parity: identical spike rasters; state within float32 rounding (the kernels' single-precision math
functions and the interpreter's may differ in the last bits: 1e-5 relative, 1e-6 absolute)."""

import ctypes

import numpy as np
import pytest
import torch

from naer2_b200 import _lib
from naer2_b200.patterns import all_to_all, fixed_indegree
from naer2_b200.transpiler import JitRuntime
from oracle import dsl_interpreter
from tests.dsl_models import DecayLIF, Izhikevich, Pacemaker, Syn, TwoPort

pytestmark = pytest.mark.gpu


def check_against_interpreter(net, steps):
    rasters, state, edges = dsl_interpreter.run(net, steps)  # before the GPU run: the same initial state and seeds
    net.record(steps)
    net.run_steps(steps)
    assert isinstance(net.runtime, JitRuntime)
    net.check()
    for k, p in enumerate(net.populations):
        got = net.runtime.raster(p)
        if not np.array_equal(got, rasters[k]):
            bad = np.nonzero((got != rasters[k]).any(1))[0]
            raise AssertionError(f"population {k}: rasters differ first at step {bad[0]}")
        for a, want in state[k].items():
            have = p.state_tensor(a).cpu().numpy()
            if want.dtype == np.float32:
                np.testing.assert_allclose(have, want, rtol=1e-5, atol=1e-6, err_msg=f"{k}.{a}")
            else:
                assert np.array_equal(have, want), f"{k}.{a}"
    return rasters


def test_decay_lif_driven_by_pacemakers(cuda):
    g = torch.Generator().manual_seed(1)
    src = Pacemaker(period=6) * 50
    tgt = DecayLIF(theta=0.6, tau=5.0) * 70
    c = src >> Syn() @ fixed_indegree(8, seed=3) >> tgt
    c.weight = torch.rand(c.shape, generator=g) * 0.3
    c.delay = (torch.randint(1, 6, c.shape, generator=g) * 0.1).double()
    src.phase = torch.randint(0, 6, (50,), generator=g, dtype=torch.int32)
    net = src.network
    net.resolution = 0.1
    r = check_against_interpreter(net, 150)
    assert r[1].sum() > 50


def test_recurrent_izhikevich_with_random_drive(cuda):
    g = torch.Generator().manual_seed(2)
    pop = Izhikevich() * 200
    c = pop >> Syn() @ fixed_indegree(10, seed=4) >> pop
    c.weight = torch.randn(c.shape, generator=g) * 2.0
    c.delay = 0.3
    pop.v = -65.0 + 10.0 * torch.rand(200, generator=g)
    net = pop.network
    net.resolution = 0.5
    r = check_against_interpreter(net, 200)
    assert r[0].sum() > 100


def test_two_receive_ports_int_and_bool_state(cuda):
    g = torch.Generator().manual_seed(5)
    exc = Pacemaker(period=3) * 20
    inh = Pacemaker(period=11) * 10
    tgt = TwoPort(theta=1.5) * 40
    ce = exc >> Syn(gain=1.5) @ "exc" @ fixed_indegree(4, seed=6) >> tgt
    ce.weight = torch.rand(ce.shape, generator=g)
    ci = inh >> Syn(weight=0.4) @ "inh" @ all_to_all() >> tgt
    ci.delay = 0.2
    exc.phase = torch.arange(20, dtype=torch.int32)
    net = exc.network + inh.network
    net.resolution = 0.1
    r = check_against_interpreter(net, 120)
    assert r[2].sum() > 10


def test_a_compile_error_carries_the_nvrtc_log(cuda):
    lib = _lib.load()
    h = ctypes.c_void_p()
    rc = lib.n2b_jit_compile(b'extern "C" __global__ void n2b_user_step(int x) { undefined_name = x; }',
                             b"n2b_user_step", None, 0, 0, ctypes.byref(h))
    assert rc == -1
    msg = lib.n2b_last_error().decode()
    assert "NVRTC compile failed" in msg and "undefined_name" in msg


def test_pair_stdp_edge_hooks_change_the_weights_as_the_interpreter_does(cuda):
    from tests.dsl_models import PairSTDP, TraceLIF

    g = torch.Generator().manual_seed(9)
    src = Pacemaker(period=5) * 40
    tgt = TraceLIF(theta=1.2) * 30
    c = src >> PairSTDP() @ fixed_indegree(10, seed=10) >> tgt
    c.weight = 0.2 + 0.6 * torch.rand(c.shape, generator=g)
    c.delay = (torch.randint(1, 4, c.shape, generator=g) * 0.1).double()
    src.phase = torch.randint(0, 5, (40,), generator=g, dtype=torch.int32)
    net = src.network
    net.resolution = 0.1
    rasters, state, edges = dsl_interpreter.run(net, 200)
    net.record(200)
    net.run_steps(200)
    net.check()
    for k, p in enumerate(net.populations):
        assert np.array_equal(net.runtime.raster(p), rasters[k]), k
    assert rasters[1].sum() > 20
    w0 = c.fabric.value("weight").numpy()
    for name in ("weight", "x_pre", "t_last"):
        got = net.runtime.edge_state(c, name).cpu().numpy()
        np.testing.assert_allclose(got, edges[(0, name)], rtol=1e-5, atol=1e-6, err_msg=name)
    moved = np.abs(net.runtime.edge_state(c, "weight").cpu().numpy() - w0)
    assert (moved > 1e-3).mean() > 0.5  # learning happened on most links


def test_event_driven_exact_times(cuda):
    """net.exact: spikes carry their times within the step; arrivals are delivered in time order, each at its
    own time, with send after each group of equal times (DecayLIF decays exactly between them)."""
    from tests.dsl_models import JitterPacemaker

    g = torch.Generator().manual_seed(11)
    src = JitterPacemaker(period=4) * 60
    tgt = DecayLIF(theta=0.5, tau=3.0, t_ref=0.25) * 50
    c1 = src >> Syn() @ fixed_indegree(6, seed=12) >> tgt
    c1.weight = 0.1 + 0.3 * torch.rand(c1.shape, generator=g)
    c1.delay = (torch.randint(1, 5, c1.shape, generator=g) * 0.1).double()
    c2 = tgt >> Syn() @ fixed_indegree(3, seed=13) >> tgt
    c2.weight = 0.15 * torch.rand(c2.shape, generator=g)
    c2.delay = 0.2
    src.phase = torch.randint(0, 4, (60,), generator=g, dtype=torch.int32)
    src.jitter = (0.1 * torch.rand(60, generator=g)).float()
    net = src.network
    net.resolution = 0.1
    net.exact = True
    rasters, state, _, offsets = dsl_interpreter.run(net, 150)
    net.record(150)
    net.run_steps(150)
    net.check()
    rt = net.runtime
    for k, p in enumerate(net.populations):
        assert np.array_equal(rt.raster(p), rasters[k]), k
        times, ids = rt.spike_times(p)
        steps, ids_o = np.nonzero(rasters[k])
        want = (steps * 0.1).astype(np.float32) + offsets[k][steps, ids_o]
        np.testing.assert_allclose(times, want, rtol=1e-6, atol=1e-6)
    v = net.populations[1].state_tensor("v").cpu().numpy()
    np.testing.assert_allclose(v, state[1]["v"], rtol=1e-5, atol=1e-6)
    assert rasters[1].sum() > 30
    frac = offsets[1][np.nonzero(rasters[1])]
    assert (np.abs(frac - 0.1) > 1e-4).mean() > 0.5  # most target spikes off the step grid


def test_brunel_with_its_drive_in_the_hooks(cuda):
    """Brunel's model A as TranspiledLIF (the built-in LIF's dynamics, its Poisson drive drawn in its update
    hook): excitatory and inhibitory populations, recurrent delayed links, one uniform draw per neuron and step."""
    from naer2_b200.networks import brunel

    net, pops = brunel.build(NE=400, NI=100, CE=40, CI=10, delay="uniform", max_delay_steps=8, seed=3,
                             transpiled=True)
    r = check_against_interpreter(net, 120)
    assert r[0].sum() > 200 and r[1].sum() > 50
