"""The kernels' bounded waits, made to give up on the GPU without a hang.

Two waits in the library spin on memory that other blocks write: the persistent step kernel's grid barrier
(n2b_device.cuh, grid_sync) and the BPTT adjoint's per-step exchange of q between the 8 CTAs of a group
(bptt.cu, group_wait). Each gives up after a limit and reports it in an error word instead of hanging. Here the
limit is set to almost nothing (1 ns of %globaltimer, 1 poll), so the waits give up while every block still
arrives and every launch still ends: the test checks the error words, that a window after the stop returns at
once, and that a reset of the error words brings a run with the normal limit back to the oracle's results."""

import numpy as np
import pytest
import torch

import oracle
from naer2_b200 import _lib
from naer2_b200.bptt import RecurrentLIF
from naer2_b200.networks import brunel, bptt_task
from naer2_b200.runtime import describe

pytestmark = pytest.mark.gpu


def _busy_network(limit_ns: int):
    """Config 0's network with a strong drive: many spikes per step, so that the blocks reach each barrier
    microseconds apart and a 1 ns limit runs out in some block."""
    net, _ = brunel.build(**brunel.CONFIG0, eta=6.0, seed=11)
    net.persistent = True
    net.window = 100
    net.barrier_limit_ns = limit_ns
    return net


def test_grid_barrier_gives_up_and_stops_the_window(cuda):
    net = _busy_network(1)
    net.run_steps(100)
    torch.cuda.synchronize()
    words = net.runtime.status()
    assert words[_lib.ERR_BARRIER] >= 1, words  # a wait gave up
    with pytest.raises(RuntimeError, match="persistent window stopped"):
        net.check()
    # the stop holds: the next window returns at once, the state does not move and no wait runs
    before = [p.state_tensor("V").clone() for p in net.populations]
    c0 = net.counters()
    net.run_steps(200)
    torch.cuda.synchronize()
    assert net.runtime.status()[_lib.ERR_BARRIER] == words[_lib.ERR_BARRIER]
    assert net.counters() == c0
    for p, v in zip(net.populations, before):
        assert torch.equal(p.state_tensor("V"), v)
    net.close()


def test_normal_limit_matches_the_oracle_after_a_stopped_run(cuda):
    """A run that stopped leaves the device usable: a fresh network with the default limit gives the oracle's
    raster, bit for bit."""
    stopped = _busy_network(1)
    stopped.run_steps(100)
    torch.cuda.synchronize()
    assert stopped.runtime.status()[_lib.ERR_BARRIER] >= 1
    stopped.close()

    net = _busy_network(0)
    desc = describe(net)
    states = oracle.states_of(net, desc)
    net.record(300)
    net.run_steps(300)
    net.check()
    expected, events = oracle.run(desc, states, 0, 300)
    for pop, want in zip(net.populations, expected):
        assert np.array_equal(net.runtime.raster(pop), want)
    assert net.counters()["events"] == events
    net.close()


def test_reset_clears_the_stop(cuda):
    net = _busy_network(1)
    net.run_steps(100)
    torch.cuda.synchronize()
    assert net.runtime.status()[_lib.ERR_BARRIER] >= 1
    net.runtime.reset_counters()
    assert net.runtime.status() == [0] * _lib.ERR_WORDS
    net.close()


def test_bptt_exchange_wait_gives_up(cuda):
    B, T, C, H, R = 8, 40, 32, 64, 5
    layer = RecurrentLIF(n_in=C, hidden=H, readouts=R, density=0.2, checkpoint=9, seed=0, device=cuda,
                         w_scale=(4.0, 0.5, 1.0))
    rates = bptt_task.templates(classes=R, channels=C, steps=T, seed=0)
    x, y = bptt_task.sample(rates, B, seed=1, device=cuda)

    def backward():
        layer.zero_grad(set_to_none=True)
        m = layer(x)
        torch.nn.functional.cross_entropy(m, y).backward()
        torch.cuda.synchronize()
        return [p.grad.detach().clone() for p in (layer.w_in, layer.w_rec, layer.w_out)]

    good = backward()
    assert layer.status(B, T) == [0, 0, 0, 0]
    layer.wait_polls = 1  # one poll: the CTAs that arrive before the group's last give up at once
    backward()
    words = layer.status(B, T)
    assert words[3] >= 1, words
    layer.wait_polls = 0  # the default limit again: the same gradients as before, no error word
    again = backward()
    assert layer.status(B, T) == [0, 0, 0, 0]
    for a, b in zip(good, again):
        assert torch.equal(a, b)
