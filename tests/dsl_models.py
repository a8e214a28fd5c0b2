"""User-defined models (no built-in kernel) for the transpiler tests: their hooks run as Python in the
oracle interpreter and as transpiled CUDA on the GPU."""

import math
import random

import naer2_b200 as n2
from naer2_b200 import receives as r


@n2.node
class DecayLIF:
    """A LIF neuron whose membrane decays exactly between its inputs (receive), thresholded in send."""

    def __init__(self, tau: float = 10.0, theta: float = 1.0, v_reset: float = 0.0, t_ref: float = 1.0):
        self.tau, self.theta, self.v_reset, self.t_ref = tau, theta, v_reset, t_ref
        self.v: float = 0.0
        self.last: float = 0.0
        self.ref_end: float = 0.0

    def update(self, time: n2.time):
        pass

    def send(self, time: n2.time):
        if self.v >= self.theta:
            n2.spike(time)
            self.v = self.v_reset
            self.ref_end = time + self.t_ref
            self.last = time + self.t_ref

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        if time >= self.ref_end:
            self.v = self.v * math.exp((self.last - time) / self.tau) + edge.weight
            self.last = time


@n2.node
class Izhikevich:
    """Izhikevich's two-variable neuron with a random drive drawn each step."""

    def __init__(self, a: float = 0.02, b: float = 0.2, c: float = -65.0, d: float = 8.0, drive: float = 12.0):
        self.a, self.b, self.c, self.d, self.drive = a, b, c, d, drive
        self.v: float = -65.0
        self.u: float = -13.0
        self.i: float = 0.0

    def update(self, time: n2.time):
        noise = self.drive if random.random() < 0.3 else 0.0
        self.v += 0.5 * (0.04 * self.v ** 2 + 5 * self.v + 140 - self.u + self.i + noise)
        self.v += 0.5 * (0.04 * self.v ** 2 + 5 * self.v + 140 - self.u + self.i + noise)
        self.u += self.a * (self.b * self.v - self.u)
        self.i = self.i * 0.5

    def send(self, time: n2.time):
        if self.v >= 30.0:
            n2.spike()
            self.v = self.c
            self.u += self.d

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        self.i += edge.weight


@n2.node(receive={"exc": "on_exc", "inh": "on_inh"})
class TwoPort:
    """Excitatory and inhibitory ports with their own edge attributes; an int counter and a bool flag."""

    def __init__(self, theta: float = 2.0, leak: float = 0.9):
        self.theta, self.leak = theta, leak
        self.g: float = 0.0
        self.count: int = 0
        self.inhibited: bool = False

    def update(self, time: n2.time):
        self.g = self.g * self.leak
        if self.count >= 3 and not self.inhibited:
            self.g += 0.25
        elif self.count % 2 == 1:
            self.g -= 0.125

    def send(self, time: n2.time):
        if self.g > self.theta:
            n2.spike(time)
            self.g = 0.0
            self.count = 0
            self.inhibited = False

    def on_exc(self, time: n2.time, edge: r.edge, source: r.source):
        self.g += edge.weight * edge.gain
        self.count += 1

    def on_inh(self, time: n2.time, edge: r.edge, source: r.source):
        self.g = max(self.g - edge.weight, -1.0)
        self.inhibited = True


@n2.node
class Pacemaker:
    """A source that fires every `period` steps, phase-shifted per neuron by its own state."""

    def __init__(self, period: int = 7):
        self.period = period
        self.phase: int = 0

    def update(self, time: n2.time):
        self.phase = self.phase + 1

    def send(self, time: n2.time):
        if self.phase % self.period == 0:
            n2.spike()

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        pass


@n2.edge
class Syn:
    def __init__(self, weight: float = 0.1, gain: float = 1.0):
        self.weight = weight
        self.gain = gain

    def forward(self):
        pass

    def backward(self):
        pass


@n2.node
class TraceLIF:
    """A leaky neuron keeping a postsynaptic trace (y_post, decaying from its last spike t_post) for STDP."""

    def __init__(self, decay: float = 0.9, theta: float = 1.0, tau_post: float = 2.0):
        self.decay, self.theta, self.tau_post = decay, theta, tau_post
        self.v: float = 0.0
        self.y_post: float = 0.0
        self.t_post: float = 0.0

    def update(self, time: n2.time):
        self.v = self.v * self.decay

    def send(self, time: n2.time):
        if self.v >= self.theta:
            n2.spike()
            self.v = 0.0
            self.y_post = self.y_post * math.exp((self.t_post - time) / self.tau_post) + 1.0
            self.t_post = time

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        self.v += edge.weight


@n2.edge
class PairSTDP:
    """Pair-based STDP: a presynaptic trace per link, the postsynaptic trace on the target; depression at a
    presynaptic arrival (forward), potentiation when the target fires (backward), weights kept in [0, w_max]."""

    def __init__(self, weight: float = 0.5, tau_pre: float = 2.0, tau_post: float = 2.0, a_plus: float = 0.05,
                 a_minus: float = 0.04, w_max: float = 1.0):
        self.weight = weight
        self.x_pre = 0.0
        self.t_last = 0.0
        self.tau_pre, self.tau_post, self.a_plus, self.a_minus, self.w_max = tau_pre, tau_post, a_plus, a_minus, w_max

    def forward(self, time: n2.time, dst: r.destination):
        self.x_pre = self.x_pre * math.exp((self.t_last - time) / self.tau_pre) + 1.0
        self.t_last = time
        y = dst.y_post * math.exp((dst.t_post - time) / self.tau_post)
        self.weight = max(self.weight - self.a_minus * y, 0.0)

    def backward(self, time: n2.time, dst: r.destination):
        x = self.x_pre * math.exp((self.t_last - time) / self.tau_pre)
        self.weight = min(self.weight + self.a_plus * x, self.w_max)


@n2.node
class JitterPacemaker:
    """Fires every `period` steps at its own time inside the step: `jitter` ms (its own state) before the step's
    end."""

    def __init__(self, period: int = 4):
        self.period = period
        self.phase: int = 0
        self.jitter: float = 0.0

    def update(self, time: n2.time):
        self.phase = self.phase + 1
        self.jitter = self.jitter * 0.9 + 0.005  # per neuron, drifting inside (0, 0.1)

    def send(self, time: n2.time):
        if self.phase % self.period == 0:
            n2.spike(time - self.jitter)

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        pass
