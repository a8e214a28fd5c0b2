"""Brunel (2000) model A, time-driven: a sparse balanced network of N_E
excitatory and N_I inhibitory LIF neurons with delta synapses, fixed
in-degree (C_E from E, C_I from I, drawn uniformly without autapses), PSP J
and -g J, an external Poisson drive of eta * nu_thr per external source
(nu_thr = theta / (J C_E tau)) from C_E sources, i.e. C_E eta nu_thr events
per ms of weight J into every neuron -- the reference's
tools/brunel_reference.py (time-driven) and test/networks/Brunel/net.py
(event-driven) at a fixed dt.

delay: one delay in ms for every link, or "uniform" -- integer delays drawn
uniformly in [1, max_delay_steps] steps per link.
"""

from __future__ import annotations

import math
import random

import numpy as np
import torch

import naer2_b200 as n2

from .. import philox
from .. import receives as _r
from ..decorators import node
from ..models import LIF
from ..patterns import fixed_indegree

POISSON_TERMS = 12  # external events per step counted up to this (P(more) < 1e-6 at config 1's 2 per step)


@node
class TranspiledLIF:
    """Brunel's LIF as `LIF` states it, with its external Poisson drive drawn in its own update hook (one uniform
    per step, counted against the Poisson CDF of ext_rate dt at POISSON_TERMS thresholds), so that it has no
    built-in kernel: a network of it steps on the transpiled, run-time compiled step kernels. Same dynamics as
    `LIF`, other random draws (its rasters are not `LIF`'s)."""

    def __init__(self, tau: float = 20.0, theta: float = 20.0, V_r: float = 10.0, t_ref: float = 2.0,
                 ext_rate: float = 0.0, ext_weight: float = 0.0, dt: float = 0.1):
        self.decay = float(np.float32(math.exp(-dt / tau)))
        self.theta, self.V_r, self.ext_weight = theta, V_r, ext_weight
        self.ref_steps = int(round(t_ref / dt))
        lam, term, cdf = ext_rate * dt, math.exp(-ext_rate * dt), 0.0
        for k in range(POISSON_TERMS):  # c<k> = P(count <= k)
            cdf += term
            term *= lam / (k + 1)
            setattr(self, f"c{k}", float(np.float32(min(cdf, 1.0))))
        self.V: float = 0.0
        self.ref: int = 0
        self.I: float = 0.0

    def receive(self, time: _r.time, edge: _r.edge, source: _r.source):
        self.I += edge.weight

    def update(self, time: _r.time):
        u = random.random()
        k = 0
        if u > self.c0:
            k += 1
        if u > self.c1:
            k += 1
        if u > self.c2:
            k += 1
        if u > self.c3:
            k += 1
        if u > self.c4:
            k += 1
        if u > self.c5:
            k += 1
        if u > self.c6:
            k += 1
        if u > self.c7:
            k += 1
        if u > self.c8:
            k += 1
        if u > self.c9:
            k += 1
        if u > self.c10:
            k += 1
        if u > self.c11:
            k += 1
        if self.ref > 0:
            self.ref -= 1
        else:
            self.V = self.V * self.decay + self.I + k * self.ext_weight
        self.I = 0.0

    def send(self, time: _r.time):
        if self.ref == 0 and self.V >= self.theta:
            n2.spike()
            self.V = self.V_r
            self.ref = self.ref_steps


CONFIG0 = dict(NE=800, NI=200, CE=80, CI=20, delay=1.5)
CONFIG1 = dict(NE=10000, NI=2500, CE=1000, CI=250, delay="uniform", max_delay_steps=20)


def build(NE: int = 800, NI: int = 200, CE: int = 80, CI: int = 20, J: float = 0.1, g: float = 5.0,
          eta: float = 2.0, delay="uniform", max_delay_steps: int = 20, tau: float = 20.0, theta: float = 20.0,
          V_r: float = 10.0, t_ref: float = 2.0, dt: float = 0.1, seed: int = 0, group_size: int = 256,
          device=None, transpiled: bool = False):
    """(network, {"E": E, "I": I}) of Brunel's model A at step dt. device: draw the connectivity and delays there
    (CUDA: torch's generator, fast at large sizes; default: numpy's Philox on the host). transpiled: the neurons
    are TranspiledLIF (the run-time compiled step kernels) instead of the built-in LIF."""
    nu_thr = theta / (J * CE * tau)
    ext_rate = CE * eta * nu_thr  # external events per ms into each neuron
    if transpiled:
        E = TranspiledLIF(tau=tau, theta=theta, V_r=V_r, t_ref=t_ref, ext_rate=ext_rate, ext_weight=J, dt=dt) * NE
        I = TranspiledLIF(tau=tau, theta=theta, V_r=V_r, t_ref=t_ref, ext_rate=ext_rate, ext_weight=J, dt=dt) * NI
    else:
        E = LIF(tau=tau, theta=theta, V_r=V_r, t_ref=t_ref, ext_rate=ext_rate, ext_weight=J) * NE
        I = LIF(tau=tau, theta=theta, V_r=V_r, t_ref=t_ref, ext_rate=ext_rate, ext_weight=J) * NI
    E.seed, I.seed = (seed << 8) | 1, (seed << 8) | 2
    E.group_size = I.group_size = group_size
    E.V = torch.from_numpy((philox.uniform(seed, NE, stream=1) * theta).astype(np.float32))
    I.V = torch.from_numpy((philox.uniform(seed, NI, stream=2) * theta).astype(np.float32))
    k = 0
    for tgt in (E, I):
        for src, C, w in ((E, CE, J), (I, CI, -g * J)):
            k += 1
            conn = src >> fixed_indegree(C, autapses=False, seed=(seed << 8) | (16 + k), device=device) >> tgt
            conn.weight = w
            if delay == "uniform":
                if device is not None and torch.device(device).type == "cuda":
                    gen = torch.Generator(device=device).manual_seed((seed << 8) | (32 + k))
                    steps_t = torch.randint(1, max_delay_steps + 1, (conn.shape[0],), generator=gen, device=device)
                    conn.delay = (steps_t * dt).to(torch.float32)
                else:
                    steps = philox.generator((seed << 8) | (32 + k)).integers(1, max_delay_steps + 1, conn.shape[0])
                    conn.delay = torch.from_numpy((steps * dt).astype(np.float32))
            else:
                conn.delay = float(delay)
    net = E.network
    net.resolution = dt
    return net, {"E": E, "I": I}
