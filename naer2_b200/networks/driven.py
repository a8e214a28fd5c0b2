"""A densely driven LIF population: the workload where gathering beats scattering.

N_in independent Poisson sources at a high rate (the merged input of many afferents, each source standing for
a bundle) drive N LIF neurons with a fixed in-degree K_in, plus a sparse recurrent E/I part of Brunel's kind.
At the default sizes the input connection carries 5M links and ~39% of its sources spike in every 0.1 ms step:
pushing them scatters ~2M arrival-slot reductions per step, ~200 into every target, while pulling streams the
5M link words (20 MB, L2-resident) once per step and sums each target in registers. The autotuner
(naer2_b200.tune) picks pull for that connection and push for the sparse recurrent ones."""

from __future__ import annotations

import numpy as np
import torch

from .. import philox
from ..models import LIF, Poisson_source
from ..patterns import fixed_indegree

CONFIG = dict(N_in=2000, rate_in=5.0, N=10000, K_in=500, J_in=0.001, NE_frac=0.8, CE=100, CI=25, J=0.1, g=5.0)


def build(N_in: int = 2000, rate_in: float = 5.0, N: int = 10000, K_in: int = 500, J_in: float = 0.001,
          NE_frac: float = 0.8, CE: int = 100, CI: int = 25, J: float = 0.1, g: float = 5.0, seed: int = 0,
          device=None, dt: float = 0.1):
    """(network, {"in", "E", "I"}). rate_in: spikes per ms of each input source; J_in: the input weight (mV), by
    default such that the mean input per step (K_in x P(spike) x J_in ~ 0.2 mV) equals Brunel's external drive
    at eta 2; delays uniform in 1-20 steps on the input and recurrent links alike."""
    src = Poisson_source(rate=rate_in) * N_in
    NE = int(round(N * NE_frac))
    NI = N - NE
    E = LIF(tau=20.0, theta=20.0, V_r=10.0, t_ref=2.0) * NE
    I = LIF(tau=20.0, theta=20.0, V_r=10.0, t_ref=2.0) * NI
    src.seed, E.seed, I.seed = (seed << 8) | 3, (seed << 8) | 1, (seed << 8) | 2
    E.V = torch.from_numpy((philox.uniform(seed, NE, stream=1) * 20.0).astype(np.float32))
    I.V = torch.from_numpy((philox.uniform(seed, NI, stream=2) * 20.0).astype(np.float32))
    k = 0
    for tgt in (E, I):
        for s, C, w in ((src, K_in, J_in), (E, CE, J), (I, CI, -g * J)):
            k += 1
            conn = s >> fixed_indegree(C, autapses=s is not tgt, seed=(seed << 8) | (16 + k), device=device) >> tgt
            conn.weight = w
            if device is not None and torch.device(device).type == "cuda":
                gen = torch.Generator(device=device).manual_seed((seed << 8) | (32 + k))
                steps = torch.randint(1, 21, (conn.shape[0],), generator=gen, device=device)
                conn.delay = (steps * dt).to(torch.float32)
            else:
                steps = philox.generator((seed << 8) | (32 + k)).integers(1, 21, conn.shape[0])
                conn.delay = torch.from_numpy((steps * dt).astype(np.float32))
    net = src.network
    net.resolution = dt
    return net, {"in": src, "E": E, "I": I}
