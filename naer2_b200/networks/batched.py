"""Many independent Brunel networks of uneven size and parameters, stepped together (the batched workload):
instance b draws N_E log-uniform in [1,000, 20,000], N_I = N_E / 4, C_E = min(0.1 N_E, 1,000), C_I = C_E / 4,
g uniform in [3, 6], eta uniform in [0.9, 4], per-link delays uniform in 1-20 steps, its own seed. All
instances joined in one Network run as one persistent launch per window (each instance's populations are
populations of that network; nothing connects instances); `build_instance(b)` gives one instance alone, the
plain one-network-at-a-time comparison."""

from __future__ import annotations

import math

import numpy as np

from . import brunel


def instance_params(b: int, seed: int = 0) -> dict:
    """Instance b's draws (deterministic in (seed, b))."""
    rng = np.random.Generator(np.random.Philox(key=(seed << 20) | (b + 1)))
    NE = int(round(math.exp(rng.uniform(math.log(1000), math.log(20000)))))
    NI = NE // 4
    CE = min(int(round(0.1 * NE)), 1000)
    CI = max(CE // 4, 1)
    return dict(NE=NE, NI=NI, CE=CE, CI=CI, g=float(rng.uniform(3.0, 6.0)), eta=float(rng.uniform(0.9, 4.0)),
                delay="uniform", max_delay_steps=20, seed=(seed << 12) | (b + 1))


def build_instance(b: int, seed: int = 0, device=None):
    """Instance b as its own network: (network, {"E", "I"})."""
    return brunel.build(**instance_params(b, seed), device=device)


def build(B: int = 64, seed: int = 0, device=None):
    """(network, [instance population dicts]) with all B instances in one network."""
    nets, parts = [], []
    for b in range(B):
        net, pops = build_instance(b, seed, device)
        nets.append(net)
        parts.append(pops)
    net = nets[0]
    for other in nets[1:]:
        net += other
    return net, parts
