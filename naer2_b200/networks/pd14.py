"""The layered cortical microcircuit of Potjans & Diesmann (2014) at a fixed dt: 8 populations (E/I of layers
2/3, 4, 5, 6) of PD14 LIF neurons with exponential current synapses, the reference's model
(test/networks/PD14/net.py, neuron.py, connection.py) with the changes of the full-size PD14 workload: an
explicit Poisson background of 8 Hz x K_bg events of weight J_E into every neuron (instead of the DC shift),
the connection matrix given target rows x source columns, inhibitory delays 0.8 +- 0.4 ms, every delay
clipped to >= dt and rounded to steps.

Connectivity: the reference's fixed-total-number rule per population pair (test/networks/PD14/
connection.py:14-24): Q = ln(1 - p) / ln(1 - 1/(N_src N_tgt)), k = round(Q / N_src) targets drawn uniformly
per source. Weights: normal, mean J_E = 87.81 pA (0.08781 nA), sd 10%, clamped to their sign; L4E -> L2/3E
doubled; inhibitory -4 J_E. Initial potentials: normal per population (the reference's V_mean / V_std).

scale: population sizes times `scale` (test sizes); device: draw the connectivity, weights and delays there
(a CUDA device builds the ~3e8 links of the full size in seconds).
"""

from __future__ import annotations

import numpy as np
import torch

from ..models import PD14_neuron
from ..patterns import fixed_outdegree

NAMES = ["E_23", "I_23", "E_4", "I_4", "E_5", "I_5", "E_6", "I_6"]
SIZES = [20683, 5834, 21915, 5479, 4850, 1065, 14395, 2948]
K_BG = [1600, 1500, 2100, 1900, 2000, 1900, 2900, 2100]
# connection probabilities, target rows x source columns
PROB = [[.1009, .1689, .0437, .0818, .0323, 0, .0076, 0],
        [.1346, .1371, .0316, .0515, .0755, 0, .0042, 0],
        [.0077, .0059, .0497, .135, .0067, .0003, .0453, 0],
        [.0691, .0029, .0794, .1597, .0033, 0, .1057, 0],
        [.1004, .0622, .0505, .0057, .0831, .3726, .0204, 0],
        [.0548, .0269, .0257, .0022, .06, .3158, .0086, 0],
        [.0156, .0066, .0211, .0166, .0572, .0197, .0396, .2252],
        [.0364, .001, .0034, .0005, .0277, .008, .0658, .1443]]
V_MEAN = [-68.28, -63.16, -63.33, -63.45, -63.11, -61.66, -66.72, -61.45]
V_STD = [5.36, 4.57, 4.74, 4.94, 4.94, 4.55, 5.46, 4.48]
J_E = 0.08781  # nA
DELAY = {"E": (1.5, 0.75), "I": (0.8, 0.4)}  # ms, mean and sd


def build(scale: float = 1.0, seed: int = 0, device=None, dt: float = 0.1, background: str = "poisson",
          group_size: int = 256):
    """(network, [populations in NAMES order])."""
    dev = torch.device(device) if device is not None else torch.device("cpu")
    gen = torch.Generator(device=dev).manual_seed(seed)
    pops = []
    for k, (n, kbg) in enumerate(zip(SIZES, K_BG)):
        n = max(1, int(round(n * scale)))
        p = PD14_neuron(K_cortical=kbg, background=background) * n
        p.seed = (seed << 8) | (k + 1)
        p.group_size = group_size
        p.potential = (torch.randn(n, generator=gen, device=dev) * V_STD[k] + V_MEAN[k]).to(torch.float32)
        pops.append(p)
    for t in range(8):
        for s in range(8):
            prob = PROB[t][s]
            if prob == 0.0:
                continue
            exc = s % 2 == 0
            pair_seed = (seed << 16) | (t << 4) | s
            c = pops[s] >> fixed_outdegree(prob, seed=pair_seed, device=dev if dev.type == "cuda" else None) >> pops[t]
            n_links = c.shape[0]
            w_mean = J_E * (2.0 if (s, t) == (2, 0) else 1.0) * (1.0 if exc else -4.0)
            g = torch.Generator(device=dev).manual_seed(pair_seed ^ 0x5A5A)
            w = torch.randn(n_links, generator=g, device=dev) * abs(w_mean) * 0.1 + w_mean
            c.weight = (w.clamp(min=0) if exc else w.clamp(max=0)).to(torch.float32)
            mu, sd = DELAY["E" if exc else "I"]
            d = torch.randn(n_links, generator=g, device=dev) * sd + mu
            c.delay = d.clamp(min=dt).to(torch.float32)
    net = pops[0].network
    net.resolution = dt
    return net, pops


def expected_synapses(scale: float = 1.0) -> int:
    """Links of the fixed-total-number rule at this scale (no draw)."""
    import math

    sizes = [max(1, int(round(n * scale))) for n in SIZES]
    total = 0
    for t in range(8):
        for s in range(8):
            p = PROB[t][s]
            if p == 0.0:
                continue
            Q = math.log(1 - p) / math.log(1 - 1 / (sizes[s] * sizes[t]))
            total += round(Q / sizes[s]) * sizes[s]
    return total
