"""The BPTT workload's synthetic classification task and layer (seeded; no dataset is read).

Input: 700 channels of Poisson spikes over T steps of 1 ms. Each of 20 classes has a rate template over
(time, channel): a sum of 4 Gaussian bumps with random centres, widths (20-80 steps, 15-60 channels) and
heights, clipped to 0-50 Hz. A sample of class k draws its spikes from the template with a 10% multiplicative
jitter on every (step, channel) rate. The layer: `naer2_b200.bptt.RecurrentLIF` with 1024 hidden neurons at 10%
recurrent density, delays 1-5 steps, 20 readouts, checkpoints every 50 steps.
"""

from __future__ import annotations

import torch

from ..bptt import RecurrentLIF

CONFIG4 = dict(batch=128, steps=500, channels=700, hidden=1024, readouts=20, density=0.1, checkpoint=50,
               classes=20)


def templates(classes: int = 20, channels: int = 700, steps: int = 500, seed: int = 0, max_rate: float = 50.0,
              bumps: int = 4) -> torch.Tensor:
    """Rate templates [classes, steps, channels] in Hz."""
    g = torch.Generator(device="cpu").manual_seed(seed)
    t = torch.arange(steps, dtype=torch.float64)[:, None]
    c = torch.arange(channels, dtype=torch.float64)[None, :]
    out = torch.zeros(classes, steps, channels, dtype=torch.float64)
    for k in range(classes):
        for _ in range(bumps):
            u = torch.rand(5, generator=g, dtype=torch.float64)
            t0, c0 = u[0] * steps, u[1] * channels
            st, sc = 20 + 60 * u[2], 15 + 45 * u[3]
            h = max_rate * (0.5 + 0.5 * u[4])
            out[k] += h * torch.exp(-0.5 * ((t - t0) / st) ** 2 - 0.5 * ((c - c0) / sc) ** 2)
    return out.clamp(0.0, max_rate).float()


def sample(rates: torch.Tensor, batch: int, seed: int = 0, dt_ms: float = 1.0, jitter: float = 0.1,
           device=None):
    """(x [T, B, C] bool spikes, y [B] int64 labels), drawn on `device` from the templates."""
    dev = torch.device(device) if device is not None else rates.device
    g = torch.Generator(device=dev).manual_seed(seed)
    classes, steps, channels = rates.shape
    y = torch.randint(0, classes, (batch,), generator=g, device=dev)
    r = rates.to(dev)[y].permute(1, 0, 2)  # [T, B, C]
    noise = 1.0 + jitter * torch.randn(r.shape, generator=g, device=dev)
    p = (r * noise).clamp(0.0, 50.0) * (dt_ms * 1e-3)
    x = torch.rand(r.shape, generator=g, device=dev) < p
    return x, y


def build(seed: int = 0, device="cuda", **overrides):
    """(layer, x, y) of the BPTT workload (CONFIG4, any key overridden)."""
    cfg = dict(CONFIG4, **overrides)
    layer = RecurrentLIF(n_in=cfg["channels"], hidden=cfg["hidden"], readouts=cfg["readouts"],
                         density=cfg["density"], checkpoint=cfg["checkpoint"], seed=seed, device=device)
    rates = templates(cfg["classes"], cfg["channels"], cfg["steps"], seed=seed)
    x, y = sample(rates, cfg["batch"], seed=seed + 7, device=device)
    return layer, x, y
