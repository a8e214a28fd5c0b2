"""naer2_b200.stats against a direct restatement of the reference's statistics (tools/brunel_reference.py:50-62:
torch on the whole list of spike times), on random rasters fed to SpikeStats in uneven chunks of packed words."""

import numpy as np
import torch

from naer2_b200.stats import SpikeStats


def reference_style(raster: np.ndarray, dt: float, cv_neurons: int):
    """The reference's computation over one population (lo = 0, hi = n): times t = (step + 1) dt."""
    steps, n = raster.shape
    T = steps * dt
    st, ids = np.nonzero(raster)
    times = torch.from_numpy((st + 1).astype(np.float64) / round(1 / dt))  # exact multiples of dt
    nodes = torch.from_numpy(ids.astype(np.int64))
    m = times >= 50.0
    rate = int(m.sum()) / n / ((T - 50.0) / 1000)
    tt, nn = times[m], nodes[m]
    cvs = []
    for j in range(0, cv_neurons):
        tj = tt[nn == j]
        if len(tj) >= 4:
            isi = tj.diff()
            cvs.append(float(isi.std() / isi.mean()))
    act = torch.histc(tt, bins=int(round(T - 50)), min=50.0, max=T)
    return rate, sum(cvs) / len(cvs), float(act.std() / act.mean())


def test_chunked_statistics_equal_the_reference_formulas():
    rng = np.random.default_rng(5)
    steps, n, dt = 3000, 300, 0.1
    p = rng.uniform(0.001, 0.02, size=n)
    raster = rng.random((steps, n)) < p
    raster[steps - 1, :7] = True  # spikes at exactly T fall into the last bin
    words = np.packbits(np.pad(raster, ((0, 0), (0, (-n) % 32))), axis=1, bitorder="little").view(np.uint32)
    s = SpikeStats(n, dt, cv_neurons=200)
    for a, b in ((0, 123), (123, 1000), (1000, 1001), (1001, steps)):
        s.add_words(words[a:b], a)
    rate, cv, act = reference_style(raster, dt, 200)
    assert abs(s.rate_hz() - rate) < 1e-9
    assert abs(s.cv_isi() - cv) < 1e-9
    assert abs(s.activity_cv() - act) < 1e-9
    assert s.summary()["spikes"] == int(raster[499:].sum())
