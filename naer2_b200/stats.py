"""Long-run spike statistics of a population, defined as the reference defines them for Brunel's network
(tools/brunel_reference.py:50-62 of the reference):
  rate      spikes at times t >= t_skip (50 ms) per neuron, over (T - t_skip), in Hz;
  CV-ISI    the mean over neurons with at least 4 such spikes of std(ISI) / mean(ISI) (std unbiased), over
            the population's first `cv_neurons` neurons (the reference samples 2,000; None: all);
  activity  std / mean (std unbiased) of the population's spike counts in 1 ms bins over [t_skip, T].
A spike of step n has time t = (n + 1) dt, as the reference stamps it.

SpikeStats accumulates these from packed raster rows chunk by chunk (uint32 words; bit j of word w is neuron
32 w + j), so a run of 100,000 steps of 77,169 neurons never holds its whole raster at once."""

from __future__ import annotations

import numpy as np


def unpack(words: np.ndarray, n: int) -> np.ndarray:
    """bool [rows, n] from uint32 raster words [rows, ceil(n / 32)]."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    bits = np.unpackbits(w.view(np.uint8).reshape(len(w), -1, 4), axis=2, bitorder="little")
    return bits.reshape(len(w), -1)[:, :n].astype(bool)


class SpikeStats:
    def __init__(self, n: int, dt: float, t_skip_ms: float = 50.0, cv_neurons: int | None = 2000,
                 bin_ms: float = 1.0):
        self.n, self.dt = int(n), float(dt)
        self.skip_time = int(round(t_skip_ms / dt))  # t >= t_skip  <=>  n + 1 >= skip_time
        self.bin_steps = max(1, int(round(bin_ms / dt)))
        self.cv_n = self.n if cv_neurons is None else min(self.n, int(cv_neurons))
        self.count = np.zeros(self.n, dtype=np.int64)
        self.last = np.full(self.n, -1, dtype=np.int64)
        self.isi_n = np.zeros(self.n, dtype=np.int64)
        self.isi_s1 = np.zeros(self.n, dtype=np.float64)
        self.isi_s2 = np.zeros(self.n, dtype=np.float64)
        self.activity = np.zeros(0, dtype=np.int64)
        self.steps = 0  # steps seen (from step 0)

    def add_words(self, words: np.ndarray, step0: int) -> None:
        self.add(unpack(words, self.n), step0)

    def add(self, raster: np.ndarray, step0: int) -> None:
        """Steps step0 .. step0 + len(raster) - 1 (bool [rows, n]), in order after the rows added before."""
        rows = len(raster)
        self.steps = max(self.steps, step0 + rows)
        st, ids = np.nonzero(raster)
        st = st.astype(np.int64) + step0
        keep = st + 1 >= self.skip_time
        st, ids = st[keep], ids[keep]
        if len(st) == 0:
            return
        np.add.at(self.count, ids, 1)
        b = (st + 1 - self.skip_time) // self.bin_steps
        if b.max() >= len(self.activity):
            grown = np.zeros(int(b.max()) + 1, dtype=np.int64)
            grown[: len(self.activity)] = self.activity
            self.activity = grown
        np.add.at(self.activity, b, 1)
        # intervals: spikes in (neuron, step) order; the first of each neuron in this chunk pairs with its last
        order = np.lexsort((st, ids))
        ids, st = ids[order], st[order]
        prev = np.empty_like(st)
        prev[1:] = st[:-1]
        first = np.ones(len(ids), dtype=bool)
        first[1:] = ids[1:] != ids[:-1]
        prev[first] = self.last[ids[first]]
        has = prev >= 0
        isi = (st - prev)[has].astype(np.float64)
        owner = ids[has]
        np.add.at(self.isi_n, owner, 1)
        np.add.at(self.isi_s1, owner, isi)
        np.add.at(self.isi_s2, owner, isi * isi)
        lastpos = np.ones(len(ids), dtype=bool)
        lastpos[:-1] = ids[1:] != ids[:-1]
        self.last[ids[lastpos]] = st[lastpos]

    def rate_hz(self) -> float:
        span_ms = self.steps * self.dt - self.skip_time * self.dt
        return float(self.count.sum()) / self.n / (span_ms / 1000.0) if span_ms > 0 and self.n else float("nan")

    def cv_isi(self) -> float:
        n, s1, s2 = self.isi_n[: self.cv_n], self.isi_s1[: self.cv_n], self.isi_s2[: self.cv_n]
        ok = n >= 3  # at least 4 spikes
        if not ok.any():
            return float("nan")
        mean = s1[ok] / n[ok]
        var = np.maximum(s2[ok] - n[ok] * mean * mean, 0.0) / (n[ok] - 1)
        return float(np.mean(np.sqrt(var) / mean))

    def activity_cv(self) -> float:
        bins = (self.steps - self.skip_time + 1) // self.bin_steps  # whole bins over [t_skip, T]
        if bins <= 1:
            return float("nan")
        a = np.zeros(bins, dtype=np.float64)
        m = min(bins, len(self.activity))
        a[:m] = self.activity[:m]
        if len(self.activity) > bins:  # a spike at exactly T falls in the last bin
            a[-1] += self.activity[bins:].sum()
        return float(a.std(ddof=1) / a.mean()) if a.mean() > 0 else float("nan")

    def summary(self) -> dict:
        return {"rate_hz": self.rate_hz(), "cv_isi": self.cv_isi(), "activity_std_over_mean": self.activity_cv(),
                "spikes": int(self.count.sum())}
