"""Long-run statistics of the oracle against the reference's own time-driven loop (CPU).

Over long runs rasters cannot be compared with the reference: its fp32 sparse matvec and its own Poisson draws
(torch.poisson) make the chaotic network diverge from any other implementation within a few hundred steps.
The statistics are the check: tests/golden/brunel_longrun_c1.json holds the rates, CV-ISI and activity
std/mean that tools/brunel_reference.py computed with its own code over 10,000 steps (1 s) of Brunel's network
at config 1's size with its single delay of 1.5 ms (the loop has no per-link delays); the oracle runs the same
network (the same drawn connectivity and V0, its own Philox Poisson drive) and must give rates within 2% and
mean CV-ISI within 0.05 of the reference's, per population, by the reference's definitions
(naer2_b200.stats). The GPU path equals the oracle bit for bit over these runs (test_longrun_gpu.py)."""

import json
import pathlib
import sys

import numpy as np

import oracle
from naer2_b200.poisson import cdf_table
from naer2_b200.stats import SpikeStats
from test_oracle import brunel_golden_desc

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from make_golden import longrun_network  # noqa: E402  (the fixture's network, drawn again here)

RATE_REL_TOL = 0.02  # population rates within 2%
CV_ABS_TOL = 0.05    # mean CV-ISI within 0.05


def test_oracle_long_run_statistics_match_the_reference_loop():
    fx = json.loads((GOLDEN / "brunel_longrun_c1.json").read_text())
    P = fx["network"]
    NE, NI, steps = P["NE"], P["NI"], P["steps"]
    src, V0 = longrun_network(NE, NI, P["CE"], P["CI"], key=P["key"])
    theta, tau = 20.0, 20.0
    lam = P["eta"] * theta / (P["J"] * tau) * P["dt_ms"]  # C_E nu_ext dt (brunel_reference.py:24-25): 2.0
    g = {"src": src, "NE": NE, "J": P["J"], "g": P["g"], "delay_steps": P["delay_steps"], "table": cdf_table(lam),
         "seed": 0x10C0}
    desc = brunel_golden_desc(g)
    N = NE + NI
    st = [oracle.State(N, desc.pops[0].acc_depth, v=V0)]
    oracle.set_threads(0)
    stats = {"E": SpikeStats(NE, P["dt_ms"]), "I": SpikeStats(NI, P["dt_ms"])}
    chunk = 1000
    for k in range(steps // chunk):
        r, _ = oracle.run(desc, st, k * chunk, chunk)
        stats["E"].add(r[0][:, :NE], k * chunk)
        stats["I"].add(r[0][:, NE:], k * chunk)
    for name in ("E", "I"):
        got, want = stats[name].summary(), fx["stats"][name]
        assert abs(got["rate_hz"] - want["rate_hz"]) <= RATE_REL_TOL * want["rate_hz"], (name, got, want)
        assert abs(got["cv_isi"] - want["cv_isi"]) <= CV_ABS_TOL, (name, got, want)
