"""The CPU oracle pinned before it is trusted: Philox4x32-10 against the
published known-answer vectors and Triton's implementation (the reference's
tl.rand), the LIF step loop against the reference's own
tools/brunel_reference.py run on the same inputs, and the PD14 neuron against
the reference's torch restatement of its hooks (fixtures: tests/golden/)."""

import json
import math
import pathlib

import numpy as np
import pytest

import oracle
from naer2_b200 import philox as host_philox
from naer2_b200.poisson import cdf_table, count
from naer2_b200.runtime import ConnDesc, NetDesc, PopDesc, fixed_shift, wfx
import torch

from naer2_b200.topology import Topology, pack_links

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"

# Random123 known-answer vectors of philox4x32-10 (counter, key, output)
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("counter,key,expected", KAT)
def test_philox_known_answers(counter, key, expected):
    assert oracle.philox(counter, key) == expected
    assert [int(x) for x in host_philox.philox4x32(*counter, *key)] == expected


def test_philox_matches_triton():
    """Triton's randint4x(seed, offset) is Philox with counter (offset, 0, 0, 0), key (seed lo, seed hi)."""
    data = json.loads((GOLDEN / "philox_triton.json").read_text())
    for case in data["cases"]:
        seed = case["seed"]
        for off, words, r in zip(case["offsets"], case["words"], case["rand"]):
            got = oracle.philox([off, 0, 0, 0], [seed & 0xFFFFFFFF, seed >> 32])
            assert got == words
            # tl.rand: the first word as int32, negatives folded, times 4.6566127342e-10
            x = np.int32(np.uint32(got[0]))
            x = -x - 1 if x < 0 else x
            assert np.float32(np.float32(x) * np.float32(4.6566127342e-10)) == np.float32(r)


def test_poisson_table_mean_and_variance():
    for lam in (0.3, 2.0, 6.7):
        table = cdf_table(lam)
        counts = oracle.poisson_counts(table, 99, 0, 200, 500).reshape(-1)
        assert abs(counts.mean() - lam) < 0.02 * lam + 0.01
        assert abs(counts.var() - lam) < 0.05 * lam + 0.01
        u = np.array(oracle.philox([3, 5, 0, 0], [99, 0])[:1], dtype=np.uint32)
        assert count(table, u)[0] == oracle.poisson_counts(table, 99, 5, 1, 4)[0, 3]


def test_fixed_point_weights():
    assert oracle.wfx(0.1, 40) == wfx(0.1, 40) == int(np.ldexp(np.float32(0.1), 40))
    assert oracle.wfx(-0.5, 40) == -(1 << 39)
    assert oracle.wfx(2.0 ** -45, 40) == 0  # below the resolution: rounds to nearest even (0)
    assert oracle.wfx(1.5 * 2.0 ** -40, 40) == 2  # a tie: to even
    assert fixed_shift(0.0) == 40 and fixed_shift(2.0 ** 30) == 31


def brunel_golden_desc(g):
    """The fixture's network as one population (the reference's own layout): LIF, one push connection with
    per-link weights (J for excitatory sources, -gJ for inhibitory ones) and the fixture's one delay."""
    src = g["src"].astype(np.int64)
    N, K = src.shape
    NE = int(g["NE"])
    J, gJ = float(g["J"]), float(g["g"]) * float(g["J"])
    tgt = np.repeat(np.arange(N), K)
    s = src.reshape(-1)
    w = np.where(s < NE, np.float32(J), np.float32(-gJ)).astype(np.float32)
    order = np.argsort(s, kind="stable")
    ptr = np.zeros(N + 1, np.int64)
    ptr[1:] = np.cumsum(np.bincount(s, minlength=N))
    topo = Topology(torch.from_numpy(ptr), torch.from_numpy(tgt[order]))
    steps = torch.full((len(s),), int(g["delay_steps"]), dtype=torch.int64)
    warr = torch.from_numpy(w[order])
    table = g["table"]
    insum = np.bincount(tgt, weights=np.abs(w.astype(np.float64)), minlength=N).max()
    sh = fixed_shift(insum + J * (len(table) - 1))
    pop = PopDesc(model=1, n=N, acc_depth=16, bit_depth=0, shift=sh, ref_steps=20, fire_threshold=0,
                  seed=int(g["seed"]), p=[float(np.float32(math.exp(-0.1 / 20))), 20.0, 10.0] + [0.0] * 5,
                  ext_table=table, ext_weight=J, ext_wfx=wfx(J, sh), state={})
    conn = ConnDesc(src=0, tgt=0, mode="push", n_links=len(s), ptr=topo.source_offsets.to(torch.int32),
                    link=pack_links(topo.target_indices, steps), weight=0.0, w=warr, split=None, topo=topo,
                    steps=steps, warr=warr)
    return NetDesc(dt=0.1, pops=[pop], conns=[conn], n_links=len(s))


def test_oracle_matches_reference_brunel_loop():
    """tools/brunel_reference.py's own loop (tests/golden/make_golden.py): identical raster over 1000 steps,
    V within 1e-6 relative (its fp32 sparse matvec against the oracle's exact sum)."""
    g = np.load(GOLDEN / "brunel_reference_c0.npz")
    desc = brunel_golden_desc(g)
    N = desc.pops[0].n
    st = [oracle.State(N, 16, v=g["V0"])]
    rasters, Vs = [], []
    for k in range(int(g["steps"]) // 100):
        r, _ = oracle.run(desc, st, 100 * k, 100)
        rasters.append(r[0])
        Vs.append(st[0].v.copy())
    raster = np.concatenate(rasters)
    expected = np.unpackbits(g["raster"], axis=1)[:, :N].astype(bool)
    assert raster.sum() > 5000
    assert np.array_equal(raster, expected)
    V = np.stack(Vs)
    np.testing.assert_allclose(V, g["V"], rtol=1e-6, atol=1e-5)


def test_oracle_matches_reference_pd14_neuron():
    """The reference's torch restatement of PD14's hooks (test/test_fused_models_gpu.py:32-52): identical
    raster over 400 steps; V and I within the reference test's own 1e-5."""
    g = np.load(GOLDEN / "pd14_neuron.npz")
    n, steps, every, K = len(g["V0"]), int(g["steps"]), int(g["every"]), int(g["K_cortical"])
    dt, t_mem, t_syn, R = 0.1, 10.0, 0.5, 40.0
    V_rest = -65.0 + R * K * 8e-3 * 0.08781 * t_syn  # the reference class's DC background
    P_V, P_I = math.exp(-dt / t_mem), math.exp(-dt / t_syn)
    P_VI = R * t_syn / (t_mem - t_syn) * (P_V - P_I)
    f = lambda x: float(np.float32(x))
    J, table = float(g["J"]), g["table"]
    sh = fixed_shift(J * (len(table) - 1))
    pop = PopDesc(model=2, n=n, acc_depth=1, bit_depth=0, shift=sh, ref_steps=19, fire_threshold=0, seed=int(g["seed"]),
                  p=[f(P_V), f(P_I), f(P_VI), f(V_rest), -50.0, -65.0, 0.0, 0.0], ext_table=table, ext_weight=J,
                  ext_wfx=wfx(J, sh), state={})
    desc = NetDesc(dt=dt, pops=[pop], conns=[], n_links=0)
    st = [oracle.State(n, 1, v=g["V0"], i=g["I0"])]
    rasters, Vs, Is = [], [], []
    for k in range(steps // every):
        r, _ = oracle.run(desc, st, k * every, every)
        rasters.append(r[0])
        Vs.append(st[0].v.copy())
        Is.append(st[0].i.copy())
    raster = np.concatenate(rasters)
    assert raster.sum() > 1000
    assert np.array_equal(raster, np.unpackbits(g["raster"], axis=1)[:, :n].astype(bool))
    np.testing.assert_allclose(np.stack(Vs), g["V"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(np.stack(Is), g["I"], rtol=1e-5, atol=1e-5)


def test_oracle_rejects_out_of_range_links():
    g = np.load(GOLDEN / "brunel_reference_c0.npz")
    desc = brunel_golden_desc(g)
    desc.pops[0].acc_depth = 8  # the delay of 15 steps no longer fits
    with pytest.raises(RuntimeError):
        oracle.run(desc, [oracle.State(desc.pops[0].n, 8, v=g["V0"])], 0, 200)


def test_a_planted_mistake_is_caught():
    """A wrong refractory period in the oracle's description changes the raster: the golden check bites."""
    g = np.load(GOLDEN / "brunel_reference_c0.npz")
    desc = brunel_golden_desc(g)
    desc.pops[0].ref_steps = 19
    st = [oracle.State(desc.pops[0].n, 16, v=g["V0"])]
    r, _ = oracle.run(desc, st, 0, 300)
    expected = np.unpackbits(g["raster"], axis=1)[:300, :desc.pops[0].n].astype(bool)
    assert not np.array_equal(r[0], expected)
