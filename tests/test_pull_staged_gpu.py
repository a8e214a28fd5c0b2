"""The staged pull intake (incoming CSR rows streamed into shared memory by bulk copies, gathered against the
source's spike-bit ring) against the oracle, bit for bit: long rows (many chunks per warp), ragged row ranges
(the unaligned head and tail loaded directly), per-link weights (staged beside the links), persistent windows
and per-step launches, and a connection whose rows are not 16-byte aligned (the plain walk instead)."""

import ctypes

import numpy as np
import pytest
import torch

import oracle
from naer2_b200 import _lib
from naer2_b200.networks import brunel
from naer2_b200.runtime import NetworkRuntime, describe
from test_parity_gpu import assert_identical, pd14_small, run_both

pytestmark = pytest.mark.gpu


def all_pull(net):
    return {id(c): "pull" for c in net.connections}


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_long_rows_all_pull_match_oracle(cuda, persistent):
    """Config 1's in-degrees (1,000 + 250 links per target): each warp streams 40,000 links in 79 chunks."""
    net, _ = brunel.build(NE=4000, NI=1000, CE=1000, CI=250, delay="uniform", max_delay_steps=20, seed=12)
    gr, orr, gs, os_, cnt, ev = run_both(net, 300, modes=all_pull(net), persistent=persistent)
    assert set(net.runtime.modes) == {"pull"}
    assert sum(r.sum() for r in gr) > 1000
    assert_identical(gr, orr, gs, os_)
    assert net.runtime.status()[_lib.ERR_PULL_STAGE] == 0


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_ragged_rows_with_weights_all_pull_match_oracle(cuda, persistent):
    """PD14's random in-degrees and per-link weights: ragged warp ranges, weights staged with the links."""
    net, _ = pd14_small(seed=21)
    gr, orr, gs, os_, cnt, ev = run_both(net, 500, chunk=170, modes=all_pull(net), persistent=persistent)
    assert sum(r.sum() for r in gr) > 100
    assert_identical(gr, orr, gs, os_)
    assert net.runtime.status()[_lib.ERR_PULL_STAGE] == 0


def sparse_rows_net(seed):
    """2,000 LIF targets pulling from two Poisson populations by fixed out-degree, delays uniform in 1-20 steps:
    300 sources x 2 links (single weight; in-degree ~0.3: most rows empty, the rest a link or two) and 3,000
    sources x 40 links with per-link weights (in-degree ~60: 59 items of the grid-wide pull, rows shorter than a
    batch and rows crossing batches, chunks and items)."""
    from naer2_b200 import philox
    from naer2_b200.models import LIF, Poisson_source
    from naer2_b200.patterns import fixed_outdegree

    rng = np.random.Generator(np.random.Philox(key=seed))
    a = Poisson_source(rate=0.5) * 300
    b = Poisson_source(rate=0.2) * 3000
    t = LIF(tau=20.0, theta=20.0, V_r=10.0, t_ref=2.0) * 2000
    a.seed, b.seed, t.seed = (seed << 8) | 1, (seed << 8) | 2, (seed << 8) | 3
    t.V = torch.from_numpy((philox.uniform(seed, 2000, stream=1) * 20.0).astype(np.float32))
    for k, (src, deg, w) in enumerate(((a, 2, 6.0), (b, 40, None))):
        c = src >> fixed_outdegree(k=deg, seed=(seed << 8) | (16 + k)) >> t
        c.weight = w if w is not None else torch.from_numpy(rng.uniform(0.05, 0.15, c.shape[0]).astype(np.float32))
        c.delay = torch.from_numpy((rng.integers(1, 21, c.shape[0]) * 0.1).astype(np.float32))
    net = t.network
    net.resolution = 0.1
    return net


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_short_and_empty_rows_all_pull_match_oracle(cuda, persistent):
    net = sparse_rows_net(seed=31)
    gr, orr, gs, os_, cnt, ev = run_both(net, 400, chunk=150, modes=all_pull(net), persistent=persistent)
    assert sum(r.sum() for r in gr[2:]) > 500  # the targets fire
    assert_identical(gr, orr, gs, os_)
    assert net.runtime.status()[_lib.ERR_PULL_STAGE] == 0


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
@pytest.mark.parametrize("grid", [1, 5, 37])
def test_grid_wide_pull_on_any_grid_matches_oracle(cuda, grid, persistent):
    """The delay >= 2 rows' items claimed by however many warps the launch has (one block: its eight warps take
    all 59+ items of the weighted connection in turn): the oracle's rasters and state for any grid."""
    net = sparse_rows_net(seed=32)
    net.grid = grid
    gr, orr, gs, os_, cnt, ev = run_both(net, 300, modes=all_pull(net), persistent=persistent)
    assert net.runtime.opt.grid == grid
    assert sum(r.sum() for r in gr[2:]) > 300
    assert_identical(gr, orr, gs, os_)


def test_unaligned_rows_walk_and_match_the_staged_path(cuda):
    """The same pull network twice through the C ABI: once as built (16-byte aligned rows: staged), once with
    every pull connection's link and weight arrays moved to an address 4 bytes past a 16-byte boundary (not
    staged: the plain walk). Identical rasters and state."""
    def build():
        net, _ = pd14_small(seed=22)
        net.tuned.update(all_pull(net))
        net.record(400)
        return net

    results = []
    for shift in (False, True):
        net = build()
        rt = NetworkRuntime(net)
        keep = []
        if shift:
            for k, c in enumerate(rt.desc.conns):
                cc = rt.cconn[k]
                for field, src in (("link", c.link), ("w", c.w)):
                    if src is None or getattr(cc, field) is None:
                        continue
                    buf = torch.zeros(src.numel() + 4, dtype=src.dtype, device=cuda)
                    buf[1:1 + src.numel()] = src.to(cuda)
                    keep.append(buf)
                    setattr(cc, field, buf.data_ptr() + 4)
            rt.close()
            lib = _lib.load()
            nbytes = ctypes.c_size_t()
            _lib.check(lib.n2b_workspace_bytes(rt.cpop, len(rt.pops), rt.cconn, len(rt.desc.conns),
                                               ctypes.byref(rt.opt), ctypes.byref(nbytes)), "workspace")
            rt.handle = ctypes.c_void_p()
            _lib.check(lib.n2b_create(rt.cpop, len(rt.pops), rt.cconn, len(rt.desc.conns), ctypes.byref(rt.opt),
                                      ctypes.c_void_p(rt.workspace.data_ptr()), nbytes.value, rt._s,
                                      ctypes.byref(rt.handle)), "create")
            _lib.check(lib.n2b_record(rt.handle, 0, rt._s), "record")
        net._runtime = rt
        net.run_steps(400)
        torch.cuda.synchronize()
        assert rt.status() == [0] * _lib.ERR_WORDS
        results.append(([rt.raster(p) for p in net.populations],
                        [p.state_tensor("potential").cpu().numpy().copy() for p in net.populations]))
        net.close()
        del keep
    (ra, va), (rb, vb) = results
    assert sum(r.sum() for r in ra) > 100
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y)
    for x, y in zip(va, vb):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_autotuner_pulls_the_dense_input_and_matches_oracle(cuda):
    """The densely driven population (5M input links, ~39% of the inputs spiking per step): the autotuner's
    measured choice pulls the input connections and pushes the sparse recurrent ones; the tuned network
    equals the oracle bit for bit."""
    from naer2_b200.networks import driven
    from naer2_b200.tune import autotune

    net, pops = driven.build(**driven.CONFIG, seed=3, device=cuda)
    report = autotune(net, steps=200, warmup=50)
    inputs = [c for c in net.connections if c._source is pops["in"]]
    assert report["chosen"]["pull"] > 0, report
    assert all(net.tuned.get(id(c)) == "pull" for c in inputs), report
    assert all(net.tuned.get(id(c), "push") == "push" for c in net.connections if c._source is not pops["in"])
    gr, orr, gs, os_, cnt, ev = run_both(net, 300, persistent=net.persistent)
    assert sum(r.sum() for r in gr[1:]) > 1000  # the driven neurons fire
    assert_identical(gr, orr, gs, os_)  # (events: a pull counts a link at its arrival, the oracle at emission)
