"""Parity of the CUDA hot path with the oracle (and through it the reference):
every raster bit-identical and every state value bit-identical -- the input
of a step is an exact integer sum on both sides and every float operation
is rounded the same way, so nothing is left to a tolerance -- and, on the
reference's own fixture (tests/golden/brunel_reference_c0.npz), the raster
of tools/brunel_reference.py itself, through the C ABI."""

import ctypes
import math

import numpy as np
import pytest
import torch

import oracle
from naer2_b200 import _lib
from naer2_b200.models import LIF, PD14_neuron, Poisson_source
from naer2_b200.networks import brunel
from naer2_b200.patterns import all_to_all, fixed_indegree, fixed_outdegree
from naer2_b200.runtime import describe
from test_oracle import GOLDEN, brunel_golden_desc

pytestmark = pytest.mark.gpu


def run_both(net, steps, chunk=None, modes=None, persistent=True):
    """Run `net` on the GPU and the oracle from the same initial state; return (gpu rasters, oracle rasters,
    gpu states, oracle states, gpu counters, oracle events)."""
    net.persistent = persistent
    desc = describe(net, modes)
    st = oracle.states_of(net, desc)
    net.record(steps)
    if modes:
        net.tuned.update(modes)
    if chunk:
        for _ in range(steps // chunk):
            net.run_steps(chunk)
        net.run_steps(steps % chunk)
    else:
        net.run_steps(steps)
    rt = net.runtime
    gpu_r = [rt.raster(p) for p in net.populations]
    ora_r, events = oracle.run(desc, st, 0, steps)
    gpu_s = [{slot: p.state_tensor(attr).cpu().numpy() for slot, attr in d.state.items()}
             for p, d in zip(net.populations, desc.pops)]
    net.check()
    return gpu_r, ora_r, gpu_s, st, rt.counters(), events


def assert_identical(gpu_r, ora_r, gpu_s, ora_s):
    for k, (g, o) in enumerate(zip(gpu_r, ora_r)):
        if not np.array_equal(g, o):
            bad = np.nonzero((g != o).any(1))[0]
            raise AssertionError(f"population {k}: rasters differ first at step {bad[0]}")
    for k, (g, o) in enumerate(zip(gpu_s, ora_s)):
        for slot, arr in g.items():
            want = getattr(o, slot)
            assert np.array_equal(arr.view(np.uint32) if arr.dtype == np.float32 else arr,
                                  want.view(np.uint32) if want.dtype == np.float32 else want), (k, slot)


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_config0_dsl_matches_oracle(cuda, persistent):
    net, pops = brunel.build(**brunel.CONFIG0, seed=1)
    gr, orr, gs, os_, cnt, ev = run_both(net, 1000, persistent=persistent)
    assert sum(r.sum() for r in gr) > 1000
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev
    assert cnt["spikes"] == sum(int(r.sum()) for r in gr)


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_config1_first_1000_steps_match_oracle(cuda, persistent):
    net, pops = brunel.build(**brunel.CONFIG1, seed=2)
    gr, orr, gs, os_, cnt, ev = run_both(net, 1000, chunk=300, persistent=persistent)
    assert sum(r.sum() for r in gr) > 10000
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev


def test_reference_brunel_fixture_through_c_abi(cuda):
    """The reference loop's raster (tests/golden), reproduced by the library called through its C ABI."""
    g = np.load(GOLDEN / "brunel_reference_c0.npz")
    desc = brunel_golden_desc(g)
    d, c = desc.pops[0], desc.conns[0]
    N, steps = d.n, int(g["steps"])
    dev = cuda
    v = torch.from_numpy(g["V0"].copy()).to(dev)
    ref = torch.zeros(N, dtype=torch.int32, device=dev)
    acc = torch.zeros(d.acc_depth * N, dtype=torch.int64, device=dev)
    words = (N + 31) // 32
    raster = torch.zeros(steps * words, dtype=torch.int32, device=dev)
    table = torch.from_numpy(d.ext_table.view(np.int32).copy()).to(dev)
    ptr = c.ptr.to(dev)
    link = c.link.to(dev)
    w = c.w.to(dev)
    P = (_lib.Population * 1)()
    p = P[0]
    p.model, p.n, p.acc_depth, p.shift, p.ref_steps = _lib.MODEL_LIF_DELTA, N, d.acc_depth, d.shift, d.ref_steps
    p.ext_len, p.seed, p.ext_wfx = len(d.ext_table), d.seed, d.ext_wfx
    for i, x in enumerate(d.p):
        p.p[i] = x
    p.v, p.ref, p.acc, p.ext_table = v.data_ptr(), ref.data_ptr(), acc.data_ptr(), table.data_ptr()
    p.raster, p.raster_steps = raster.data_ptr(), steps
    C = (_lib.Connection * 1)()
    C[0].src, C[0].tgt, C[0].mode, C[0].n_links = 0, 0, _lib.PUSH, c.n_links
    C[0].ptr, C[0].link, C[0].w = ptr.data_ptr(), link.data_ptr(), w.data_ptr()
    lib = _lib.load()
    opt = _lib.Options(block=128, device=0)
    nbytes = ctypes.c_size_t()
    _lib.check(lib.n2b_workspace_bytes(P, 1, C, 1, ctypes.byref(opt), ctypes.byref(nbytes)), "workspace")
    ws = torch.zeros(nbytes.value, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    s = ctypes.c_void_p(stream.cuda_stream)
    h = ctypes.c_void_p()
    torch.cuda.synchronize()
    _lib.check(lib.n2b_create(P, 1, C, 1, ctypes.byref(opt), ctypes.c_void_p(ws.data_ptr()), nbytes.value, s,
                              ctypes.byref(h)), "create")
    try:
        _lib.check(lib.n2b_capture(h, 100, s), "capture")
        _lib.check(lib.n2b_replay(h, steps // 100, s), "replay")
        stream.synchronize()
        got = np.unpackbits(raster.cpu().numpy().view(np.uint8).reshape(steps, words, 4), axis=2,
                            bitorder="little").reshape(steps, -1)[:, :N].astype(bool)
        expected = np.unpackbits(g["raster"], axis=1)[:, :N].astype(bool)
        assert np.array_equal(got, expected)
        st = [oracle.State(N, d.acc_depth, v=g["V0"])]
        oracle.run(desc, st, 0, steps, record=False)
        assert np.array_equal(v.cpu().numpy().view(np.uint32), st[0].v.view(np.uint32))
        np.testing.assert_allclose(v.cpu().numpy(), g["V"][-1], rtol=1e-6, atol=1e-5)
        words_ = (ctypes.c_int32 * _lib.ERR_WORDS)()
        _lib.check(lib.n2b_status(h, words_, _lib.ERR_WORDS, s), "status")
        assert list(words_) == [0] * _lib.ERR_WORDS
    finally:
        lib.n2b_destroy(h)


@pytest.mark.parametrize("mode", ["pull", "mixed"])
def test_pull_matches_push_and_oracle(cuda, mode):
    net, pops = brunel.build(NE=400, NI=100, CE=40, CI=10, delay="uniform", max_delay_steps=12, seed=3)
    conns = net.connections
    modes = {id(c): ("pull" if (mode == "pull" or k % 2 == 0) else "push") for k, c in enumerate(conns)}
    gr, orr, gs, os_, cnt, ev = run_both(net, 600, modes=modes)
    assert [m for m in net.runtime.modes] == [modes[id(c)] for c in conns]
    assert sum(r.sum() for r in gr) > 100
    assert_identical(gr, orr, gs, os_)


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_graph_windows_match_single_steps(cuda, persistent):
    a, _ = brunel.build(**brunel.CONFIG0, seed=4)
    b, _ = brunel.build(**brunel.CONFIG0, seed=4)
    a.persistent = b.persistent = persistent
    a.window, b.window = 50, 10_000
    a.record(730)
    b.record(730)
    a.run_steps(730)  # 14 windows + 30 single steps
    b.run_steps(730)  # 730 single steps
    for pa, pb in zip(a.populations, b.populations):
        assert np.array_equal(a.runtime.raster(pa), b.runtime.raster(pb))
        assert torch.equal(pa.V, pb.V)


def pd14_small(seed=5, per_link=True):
    sizes = [207, 58, 219, 55, 49, 11, 144, 30]
    K = [1600, 1500, 2100, 1900, 2000, 1900, 2900, 2100]
    prob = np.array([[.1009, .1689, .0437, .0818, .0323, 0, .0076, 0], [.1346, .1371, .0316, .0515, .0755, 0, .0042, 0],
                     [.0077, .0059, .0497, .135, .0067, .0003, .0453, 0], [.0691, .0029, .0794, .1597, .0033, 0, .1057, 0],
                     [.1004, .0622, .0505, .0057, .0831, .3726, .0204, 0], [.0548, .0269, .0257, .0022, .06, .3158, .0086, 0],
                     [.0156, .0066, .0211, .0166, .0572, .0197, .0396, .2252], [.0364, .001, .0034, .0005, .0277, .008, .0658, .1443]])
    rng = np.random.Generator(np.random.Philox(key=seed))
    pops = []
    for k, (n, kc) in enumerate(zip(sizes, K)):
        p = PD14_neuron(K_cortical=kc) * n
        p.potential = torch.from_numpy(rng.normal(-58.0, 5.0, n).astype(np.float32))
        p.seed = 100 + k
        pops.append(p)
    for t in range(8):
        for s in range(8):
            if prob[t, s] == 0:
                continue
            c = pops[s] >> fixed_outdegree(min(0.9, prob[t, s] * 30), seed=1000 + 8 * t + s) >> pops[t]
            n_links = c.shape[0]
            w_mean = 0.08781 * (2 if (s, t) == (2, 0) else 1) * (-4 if s % 2 else 1)
            if per_link:
                w = rng.normal(w_mean, abs(w_mean) * 0.1, n_links).astype(np.float32)
                c.weight = torch.from_numpy(np.clip(w, 0, None) if w_mean > 0 else np.clip(w, None, 0))
            else:
                c.weight = w_mean
            d = rng.normal(1.5 if s % 2 == 0 else 0.8, 0.75 if s % 2 == 0 else 0.4, n_links)
            c.delay = torch.from_numpy(np.maximum(d, 0.1).astype(np.float32))
    net = pops[0].network
    return net, pops


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
def test_pd14_small_matches_oracle(cuda, persistent):
    net, pops = pd14_small()
    gr, orr, gs, os_, cnt, ev = run_both(net, 800, chunk=250, persistent=persistent)
    assert sum(r.sum() for r in gr) > 100
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev


@pytest.mark.parametrize("n", [1, 31, 33, 129, 300])
def test_ragged_sizes_and_sources(cuda, n):
    """Sizes off the warp and block grid, a Poisson source population driving them, all-to-all links with
    the deepest delay the ring allows."""
    src = Poisson_source(rate=0.2) * 37
    tgt = LIF(theta=1.0, V_r=0.0, t_ref=0.3, ext_rate=0.5, ext_weight=0.3) * n
    src.seed, tgt.seed = 11, 12
    c = src >> all_to_all() >> tgt
    c.weight = 0.25
    c.delay = torch.from_numpy(np.random.default_rng(n).integers(1, 16, c.shape[0]).astype(np.float32) * 0.1)
    c2 = tgt >> all_to_all() >> tgt
    c2.weight = -0.05
    c2.delay = 1.5  # 15 steps: a ring of 16, its deepest slot
    net = src.network
    net.block = 64
    gr, orr, gs, os_, cnt, ev = run_both(net, 400)
    assert gr[0].sum() > 0 and gr[1].sum() > 0
    assert_identical(gr, orr, gs, os_)


def test_silent_and_saturated_networks(cuda):
    quiet = LIF() * 500  # no drive at all: nothing fires
    c = quiet >> fixed_indegree(10, seed=9) >> quiet
    c.weight = 0.1
    c.delay = 0.2
    gr, orr, gs, os_, cnt, ev = run_both(quiet.network, 200)
    assert cnt["spikes"] == 0 and cnt["events"] == 0
    loud = LIF(theta=0.5, V_r=0.0, t_ref=0.1, ext_rate=50.0, ext_weight=1.0) * 640  # every neuron, every 2nd step
    c = loud >> fixed_indegree(64, seed=10) >> loud
    c.weight = 0.01
    c.delay = 0.1
    gr, orr, gs, os_, cnt, ev = run_both(loud.network, 200)
    assert gr[0].sum() > 0.4 * 640 * 200
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev


def test_barrier_status_is_clean_after_persistent_windows(cuda):
    net, pops = brunel.build(**brunel.CONFIG0, seed=12)
    net.persistent = True
    net.run_steps(2345)
    assert net.runtime.status() == [0] * _lib.ERR_WORDS


def test_counters_count_events(cuda):
    net, pops = brunel.build(**brunel.CONFIG0, seed=6)
    net.run_steps(300)
    c = net.counters()
    assert c["spikes"] == sum(c["per_population"]) > 0
    assert c["events"] > 0
    net.runtime.reset_counters()
    assert net.counters()["events"] == 0


@pytest.mark.parametrize("persistent", [True, False], ids=["persistent", "per-step"])
@pytest.mark.parametrize("grid", [1, 7, 1000])
def test_grid_size_does_not_change_results(cuda, grid, persistent):
    """Far links are shared by however many blocks the launch has (a persistent block looping over several
    tiles when there are fewer blocks than tiles): the same sums for any grid."""
    kw = dict(brunel.CONFIG0, delay="uniform", max_delay_steps=9, seed=8)
    a, _ = brunel.build(**kw)
    b, _ = brunel.build(**kw)
    a.grid = grid
    a.persistent = persistent
    b.persistent = False
    a.record(500)
    b.record(500)
    a.run_steps(500)
    b.run_steps(500)
    assert a.runtime.raster(a.populations[0]).sum() > 0
    for pa, pb in zip(a.populations, b.populations):
        assert np.array_equal(a.runtime.raster(pa), b.runtime.raster(pb))
        assert torch.equal(pa.V, pb.V)
    assert a.counters()["events"] == b.counters()["events"]


def test_pd14_builder_scaled_matches_oracle(cuda):
    """The config-2 builder (explicit Poisson background, per-link normal weights and delays) at 2% size."""
    from naer2_b200.networks import pd14

    net, pops = pd14.build(scale=0.02, seed=3)
    gr, orr, gs, os_, cnt, ev = run_both(net, 600, chunk=250)
    assert sum(r.sum() for r in gr) > 1000
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev


def test_pd14_drawn_on_the_gpu_matches_oracle(cuda):
    """Connectivity, weights and delays drawn on the device (the full-size path), checked at 2% size."""
    from naer2_b200.networks import pd14

    net, pops = pd14.build(scale=0.02, seed=4, device=cuda)
    assert net.connections[0].fabric.topology.target_indices.is_cuda
    gr, orr, gs, os_, cnt, ev = run_both(net, 400)
    assert_identical(gr, orr, gs, os_)
    assert cnt["events"] == ev
