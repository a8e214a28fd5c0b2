"""The DSL and host-side logic on CPU (the reference's unit/ and test/ integration areas: decorators and
hooks, the connection chain, patterns and topology, delays, the kernels' description of a network)."""

import math

import numpy as np
import pytest
import torch

import naer2_b200 as n2
from naer2_b200 import receives as r
from naer2_b200.models import LIF, PD14_neuron, Poisson_source, params_of
from naer2_b200.networks import brunel
from naer2_b200.patterns import all_to_all, fixed_indegree, fixed_outdegree, one_to_one
from naer2_b200.runtime import describe, fixed_shift, next_pow2
from naer2_b200.topology import Topology, delay_steps, pull_form, pull_split_form, push_form
from naer2_b200.types import IndexBox, Points, Region


@n2.node
class Relay:
    def __init__(self):
        self.x: float = 0.0

    def update(self, time: n2.time):
        pass

    def send(self, time: n2.time):
        pass

    def receive(self, time: n2.time, edge: r.edge, source: r.source):
        self.x += edge.weight


@n2.edge
class Static:
    def __init__(self, weight: float):
        self.weight = weight

    def forward(self):
        pass

    def backward(self):
        pass


@n2.pattern
def every_other(position: n2.Position, source_region: n2.Region, target_region=None):
    """Targets 0, 2, 4, ... of a flat target region."""
    n = len(target_region)
    return Points(torch.arange(0, n, 2, dtype=torch.int64).unsqueeze(1))


def test_hook_verification():
    class Bad:
        def update(self, time: int):
            pass

    with pytest.raises(TypeError):
        n2.node(type("B", (), {"update": Bad.update, "send": Bad.update, "receive": Bad.update}))

    class Unannotated:
        def update(self, t):
            pass

    with pytest.raises(TypeError):
        n2.node(type("U", (), {"update": Unannotated.update, "send": Unannotated.update,
                              "receive": Unannotated.update}))
    with pytest.raises(ValueError):
        n2.node(42)


def test_population_and_dynamic_attrs():
    p = Relay() * 10
    assert isinstance(p, n2.Population) and len(p) == 10
    assert set(p.dynamic_attrs) == {"x"}
    assert torch.equal(p.x, torch.zeros(10))
    p.x = 2.0
    assert torch.equal(p.x, torch.full((10,), 2.0))
    p.x = torch.arange(10.0)
    assert p.x[3] == 3.0
    with pytest.raises(ValueError):
        p.x = torch.zeros(3)
    q = LIF() * 5
    assert q.ref.dtype == torch.int32 and q.V.dtype == torch.float32


def test_connection_chain_forms():
    a, b = Relay() * 6, Relay() * 8
    c1 = a >> Static(0.5) @ every_other >> b
    assert c1.shape == (6 * 4,) and c1.fabric.instance.weight == 0.5
    c2 = a >> every_other >> b
    c2.weight = torch.ones(c2.shape)
    c3 = a >> Static(0.1) @ "receive" @ every_other >> b
    assert c3._target_port == "receive"
    assert a.network is b.network and len(a.network.connections) == 3
    assert a.network.populations == [a, b]  # creation order
    with pytest.raises(ValueError):
        a >> Static(0.1) @ "nope" @ every_other >> b
    with pytest.raises(ValueError):
        c2.not_read_by_receive = 1.0  # the receive hook reads edge.weight only
    with pytest.raises(ValueError):
        a >> every_other >> b @ {"weight": "w"}  # needs parentheses


def test_connection_mapping_renames_edge_attrs():
    a, b = Relay() * 3, Relay() * 3
    c = (a >> Static(0.2) @ one_to_one() >> b) @ {"w": "weight"}  # edge attr w read as edge.weight
    c.w = 0.7
    assert c.fabric.w == 0.7


def test_delay_setting_and_steps():
    a, b = Relay() * 4, Relay() * 4
    c = a >> all_to_all() >> b | 1.5
    assert c.fabric.delay == 1.5
    c.delay = torch.full(c.shape, 0.3)
    assert delay_steps(c.fabric.value("delay"), 16, 0.1).tolist() == [3] * 16
    assert delay_steps(0.01, 3, 0.1).tolist() == [1, 1, 1]  # at least one step
    assert delay_steps(torch.tensor([0.05, 0.15, 0.25]), 3, 0.1).tolist() == [1, 2, 2]  # half to even
    with pytest.raises(ValueError):
        delay_steps(30.0, 1, 0.1)  # 300 steps: beyond the link word's 8-bit delay
    with pytest.raises(ValueError):
        c.delay = torch.ones(3)


def test_fixed_indegree_without_autapses():
    e = LIF() * 300
    c = e >> fixed_indegree(25, autapses=False, seed=3) >> e
    t = c.fabric.topology
    off, tgt = t.source_offsets.numpy(), t.target_indices.numpy()
    src = np.repeat(np.arange(300), np.diff(off))
    assert (np.bincount(tgt, minlength=300) == 25).all()
    assert not (src == tgt).any()
    for s in range(300):  # rows ordered by target
        row = tgt[off[s]:off[s + 1]]
        assert (np.diff(row) >= 0).all()
    e2 = LIF() * 300
    c2 = e2 >> fixed_indegree(25, autapses=False, seed=3) >> e2
    assert torch.equal(c2.fabric.topology.target_indices, t.target_indices)  # seeded


def test_fixed_outdegree_follows_the_reference_rule():
    a, b = LIF() * 200, LIF() * 300
    c = a >> fixed_outdegree(0.1, seed=5) >> b
    Q = math.log(1 - 0.1) / math.log(1 - 1 / (200 * 300))
    k = round(Q / 200)
    assert len(c.fabric.topology) == 200 * k
    assert (np.diff(c.fabric.topology.source_offsets.numpy()) == k).all()


def test_per_position_patterns_match_bulk_links():
    pat = fixed_indegree(4, seed=11)
    src = Region(20)
    offsets, targets = pat.links(20, 30)
    pat2 = fixed_indegree(4, seed=11)
    rows = [pat2(pos, src, Region(30)).coords[:, 0].numpy() for pos in src]
    assert np.array_equal(np.concatenate(rows), targets)
    topo = Topology.build(every_other, Region(5), Region(9))
    assert len(topo) == 5 * 5 and topo.target_indices[:5].tolist() == [0, 2, 4, 6, 8]


def test_region_types():
    box = Region((3, 4))
    assert isinstance(box, IndexBox) and len(box) == 12 and isinstance(box, Region)
    assert box.position_at(5).coords.tolist() == [1, 1]
    pts = Points(torch.tensor([[1.0, 2.0], [3.0, 4.0]]))
    assert len(pts) == 2 and isinstance(pts, Region)
    assert Region(box) is box


def test_push_and_pull_forms():
    topo = Topology(torch.tensor([0, 3, 5, 5]), torch.tensor([2, 0, 1, 2, 0]))
    steps = np.array([3, 1, 2, 1, 4])
    ptr, link, perm, split = push_form(topo, torch.from_numpy(steps), 3)
    assert ptr.tolist() == [0, 3, 5, 5]
    word = link.to(torch.int64) & 0xFFFFFFFF
    d, t = (word >> 24).tolist(), (word & 0xFFFFFF).tolist()
    assert d == [1, 3, 2, 1, 4] and t == [0, 2, 1, 2, 0]  # delay-1 links first within each row
    assert split.tolist() == [1, 4, 5]
    assert perm.tolist() == [1, 0, 2, 3, 4]
    pptr, plink, pperm = pull_form(topo, torch.from_numpy(steps), 3)
    assert pptr.tolist() == [0, 2, 3, 5]
    assert (plink & 0xFFFFFF).tolist() == [0, 1, 0, 0, 1]  # sources, target order, canonical order within
    assert pperm.tolist() == [1, 4, 2, 0, 3]
    with pytest.raises(ValueError):
        push_form(topo, torch.from_numpy(steps), 2)  # a target outside the population
    # the split pull form: every target's delay-1 links, then every target's delay >= 2 links
    sptr, slink, sperm, fptr = pull_split_form(topo, torch.from_numpy(steps), 3)
    assert sptr.tolist() == [0, 1, 1, 2] and fptr.tolist() == [2, 3, 4, 5]
    sw = slink.to(torch.int64) & 0xFFFFFFFF
    assert (sw >> 24).tolist() == [1, 1, 4, 2, 3] and (sw & 0xFFFFFF).tolist() == [0, 1, 1, 0, 0]
    assert sperm.tolist() == [1, 3, 4, 2, 0]
    assert sorted(sperm.tolist()) == list(range(5))


def test_describe_brunel():
    net, pops = brunel.build(**brunel.CONFIG0, seed=1)
    d = describe(net)
    assert [p.n for p in d.pops] == [800, 200]
    for p in d.pops:
        assert p.acc_depth == 16 and p.ref_steps == 20 and p.shift == 40
        assert p.p[0] == float(np.float32(math.exp(-0.1 / 20)))
        assert len(p.ext_table) > 10 and p.ext_wfx == int(np.ldexp(np.float32(0.1), 40))
    assert [c.mode for c in d.conns] == ["push"] * 4
    assert all(c.w is None for c in d.conns)  # single-weight connections carry no weight array
    assert d.n_links == 1000 * 100
    assert all(torch.equal(c.split, c.ptr[:-1]) for c in d.conns)  # delay 15: no delay-1 link


def test_describe_pd14_and_sources():
    a = PD14_neuron(K_cortical=2000) * 50
    s = Poisson_source(0.05) * 10
    c = s >> all_to_all() >> a
    c.weight = torch.linspace(0.01, 0.2, c.shape[0])
    c.delay = 0.25
    net = a.network
    d = describe(net)
    pa, ps = d.pops
    assert pa.ref_steps == 19 and pa.acc_depth == 4
    P_V = math.exp(-0.1 / 10.0)
    assert pa.p[0] == float(np.float32(P_V)) and pa.p[3] == -65.0
    assert ps.fire_threshold == int(math.floor((1 - math.exp(-0.005)) * 2 ** 32))
    assert d.conns[0].w is not None and len(d.conns[0].w) == 500
    w = c.fabric.value("weight").numpy()  # (describe's weights: the same values, as a tensor)
    tgt = c.fabric.topology.target_indices.numpy()
    max_in = np.bincount(tgt, weights=np.abs(w.astype(np.float64)), minlength=50).max()
    assert pa.shift == fixed_shift(max_in + 0.08781 * (len(pa.ext_table) - 1))


def test_fixed_point_shift_and_depth_helpers():
    assert next_pow2(16) == 16 and next_pow2(17) == 32 and next_pow2(1) == 1
    assert fixed_shift(1000.0) == 40  # min(40, 61 - 10)
    assert fixed_shift(2.0 ** 40) == 21
    assert fixed_shift(0.0) == 40


def test_user_models_need_the_transpiler():
    p = Relay() * 3
    with pytest.raises(NotImplementedError):
        params_of(p, 0.1)


def test_no_cpu_fallback():
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    net, _ = brunel.build(**brunel.CONFIG0)
    with pytest.raises(RuntimeError, match="CUDA"):
        net.step(1.0)


def test_step_length_must_be_whole_steps():
    net, _ = brunel.build(**brunel.CONFIG0)
    assert net.steps_for(1.5) == 15
    with pytest.raises(ValueError):
        net.steps_for(0.15 + 0.01)
