"""The transpiler on CPU: hook lowering (what each construct becomes, what is refused), the generated source
compiled by nvcc for sm_100a, and the DSL interpreter that checks the compiled kernels on the GPU."""

import ast
import math
import shutil
import subprocess

import numpy as np
import pytest
import torch

import naer2_b200 as n2
from naer2_b200 import receives as r
from naer2_b200.patterns import fixed_indegree
from naer2_b200.transpiler.cuda import HookContext, lower_hook
from naer2_b200.transpiler.template import build_source, hook_context
from oracle import dsl_interpreter
from tests.dsl_models import DecayLIF, Izhikevich, Pacemaker, Syn, TwoPort


def lower(src: str, **ctx) -> str:
    fn = ast.parse(src).body[0]
    base = dict(self_attrs={"v": float, "n": int, "on": bool}, self_static={"tau": 20.0}, time_name="time",
                edge_name="edge", edge_dynamic={"weight"}, edge_static={"gain": 2.0})
    base.update(ctx)
    return lower_hook(fn, HookContext(**base), "test")


def test_lowering_of_statements_and_expressions():
    out = lower("""def h(self, time, edge):
    x = self.v / self.tau
    if x > 1 and not self.on:
        self.v -= x ** 2
    elif x < -1 or self.n % 3 == 1:
        self.n += 1
    else:
        self.on = x >= 0.5
    self.v = math.exp(-time / self.tau) * edge.weight * edge.gain if self.v > 0 else abs(self.v) // 2
    return
""")
    assert "float l_x = 0.f;" in out and "l_x = (float)(((float)(s_v) / (float)(20.0f)));" in out
    assert "((float)(l_x) * (float)(l_x))" in out and "n2_pymod" in out
    assert "s_on = ((((l_x >= 0.5f))) != 0);" in out and "s_n = (int)((s_n + 1.0f));" in out
    assert "expf" in out and "e_weight" in out and "2.0f" in out and "floorf" in out and "break;" in out


@pytest.mark.parametrize("src, what", [
    ("def h(self):\n    for i in range(3):\n        self.v += 1\n", "For"),
    ("def h(self, time, edge, source):\n    self.v = source.v\n", "source"),
    ("def h(self):\n    self.v = print(1)\n", "print"),
    ("def h(self):\n    self.tau = 1.0\n", "not a dynamic attribute"),
    ("def h(self):\n    self.v = self.w\n", "self.w"),
])
def test_unsupported_constructs_are_refused(src, what):
    with pytest.raises(NotImplementedError, match=what):
        lower(src, source_name="source")


def _source_of(pop, incoming):
    node = pop.node
    hooks = {"update": (node.update.ast, hook_context(pop, node.update)),
             "send": (node.send.ast, hook_context(pop, node.send))}
    return build_source(type(pop.instance).__name__, dict(pop.dynamic_attrs), hooks, incoming)


@pytest.mark.skipif(shutil.which("nvcc") is None and not __import__("os").path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not found")
def test_generated_sources_compile_for_sm100a(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    from naer2_b200.networks.brunel import TranspiledLIF

    pops = [Izhikevich() * 40, DecayLIF() * 40, TwoPort() * 40, TranspiledLIF(ext_rate=20.0, ext_weight=0.1) * 40]
    for k, p in enumerate(pops):
        incoming = []
        for port, hook in p.node.receive.items():
            dyn = ["weight"] if "weight" in ast.unparse(hook.ast) else []
            stat = {"gain": 1.5} if "gain" in ast.unparse(hook.ast) else {}
            incoming.append({"receive": (hook.ast, hook_context(p, hook, dyn, stat, site_base=32 * len(incoming))),
                             "edge_dynamic": dyn})
        for exact in (False, True):
            node = p.node
            hooks = {"update": (node.update.ast, hook_context(p, node.update)),
                     "send": (node.send.ast, hook_context(p, node.send))}
            src, fields = build_source(type(p.instance).__name__, dict(p.dynamic_attrs), hooks, incoming, exact)
            f = tmp_path / f"k{k}{int(exact)}.cu"
            f.write_text(src)
            subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c", str(f), "-o",
                            str(tmp_path / f"k{k}{int(exact)}.o")], check=True, capture_output=True)


def test_interpreter_runs_a_small_network():
    src = Pacemaker(period=5) * 8
    tgt = DecayLIF(theta=0.25) * 6
    c = src >> Syn(weight=0.3) @ fixed_indegree(3, seed=2) >> tgt
    c.delay = 0.2
    src.phase = torch.arange(8, dtype=torch.int32)
    net = src.network
    net.resolution = 0.1
    rasters, state, _ = dsl_interpreter.run(net, 30)
    assert rasters[0].sum() == sum(((np.arange(8) + n + 1) % 5 == 0).sum() for n in range(30))
    assert rasters[1].sum() > 0 and (state[1]["v"] < 0.25).all()


def test_edge_hooks_lower_and_refuse_the_source():
    from tests.dsl_models import PairSTDP, TraceLIF

    tgt = TraceLIF() * 4
    src = Pacemaker() * 4
    c = src >> PairSTDP() @ fixed_indegree(2, seed=1) >> tgt
    from naer2_b200.transpiler.runtime import EdgePlan
    from naer2_b200.transpiler.template import edge_hook_context

    plan = EdgePlan(c, tgt.node.receive["receive"])
    assert plan.per_link == ["t_last", "weight", "x_pre"] and plan.written == ["t_last", "weight", "x_pre"]
    assert plan.static["tau_pre"] == 2.0 and plan.forward is not None and plan.backward is not None
    out = lower_hook(plan.forward.ast, edge_hook_context(tgt, plan.forward, plan.per_link, plan.static), "fwd")
    assert "e_x_pre = " in out and "s_y_post" in out and "e_weight = " in out
    bad = ast.parse("def forward(self, time, src):\n    x = src.v\n").body[0]
    ctx = HookContext(time_name="time", source_name="src", roots={}, random=False)
    with pytest.raises(NotImplementedError, match="sending neuron"):
        lower_hook(bad, ctx, "fwd")


def test_clocked_kernel_geometry_by_population_size():
    """The clocked intake's threads per neuron (scan(n)): 32 for populations of at most 4,096 neurons, else 8;
    the block (32 neurons) stays within 1,024 threads and the arrival lists within LIST_WORDS, as the generated
    source states them."""
    from naer2_b200.transpiler.template import LIST_WORDS, NPB_C, scan

    for n, want in ((1, 32), (4096, 32), (4097, 8), (10000, 8)):
        assert scan(n) == want
        pop = DecayLIF() * 8
        node = pop.node
        hooks = {"update": (node.update.ast, hook_context(pop, node.update)),
                 "send": (node.send.ast, hook_context(pop, node.send))}
        inc = [{"receive": (node.receive["receive"].ast, hook_context(pop, node.receive["receive"], ["weight"], {})),
                "edge_dynamic": ["weight"]}]
        src, _ = build_source("DecayLIF", dict(pop.dynamic_attrs), hooks, inc, exact=False, n=n)
        cap = LIST_WORDS // (NPB_C * want)
        assert f"__launch_bounds__({want * NPB_C})" in src and want * NPB_C <= 1024
        assert f"constexpr int SCAN = {want}, NPB_C = {NPB_C}, CAP = {cap};" in src and cap >= 4


def test_transpiled_lif_thresholds_are_the_poisson_cdf():
    """TranspiledLIF counts external events by comparing one uniform with P(count <= k), k < 12: the counts of
    many uniforms have the Poisson mean and variance of ext_rate dt."""
    from naer2_b200.networks.brunel import POISSON_TERMS, TranspiledLIF

    m = TranspiledLIF(ext_rate=20.0, ext_weight=0.1, dt=0.1)
    c = np.array([getattr(m, f"c{k}") for k in range(POISSON_TERMS)])
    lam = 2.0
    k = np.arange(POISSON_TERMS)
    cdf = np.cumsum(np.exp(-lam) * lam ** k / np.array([math.factorial(int(i)) for i in k]))
    np.testing.assert_allclose(c, cdf, rtol=1e-6)
    u = np.random.default_rng(1).random(400_000)
    counts = (u[:, None] > c[None, :]).sum(1)
    assert abs(counts.mean() - lam) < 0.01 and abs(counts.var() - lam) < 0.02
