"""Regenerate the golden fixtures of this directory from the reference itself.

    python tests/golden/make_golden.py --reference PATH   (or NAER2_REFERENCE=PATH)

Runs only where the reference source tree is available (PATH: the root of
its checkout); the fixtures it writes are committed, and the tests read only
them. What each fixture pins:

brunel_reference_c0.npz
    The reference's time-driven Brunel loop, tools/brunel_reference.py:34-48,
    executed here on CPU from its own source text with these substitutions:
    dev "cpu", dt 0.1, T 100 ms, N_E/N_I 800/200, C_E/C_I 80/20, the
    connectivity (`src`) drawn here (fixed in-degree, no autapses), V0 drawn
    here, and the Poisson counts `torch.poisson(...)` replaced by the counts
    the hot path draws itself (Philox4x32-10 key `seed`, counter
    (j, step, 0, 0), inverted against the fp64 table `table`). Everything
    else -- the delay buffer, refractory test, update, reset, the sparse
    matvec -- is the reference's code as written. Outputs: the spike raster
    (packed bits) and V after every 100 steps.

pd14_neuron.npz
    The PD14 neuron update + send restated in torch by the reference's own
    GPU test, _neuron_reference in test/test_fused_models_gpu.py:32-52,
    extracted from its source and run here on CPU step by step over a fixed
    dt of 0.1 ms, with a per-step input current (count * J) injected as
    `received`. Outputs: the raster and the state after every 10th step.

brunel_longrun_c1.json
    The same loop at config 1's size (N_E/N_I 10,000/2,500, C_E/C_I
    1,000/250) over 10,000 steps of 0.1 ms (1 s), with the reference's own
    connectivity rule (with replacement, autapses kept; drawn here so that the
    oracle can run the same network: longrun_network), its one delay of
    1.5 ms, V0 drawn here, and its own Poisson drive (torch.poisson, torch's
    generator seeded). Its statistics are computed by its own code
    (lines 50-62: rate after 50 ms, CV-ISI over the first 2,000 neurons with
    at least 4 spikes, activity std/mean in 1 ms bins), captured instead of
    printed; plus the loop's wall time on this machine's cores.

refmodel_pd14.npz, refmodel_brunel.npz
    The reference's own neuron models -- PD14_neuron (test/networks/PD14/neuron.py) and Brunel_neuron
    (test/networks/Brunel/neuron.py), imported from their files with `naer2` resolving to this package's DSL
    -- in small networks built here, lowered by this package's transpiler: the plan (naer2_b200.transpiler.
    plan_of: the generated CUDA sources, Params fields and values, pull CSR), the initial state, and the
    rasters and final state of the same networks run by the DSL interpreter (oracle/dsl_interpreter.py,
    which calls the models' own hook functions). PD14_neuron clocked (its DC background, two populations,
    per-link normal weights and delays); Brunel_neuron event-driven at exact spike times (net.exact), driven
    by jittered pacemakers (tests/dsl_models.py) and recurrent links. The GPU test steps the plan where the
    models' files are not, and compares.

philox_triton.json
    tl.randint4x / tl.rand of Triton (the reference's random lowering calls
    tl.rand, naer2/transpiler/transformers/random_lowering_transformer.py:
    74-86) under TRITON_INTERPRET=1 on CPU, for a few seeds and offsets.
"""

from __future__ import annotations

import argparse
import ast
import json
import math
import os
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402  (test infrastructure: the shared Philox counts and tables)
from naer2_b200.poisson import cdf_table  # noqa: E402

SEED_C0 = 0x0C0FFEE
SEED_PD14 = 0x0D14


def _sub(src: str, old: str, new: str) -> str:
    if src.count(old) != 1:
        raise RuntimeError(f"expected exactly one {old!r} in the reference source")
    return src.replace(old, new)


def brunel_c0(reference: pathlib.Path, steps: int = 1000):
    import torch

    NE, NI, CE, CI = 800, 200, 80, 20
    N = NE + NI
    rng = np.random.Generator(np.random.Philox(key=7))
    # fixed in-degree without autapses, per target: CE sources from E, CI from I (with replacement)
    tgt = np.arange(N)
    e_src = rng.integers(0, NE - 1, size=(N, CE))
    e_src += (e_src >= tgt[:, None]) & (tgt[:, None] < NE)
    i_src = rng.integers(0, NI - 1, size=(N, CI))
    i_src += (i_src >= (tgt[:, None] - NE)) & (tgt[:, None] >= NE)
    src = np.concatenate([e_src, NE + i_src], axis=1).astype(np.int64)
    V0 = (rng.random(N, dtype=np.float32) * np.float32(20.0)).astype(np.float32)
    table = cdf_table(2.0)  # lam = C_E nu_ext dt = 2.0 per step at eta 2 (brunel_reference.py:24-25)
    counts = oracle.poisson_counts(table, SEED_C0, 0, steps, N)

    text = (reference / "tools" / "brunel_reference.py").read_text()
    text = text[: text.index("times = torch.cat")]  # the statistics after the loop are not needed
    text = _sub(text, 'dt = float(sys.argv[1]) if len(sys.argv) > 1 else 0.05', "dt = 0.1")
    text = _sub(text, "T = 400.0", f"T = {steps * 0.1!r}")
    text = _sub(text, 'dev = "cuda"', 'dev = "cpu"')
    text = _sub(text, "NE, NI = 10000, 2500", f"NE, NI = {NE}, {NI}")
    text = _sub(text, "CE, CI = 1000, 250", f"CE, CI = {CE}, {CI}")
    text = _sub(text, "src = torch.cat([torch.randint(0, NE, (N, CE), generator=gen), NE + torch.randint(0, NI, "
                      "(N, CI), generator=gen)], 1).flatten()", "src = _golden_src.flatten()")
    text = _sub(text, "V = torch.rand(N, generator=gen).to(dev) * theta", "V = _golden_V0.clone()")
    text = _sub(text, "torch.poisson(torch.full((N,), lam, device=dev))", "_golden_counts[n]")
    text = _sub(text, "torch.cuda.synchronize()", "pass")
    # V every 100 steps, taken inside the loop after the reference's own statements
    text = _sub(text, "        spk_t.append(torch.full((len(idx),), t, device=dev)); spk_i.append(idx)",
                "        spk_t.append(torch.full((len(idx),), t, device=dev)); spk_i.append(idx)\n"
                "    if (n + 1) % 100 == 0:\n        _golden_V.append(V.clone())")
    ns = {"_golden_src": torch.from_numpy(src), "_golden_V0": torch.from_numpy(V0),
          "_golden_counts": torch.from_numpy(counts.astype(np.float32)), "_golden_V": [], "__name__": "golden"}
    exec(compile(text, str(reference / "tools" / "brunel_reference.py"), "exec"), ns)
    raster = np.zeros((steps, N), dtype=bool)
    for t_, idx in zip(ns["spk_t"], ns["spk_i"]):
        n = int(round(float(t_[0]) / 0.1)) - 1  # the reference stamps step n with t = (n + 1) dt
        raster[n, idx.numpy()] = True
    V = np.stack([v.numpy() for v in ns["_golden_V"]]).astype(np.float32)
    np.savez_compressed(HERE / "brunel_reference_c0.npz", src=src.astype(np.int32), V0=V0, seed=np.uint64(SEED_C0),
                        table=table, steps=np.int64(steps), NE=np.int64(NE), NI=np.int64(NI), J=np.float32(0.1),
                        g=np.float32(5.0), delay_steps=np.int64(15), raster=np.packbits(raster, axis=1), V=V)
    print(f"brunel_reference_c0: {raster.sum()} spikes in {steps} steps")


LONGRUN_KEY = 23
LONGRUN = dict(NE=10000, NI=2500, CE=1000, CI=250, delay_steps=15, steps=10000)


def longrun_network(NE: int, NI: int, CE: int, CI: int, key: int = LONGRUN_KEY):
    """(src int64 [N, C_E + C_I], V0 fp32 [N]) of the long-run fixture: per target C_E sources from E and C_I from
    I, uniform with replacement, autapses kept (the reference's rule, tools/brunel_reference.py:20-21);
    V0 uniform in [0, 20) mV. Numpy's Philox under `key`: the test draws the same network."""
    rng = np.random.Generator(np.random.Philox(key=key))
    N = NE + NI
    src = np.concatenate([rng.integers(0, NE, size=(N, CE)), NE + rng.integers(0, NI, size=(N, CI))], axis=1)
    V0 = (rng.random(N, dtype=np.float32) * np.float32(20.0)).astype(np.float32)
    return src.astype(np.int64), V0


def brunel_longrun(reference: pathlib.Path):
    import time

    import torch

    P = LONGRUN
    NE, NI, CE, CI, steps = P["NE"], P["NI"], P["CE"], P["CI"], P["steps"]
    src, V0 = longrun_network(NE, NI, CE, CI)
    text = (reference / "tools" / "brunel_reference.py").read_text()
    text = _sub(text, 'dt = float(sys.argv[1]) if len(sys.argv) > 1 else 0.05', "dt = 0.1")
    text = _sub(text, "T = 400.0", f"T = {steps * 0.1!r}")
    text = _sub(text, 'dev = "cuda"', 'dev = "cpu"')
    text = _sub(text, "src = torch.cat([torch.randint(0, NE, (N, CE), generator=gen), NE + torch.randint(0, NI, "
                      "(N, CI), generator=gen)], 1).flatten()", "src = _golden_src.flatten()")
    text = _sub(text, "V = torch.rand(N, generator=gen).to(dev) * theta", "V = _golden_V0.clone()")
    text = _sub(text, "torch.cuda.synchronize()", "_golden_wall.append(time.time() - t0)")
    text = _sub(text, '    print(f"{name}: rate {rate:.2f} Hz, CV(ISI) {sum(cvs)/len(cvs):.2f}, activity std/mean '
                      '{float(act.std()/act.mean()):.2f}")',
                '    _golden_stats[name] = dict(rate_hz=rate, cv_isi=sum(cvs) / len(cvs), '
                'activity_std_over_mean=float(act.std() / act.mean()), spikes=int(m.sum()))')
    torch.manual_seed(LONGRUN_KEY)  # the reference's torch.poisson draws from torch's default generator
    ns = {"_golden_src": torch.from_numpy(src), "_golden_V0": torch.from_numpy(V0), "_golden_stats": {},
          "_golden_wall": [], "__name__": "golden"}
    exec(compile(text, str(reference / "tools" / "brunel_reference.py"), "exec"), ns)
    spikes = int(sum(len(i) for i in ns["spk_i"]))
    wall = ns["_golden_wall"][0]
    out = {"network": dict(P, key=LONGRUN_KEY, J=0.1, g=5.0, eta=2.0, dt_ms=0.1, autapses=True),
           "stats": ns["_golden_stats"], "loop_wall_s": wall, "spikes": spikes,
           "events_per_s": spikes * (CE + CI) / wall, "torch_threads": torch.get_num_threads(),
           "nproc": os.cpu_count(), "torch": torch.__version__}
    (HERE / "brunel_longrun_c1.json").write_text(json.dumps(out, indent=1))
    print(f"brunel_longrun_c1: {spikes} spikes, {ns['_golden_stats']}, loop {wall:.1f} s")


def _import_reference_model(reference: pathlib.Path, rel: str, cls: str):
    """A model class of the reference, loaded from its file with `import naer2` resolving to this package."""
    import importlib.util

    import naer2_b200

    sys.modules.setdefault("naer2", naer2_b200)
    spec = importlib.util.spec_from_file_location(f"refmodel_{cls}", reference / rel)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return getattr(mod, cls)


def reference_models(reference: pathlib.Path, steps: int = 300):
    import torch

    from naer2_b200.patterns import fixed_indegree
    from naer2_b200.transpiler import plan_of, save_plan
    from oracle import dsl_interpreter
    from tests.dsl_models import JitterPacemaker, Syn

    PD14 = _import_reference_model(reference, "test/networks/PD14/neuron.py", "PD14_neuron")
    Brunel = _import_reference_model(reference, "test/networks/Brunel/neuron.py", "Brunel_neuron")
    g = torch.Generator().manual_seed(31)

    def pd14_net():
        E = PD14(K_cortical=1600) * 240
        I = PD14(K_cortical=1500) * 60
        E.potential = (torch.randn(240, generator=g) * 4.0 - 58.0).float()
        I.potential = (torch.randn(60, generator=g) * 4.0 - 58.0).float()
        for s_, t_, k, w in ((E, E, 40, 0.08781), (E, I, 40, 0.08781), (I, E, 10, -0.35124), (I, I, 10, -0.35124)):
            c = s_ >> fixed_indegree(k, seed=int(torch.randint(0, 1 << 30, (1,), generator=g))) >> t_
            c.weight = (torch.randn(c.shape, generator=g) * abs(w) * 0.1 + w).float()
            c.delay = torch.clamp(torch.randn(c.shape, generator=g) * 0.4 + 1.0, min=0.1).double()
        net = E.network
        net.resolution = 0.1
        return net

    def brunel_net():
        src = JitterPacemaker(period=3) * 80
        tgt = Brunel(tau=10.0, theta=1.0, V_r=0.0, t_ref=0.5) * 120
        c1 = src >> Syn() @ fixed_indegree(8, seed=41) >> tgt
        c1.weight = (0.1 + 0.25 * torch.rand(c1.shape, generator=g)).float()
        c1.delay = (torch.randint(1, 5, c1.shape, generator=g) * 0.1).double()
        c2 = tgt >> Syn() @ fixed_indegree(4, seed=42) >> tgt
        c2.weight = (0.2 * torch.rand(c2.shape, generator=g) - 0.05).float()
        c2.delay = 0.3
        src.phase = torch.randint(0, 3, (80,), generator=g, dtype=torch.int32)
        src.jitter = (0.1 * torch.rand(80, generator=g)).float()
        net = src.network
        net.resolution = 0.1
        net.exact = True
        return net

    for name, make in (("pd14", pd14_net), ("brunel", brunel_net)):
        net = make()
        pops = list(net.populations)
        init = {}
        for k, p in enumerate(pops):
            for a in p.dynamic_attrs:
                init[f"p{k}_{a}_0"] = p.state_tensor(a).detach().cpu().numpy().copy()
        plan = plan_of(net)
        out = dsl_interpreter.run(net, steps)
        rasters, state = out[0], out[1]
        arrays = dict(init)
        for k, p in enumerate(pops):
            arrays[f"p{k}_raster"] = np.packbits(rasters[k], axis=1)
            for a, v in state[k].items():
                arrays[f"p{k}_{a}_end"] = v
        if len(out) > 3:  # exact times: each spike's offset within its step
            for k in range(len(pops)):
                arrays[f"p{k}_offsets"] = out[3][k]
        arrays["steps"] = np.int64(steps)
        save_plan(plan, HERE / f"refmodel_{name}_plan.npz")
        np.savez_compressed(HERE / f"refmodel_{name}.npz", **arrays)
        print(f"refmodel_{name}: spikes per population {[int(r.sum()) for r in rasters]} in {steps} steps")


def _reference_function(path: pathlib.Path, name: str):
    """A top-level function of a reference module, compiled from its source alone (its imports not run)."""
    tree = ast.parse(path.read_text())
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == name)
    mod = ast.Module(body=[fn], type_ignores=[])
    import torch

    ns = {"torch": torch, "math": math}
    exec(compile(mod, str(path), "exec"), ns)
    return ns[name]


def pd14_neuron(reference: pathlib.Path, steps: int = 400, n: int = 256, every: int = 10):
    import torch

    sys.path.insert(0, str(reference))
    try:
        from test.networks.PD14.neuron import PD14_neuron
    finally:
        sys.path.pop(0)
    neuron = PD14_neuron(K_cortical=2100)  # the reference's own class: its parameters and V_rest
    ref_fn = _reference_function(reference / "test" / "test_fused_models_gpu.py", "_neuron_reference")
    rng = np.random.Generator(np.random.Philox(key=11))
    V0 = rng.normal(-58.0, 4.0, n).astype(np.float32)
    I0 = (rng.random(n) * 0.5).astype(np.float32)
    J = np.float32(0.08781)
    table = cdf_table(8e-3 * 2100 * 0.1 * 4.0)  # a strong drive: ~6.7 events a step
    counts = oracle.poisson_counts(table, SEED_PD14, 0, steps, n)
    state = dict(potential=torch.from_numpy(V0), current=torch.from_numpy(I0),
                 t_ref_end=torch.zeros(n), last_time=torch.zeros(n))
    raster = np.zeros((steps, n), dtype=bool)
    Vs, Is = [], []
    for k in range(steps):
        time = float(np.float32((k + 1) * 0.1))
        received = torch.from_numpy(counts[k].astype(np.float32)) * torch.tensor(J)
        state, fires = ref_fn(neuron, state, time, received)
        raster[k] = fires.numpy()
        if (k + 1) % every == 0:
            Vs.append(state["potential"].numpy().copy())
            Is.append(state["current"].numpy().copy())
    np.savez_compressed(HERE / "pd14_neuron.npz", V0=V0, I0=I0, seed=np.uint64(SEED_PD14), table=table,
                        J=J, steps=np.int64(steps), every=np.int64(every), raster=np.packbits(raster, axis=1),
                        V=np.stack(Vs).astype(np.float32), I=np.stack(Is).astype(np.float32),
                        K_cortical=np.int64(2100))
    print(f"pd14_neuron: {raster.sum()} spikes in {steps} steps")


def philox_triton():
    os.environ["TRITON_INTERPRET"] = "1"
    import torch
    import triton
    import triton.language as tl

    @triton.jit
    def kernel(out_ptr, f_ptr, seed, N: tl.constexpr):
        offs = tl.arange(0, N)
        a, b, c, d = tl.randint4x(seed, offs)
        tl.store(out_ptr + offs * 4 + 0, a)
        tl.store(out_ptr + offs * 4 + 1, b)
        tl.store(out_ptr + offs * 4 + 2, c)
        tl.store(out_ptr + offs * 4 + 3, d)
        tl.store(f_ptr + offs, tl.rand(seed, offs))

    cases = []
    for seed in (0, 1, 0x1234567890, 0xDEADBEEF00C0FFEE & 0x7FFFFFFFFFFFFFFF):
        out = torch.zeros(16 * 4, dtype=torch.int32)
        f = torch.zeros(16, dtype=torch.float32)
        kernel[(1,)](out, f, seed, 16)
        words = [[int(x) & 0xFFFFFFFF for x in out[4 * i:4 * i + 4].tolist()] for i in range(16)]
        cases.append({"seed": seed, "offsets": list(range(16)), "words": words,
                      "rand": [float(x) for x in f.tolist()]})
    (HERE / "philox_triton.json").write_text(json.dumps({"triton": triton.__version__, "cases": cases}, indent=1))
    print(f"philox_triton: {len(cases)} seeds x 16 offsets (triton {triton.__version__})")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NAER2_REFERENCE"),
                    help="root of the reference checkout (or the NAER2_REFERENCE environment variable)")
    ap.add_argument("--only", choices=["brunel", "pd14", "philox", "longrun", "refmodels"])
    args = ap.parse_args()
    if not args.reference:
        raise SystemExit("give --reference PATH (or NAER2_REFERENCE): the root of the reference checkout")
    ref = pathlib.Path(args.reference)
    if not ref.exists():
        raise SystemExit(f"the reference tree is not at {ref}: the committed fixtures stand")
    if args.only in (None, "philox"):
        philox_triton()
    if args.only in (None, "brunel"):
        brunel_c0(ref)
    if args.only in (None, "pd14"):
        pd14_neuron(ref)
    if args.only in (None, "longrun"):
        brunel_longrun(ref)
    if args.only in (None, "refmodels"):
        reference_models(ref)


if __name__ == "__main__":
    main()
