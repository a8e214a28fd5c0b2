"""The reference's own neuron models through the transpiler: tests/golden/refmodel_*.npz hold the plans that
tests/golden/make_golden.py made from the reference's PD14_neuron (test/networks/PD14/neuron.py, clocked) and
Brunel_neuron (test/networks/Brunel/neuron.py, event-driven at exact times) with this package's transpiler,
and the DSL interpreter's results of the same networks (the models' own hook functions run in Python).

CPU: the plans load, and their generated sources compile with nvcc for sm_100a. GPU: PlannedNetwork steps each
plan on the device (NVRTC-compiled) with no model class present, and must give the interpreter's rasters bit for
bit and its state within float32 rounding of the single-precision math functions (1e-5 relative, 1e-6
absolute, as for the other transpiled models); in the event-driven case also each spike's time within its step
(1e-6)."""

import pathlib
import shutil
import subprocess

import numpy as np
import pytest
import torch

from naer2_b200.transpiler import PlannedNetwork, load_plan

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
CASES = ["pd14", "brunel"]


def _load(case):
    return load_plan(GOLDEN / f"refmodel_{case}_plan.npz"), np.load(GOLDEN / f"refmodel_{case}.npz")


@pytest.mark.parametrize("case", CASES)
def test_reference_model_plans_compile_for_sm100a(tmp_path, case):
    plan, exp = _load(case)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    for k, p in enumerate(plan["pops"]):
        assert p["fields"][0][0] == "step" and any(f == "s_" + a for a in p["attrs"] for f, _ in p["fields"])
        f = tmp_path / f"{case}{k}.cu"
        f.write_text(p["source"])
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c", str(f), "-o",
                        str(tmp_path / f"{case}{k}.o")], check=True, capture_output=True)
    assert plan["pops"][-1]["name"] == {"pd14": "PD14_neuron", "brunel": "Brunel_neuron"}[case]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_reference_models_on_the_gpu_match_the_interpreter(cuda, case):
    plan, exp = _load(case)
    steps = int(exp["steps"])
    states = [{a: torch.from_numpy(exp[f"p{k}_{a}_0"].copy()) for a in p["attrs"]} for k, p in enumerate(plan["pops"])]
    net = PlannedNetwork(plan, states, cuda, record_steps=steps)
    net.run_steps(steps)
    rt = net.runtime
    rt.check()
    for k, (pop, p) in enumerate(zip(net.populations, plan["pops"])):
        want = np.unpackbits(exp[f"p{k}_raster"], axis=1)[:, :p["n"]].astype(bool)
        got = rt.raster(pop)
        if not np.array_equal(got, want):
            bad = np.nonzero((got != want).any(1))[0]
            raise AssertionError(f"{case} population {k}: rasters differ first at step {bad[0]}")
        for a in p["attrs"]:
            have, w = pop.state_tensor(a).cpu().numpy(), exp[f"p{k}_{a}_end"]
            if w.dtype == np.float32:
                np.testing.assert_allclose(have, w, rtol=1e-5, atol=1e-6, err_msg=f"{case} {k}.{a}")
            else:
                assert np.array_equal(have, w), f"{case} {k}.{a}"
        if f"p{k}_offsets" in exp.files:
            times, ids = rt.spike_times(pop)
            st, ids_o = np.nonzero(want)
            np.testing.assert_allclose(times, (st * plan["dt"]).astype(np.float32) + exp[f"p{k}_offsets"][st, ids_o],
                                       rtol=1e-6, atol=1e-6)
    assert sum(int(np.unpackbits(exp[f"p{k}_raster"]).sum()) for k in range(len(plan["pops"]))) > 500
    net.close()
