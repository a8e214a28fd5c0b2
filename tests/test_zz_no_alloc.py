"""n2b_run_static, the entry point that allocates no device memory (its workspace is a fixed array inside the
library), against the handle-based entry points (n2b_create + n2b_capture/n2b_replay/n2b_step on a workspace the
caller allocated) on the same network from the same initial state: two static calls in a row must give the same
spike rasters and the same neuron state, bit for bit, as one run through the handle. The second call only
matches if the first delivered its last step's far links before returning.

Collected last (the file name), so it runs both alone in a fresh process and after the other tests, whose
calls leave other contents in the shared array."""

import ctypes

import numpy as np
import pytest
import torch

from naer2_b200 import _lib
from naer2_b200.networks import brunel, pd14
from naer2_b200.runtime import NetworkRuntime


def _run_handle(net, steps: int, calls: int):
    """The handle path: `calls` runs of `steps` steps; (rasters per call, states per call)."""
    net.record(steps * calls)
    states = []
    for _ in range(calls):
        net.run_steps(steps)
        torch.cuda.synchronize()
        states.append(_state(net))
    rt = net.runtime
    rasters = [rt.raster(p) for p in net.populations]
    net.check()
    per_call = [[r[k * steps:(k + 1) * steps] for r in rasters] for k in range(calls)]
    return per_call, states


def _state(net):
    out = []
    for p in net.populations:
        d = {}
        for attr in p.dynamic_attrs:
            t = p._state.get(attr)
            if t is not None:
                d[attr] = t.detach().cpu().numpy().copy()
        out.append(d)
    return out


def _run_static(net, steps: int, calls: int):
    """The static path: `calls` calls of n2b_run_static over the buffers of a runtime that is never stepped
    (its struct arrays point at this network's state tensors and zeroed arrival rings)."""
    net.record(steps)
    rt = NetworkRuntime(net)
    lib = _lib.load()
    status = (ctypes.c_int32 * _lib.ERR_WORDS)()
    rasters, states = [], []
    try:
        for k in range(calls):
            torch.cuda.synchronize()
            _lib.check(lib.n2b_run_static(rt.cpop, len(rt.pops), rt.cconn, len(rt.desc.conns), ctypes.byref(rt.opt),
                                          k * steps, steps, status, rt._s), "n2b_run_static")
            assert list(status) == [0] * _lib.ERR_WORDS
            rt.stream.synchronize()
            rows = []
            for p, raster, words in zip(rt.pops, rt.rasters, rt.words):
                w = raster[: steps * words].cpu().numpy().view(np.uint32).reshape(steps, words)
                bits = np.unpackbits(w.view(np.uint8).reshape(steps, -1, 4), axis=2, bitorder="little")
                rows.append(bits.reshape(steps, -1)[:, :len(p.shape)].astype(bool))
            rasters.append(rows)
            states.append(_state(net))
    finally:
        rt.close()
    return rasters, states


def _compare(handle, static):
    (hr, hs), (sr, ss) = handle, static
    for call, (a, b) in enumerate(zip(hr, sr)):
        for k, (x, y) in enumerate(zip(a, b)):
            assert np.array_equal(x, y), f"call {call}, population {k}: rasters differ"
    for call, (a, b) in enumerate(zip(hs, ss)):
        for k, (x, y) in enumerate(zip(a, b)):
            for attr in x:
                # tolerance: none -- fixed-point input sums make every path bit-identical
                assert np.array_equal(x[attr].view(np.uint32), y[attr].view(np.uint32)), (call, k, attr)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["brunel_delay15_persistent", "brunel_uniform_per_step", "pd14_small"])
def test_static_entry_matches_handle_on_two_calls(cuda, case):
    steps = 300

    def make():
        if case == "brunel_delay15_persistent":  # every link deferred: the work list carries all deliveries
            net, _ = brunel.build(**brunel.CONFIG0, seed=7)
            net.persistent = True
        elif case == "brunel_uniform_per_step":  # delay-1 links in the step itself, the rest deferred
            net, _ = brunel.build(NE=800, NI=200, CE=80, CI=20, delay="uniform", max_delay_steps=12, seed=8)
            net.persistent = False
        else:  # per-link weights, Poisson background, eight populations
            net, _ = pd14.build(scale=0.02, seed=9, device=cuda)
            net.persistent = True
        return net

    handle = _run_handle(make(), steps, 2)
    static = _run_static(make(), steps, 2)
    assert sum(r.sum() for r in handle[0][1]) > 50  # the second call has spikes to compare
    _compare(handle, static)


def test_static_entry_rejects_networks_beyond_its_scratch():
    """A workspace above N2B_STATIC_SCRATCH_BYTES is refused before any device work (no GPU needed): a push
    connection with deferred links needs one work-list entry per source neuron, 48 bytes each."""
    lib = _lib.load()
    n = 1 << 20  # 1M sources: 48 MiB of work list
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the call stops at the size check
    P = (_lib.Population * 1)()
    P[0].model, P[0].n, P[0].acc_depth, P[0].shift, P[0].ref_steps = _lib.MODEL_LIF_DELTA, n, 16, 40, 20
    P[0].v = P[0].ref = P[0].acc = fake
    C = (_lib.Connection * 1)()
    C[0].src, C[0].tgt, C[0].mode, C[0].n_links = 0, 0, _lib.PUSH, n
    C[0].ptr = C[0].link = C[0].split = fake
    opt = _lib.Options(block=256, device=0)
    nbytes = ctypes.c_size_t()
    _lib.check(lib.n2b_workspace_bytes(P, 1, C, 1, ctypes.byref(opt), ctypes.byref(nbytes)), "workspace")
    assert nbytes.value > _lib.STATIC_SCRATCH_BYTES
    rc = lib.n2b_run_static(P, 1, C, 1, ctypes.byref(opt), 0, 10, None, None)
    assert rc == -4  # N2B_ESPACE
    assert b"static scratch" in lib.n2b_last_error()
    assert lib.n2b_run_static(P, 1, C, 1, ctypes.byref(opt), -1, 10, None, None) == -1  # N2B_EINVAL
