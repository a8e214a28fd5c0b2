"""The C-ABI library without a GPU: it loads, exports every entry point
include/naer2b.h declares, its structs have the header's layout, and its
host-side validation (n2b_workspace_bytes touches no device) rejects bad
descriptions with the documented codes."""

import ctypes
import pathlib
import re
import subprocess

import pytest

from naer2_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "naer2b.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(n2b_[a-z_]+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 12
    assert set(names) == set(_lib.SIGNATURES)
    for name in names:
        assert hasattr(lib, name), name
    assert lib.n2b_abi_version() == _lib.ABI_VERSION


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    fields = {"n2b_population": [f[0] for f in _lib.Population._fields_],
              "n2b_connection": [f[0] for f in _lib.Connection._fields_],
              "n2b_options": [f[0] for f in _lib.Options._fields_],
              "n2b_bptt_desc": [f[0] for f in _lib.BpttDesc._fields_]}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', 'int main(void) {']
    for s, fs in fields.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fs:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines += ['return 0;', '}']
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for s, cls in (("n2b_population", _lib.Population), ("n2b_connection", _lib.Connection),
                   ("n2b_options", _lib.Options), ("n2b_bptt_desc", _lib.BpttDesc)):
        assert int(out[s]) == ctypes.sizeof(cls), s
        for f in fields[s]:
            assert int(out[f"{s}.{f}"]) == getattr(cls, f).offset, f"{s}.{f}"


def _pop(**kw):
    p = _lib.Population()
    p.model, p.n, p.acc_depth, p.shift = _lib.MODEL_LIF_DELTA, 100, 16, 40
    p.v = p.ref = p.acc = 0x1000  # never dereferenced by the host
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _bytes(pops, conns=(), block=128):
    lib = _lib.load()
    P = (_lib.Population * max(len(pops), 1))(*pops)
    C = (_lib.Connection * max(len(conns), 1))(*conns)
    opt = _lib.Options(block=block, device=0)
    n = ctypes.c_size_t()
    rc = lib.n2b_workspace_bytes(P, len(pops), C, len(conns), ctypes.byref(opt), ctypes.byref(n))
    return rc, n.value, lib.n2b_last_error().decode()


def test_workspace_size_grows_with_the_network():
    rc, small, _ = _bytes([_pop()])
    assert rc == 0 and small > 0 and small % 256 == 0
    rc, big, _ = _bytes([_pop(n=100000)])
    assert rc == 0 and big > small


@pytest.mark.parametrize("kw,msg", [
    (dict(model=9), "unknown model"),
    (dict(acc_depth=12), "power of two"),
    (dict(n=(1 << 24) + 1), "n must be"),
    (dict(shift=63), "shift"),
    (dict(bit_depth=3, bits=0x1000), "bit_depth"),
    (dict(ext_len=4), "ext_table"),
    (dict(raster_steps=10), "raster"),
])
def test_invalid_population_is_rejected(kw, msg):
    rc, _, err = _bytes([_pop(**kw)])
    assert rc == -1 and msg in err


def test_invalid_connection_is_rejected():
    c = _lib.Connection(src=0, tgt=1, mode=_lib.PUSH, n_links=10)
    c.ptr = c.link = 0x1000
    rc, _, err = _bytes([_pop()], [c])
    assert rc == -1 and "out of range" in err
    c.tgt = 0
    c.mode = _lib.PULL  # the source has no spike-bit ring
    rc, _, err = _bytes([_pop()], [c])
    assert rc == -1 and "bit ring" in err
    src = _pop(model=_lib.MODEL_POISSON_SOURCE)
    c2 = _lib.Connection(src=0, tgt=0, mode=_lib.PUSH, n_links=1)
    c2.ptr = c2.link = 0x1000
    rc, _, err = _bytes([src], [c2])
    assert rc == -1 and "takes no input" in err
    rc, _, err = _bytes([_pop()], block=96)
    assert rc == -1 and "block" in err


def test_null_handle_is_an_error_not_a_crash():
    lib = _lib.load()
    assert lib.n2b_step(None, 1, None) == -1
    assert lib.n2b_replay(None, 1, None) == -1
    assert lib.n2b_destroy(None) == 0


def test_projection_and_bptt_entry_points_reject_bad_arguments():
    """Host-side checks of n2b_project_* and n2b_bptt_workspace_bytes, made before any device work (the
    pointers here are never dereferenced)."""
    lib = _lib.load()
    P = 0x1000
    err = lambda: lib.n2b_last_error().decode()  # noqa: E731
    assert lib.n2b_project_forward(P, P, 10, 5, 6, P, P, None) == -1 and "hidden" in err()
    assert lib.n2b_project_forward(P, P, -1, 5, 8, P, P, None) == -1 and "rows" in err()
    assert lib.n2b_project_forward(None, P, 10, 5, 8, P, P, None) == -1 and "missing" in err()
    assert lib.n2b_project_forward(P, P, 10, 5, 8, 0x1004, P, None) == -1 and "aligned" in err()
    assert lib.n2b_project_forward(None, None, 0, 5, 8, None, None, None) == 0  # nothing to do
    assert lib.n2b_project_backward(P, 3, P, P, 5, 10, 2000, P, P, P, None) == -1 and "hidden" in err()
    assert lib.n2b_project_backward(P, 3, None, P, 5, 10, 8, P, P, P, None) == -1 and "missing" in err()
    d = _lib.BpttDesc(batch=12, steps=10, hidden=64, readouts=4, checkpoint=5)
    d.in_ptr = d.out_grp = P
    n = ctypes.c_size_t()
    assert lib.n2b_bptt_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == -1 and "multiple of 8" in err()
    d.batch, d.hidden = 16, 2048
    assert lib.n2b_bptt_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == -1 and "hidden" in err()
    d.hidden = 64
    assert lib.n2b_bptt_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == 0 and n.value > 0
