"""ctypes binding of libnaer2b.so (include/naer2b.h): the structs and entry
points, loaded from the package directory. There is no CPU fallback: a
missing or unloadable library raises."""

from __future__ import annotations

import ctypes
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libnaer2b.so"

ABI_VERSION = 2
MODEL_LIF_DELTA, MODEL_PD14, MODEL_POISSON_SOURCE = 1, 2, 3
PUSH, PULL = 0, 1
ERR_PUSH_LINK, ERR_PULL_LINK, ERR_SPLIT, ERR_ITEMS, ERR_BARRIER, ERR_PULL_STAGE, ERR_WORDS = 0, 1, 2, 3, 4, 5, 8
STATIC_SCRATCH_BYTES = 32 << 20  # N2B_STATIC_SCRATCH_BYTES: the workspace limit of n2b_run_static


class Population(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int32), ("n", ctypes.c_int32), ("acc_depth", ctypes.c_int32),
        ("bit_depth", ctypes.c_int32), ("shift", ctypes.c_int32), ("ref_steps", ctypes.c_int32),
        ("fire_threshold", ctypes.c_uint32), ("ext_len", ctypes.c_int32), ("seed", ctypes.c_uint64),
        ("ext_wfx", ctypes.c_int64), ("p", ctypes.c_float * 8),
        ("v", ctypes.c_void_p), ("i", ctypes.c_void_p), ("ref", ctypes.c_void_p), ("acc", ctypes.c_void_p),
        ("bits", ctypes.c_void_p), ("ext_table", ctypes.c_void_p), ("raster", ctypes.c_void_p),
        ("raster_steps", ctypes.c_int64),
    ]


class Connection(ctypes.Structure):
    _fields_ = [
        ("src", ctypes.c_int32), ("tgt", ctypes.c_int32), ("mode", ctypes.c_int32), ("n_links", ctypes.c_int32),
        ("weight", ctypes.c_float), ("reserved", ctypes.c_int32),
        ("ptr", ctypes.c_void_p), ("link", ctypes.c_void_p), ("w", ctypes.c_void_p), ("split", ctypes.c_void_p),
    ]


class Options(ctypes.Structure):
    _fields_ = [("block", ctypes.c_int32), ("device", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("persistent", ctypes.c_int32), ("reserved", ctypes.c_int32), ("barrier_limit_ns", ctypes.c_int64)]


BPTT_ERR_WORDS = 4  # N2B_BPTT_ERR_WORDS


class BpttDesc(ctypes.Structure):
    _fields_ = [
        ("batch", ctypes.c_int32), ("steps", ctypes.c_int32), ("hidden", ctypes.c_int32),
        ("readouts", ctypes.c_int32), ("checkpoint", ctypes.c_int32), ("smooth", ctypes.c_int32),
        ("nnz", ctypes.c_int32), ("in_cta_max", ctypes.c_int32), ("out_cta_max", ctypes.c_int32),
        ("alpha", ctypes.c_float), ("beta", ctypes.c_float), ("theta", ctypes.c_float), ("slope", ctypes.c_float),
        ("in_ptr", ctypes.c_void_p), ("in_code", ctypes.c_void_p), ("out_grp", ctypes.c_void_p),
        ("out_code", ctypes.c_void_p), ("out_perm", ctypes.c_void_p), ("wait_polls", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


# every entry point include/naer2b.h declares: (name, restype, argtypes)
_P = ctypes.c_void_p
SIGNATURES = {
    "n2b_abi_version": (ctypes.c_int32, []),
    "n2b_last_error": (ctypes.c_char_p, []),
    "n2b_workspace_bytes": (ctypes.c_int, [ctypes.POINTER(Population), ctypes.c_int32, ctypes.POINTER(Connection),
                                           ctypes.c_int32, ctypes.POINTER(Options), ctypes.POINTER(ctypes.c_size_t)]),
    "n2b_create": (ctypes.c_int, [ctypes.POINTER(Population), ctypes.c_int32, ctypes.POINTER(Connection),
                                  ctypes.c_int32, ctypes.POINTER(Options), _P, ctypes.c_size_t, _P,
                                  ctypes.POINTER(_P)]),
    "n2b_step": (ctypes.c_int, [_P, ctypes.c_int64, _P]),
    "n2b_capture": (ctypes.c_int, [_P, ctypes.c_int32, _P]),
    "n2b_replay": (ctypes.c_int, [_P, ctypes.c_int64, _P]),
    "n2b_set_step": (ctypes.c_int, [_P, ctypes.c_int64, _P]),
    "n2b_record": (ctypes.c_int, [_P, ctypes.c_int64, _P]),
    "n2b_status": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P]),
    "n2b_counters": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32, _P]),
    "n2b_reset_counters": (ctypes.c_int, [_P, _P]),
    "n2b_destroy": (ctypes.c_int, [_P]),
    "n2b_bptt_workspace_bytes": (ctypes.c_int, [ctypes.POINTER(BpttDesc), ctypes.POINTER(ctypes.c_size_t)]),
    "n2b_bptt_forward": (ctypes.c_int, [ctypes.POINTER(BpttDesc), _P, _P, _P, ctypes.c_int32, _P, _P, _P,
                                        ctypes.c_size_t, _P]),
    "n2b_bptt_backward": (ctypes.c_int, [ctypes.POINTER(BpttDesc), _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                         ctypes.c_size_t, _P]),
    "n2b_bptt_status": (ctypes.c_int, [ctypes.POINTER(BpttDesc), _P, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_int32), _P]),
    "n2b_bptt_spikes": (ctypes.c_int, [ctypes.POINTER(BpttDesc), _P, ctypes.c_size_t, _P, _P]),
    "n2b_project_forward": (ctypes.c_int, [_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, _P, _P]),
    "n2b_project_backward": (ctypes.c_int, [_P, ctypes.c_int32, _P, _P, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32, _P, _P, _P, _P]),
    "n2b_jit_compile": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p),
                                       ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(_P)]),
    "n2b_jit_launch": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_size_t, _P]),
    "n2b_jit_launch_window": (ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int64, ctypes.c_int64,
                                             ctypes.c_double, _P]),
    "n2b_jit_destroy": (ctypes.c_int, [_P]),
    "n2b_run_static": (ctypes.c_int, [ctypes.POINTER(Population), ctypes.c_int32, ctypes.POINTER(Connection),
                                      ctypes.c_int32, ctypes.POINTER(Options), ctypes.c_int64, ctypes.c_int64,
                                      ctypes.POINTER(ctypes.c_int32), _P]),
}

_lib = None


def load() -> ctypes.CDLL:
    """The library, loaded once with every signature declared; raises if it is missing or its ABI differs."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built: run `python -m naer2_b200.build` (no CPU fallback)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        if lib.n2b_abi_version() != ABI_VERSION:
            raise RuntimeError(f"{LIB_PATH.name} has ABI {lib.n2b_abi_version()}, this package {ABI_VERSION}")
        _lib = lib
    return _lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = load().n2b_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed ({rc}): {msg}")
