"""Build the in-tree CUDA libraries for sm_100a: naer2_b200/libnaer2b.so (the hot path and its C ABI) and
naer2_b200/libn2b_peak.so (the L2 atomic throughput measurement bench.py reports against).

    python -m naer2_b200.build          # compile if a source is newer than the library
    python -m naer2_b200.build --force  # always compile

nvcc cross-compiles without a GPU. The library links the CUDA runtime
statically, so it loads next to PyTorch's own runtime on any box with the
driver; it is built in the package directory (not a JIT cache) so that it
travels with the source tree.
"""

import argparse
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libnaer2b.so"
SOURCES = [CSRC / "naer2b.cu", CSRC / "bptt.cu", CSRC / "jit.cu"]
HEADERS = [CSRC / "n2b_device.cuh", ROOT / "include" / "naer2b.h"]
PEAK_LIB = HERE / "libn2b_peak.so"
PEAK_SOURCES = [CSRC / "l2_peak.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-O2", "-shared",
         "-cudart", "static", "-Xptxas", "-v", "-ldl"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build naer2_b200")


def stale(lib=LIB, sources=None, headers=None) -> bool:
    sources = SOURCES if sources is None else sources
    headers = HEADERS if headers is None else headers
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources + headers)


def _compile(lib, sources, verbose: bool) -> None:
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-o", str(tmp), *map(str, sources)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    if verbose:
        sys.stdout.write(proc.stdout + proc.stderr)
    os.replace(tmp, lib)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile libnaer2b.so and libn2b_peak.so if needed; return libnaer2b.so's path."""
    if force or stale():
        _compile(LIB, SOURCES, verbose)
    if force or stale(PEAK_LIB, PEAK_SOURCES, []):
        _compile(PEAK_LIB, PEAK_SOURCES, verbose)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--quiet", action="store_true")
    args = ap.parse_args(argv)
    path = build(force=args.force, verbose=not args.quiet)
    print(path)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
