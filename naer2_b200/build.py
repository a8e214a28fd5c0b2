"""Build the in-tree CUDA library naer2_b200/libnaer2b.so for sm_100a.

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
SOURCES = [CSRC / "naer2b.cu"]
HEADERS = [CSRC / "n2b_device.cuh", ROOT / "include" / "naer2b.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-O2", "-shared",
         "-cudart", "static", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build naer2_b200")


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compile libnaer2b.so if needed; return its path."""
    if not force and not stale():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-o", str(tmp), *map(str, SOURCES)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    if verbose:
        sys.stdout.write(proc.stdout + proc.stderr)
    os.replace(tmp, LIB)
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
