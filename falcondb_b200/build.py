"""Build the engine's shared library (CUDA kernels + C++ host) for sm_100a.

The library is built in-tree as ``falcondb_b200/libfalcondb_b200.so`` with nvcc:
every ``csrc/*.cu`` and ``csrc/*.cpp`` is compiled to an object under
``falcondb_b200/_build/`` and linked with the static CUDA runtime, so the .so
depends on no torch or Python symbols.  Objects are rebuilt when a source or any
header is newer than the object.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libfalcondb_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
# Extra nvcc flags (e.g. -D overrides of launch-shape constants for tuning sweeps).
COMMON += os.environ.get("FDB_NVCC_FLAGS", "").split()


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "falcondb_b200.h"]


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    cmd = [NVCC, *COMMON, *ARCH, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"] if verbose else []
    else:
        cmd += ["-x", "cu"]  # host C++ also goes through nvcc (same flags, CUDA headers)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        (BUILD / (src.name + ".ptxas.txt")).write_text(r.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile (if stale) and link the library; return its path."""
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    newest = max(p.stat().st_mtime for p in _headers())
    todo = [s for s in srcs if force or _stale(BUILD / (s.name + ".o"), s, newest)]
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, verbose), todo))
    objs = [BUILD / (s.name + ".o") for s in srcs]
    if todo or not LIB.exists() or force:
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
