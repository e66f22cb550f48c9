"""Build libgdock.so (the sm_100a kernels and the C ABI) in-tree with nvcc.

The library is built next to this file, so it travels with the source tree;
object files go to geauxdock_b200/_build/.  Sources are compiled in parallel
and only when they (or a header) changed.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgdock.so"
# the bounds-checking build: the kernel source compiled with -DGD_CHECK (test use)
CHECK_LIB = PKG / "libgdock_check.so"
CHECK_SRC = "gd_mc.cu"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "-I", str(ROOT / "include"), "-I", str(CSRC)]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list[str]:
    # the system g++ (an unrelated compiler wrapper may be first in $CXX)
    return ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, obj: Path, verbose: bool, extra: tuple = ()) -> None:
    cmd = [_nvcc(), *_host_cxx(), *ARCH, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every CUDA source for sm_100a and link libgdock.so (and the
    bounds-checking libgdock_check.so); returns the product library's path."""
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hm = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or not o.exists() or o.stat().st_mtime < max(s.stat().st_mtime, hm):
            todo.append((s, o))
    chk = BUILD / (Path(CHECK_SRC).stem + "_check.o")
    chk_src = CSRC / CHECK_SRC
    chk_todo = force or not chk.exists() or chk.stat().st_mtime < max(chk_src.stat().st_mtime, hm)
    jobs = [(s, o, ()) for s, o in todo] + ([(chk_src, chk, ("-DGD_CHECK",))] if chk_todo else [])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(lambda j: _compile(j[0], j[1], verbose, j[2]), jobs))
    check_objs = [chk if o.stem == Path(CHECK_SRC).stem else o for o in objs]
    for lib, ob, stale in ((LIB, objs, bool(todo)), (CHECK_LIB, check_objs, bool(todo) or chk_todo)):
        if force or stale or not lib.exists():
            cmd = [_nvcc(), *_host_cxx(), *ARCH, "-shared", "-o", str(lib), *map(str, ob)]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
