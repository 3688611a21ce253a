"""Compile libafqmc_b200.so for sm_100a with nvcc (in-tree, no JIT cache).

    python -m ad_afqmc_b200.build          # incremental
    python -m ad_afqmc_b200.build --force  # rebuild everything

Objects go to ad_afqmc_b200/_build/, the library to ad_afqmc_b200/lib/.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libafqmc_b200.so")
LIB_CHECKS = os.path.join(LIBDIR, "libafqmc_b200_checks.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-fmad=true",
         "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the sm_100a library cannot be built")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src: str, force: bool, checks: bool = False) -> str:
    bdir = BUILD + ("_checks" if checks else "")
    obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= _deps_mtime():
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, *(["-DAFQ_CHECKS"] if checks else []), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False, checks: bool = False) -> str:
    """Build the library; ``checks`` builds the debug variant
    (libafqmc_b200_checks.so, -DAFQ_CHECKS: host pointers rejected before any
    launch, out-of-range GEMM tiles reported as AFQ_ERR_BOUNDS), which
    ``_lib`` loads when the environment sets AFQ_CHECKS=1."""
    bdir = BUILD + ("_checks" if checks else "")
    lib_path = LIB_CHECKS if checks else LIB
    os.makedirs(bdir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, checks), srcs))
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(lib_path) or os.path.getmtime(lib_path) < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib_path, *objs, "-cudart=static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    if verbose:
        print(lib_path)
    return lib_path


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, checks="--checks" in sys.argv)
