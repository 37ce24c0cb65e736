"""In-tree build of the CUDA library ``_lib/libparflexdtw_b200.so``.

    python -m parflexdtw_b200.build [--verbose]

nvcc compiles every ``csrc/*.cu`` for sm_100a (B200), one object per source
file in parallel (``_build/``), and links them into one shared library
exposing the C ABI declared in ``include/parflexdtw_b200.h``.  The library is
built next to the package so that it travels with the source tree; nothing is
installed into site-packages.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "_lib")
LIB_NAME = "libparflexdtw_b200.so"
LIB_PATH = os.path.join(LIB_DIR, LIB_NAME)
OBJ_DIR = os.path.join(PKG, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def _compile(src: str, obj: str, verbose: bool) -> None:
    cmd = [nvcc_path(), *ARCH, "-lineinfo", "-O3", "-std=c++17",
           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(obj + ".tmp", obj)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every csrc/*.cu into its own object (in parallel, objects in
    _build/ next to the sources) and links them into the library."""
    if not force and not _stale():
        return LIB_PATH
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    heads = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    newest_head = max((os.path.getmtime(h) for h in heads), default=0.0)
    jobs = []
    for src in sources():
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
        if (force or not os.path.exists(obj) or
                os.path.getmtime(obj) < max(os.path.getmtime(src), newest_head)):
            jobs.append((src, obj))
    if jobs:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
            for f in [ex.submit(_compile, s, o, verbose) for s, o in jobs]:
                f.result()
    tmp = LIB_PATH + ".tmp"
    objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + ".o") for s in sources()]
    subprocess.check_call([nvcc_path(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv or "--verbose" in sys.argv,
                verbose="--verbose" in sys.argv))
