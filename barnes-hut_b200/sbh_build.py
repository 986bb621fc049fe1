"""Build recipe of the sbh_b200 CUDA library (sm_100a only).

Compiles every ``csrc/*.cu`` with nvcc into ``libsbh_b200.so`` next to this
file, in-tree, so the built library travels with the source tree:

* ``sbh_compat.cu`` and ``sbh_tree.cu`` carry ``--use_fast_math``, the
  reference's own CUDA flag (CMakeLists.txt:34,39), so that Morton
  quantisation and opening tests of the reference-layout paths round exactly
  like the reference's kernels;
* the native-tree sources are built without it: their quantisation and
  acceptance tests use IEEE operations that the CPU oracle reproduces bit for
  bit, and their fast paths use explicit intrinsics instead.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsbh_b200.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
FAST_MATH_SOURCES = {"sbh_compat.cu", "sbh_tree.cu"}


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[str]:
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _compile(src: str, extra: list[str]) -> str:
    obj = os.path.join(OBJ, src[:-3] + ".o")
    cmd = [_nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + ARCH + COMMON + extra
    if src in FAST_MATH_SOURCES:
        cmd.append("--use_fast_math")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-6000:]}")
    return obj


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", f) for f in
                                                                 os.listdir(os.path.join(ROOT, "include"))]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile (when stale or forced) and link libsbh_b200.so; returns its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    extra = list(extra or [])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra), sources()))
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart", "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB, file=sys.stderr)
    return LIB


def ptxas_report(src: str) -> str:
    """Registers / spills / shared memory per kernel of one source (-Xptxas -v)."""
    cmd = [_nvcc(), "-c", os.path.join(CSRC, src), "-o", os.devnull] + ARCH + COMMON + ["-Xptxas", "-v"]
    if src in FAST_MATH_SOURCES:
        cmd.append("--use_fast_math")
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stderr


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
