"""Build recipe of libnwgr_b200.so (in-tree, sm_100a only).

    python nwgr_b200/build.py            # build if sources are newer
    python nwgr_b200/build.py --force

Run it as a script (or load it by path, as __graft_entry__.build() and the
test suite do): importing the nwgr_b200 package loads the library it builds.

The library is compiled straight with nvcc for sm_100a (no PTX for other
architectures, no JIT cache): every .cu under nwgr_b200/csrc goes into one
shared object with hidden visibility except the extern "C" API of
include/nwg_bfs.h.  The CUDA runtime is linked statically.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libnwgr_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O3",
    "-Xptxas", "-v",
    "-shared",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, *sources(), "-o", LIB + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(PKG, "_build_ptxas.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc failed (exit {res.returncode}); see {log}")
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stdout.write(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)

