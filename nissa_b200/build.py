"""Build the CUDA library in place: nissa_b200/libtmsolve.so (sm_100a).

    python -m nissa_b200.build [--force]

The library is compiled with nvcc for sm_100a only (B200) and placed next to
this file so that it travels with the source tree.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libtmsolve.so")
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC_FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", "--split-compile", "0"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + sorted(glob.glob(os.path.join(INCLUDE, "*.h")))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in deps())


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu of csrc/ to an object in parallel, then link the shared library."""
    if not force and not stale():
        return LIB
    import concurrent.futures
    import tempfile
    with tempfile.TemporaryDirectory(prefix="tms_build_") as d:
        objs = []
        cmds = []
        for src in sources():
            obj = os.path.join(d, os.path.basename(src) + ".o")
            objs.append(obj)
            cmds.append([nvcc()] + [f for f in NVCC_FLAGS if f != "-shared"] + ["-I" + INCLUDE, "-I" + CSRC, "-c", src,
                                                                               "-o", obj])
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
            for cmd, rc in zip(cmds, ex.map(lambda c: subprocess.call(c), cmds)):
                if verbose:
                    print(" ".join(cmd))
                if rc != 0:
                    raise subprocess.CalledProcessError(rc, cmd)
        tmp = LIB + ".tmp%d" % os.getpid()
        subprocess.check_call([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a"] + objs + ["-o", tmp])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
