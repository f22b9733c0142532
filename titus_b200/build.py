"""Build libtitus.so in-tree with nvcc for sm_100a.

    python -m titus_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("titus_api.cu", "titus_noalloc.cu", "titus_adaptive.cu", "titus_adaptive3d.cu", "titus_flux.cu", "titus_pn_full.cu", "titus_pn3d.cu", "titus_tc_probe.cu")]
DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))] + \
    [os.path.join(ROOT, "include", "titus.h")]
TARGET = os.path.join(HERE, "libtitus.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def up_to_date() -> bool:
    if not os.path.exists(TARGET):
        return False
    t = os.path.getmtime(TARGET)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile each translation unit to an object in parallel, then link the .so."""
    if not force and up_to_date():
        return TARGET
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(os.path.basename(src))[0] + ".o")
        cmd = ["nvcc", *compile_flags, "-c", "-o", obj, src]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd)))
        objs.append(obj)
    for cmd, pr in procs:
        if pr.wait() != 0:
            raise subprocess.CalledProcessError(pr.returncode, cmd)
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", TARGET, *objs],
                   check=True)
    return TARGET


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
