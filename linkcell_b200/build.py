"""Builds liblinkcell_b200.so in-tree with nvcc for sm_100a.

Usage: python -m linkcell_b200.build [--verbose]

All CUDA sources and the C ABI go into one shared library next to this file.
Host code is compiled with -ffp-contract=off, because the host cell set-up
must round exactly as the reference Rust code does. Device code keeps FMA
contraction on; the exact FP64 paths use the __d*_rn intrinsics, which are
never contracted. plan.cu, whose cell planner also runs on the device, is
built with -fmad=false.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblinkcell_b200.so")
SOURCES = ["kernels_prep.cu", "kernels_walk.cu", "workspace.cu", "capi.cu", "mlp.cu", "noalloc.cu",
           "neighbors.cu", "plan.cu"]
# plan.cu: the cell planner runs on the host and on the device and must round
# the same way on both, so its device code is built without FMA contraction.
EXTRA = {"plan.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for root in (CSRC, os.path.join(HERE, "..", "include")):
        for name in os.listdir(root):
            if os.path.getmtime(os.path.join(root, name)) > t:
                return True
    return False


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    common = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-I", CSRC, "-I", os.path.join(HERE, "..", "include")]
    if verbose:
        common += ["-Xptxas", "-v"]
    objs = []
    procs = []
    for s in srcs:
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        cmd = [nvcc, *common, *EXTRA.get(s, []), "-c", os.path.join(CSRC, s), "-o", obj]
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        text = out.decode(errors="replace")
        if p.returncode != 0:
            failed.append((s, text))
        elif verbose and text:
            print(f"== {s}\n{text}")
    if failed:
        for s, text in failed:
            sys.stderr.write(f"nvcc failed on {s}:\n{text}\n")
        raise RuntimeError("nvcc build failed")
    link = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-ldl", "-lrt", "-lpthread"]
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
