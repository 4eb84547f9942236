"""The C++ entry points through a small C++ program
(tests/cpp/batch_driver.cpp) built against include/linkcell_gpu.hpp,
include/linkcell.hpp and the in-tree library.

The CPU test checks that the headers compile and the program links. The GPU
test runs a heterogeneous batch (own cell, n, k, hint and mask per frame)
through linkcell::gpu::Workspace::knearest_into_batch. It then runs the first
frame through Workspace::knearest_into, Workspace::knearest_into_many_dcell
and the host linkcell::knearest, and compares every result with the
oracle."""

from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT

CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIBDIR = os.path.join(ROOT, "linkcell_b200")


def build_driver(out_dir) -> str:
    from linkcell_b200 import build as B
    B.build()
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not on PATH")
    exe = os.path.join(str(out_dir), "batch_driver")
    cmd = [gxx, "-std=c++17", "-O2", "-Wall", "-Werror",
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(CUDA, "include"),
           os.path.join(ROOT, "tests", "cpp", "batch_driver.cpp"),
           "-L" + LIBDIR, "-llinkcell_b200", "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def write_batch(path, frames):
    from gpu_helpers import lc_cell_of
    masks = [f.get("mask") for f in frames]
    mask_parts, moff = [], 0
    with open(path, "wb") as fh:
        mlen = sum(len(m) for m in masks if m is not None)
        np.array([len(frames), mlen], dtype=np.int64).tofile(fh)
        for f, m in zip(frames, masks):
            off = -1
            if m is not None:
                off = moff
                mask_parts.append(np.asarray(m, dtype=np.int32))
                moff += len(m)
            np.array([len(f["xyz"]), f["k"], off], dtype=np.int64).tofile(fh)
            c = lc_cell_of(f["cell"])
            vals = [getattr(c, name) for name, _ in c._fields_]
            np.array(vals + [float(f.get("cell_hint", 0.0))], dtype=np.float64).tofile(fh)
        np.concatenate([np.asarray(f["xyz"], dtype=np.float64).reshape(-1, 3)
                        for f in frames]).tofile(fh)
        if mask_parts:
            np.concatenate(mask_parts).tofile(fh)


def test_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_driver(tmp_path))


@pytest.mark.gpu
def test_cpp_batch_matches_oracle(gpu, oracle_mod, tmp_path):
    from gpu_helpers import assert_same
    from linkcell_b200 import workloads as W
    exe = build_driver(tmp_path)
    frames = W.frames_batch(n_frames=10, seed=29, n_min=40, n_max=2500)
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    write_batch(src, frames)
    r = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    total = sum(len(f["xyz"]) * f["k"] for f in frames)
    r0 = len(frames[0]["xyz"]) * frames[0]["k"]
    raw = np.fromfile(dst, dtype=np.uint8)
    assert raw.size == total * 12 + 3 * r0 * 12
    nn = raw[:total * 4].view(np.int32)
    d2 = raw[total * 4:total * 12].view(np.float64)
    off = 0
    for i, f in enumerate(frames):
        n, k = len(f["xyz"]), f["k"]
        want = oracle_mod.knearest(f["xyz"], f["cell"], k, mask=f.get("mask"),
                                   cell_hint=f.get("cell_hint", 0.0))
        got = (nn[off:off + n * k].reshape(n, k), d2[off:off + n * k].reshape(n, k))
        assert_same(got, want, f"frame {i}")
        off += n * k
    # frame 0 through Workspace::knearest_into, knearest_into_many_dcell and
    # the host linkcell::knearest
    f = frames[0]
    n, k = len(f["xyz"]), f["k"]
    want = oracle_mod.knearest(f["xyz"], f["cell"], k, mask=f.get("mask"),
                               cell_hint=f.get("cell_hint", 0.0))
    pos = total * 12
    for name in ("knearest_into", "knearest_into_many_dcell", "linkcell::knearest"):
        got = (raw[pos:pos + 4 * r0].view(np.int32).reshape(n, k),
               raw[pos + 4 * r0:pos + 12 * r0].view(np.float64).reshape(n, k))
        assert_same(got, want, name)
        pos += 12 * r0
