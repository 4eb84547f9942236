"""The host-pointer C ABI (lc_knearest*) on the GPU: page-locked output
buffers take the row-range path (each range of rows copied back while the
next is searched) or, with LINKCELL_HOST_ROWS=2, the mapped-row path (rows
written straight to host memory); pageable ones the device copy. All must
give the reference rows. A fresh host thread reads LINKCELL_MODE and
LINKCELL_HOST_ROWS when its workspace is made, so the learned mode (with the
shipped network found beside the library) is checked the same way."""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np
import pytest

from gpu_helpers import assert_same, lc_cell_of

pytestmark = pytest.mark.gpu


def _host_call(L, xyz, cell, k, nn, d2):
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    c = lc_cell_of(cell)
    return L.lc_knearest_d2(ctypes.cast(xyz.ctypes.data, dp), xyz.shape[0], ctypes.byref(c), k,
                            None, 0.0, ctypes.cast(nn, ip), ctypes.cast(d2, dp))


def _in_thread(fn):
    out = {}

    def body():
        out["v"] = fn()
    t = threading.Thread(target=body)
    t.start()
    t.join()
    return out["v"]


def _with_env(env, fn):
    old = {key: os.environ.get(key) for key in env}
    os.environ.update(env)
    try:
        return _in_thread(fn)
    finally:
        for key, v in old.items():
            if v is None:
                os.environ.pop(key, None)
            else:
                os.environ[key] = v


@pytest.mark.parametrize("pinned,rows", [(True, "1"), (True, "2"), (False, "1")])
@pytest.mark.parametrize("mode", ["0", "2"])
def test_host_abi_pinned_and_pageable_outputs(gpu, lib, oracle_mod, pinned, rows, mode):
    import torch
    rng = np.random.default_rng(21)
    n, k = 30000, 16
    cell = np.array([[34.0, 0.0, 0.0], [8.0, 32.0, 0.0], [3.0, 5.0, 33.0]])
    xyz = np.ascontiguousarray(rng.random((n, 3)) @ cell)
    want = oracle_mod.knearest(xyz, cell, k)
    if pinned:
        nn_t = torch.full((n, k), -9, dtype=torch.int32).pin_memory()
        d2_t = torch.zeros((n, k), dtype=torch.float64).pin_memory()
        nn_p, d2_p = nn_t.data_ptr(), d2_t.data_ptr()
    else:
        nn_a = np.full((n, k), -9, dtype=np.int32)
        d2_a = np.zeros((n, k))
        nn_p, d2_p = nn_a.ctypes.data, d2_a.ctypes.data
    # two calls: the first one tunes the walk (whole searches), the second
    # takes the configured host-row path
    for _ in range(2):
        rc = _with_env({"LINKCELL_MODE": mode, "LINKCELL_HOST_ROWS": rows},
                       lambda: [_host_call(lib, xyz, cell, k, nn_p, d2_p) for _ in range(2)])
        assert rc == [0, 0]
    got = (nn_t.numpy(), d2_t.numpy()) if pinned else (nn_a, d2_a)
    assert_same(got, want, f"host abi pinned={pinned} rows={rows} mode={mode}")


@pytest.mark.parametrize("rows", ["1", "2"])
def test_host_abi_many_frames_with_mask_pinned(gpu, lib, oracle_mod, rows):
    """lc_knearest_many (shared cell and mask, three frames) through the
    row-range and mapped paths: masked rows keep -1 / NaN, every frame's
    rows match the reference."""
    import torch
    rng = np.random.default_rng(8)
    n, nf, k = 9000, 3, 12
    cell = np.array([[28.0, 0.0, 0.0], [5.0, 27.0, 0.0], [-3.0, 4.0, 29.0]])
    xyz = np.ascontiguousarray(rng.random((n * nf, 3)) @ cell)
    mask = (rng.random(n) < 0.9).astype(np.int32)
    want = oracle_mod.knearest(xyz, cell, k, mask=mask, n_frames=nf)
    nn_t = torch.full((n * nf, k), -9, dtype=torch.int32).pin_memory()
    d2_t = torch.zeros((n * nf, k), dtype=torch.float64).pin_memory()
    c = lc_cell_of(cell)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)

    def call():
        return [lib.lc_knearest_many(ctypes.cast(xyz.ctypes.data, dp), n, nf, ctypes.byref(c), k,
                                     ctypes.cast(mask.ctypes.data, ip), 0.0,
                                     ctypes.cast(nn_t.data_ptr(), ip),
                                     ctypes.cast(d2_t.data_ptr(), dp)) for _ in range(3)]
    assert _with_env({"LINKCELL_MODE": "2", "LINKCELL_HOST_ROWS": rows}, call) == [0, 0, 0]
    assert_same((nn_t.numpy(), d2_t.numpy()), want, f"many frames rows={rows}")


@pytest.mark.parametrize("pinned", [True, False])
def test_host_batch_heterogeneous_frames(gpu, lib, oracle_mod, pinned):
    """lc_knearest_batch: frames with their own cell, n, k and mask, host
    pointers. With page-locked outputs the rows come back in row ranges that
    cross frame boundaries, where k changes."""
    import torch
    from gpu_helpers import lc_cell_of
    from linkcell_b200 import LcFrame
    from linkcell_b200 import workloads as W
    frames = W.frames_batch(n_frames=12, seed=17, n_min=500, n_max=20000)
    arr = (LcFrame * len(frames))()
    total, moff = 0, 0
    for i, f in enumerate(frames):
        arr[i].n, arr[i].k = len(f["xyz"]), f["k"]
        arr[i].cell = lc_cell_of(f["cell"])
        arr[i].cell_hint = float(f["cell_hint"])
        arr[i].mask_offset = moff
        moff += len(f["xyz"])
        total += len(f["xyz"]) * f["k"]
    assert moff > 2 * 16384  # several row ranges
    xyz = np.ascontiguousarray(np.concatenate([f["xyz"] for f in frames]), dtype=np.float64)
    mask = np.ascontiguousarray(np.concatenate([f["mask"] for f in frames]), dtype=np.int32)
    if pinned:
        nn_t = torch.full((total,), -9, dtype=torch.int32).pin_memory()
        d2_t = torch.zeros((total,), dtype=torch.float64).pin_memory()
        nn_p, d2_p = nn_t.data_ptr(), d2_t.data_ptr()
    else:
        nn_a = np.full(total, -9, dtype=np.int32)
        d2_a = np.zeros(total)
        nn_p, d2_p = nn_a.ctypes.data, d2_a.ctypes.data

    def call():
        return lib.lc_knearest_batch(xyz.ctypes.data, arr, len(frames), mask.ctypes.data, nn_p,
                                     d2_p)
    rc = _in_thread(lambda: [call(), call()])  # the first call tunes the walk
    assert rc == [0, 0], lib.lc_last_error()
    nn, d2 = (nn_t.numpy(), d2_t.numpy()) if pinned else (nn_a, d2_a)
    off = 0
    for i, f in enumerate(frames):
        n, k = len(f["xyz"]), f["k"]
        want = oracle_mod.knearest(f["xyz"], f["cell"], k, mask=f["mask"],
                                   cell_hint=f["cell_hint"])
        got = (nn[off:off + n * k].reshape(n, k), d2[off:off + n * k].reshape(n, k))
        assert_same(got, want, f"host batch pinned={pinned} frame {i}")
        off += n * k
