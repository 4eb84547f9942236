"""The host-pointer C ABI (lc_knearest*) on the GPU: page-locked output
buffers take the mapped-row path (rows written straight to host memory),
pageable ones the device copy; both must give the reference rows. A fresh
host thread reads LINKCELL_MODE when its workspace is made, so the learned
mode (with the shipped network found beside the library) is checked the
same way."""

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


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("mode", ["0", "2"])
def test_host_abi_pinned_and_pageable_outputs(gpu, lib, oracle_mod, pinned, mode):
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
    old = os.environ.get("LINKCELL_MODE")
    os.environ["LINKCELL_MODE"] = mode
    try:
        rc = _in_thread(lambda: _host_call(lib, xyz, cell, k, nn_p, d2_p))
    finally:
        if old is None:
            os.environ.pop("LINKCELL_MODE", None)
        else:
            os.environ["LINKCELL_MODE"] = old
    assert rc == 0
    got = (nn_t.numpy(), d2_t.numpy()) if pinned else (nn_a, d2_a)
    assert_same(got, want, f"host abi pinned={pinned} mode={mode}")
