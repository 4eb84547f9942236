"""The allocation-free entry point lc_gpu_knearest_noalloc.

Callers that cannot call cudaMalloc (a host whose pool allocator owns the
device memory, a real-time loop that must not allocate, a plug-in inside a
framework that owns the allocator) use this entry point: all of its scratch
sits in a fixed static device array. Its rows must equal those of the
regular entry point, lc_gpu_knearest_many, on two calls in a row, and it
must refuse searches above its stated limits.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(seed, n, k, rows):
    rng = np.random.default_rng(seed)
    frac = rng.random((n, 3))
    xyz = frac @ np.asarray(rows) + rng.integers(-2, 3, size=(n, 3)) @ np.asarray(rows)
    mask = (rng.random(n) < 0.9).astype(np.int32)
    return xyz, mask


def _noalloc(L, torch, xyz, rows, k, mask, hint):
    from gpu_helpers import lc_cell_of
    x = torch.as_tensor(np.ascontiguousarray(xyz), device="cuda")
    m = torch.as_tensor(mask, device="cuda")
    n = x.shape[0]
    nn = torch.full((n, k), -9, dtype=torch.int32, device="cuda")
    d2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    c = lc_cell_of(rows)
    rc = L.lc_gpu_knearest_noalloc(x.data_ptr(), n, ctypes.byref(c), k, m.data_ptr(), hint,
                                   nn.data_ptr(), d2.data_ptr(), None, 1)
    return rc, nn.cpu().numpy(), d2.cpu().numpy()


def test_noalloc_matches_regular_entry_on_two_calls(gpu, lib):
    import torch
    from gpu_helpers import DeviceRunner, assert_same
    from linkcell_b200 import _capi
    runner = DeviceRunner(mode=0)
    try:
        cases = [
            (11, 20000, 16, [[40.0, 0, 0], [12.0, 38.0, 0], [4.0, 8.0, 39.0]], 3.0),
            (12, 9000, 33, [[30.0, 0, 0], [0, 27.0, 0], [0, 0, 33.0]], 2.5),
        ]
        for seed, n, k, rows, hint in cases:
            xyz, mask = _inputs(seed, n, k, rows)
            rc, nn, d2 = _noalloc(lib, torch, xyz, rows, k, mask, hint)
            assert rc == 0, _capi.gpu_error()
            want = runner.run(xyz, rows, k, mask, hint)
            assert_same((nn, d2), want, f"no-alloc seed {seed}")
    finally:
        runner.close()


def test_noalloc_rejects_sizes_above_its_limits(gpu, lib):
    import torch
    from linkcell_b200 import _capi
    rows = [[400.0, 0, 0], [0, 400.0, 0], [0, 0, 400.0]]
    xyz, mask = _inputs(3, 65537, 4, rows)
    rc, _, _ = _noalloc(lib, torch, xyz, rows, 4, mask, 3.0)
    assert rc != 0 and "65536 points" in _capi.gpu_error()
    xyz, mask = _inputs(4, 100, 65, [[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]])
    rc, _, _ = _noalloc(lib, torch, xyz, [[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]], 65, mask, 3.0)
    assert rc != 0 and "k <= 64" in _capi.gpu_error()
    xyz, mask = _inputs(5, 1000, 4, rows)
    rc, _, _ = _noalloc(lib, torch, xyz, rows, 4, mask, 3.0)  # 133^3 cells
    assert rc != 0 and "65536 cells" in _capi.gpu_error()
