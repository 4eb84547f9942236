"""Failure detection on the device: the cell-count scan's bounded wait.

k_scan_cells is a single-pass scan in which each tile of cells waits for the
tiles before it to publish their prefix. Every such wait is bounded; when it
runs out, the scan records kStatusScanTimeout and the search fails with
"device search failed" where it is waited for, instead of hanging. The test
makes a wait run out on purpose without faulting anything: through
lc_gpu_set_scan_limit one scan tile never publishes (a flag that nothing
sets) and the wait bound is a few dozen loads. A tile whose wait ran out
sums its prefix from the cell counts, so the rows stay exact, and the same
workspace searches normally once the hook is cleared.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _search(L, ws, x, n, cell, k, wait):
    import torch
    nn = torch.full((n, k), -9, dtype=torch.int32, device="cuda")
    d2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k, None, 3.0,
                                nn.data_ptr(), d2.data_ptr(), wait)
    return rc, nn, d2


@pytest.mark.parametrize("mode", [0, 2])
def test_scan_wait_runs_out_and_is_reported(gpu, lib, oracle_mod, mode):
    import torch
    from gpu_helpers import assert_same, lc_cell_of
    from linkcell_b200 import _capi
    box = [90.0, 90.0, 90.0]  # 30^3 = 27,000 cells: seven scan tiles of 4,096
    xyz = np.random.default_rng(8).random((20000, 3)) * 90.0
    want = oracle_mod.knearest(xyz, box, 12, cell_hint=3.0)
    cell = lc_cell_of(box)
    x = torch.as_tensor(xyz, device="cuda")
    ws = lib.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    try:
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        assert lib.lc_gpu_set_scan_limit(ws, 32, 1) == 0  # tile 1 stays silent: tile 2 gives up
        rc, nn, d2 = _search(lib, ws, x, 20000, cell, 12, 1)
        assert rc != 0 and "device search failed" in _capi.gpu_error()
        assert_same((nn.cpu().numpy(), d2.cpu().numpy()), want, "rows after a scan timeout")
        # without a wait, the call is accepted and lc_gpu_wait reports the timeout
        rc, nn, d2 = _search(lib, ws, x, 20000, cell, 12, 0)
        assert rc == 0
        lib.lc_gpu_wait(ws)
        assert "device search failed" in _capi.gpu_error()
        # the hook cleared, the same workspace searches normally
        assert lib.lc_gpu_set_scan_limit(ws, 0, -1) == 0
        rc, nn, d2 = _search(lib, ws, x, 20000, cell, 12, 1)
        assert rc == 0, _capi.gpu_error()
        assert_same((nn.cpu().numpy(), d2.cpu().numpy()), want, "rows after the hook")
    finally:
        lib.lc_gpu_workspace_free(ws)
