"""lc_gpu_neighbors_within: the n x k rows of a search filtered by a cutoff
into CSR on the device, checked against the same filter in numpy over the
reference rows."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from gpu_helpers import lc_cell_of

pytestmark = pytest.mark.gpu


def _csr_numpy(nn, d2, cutoff):
    keep = (nn >= 0) & (d2 <= cutoff * cutoff)
    counts = keep.sum(axis=1)
    row_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return row_ptr, nn[keep], d2[keep]


@pytest.mark.parametrize("cutoff", [0.0, 2.5, 4.0, 1e9])
def test_csr_matches_numpy_filter(gpu, lib, oracle_mod, cutoff):
    import torch
    rng = np.random.default_rng(13)
    n, k = 20000, 16
    cell = np.array([[30.0, 0.0, 0.0], [6.0, 29.0, 0.0], [2.0, -4.0, 31.0]])
    xyz = rng.random((n, 3)) @ cell
    xyz[:50] = xyz[50:100]  # exact duplicates: zero distances
    mask = (rng.random(n) < 0.9).astype(np.int32)
    want_nn, want_d2 = oracle_mod.knearest(xyz, cell, k, mask=mask)
    ws = lib.lc_gpu_workspace_new()
    try:
        x = torch.as_tensor(xyz, device="cuda")
        m = torch.as_tensor(mask, device="cuda")
        nn = torch.empty((n, k), dtype=torch.int32, device="cuda")
        d2 = torch.empty((n, k), dtype=torch.float64, device="cuda")
        c = lc_cell_of(cell)
        torch.cuda.synchronize()
        assert lib.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(c), k, m.data_ptr(),
                                        0.0, nn.data_ptr(), d2.data_ptr(), 1) == 0
        rp_w, col_w, dist_w = _csr_numpy(want_nn, want_d2, cutoff)
        cap = n * k
        row_ptr = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        col = torch.empty(cap, dtype=torch.int32, device="cuda")
        dist = torch.empty(cap, dtype=torch.float64, device="cuda")
        nnz = ctypes.c_size_t()
        assert lib.lc_gpu_neighbors_within(ws, nn.data_ptr(), d2.data_ptr(), n, k, cutoff,
                                           row_ptr.data_ptr(), col.data_ptr(), dist.data_ptr(),
                                           cap, ctypes.byref(nnz)) == 0
        assert nnz.value == len(col_w)
        assert np.array_equal(row_ptr.cpu().numpy(), rp_w)
        assert np.array_equal(col.cpu().numpy()[:nnz.value], col_w)
        assert np.array_equal(dist.cpu().numpy()[:nnz.value], dist_w)
        if nnz.value > 1:
            small = nnz.value // 2
            rc = lib.lc_gpu_neighbors_within(ws, nn.data_ptr(), d2.data_ptr(), n, k, cutoff,
                                             row_ptr.data_ptr(), col.data_ptr(), None, small,
                                             ctypes.byref(nnz))
            assert rc != 0 and nnz.value == len(col_w)
            assert b"longer than its buffer" in lib.lc_gpu_last_error()
    finally:
        lib.lc_gpu_workspace_free(ws)
