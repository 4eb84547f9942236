"""CUDA-graph replay and the walk autotuner, checked against the oracle.

A workspace with graphs on captures its launch sequence once per batch
signature (sizes, pointers, configuration) and replays it; the frame table
(the cell) is re-read at every replay, so a new cell of the same sizes must
give that cell's reference rows without a new capture."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from gpu_helpers import assert_same, lc_cell_of

pytestmark = pytest.mark.gpu


class Fixed:
    """One set of device buffers reused across calls (stable pointers)."""

    def __init__(self, L, ws, n, k):
        import torch
        self.torch, self.L, self.ws, self.n, self.k = torch, L, ws, n, k
        self.x = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        self.nn = torch.zeros((n, k), dtype=torch.int32, device="cuda")
        self.d2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")

    def run(self, xyz, cell):
        self.x.copy_(self.torch.as_tensor(np.asarray(xyz, dtype=np.float64)))
        self.nn.fill_(-9)
        self.torch.cuda.synchronize()
        c = lc_cell_of(cell)
        rc = self.L.lc_gpu_knearest_many(self.ws, self.x.data_ptr(), self.n, 1, ctypes.byref(c),
                                         self.k, None, 0.0, self.nn.data_ptr(),
                                         self.d2.data_ptr(), 1)
        assert rc == 0
        return self.nn.cpu().numpy(), self.d2.cpu().numpy()


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_graph_replay_follows_new_cells(gpu, lib, oracle_mod, mode):
    rng = np.random.default_rng(11 + mode)
    n, k = 3000, 12
    ws = lib.lc_gpu_workspace_new()
    try:
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        if mode == 2:
            assert lib.lc_gpu_set_proposal(ws, 2) == 0
        assert lib.lc_gpu_set_graph(ws, 1) == 0
        buf = Fixed(lib, ws, n, k)
        for step in range(4):
            L = 14.0 + 0.01 * step  # same cell grid: the graph is replayed
            cell = np.array([[L, 0.3, -0.2], [0.0, L - 1.0, 0.4], [0.0, 0.0, L + 0.5]])
            xyz = rng.random((n, 3)) @ cell
            want = oracle_mod.knearest(xyz, cell, k)
            assert_same(buf.run(xyz, cell), want, f"graph step {step}")
        assert lib.lc_gpu_graph_captures(ws) == 1
        # new sizes: a new capture
        buf2 = Fixed(lib, ws, n - 7, k)
        xyz = rng.random((n - 7, 3)) * 15.0
        assert_same(buf2.run(xyz, [15.0, 15.0, 15.0]),
                    oracle_mod.knearest(xyz, [15.0, 15.0, 15.0], k), "recapture")
        assert lib.lc_gpu_graph_captures(ws) == 2
    finally:
        lib.lc_gpu_workspace_free(ws)


def test_graph_stats_report_total_time(gpu, lib):
    rng = np.random.default_rng(3)
    ws = lib.lc_gpu_workspace_new()
    try:
        assert lib.lc_gpu_set_graph(ws, 1) == 0
        buf = Fixed(lib, ws, 2000, 8)
        for _ in range(2):
            buf.run(rng.random((2000, 3)) * 12.0, [12.0, 12.0, 12.0])
        counters = (ctypes.c_longlong * 16)()
        ms = ctypes.c_double()
        assert lib.lc_gpu_stats(ws, counters, 16, ctypes.byref(ms)) == 16
        assert ms.value > 0.0
    finally:
        lib.lc_gpu_workspace_free(ws)


@pytest.mark.parametrize("mode", [0, 1])
def test_autotuner_picks_a_design_and_stays_exact(gpu, lib, oracle_mod, mode):
    rng = np.random.default_rng(5)
    n, k = 20000, 16
    xyz = rng.random((n, 3)) * 40.0
    cell = [40.0, 40.0, 40.0]
    want = oracle_mod.knearest(xyz, cell, k)
    ws = lib.lc_gpu_workspace_new()
    try:
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        assert lib.lc_gpu_set_tpp(ws, 0) == 0  # autotune even under LINKCELL_TPP
        buf = Fixed(lib, ws, n, k)
        assert_same(buf.run(xyz, cell), want, "autotuned first batch")
        first = lib.lc_gpu_get_tpp(ws)
        assert first in (1, 32)
        assert_same(buf.run(xyz, cell), want, "autotuned second batch")
        assert lib.lc_gpu_get_tpp(ws) == first
        assert lib.lc_gpu_set_tpp(ws, 1) == 0
        assert_same(buf.run(xyz, cell), want, "forced tpp 1")
        assert lib.lc_gpu_get_tpp(ws) == 1
    finally:
        lib.lc_gpu_workspace_free(ws)
