"""What the shell-proposal network gains over the same walk without it.

The learned mode's cube select walk opens the proposed shell's cube at once.
Without the network the best it can do is one constant shell for every
source (lc_gpu_set_proposal): a short one sends the sparse sources to the
literal replay, a long one gathers far more candidates for the dense ones.
On a bimodal frame (dense and sparse halves, 1M points, k = 32) the network's
search must beat the fastest constant shell (1 .. 6) in device time, or at
least evaluate fewer candidate pairs -- with identical rows in every case.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_network_beats_the_best_constant_shell(gpu, lib):
    import torch
    from linkcell_b200 import _capi, _cell_struct, learn, workloads as W
    w = W.bimodal_triclinic(n=1_000_000, seed=12, k=32)
    n, k = w["xyz"].shape[0], 32
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    x = torch.as_tensor(w["xyz"], device="cuda")
    nn = torch.empty((n, k), dtype=torch.int32, device="cuda")
    d2 = torch.empty((n, k), dtype=torch.float64, device="cuda")
    ws = lib.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()

    def search():
        rc = lib.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k, None, 3.0,
                                      nn.data_ptr(), d2.data_ptr(), 1)
        assert rc == 0, _capi.gpu_error()

    def measure(shell):
        assert lib.lc_gpu_set_proposal(ws, shell) == 0
        for _ in range(2):
            search()
        times = []
        for _ in range(5):
            search()
            ms = ctypes.c_double()
            buf = (ctypes.c_longlong * 16)()
            lib.lc_gpu_stats(ws, buf, 16, ctypes.byref(ms))
            times.append(ms.value)
        assert lib.lc_gpu_set_stats(ws, 1) == 0
        search()
        assert lib.lc_gpu_set_stats(ws, 0) == 0
        buf = (ctypes.c_longlong * 16)()
        lib.lc_gpu_stats(ws, buf, 16, None)
        return sorted(times)[2], int(buf[0]), int(buf[2]), nn.clone(), d2.clone()

    try:
        learn.attach(ws)
        assert lib.lc_gpu_set_mode(ws, 2) == 0
        assert lib.lc_gpu_set_tpp(ws, 32) == 0
        net_ms, net_pairs, net_replays, want_nn, want_d2 = measure(0)
        consts = {}
        for shell in range(1, 7):
            ms, pairs, replays, got_nn, got_d2 = measure(shell)
            assert torch.equal(got_nn, want_nn) and torch.equal(got_d2.view(torch.int64),
                                                                want_d2.view(torch.int64))
            consts[shell] = (ms, pairs, replays)
    finally:
        lib.lc_gpu_workspace_free(ws)
    best = min(consts, key=lambda s: consts[s][0])
    b_ms, b_pairs, _ = consts[best]
    assert net_ms < b_ms or net_pairs < b_pairs, (
        f"network {net_ms:.3f} ms / {net_pairs} pairs vs best constant shell {best}: "
        f"{b_ms:.3f} ms / {b_pairs} pairs ({consts})")
