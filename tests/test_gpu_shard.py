"""The split search (lc_gpu_knearest_shard) on one GPU: every rank's share
of world = 2, 3 and 4 is run in turn on cuda:0 (each share is an ordinary
search of the whole input that walks one range of sources; nothing waits on
another rank), and the shares are combined as the all-reduce would combine
them. Every row must be owned by exactly one rank, the shares must carry
comparable work, and the combined rows must equal the one-rank search and
the oracle bit for bit."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _shares(lib, x, n, cell, k, mask, world, mode):
    import torch
    from linkcell_b200 import _capi, learn
    ws = lib.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    out = []
    try:
        if mode == 2:
            learn.attach(ws)
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        for rank in range(world):
            nn = torch.full((n, k), 555, dtype=torch.int32, device="cuda")
            d2 = torch.full((n, k), 2.5, dtype=torch.float64, device="cuda")
            owned = torch.full((n,), 7, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            rc = lib.lc_gpu_knearest_shard(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k,
                                           None if mask is None else mask.data_ptr(), 3.0, rank,
                                           world, nn.data_ptr(), d2.data_ptr(), owned.data_ptr(),
                                           1)
            assert rc == 0, _capi.gpu_error()
            out.append((nn, d2, owned))
    finally:
        lib.lc_gpu_workspace_free(ws)
    return out


@pytest.mark.parametrize("mode", [0, 2])
def test_split_search_equals_the_whole_search(gpu, lib, oracle_mod, mode):
    import torch
    from gpu_helpers import DeviceRunner, assert_same
    from linkcell_b200 import _cell_struct, workloads as W
    from linkcell_b200.shard import combine
    w = W.bimodal_triclinic(n=200_000, seed=5, k=16)
    xyz, k = w["xyz"], 16
    n = xyz.shape[0]
    mask_h = (np.random.default_rng(5).random(n) < 0.9).astype(np.int32)
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    x = torch.as_tensor(xyz, device="cuda")
    mask = torch.as_tensor(mask_h, device="cuda")
    runner = DeviceRunner(mode=mode)
    try:
        whole = runner.run(xyz, w["cell"], k, mask_h, 3.0)
    finally:
        runner.close()
    src = np.sort(np.random.default_rng(6).choice(n, 4000, replace=False))
    want = oracle_mod.knearest_subset(xyz, w["cell"], k, src, mask=mask_h, cell_hint=3.0)
    assert_same((whole[0][src], whole[1][src]), want, "one-rank search")
    for world in (2, 3, 4):
        shares = _shares(lib, x, n, cell, k, mask, world, mode)
        owners = sum((o != 0).to(torch.int32) for _, _, o in shares)
        assert bool((owners == 1).all()), f"world {world}: a row has no owner or two"
        rows = [int(((o != 0) & (mask != 0)).sum()) for _, _, o in shares]
        assert min(rows) > 0.5 * sum(rows) / world, f"world {world}: unbalanced {rows}"
        nn = sum(combine(a, b, o)[0] for a, b, o in shares)
        d2 = sum(combine(a, b, o)[1] for a, b, o in shares)
        assert_same((nn.cpu().numpy(), d2.cpu().numpy()), whole, f"world {world}, mode {mode}")
