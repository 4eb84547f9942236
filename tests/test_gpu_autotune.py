"""The walk autotuner: on the first batch of each kind a workspace times
every candidate design and shape -- the cube select walk in two block sizes
and three work-grab sizes, and the thread-per-source walk -- and keeps the
fastest (the reference picks its block size among 256, 128, 64 and 512
under a shared-memory cap, src/gpu/knearest.cpp:923-960). The shape it picks
must be one of the candidates it timed, and every candidate, forced, must
give the same rows."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _search(lib, ws, x, n, cell, k):
    import torch
    from linkcell_b200 import _capi
    nn = torch.full((n, k), -9, dtype=torch.int32, device="cuda")
    d2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k, None, 3.0,
                                  nn.data_ptr(), d2.data_ptr(), 1)
    assert rc == 0, _capi.gpu_error()
    return nn, d2


@pytest.mark.parametrize("k", [32, 64])
def test_autotuned_shape_is_a_timed_candidate_with_the_same_rows(gpu, lib, oracle_mod, k):
    import torch
    from gpu_helpers import assert_same
    from linkcell_b200 import _capi, _cell_struct, learn, workloads as W
    w = W.bimodal_triclinic(n=300_000, seed=9, k=k)
    n = w["xyz"].shape[0]
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    x = torch.as_tensor(w["xyz"], device="cuda")
    ws = lib.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    try:
        learn.attach(ws)
        assert lib.lc_gpu_set_mode(ws, 2) == 0
        nn, d2 = _search(lib, ws, x, n, cell, k)
        shape = (ctypes.c_int * 3)()
        trials = (ctypes.c_int * 48)()
        count = lib.lc_gpu_walk_shape(ws, shape, trials, 16)
        cands = [tuple(trials[3 * i:3 * i + 3]) for i in range(count)]
        assert count == 7, cands  # 2 block sizes x 3 grabs of the select walk, + thread per source
        assert tuple(shape) in cands
        assert (1, 0, 0) in cands
        for tpp, warps, grab in cands:
            assert lib.lc_gpu_set_tpp(ws, tpp) == 0
            assert lib.lc_gpu_set_walk_shape(ws, warps, grab) == 0
            got = _search(lib, ws, x, n, cell, k)
            used = (ctypes.c_int * 3)()
            lib.lc_gpu_walk_shape(ws, used, None, 0)
            assert tuple(used) == (tpp, warps, grab)
            assert torch.equal(got[0], nn), f"shape {(tpp, warps, grab)}: indices differ"
            assert torch.equal(got[1].view(torch.int64), d2.view(torch.int64))
    finally:
        lib.lc_gpu_workspace_free(ws)
    src = np.sort(np.random.default_rng(10).choice(n, 3000, replace=False))
    want = oracle_mod.knearest_subset(w["xyz"], w["cell"], k, src, cell_hint=3.0)
    assert_same((nn.cpu().numpy()[src], d2.cpu().numpy()[src]), want, f"autotuned k={k}")
