"""The benchmark configurations at full size.

The 1M FCC frame (k = 16, Bernoulli(0.9) mask) and the 4M bimodal frame at
k = 32 and k = 64 are too large for the oracle to check every source in a
test, so every source is checked through properties that hold at any size,
and a sample of sources against the oracle:

- the learned walk and the plain FP64 walk, two independent walks, give the
  same rows bit for bit over the whole frame;
- every active row is full (n > k) and ordered by (dist2, index) with
  distinct indices; every masked row is -1 / NaN;
- 20,000 sources drawn with a fixed seed get exactly the oracle's rows
  (oracle.knearest_subset runs the reference walk for those sources only).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SAMPLE = 20_000


def _configs():
    from linkcell_b200 import workloads as W
    return {
        "fcc_1M_k16": lambda: W.fcc_triclinic(),
        "bimodal_4M_k32": lambda: W.bimodal_triclinic(),
        "bimodal_4M_k64": lambda: W.bimodal_triclinic(k=64),
    }


def _search(L, ws, mode, x, n, cell, k, mask, hint):
    import torch
    from linkcell_b200 import _capi
    assert L.lc_gpu_set_mode(ws, mode) == 0
    nn = torch.empty((n, k), dtype=torch.int32, device="cuda")
    d2 = torch.empty((n, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k,
                                None if mask is None else mask.data_ptr(), hint, nn.data_ptr(),
                                d2.data_ptr(), 1)
    assert rc == 0, _capi.gpu_error()
    return nn, d2


@pytest.mark.parametrize("name", ["fcc_1M_k16", "bimodal_4M_k32", "bimodal_4M_k64"])
def test_full_size_configuration(gpu, lib, oracle_mod, name):
    import torch
    from linkcell_b200 import _cell_struct
    w = _configs()[name]()
    xyz, k, hint = w["xyz"], w["k"], w["cell_hint"]
    n = xyz.shape[0]
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    x = torch.as_tensor(xyz, device="cuda")
    mask = None if w["mask"] is None else torch.as_tensor(w["mask"], device="cuda")
    ws = lib.lc_gpu_workspace_new()
    try:
        nn_l, d2_l = _search(lib, ws, 2, x, n, cell, k, mask, hint)
        nn_p, d2_p = _search(lib, ws, 0, x, n, cell, k, mask, hint)
    finally:
        lib.lc_gpu_workspace_free(ws)
    # two walks, one answer
    assert torch.equal(nn_l, nn_p), f"{name}: learned and plain indices differ"
    assert torch.equal(d2_l.view(torch.int64), d2_p.view(torch.int64)), f"{name}: dist2 differs"
    # row structure
    active = torch.ones(n, dtype=torch.bool, device="cuda") if mask is None else mask != 0
    act_nn, act_d2 = nn_l[active], d2_l[active]
    assert bool((act_nn >= 0).all()) and bool(torch.isfinite(act_d2).all())
    ordered = (act_d2[:, 1:] > act_d2[:, :-1]) | (
        (act_d2[:, 1:] == act_d2[:, :-1]) & (act_nn[:, 1:] > act_nn[:, :-1]))
    assert bool(ordered.all()), f"{name}: a row is not ordered by (dist2, index)"
    srt = torch.sort(act_nn, dim=1).values
    assert bool((srt[:, 1:] != srt[:, :-1]).all()), f"{name}: repeated index in a row"
    if mask is not None:
        assert bool((nn_l[~active] == -1).all()) and bool(torch.isnan(d2_l[~active]).all())
    # a sample against the reference walk
    rng = np.random.default_rng(12345)
    src = np.sort(rng.choice(n, size=SAMPLE, replace=False)).astype(np.int64)
    want_nn, want_d2 = oracle_mod.knearest_subset(xyz, w["cell"], k, src, mask=w["mask"],
                                                  cell_hint=hint)
    got_nn = nn_l[torch.as_tensor(src, device="cuda")].cpu().numpy()
    got_d2 = d2_l[torch.as_tensor(src, device="cuda")].cpu().numpy()
    assert np.array_equal(got_nn, want_nn), f"{name}: sampled indices differ from the oracle"
    assert np.array_equal(got_d2.view(np.int64), want_d2.view(np.int64)), \
        f"{name}: sampled dist2 differs from the oracle"
