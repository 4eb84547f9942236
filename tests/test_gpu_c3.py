"""The batched-frames configuration at its full size: 256 frames (seed 3) of
their own sheared cells, densities, n (1,288 .. 150,061 points, 7.36M in
all), k in {4, 8, 16, 32} and Bernoulli(0.95) masks, searched by one
lc_gpu_knearest_batch call in the learned mode with the launch sequence
captured in a CUDA graph and replayed.

The reference searches one frame per call (src/gpu/knearest.cpp:705-816 for
its device batch of one shared cell; src/knearest.rs:225-273 on the CPU),
so every frame's rows must equal the reference walk's for that frame:

- frames of up to 6,000 points are checked whole against the oracle;
- every larger frame on 1,500 sources drawn with a fixed seed
  (oracle.knearest_subset runs the reference walk for those only);
- over all 7.36M rows, the graph replay equals the first (captured) run
  and the plain FP64 walk bit for bit, rows are ordered by (dist2, index)
  with distinct indices, and masked rows are -1 / NaN.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WHOLE = 6000
SAMPLE = 1500


def test_batched_frames_full_size(gpu, lib, oracle_mod):
    import torch
    from gpu_helpers import lc_cell_of
    from linkcell_b200 import LcFrame, _capi, learn, workloads as W
    frames = W.frames_batch(256, seed=3)
    arr = (LcFrame * len(frames))()
    bases, out_total, moff = [], 0, 0
    for f, fr in enumerate(frames):
        arr[f].n, arr[f].k = fr["n"], fr["k"]
        arr[f].cell = lc_cell_of(fr["cell"])
        arr[f].cell_hint = fr["cell_hint"]
        arr[f].mask_offset = moff
        bases.append(out_total)
        out_total += fr["n"] * fr["k"]
        moff += fr["n"]
    x = torch.as_tensor(np.concatenate([fr["xyz"] for fr in frames]), device="cuda")
    m = torch.as_tensor(np.concatenate([fr["mask"] for fr in frames]).astype(np.int32),
                        device="cuda")
    ws = lib.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    try:
        learn.attach(ws)
        assert lib.lc_gpu_set_graph(ws, 1) == 0
        # one pair of output buffers: a graph replays while pointers and sizes repeat
        nn = torch.empty((out_total,), dtype=torch.int32, device="cuda")
        d2 = torch.empty((out_total,), dtype=torch.float64, device="cuda")

        def run(mode):
            assert lib.lc_gpu_set_mode(ws, mode) == 0
            nn.fill_(-9)
            d2.zero_()
            torch.cuda.synchronize()
            rc = lib.lc_gpu_knearest_batch(ws, x.data_ptr(), arr, len(frames), m.data_ptr(),
                                           nn.data_ptr(), d2.data_ptr(), 1)
            assert rc == 0, _capi.gpu_error()
            return nn.clone(), d2.clone()

        nn1, d21 = run(2)
        nn2, d22 = run(2)  # replays the graph captured by the first call
        captures = int(lib.lc_gpu_graph_captures(ws))
        nn0, d20 = run(0)
    finally:
        lib.lc_gpu_workspace_free(ws)
    assert captures == 1
    assert torch.equal(nn1, nn2) and torch.equal(d21.view(torch.int64), d22.view(torch.int64))
    assert torch.equal(nn1, nn0), "learned and plain walks differ"
    assert torch.equal(d21.view(torch.int64), d20.view(torch.int64))
    nn, d2 = nn1.cpu().numpy(), d21.cpu().numpy()
    rng = np.random.default_rng(33)
    checked = 0
    for f, fr in enumerate(frames):
        n, k = fr["n"], fr["k"]
        rows_nn = nn[bases[f]:bases[f] + n * k].reshape(n, k)
        rows_d2 = d2[bases[f]:bases[f] + n * k].reshape(n, k)
        act = fr["mask"] != 0
        assert (rows_nn[~act] == -1).all() and np.isnan(rows_d2[~act]).all()
        a_nn, a_d2 = rows_nn[act], rows_d2[act]
        full = a_nn >= 0
        assert (full | (a_nn == -1)).all()
        ordered = (a_d2[:, 1:] > a_d2[:, :-1]) | ((a_d2[:, 1:] == a_d2[:, :-1]) &
                                                  (a_nn[:, 1:] > a_nn[:, :-1]))
        assert (ordered | ~full[:, 1:]).all(), f"frame {f}: a row is not ordered"
        if n <= WHOLE:
            want = oracle_mod.knearest(fr["xyz"], fr["cell"], k, mask=fr["mask"],
                                       cell_hint=fr["cell_hint"])
            src = np.arange(n)
        else:
            src = np.sort(rng.choice(n, size=SAMPLE, replace=False))
            want = oracle_mod.knearest_subset(fr["xyz"], fr["cell"], k, src, mask=fr["mask"],
                                              cell_hint=fr["cell_hint"])
        got_nn, got_d2 = rows_nn[src], rows_d2[src]
        assert np.array_equal(got_nn, want[0]), f"frame {f} (n {n}, k {k}): indices differ"
        same = (got_d2 == want[1]) | (np.isnan(got_d2) & np.isnan(want[1]))
        assert same.all(), f"frame {f}: dist2 differs"
        checked += src.size
    assert checked > 250_000
