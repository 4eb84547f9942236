"""The allocation-free entry point lc_gpu_knearest_noalloc.

Callers that cannot call cudaMalloc (a host whose pool allocator owns the
device memory, a real-time loop that must not allocate, a plug-in inside a
framework that owns the allocator) use this entry point: all of its scratch
sits in a fixed static device array that every call reuses. Its rows must be
the reference walk's (the CPU oracle), bit for bit, on two calls in a row
and on a call enqueued on the caller's own stream; an all-masked search on a
mesh past its limits must give -1 / NaN rows as the reference does; and it
must refuse searches above its stated limits.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    (11, 20000, 16, [[40.0, 0, 0], [12.0, 38.0, 0], [4.0, 8.0, 39.0]], 3.0),
    (12, 9000, 33, [[30.0, 0, 0], [0, 27.0, 0], [0, 0, 33.0]], 2.5),
]


def _inputs(seed, n, rows):
    rng = np.random.default_rng(seed)
    frac = rng.random((n, 3))
    xyz = frac @ np.asarray(rows) + rng.integers(-2, 3, size=(n, 3)) @ np.asarray(rows)
    xyz[5] = xyz[17]  # an exact duplicate: tie order at dist2 = 0
    mask = (rng.random(n) < 0.9).astype(np.int32)
    return xyz, mask


def _noalloc(L, torch, xyz, rows, k, mask, hint, stream=None, wait=1, with_d2=True):
    from gpu_helpers import lc_cell_of
    x = torch.as_tensor(np.ascontiguousarray(xyz), device="cuda")
    m = None if mask is None else torch.as_tensor(mask, device="cuda")
    n = x.shape[0]
    nn = torch.full((n, k), -9, dtype=torch.int32, device="cuda")
    d2 = torch.zeros((n, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    c = lc_cell_of(rows)
    rc = L.lc_gpu_knearest_noalloc(x.data_ptr(), n, ctypes.byref(c), k,
                                   None if m is None else m.data_ptr(), hint, nn.data_ptr(),
                                   d2.data_ptr() if with_d2 else None, stream, wait)
    torch.cuda.synchronize()
    return rc, nn.cpu().numpy(), d2.cpu().numpy()


def test_noalloc_matches_the_oracle_on_two_calls(gpu, lib, oracle_mod):
    import torch
    from gpu_helpers import assert_same
    from linkcell_b200 import _capi
    for seed, n, k, rows, hint in CASES:
        xyz, mask = _inputs(seed, n, rows)
        want = oracle_mod.knearest(xyz, rows, k, mask=mask, cell_hint=hint)
        assert (want[0] == -1).any()  # k past the neighbours of masked rows: padding checked
        for call in range(2):  # the second call reuses the array the first left behind
            rc, nn, d2 = _noalloc(lib, torch, xyz, rows, k, mask, hint)
            assert rc == 0, _capi.gpu_error()
            assert_same((nn, d2), want, f"no-alloc seed {seed} call {call}")


def test_noalloc_on_a_user_stream_without_wait_and_without_d2(gpu, lib, oracle_mod):
    import torch
    from gpu_helpers import assert_same
    from linkcell_b200 import _capi
    seed, n, k, rows, hint = CASES[0]
    xyz, mask = _inputs(seed, n, rows)
    want = oracle_mod.knearest(xyz, rows, k, mask=mask, cell_hint=hint)
    s = torch.cuda.Stream()
    rc, nn, d2 = _noalloc(lib, torch, xyz, rows, k, mask, hint, stream=s.cuda_stream, wait=0)
    assert rc == 0, _capi.gpu_error()
    assert_same((nn, d2), want, "no-alloc on a user stream, wait = 0")
    rc, nn, d2 = _noalloc(lib, torch, xyz, rows, k, mask, hint, with_d2=False)
    assert rc == 0, _capi.gpu_error()
    assert np.array_equal(nn, want[0])
    assert (d2 == 0.0).all()  # out_d2 = NULL: the distance buffer is never written


def test_noalloc_all_masked_past_its_mesh_limits(gpu, lib, oracle_mod):
    """src/knearest.rs:370-375: an all-masked search returns -1 / NaN rows
    before it sizes the mesh, so neither a too-fine mesh nor one above the
    entry point's cell limit is an error then; one active point makes it one."""
    import torch
    from linkcell_b200 import _capi
    box = [[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]]
    big = [[400.0, 0, 0], [0, 400.0, 0], [0, 0, 400.0]]
    for rows, hint, msg in ((box, 1e-9, "too many cells"), (big, 3.0, "65536 cells")):
        xyz, _ = _inputs(6, 500, rows)
        none = np.zeros(500, dtype=np.int32)
        want = oracle_mod.knearest(xyz, rows, 3, mask=none, cell_hint=hint)
        rc, nn, d2 = _noalloc(lib, torch, xyz, rows, 3, none, hint)
        assert rc == 0, _capi.gpu_error()
        assert (nn == -1).all() and np.isnan(d2).all() and (want[0] == -1).all()
        one = none.copy()
        one[7] = 1
        rc, _, _ = _noalloc(lib, torch, xyz, rows, 3, one, hint)
        assert rc != 0 and msg in _capi.gpu_error()


def test_noalloc_rejects_sizes_above_its_limits(gpu, lib):
    import torch
    from linkcell_b200 import _capi
    rows = [[400.0, 0, 0], [0, 400.0, 0], [0, 0, 400.0]]
    xyz, mask = _inputs(3, 65537, rows)
    rc, _, _ = _noalloc(lib, torch, xyz, rows, 4, mask, 3.0)
    assert rc != 0 and "65536 points" in _capi.gpu_error()
    small = [[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]]
    xyz, mask = _inputs(4, 100, small)
    rc, _, _ = _noalloc(lib, torch, xyz, small, 65, mask, 3.0)
    assert rc != 0 and "k <= 64" in _capi.gpu_error()
    xyz, mask = _inputs(5, 1000, rows)
    rc, _, _ = _noalloc(lib, torch, xyz, rows, 4, mask, 3.0)  # 133^3 cells
    assert rc != 0 and "65536 cells" in _capi.gpu_error()
    rc, _, _ = _noalloc(lib, torch, xyz, rows, 4, None, 3.0)
    assert rc != 0 and "65536 cells" in _capi.gpu_error()
