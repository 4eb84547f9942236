"""The device-cell entry, lc_gpu_knearest_many_dcell, planned on the device.

Up to 16 frames the cell is never read by the host: a one-block kernel
plans the mesh from the device doubles and writes the frame table, and the
cell arrays are sized for the largest mesh a frame may have. The rows must
equal the oracle's for every cell layout (3, 9 or 12 doubles), with masks
and several frames; a CUDA graph captured once must follow the device cell
as it changes, mesh included; the call must not wait for the device; and a
rejected cell must be reported when the batch is waited for."""

from __future__ import annotations

import ctypes
import time

import numpy as np
import pytest

from gpu_helpers import assert_same

pytestmark = pytest.mark.gpu


def _cell_doubles(cell, cell_n):
    c = np.asarray(cell, dtype=np.float64)
    if cell_n == 3:
        return np.diag(c) if c.shape == (3, 3) else c
    rows = c if c.shape == (3, 3) else np.diag(c)
    if cell_n == 9:
        return rows.reshape(-1)
    return np.concatenate([rows.reshape(-1), np.zeros(3)])


class DeviceCellRun:
    """Fixed device buffers (stable pointers) for repeated dcell calls."""

    def __init__(self, L, ws, n, frames, k, cell_n):
        import torch
        self.torch, self.L, self.ws = torch, L, ws
        self.n, self.frames, self.k, self.cell_n = n, frames, k, cell_n
        self.x = torch.zeros((frames * n, 3), dtype=torch.float64, device="cuda")
        self.cell = torch.zeros(cell_n, dtype=torch.float64, device="cuda")
        self.nn = torch.zeros((frames * n, k), dtype=torch.int32, device="cuda")
        self.d2 = torch.zeros((frames * n, k), dtype=torch.float64, device="cuda")
        self.mask = None

    def load(self, xyz, cell_vals, mask=None):
        torch = self.torch
        self.x.copy_(torch.as_tensor(np.asarray(xyz, dtype=np.float64).reshape(-1, 3)))
        self.cell.copy_(torch.as_tensor(np.array(cell_vals, dtype=np.float64)))
        if mask is not None:
            self.mask = torch.as_tensor(np.asarray(mask, dtype=np.int32), device="cuda")
        self.nn.fill_(-9)
        torch.cuda.synchronize()

    def call(self, hint=0.0, wait=1):
        return self.L.lc_gpu_knearest_many_dcell(
            self.ws, self.x.data_ptr(), self.n, self.frames, self.cell.data_ptr(), self.cell_n,
            self.k, None if self.mask is None else self.mask.data_ptr(), float(hint),
            self.nn.data_ptr(), self.d2.data_ptr(), wait)

    def rows(self):
        self.torch.cuda.synchronize()
        return self.nn.cpu().numpy(), self.d2.cpu().numpy()


def _error(L):
    from linkcell_b200 import _capi
    return _capi.gpu_error() or ""


@pytest.mark.parametrize("cell_n", [3, 9, 12])
@pytest.mark.parametrize("mode", [0, 2])
def test_device_cell_matches_oracle(gpu, lib, oracle_mod, cell_n, mode):
    rng = np.random.default_rng(40 + cell_n + mode)
    n, frames, k = 4000, 3, 12
    if cell_n == 3:
        cell = np.diag([21.0, 18.5, 24.0])
        origin = np.zeros(3)
    else:
        cell = np.array([[21.0, 0.0, 0.0], [4.0, 18.5, 0.0], [-3.0, 2.5, 24.0]])
        origin = np.array([1.5, -2.0, 0.25]) if cell_n == 12 else np.zeros(3)
    vals = _cell_doubles(cell, cell_n)
    if cell_n == 12:
        vals[9:] = origin
    xyz = rng.random((frames * n, 3)) @ cell + origin + rng.normal(0, 3.0, (frames * n, 3))
    mask = (rng.random(n) < 0.9).astype(np.int32)
    full = np.vstack([cell, origin]) if cell_n == 12 else cell
    want = oracle_mod.knearest(xyz, full, k, mask=mask, cell_hint=2.5, n_frames=frames)
    ws = lib.lc_gpu_workspace_new()
    try:
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        run = DeviceCellRun(lib, ws, n, frames, k, cell_n)
        run.load(xyz, vals, mask)
        assert run.call(hint=2.5) == 0, _error(lib)
        assert_same(run.rows(), want, f"dcell cell_n={cell_n} mode={mode}")
    finally:
        lib.lc_gpu_workspace_free(ws)


@pytest.mark.parametrize("mode", [0, 2])
def test_graph_replay_follows_device_cell_and_mesh(gpu, lib, oracle_mod, mode):
    """One capture, then replays while the device cell changes: the mesh
    (nx, ny, nz) changes with it, which the host never sees."""
    rng = np.random.default_rng(7 + mode)
    n, k = 6000, 10
    ws = lib.lc_gpu_workspace_new()
    try:
        assert lib.lc_gpu_set_mode(ws, mode) == 0
        assert lib.lc_gpu_set_graph(ws, 1) == 0
        run = DeviceCellRun(lib, ws, n, 1, k, 9)
        for step, L in enumerate([30.0, 30.0, 22.0, 41.0, 17.5]):
            cell = np.array([[L, 0.0, 0.0], [0.3 * L, L * 0.9, 0.0], [0.1, -0.2 * L, L * 1.1]])
            xyz = rng.random((n, 3)) @ cell
            run.load(xyz, cell.reshape(-1))
            assert run.call() == 0, _error(lib)
            assert_same(run.rows(), oracle_mod.knearest(xyz, cell, k), f"graph step {step}")
        assert lib.lc_gpu_graph_captures(ws) == 1
    finally:
        lib.lc_gpu_workspace_free(ws)


def test_device_cell_call_does_not_wait(gpu, lib, oracle_mod):
    """With wait = 0 the call returns while the stream is still busy with
    earlier work (a 0.4 s device sleep); the blocking read of the mesh the
    reference makes would have waited for it."""
    import torch
    rng = np.random.default_rng(2)
    n, k = 3000, 8
    cell = np.diag([16.0, 17.0, 18.0])
    xyz = rng.random((n, 3)) @ cell
    ws = lib.lc_gpu_workspace_new()
    try:
        run = DeviceCellRun(lib, ws, n, 1, k, 3)
        run.load(xyz, [16.0, 17.0, 18.0])
        assert run.call() == 0, _error(lib)  # first call: buffers, walk tuning
        stream = torch.cuda.ExternalStream(lib.lc_gpu_queue(ws))
        rate = torch.cuda.get_device_properties(0).clock_rate * 1000.0  # Hz
        with torch.cuda.stream(stream):
            torch.cuda._sleep(int(0.4 * rate))
        t0 = time.perf_counter()
        assert run.call(wait=0) == 0, _error(lib)
        host_s = time.perf_counter() - t0
        lib.lc_gpu_wait(ws)
        assert lib.lc_gpu_last_error() is None
        assert_same(run.rows(), oracle_mod.knearest(xyz, cell, k), "async dcell")
        assert host_s < 0.2, f"dcell call took {host_s:.3f} s with a busy stream"
    finally:
        lib.lc_gpu_workspace_free(ws)


def test_device_cell_rejections_surface_at_wait(gpu, lib):
    import torch
    rng = np.random.default_rng(3)
    n, k = 500, 4
    ws = lib.lc_gpu_workspace_new()
    try:
        run = DeviceCellRun(lib, ws, n, 2, k, 9)
        # singular cell
        run.load(rng.random((2 * n, 3)), [1.0, 0, 0, 2.0, 0, 0, 0, 0, 1.0])
        assert run.call(wait=1) != 0
        assert "bad cell" in _error(lib)
        nn, _ = run.rows()
        assert (nn == -1).all()
        # the same, waited for later
        assert run.call(wait=0) == 0
        lib.lc_gpu_wait(ws)
        assert "bad cell" in _error(lib)
        # a mesh over the cell cap
        run.load(rng.random((2 * n, 3)) * 1000.0, [1000.0, 0, 0, 0, 1000.0, 0, 0, 0, 1000.0])
        assert run.call(hint=1e-3, wait=1) != 0
        assert "too many cells" in _error(lib)
        # ... which an all-zero mask excuses, as on the host-cell path
        run.mask = torch.zeros(n, dtype=torch.int32, device="cuda")
        assert run.call(hint=1e-3, wait=1) == 0, _error(lib)
        nn, d2 = run.rows()
        assert (nn == -1).all() and np.isnan(d2).all()
        # and the workspace still searches a good cell afterwards
        run.mask = None
        cell = np.diag([12.0, 12.0, 12.0])
        xyz = rng.random((2 * n, 3)) * 12.0
        run.load(xyz, cell.reshape(-1))
        assert run.call() == 0, _error(lib)
    finally:
        lib.lc_gpu_workspace_free(ws)


def test_many_frames_read_the_cell(gpu, lib, oracle_mod):
    """Past 16 frames the entry reads the cell and plans on the host."""
    rng = np.random.default_rng(5)
    n, frames, k = 300, 17, 6
    cell = np.array([[9.0, 0.0, 0.0], [1.0, 9.5, 0.0], [0.5, 0.5, 10.0]])
    xyz = rng.random((frames * n, 3)) @ cell
    ws = lib.lc_gpu_workspace_new()
    try:
        run = DeviceCellRun(lib, ws, n, frames, k, 9)
        run.load(xyz, cell.reshape(-1))
        assert run.call() == 0, _error(lib)
        assert_same(run.rows(), oracle_mod.knearest(xyz, cell, k, n_frames=frames), "17 frames")
    finally:
        lib.lc_gpu_workspace_free(ws)
