"""Helpers of the GPU parity tests: run the product through its C ABI and
compare with the CPU oracle."""

from __future__ import annotations

import ctypes

import numpy as np

from linkcell_b200 import LcCell, LcFrame, _capi


def lc_cell_of(cell) -> LcCell:
    c = np.asarray(cell, dtype=np.float64)
    if c.shape == (3,):
        vals = [c[0], 0, 0, 0, c[1], 0, 0, 0, c[2], 0, 0, 0]
    elif c.shape == (3, 3):
        vals = list(c.reshape(-1)) + [0, 0, 0]
    else:
        vals = list(c.reshape(-1))
    return LcCell(*[float(v) for v in vals])


def host_abi(xyz, cell, k, mask=None, hint=0.0, n_frames=1):
    """lc_knearest_many with host pointers."""
    L = _capi.load()
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = x.shape[0] // n_frames
    nn = np.full((x.shape[0], k), -9, dtype=np.int32)
    d2 = np.zeros((x.shape[0], k))
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    c = lc_cell_of(cell)
    rc = L.lc_knearest_many(x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n, n_frames,
                            ctypes.byref(c), k,
                            None if m is None else m.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                            float(hint), nn.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                            d2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert rc == 0, _capi.cpu_error()
    return nn, d2


class DeviceRunner:
    """lc_gpu_* with device buffers from torch."""

    def __init__(self, mode=0):
        import torch
        self.torch = torch
        self.L = _capi.load()
        self.ws = self.L.lc_gpu_workspace_new()
        assert self.ws, _capi.gpu_error()
        assert self.L.lc_gpu_set_mode(self.ws, mode) == 0

    def close(self):
        if self.ws:
            self.L.lc_gpu_workspace_free(self.ws)
            self.ws = None

    def set_mode(self, mode):
        assert self.L.lc_gpu_set_mode(self.ws, mode) == 0

    def set_tpp(self, tpp):
        assert self.L.lc_gpu_set_tpp(self.ws, tpp) == 0

    def set_proposal(self, shell):
        assert self.L.lc_gpu_set_proposal(self.ws, shell) == 0

    def set_stats(self, on):
        assert self.L.lc_gpu_set_stats(self.ws, 1 if on else 0) == 0

    def run(self, xyz, cell, k, mask=None, hint=0.0, n_frames=1, wait=1):
        torch = self.torch
        x = torch.as_tensor(np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3),
                            device="cuda")
        n = x.shape[0] // n_frames
        nn = torch.full((x.shape[0], k), -9, dtype=torch.int32, device="cuda")
        d2 = torch.zeros((x.shape[0], k), dtype=torch.float64, device="cuda")
        m = None if mask is None else torch.as_tensor(np.asarray(mask, dtype=np.int32),
                                                      device="cuda")
        torch.cuda.synchronize()
        c = lc_cell_of(cell)
        rc = self.L.lc_gpu_knearest_many(self.ws, x.data_ptr(), n, n_frames, ctypes.byref(c), k,
                                         None if m is None else m.data_ptr(), float(hint),
                                         nn.data_ptr(), d2.data_ptr(), wait)
        assert rc == 0, _capi.gpu_error()
        if not wait:
            self.L.lc_gpu_wait(self.ws)
        return nn.cpu().numpy(), d2.cpu().numpy()

    def batch(self, frames):
        torch = self.torch
        xyz = np.concatenate([f["xyz"] for f in frames]).astype(np.float64)
        masks = [f.get("mask") for f in frames]
        arr = (LcFrame * len(frames))()
        moff = 0
        mask_parts = []
        total = 0
        for i, f in enumerate(frames):
            arr[i].n = len(f["xyz"])
            arr[i].k = f["k"]
            arr[i].cell = lc_cell_of(f["cell"])
            arr[i].cell_hint = float(f.get("cell_hint", 0.0))
            if masks[i] is not None:
                arr[i].mask_offset = moff
                mask_parts.append(np.asarray(masks[i], dtype=np.int32))
                moff += len(masks[i])
            else:
                arr[i].mask_offset = -1
            total += arr[i].n * arr[i].k
        x = torch.as_tensor(xyz, device="cuda")
        m = torch.as_tensor(np.concatenate(mask_parts), device="cuda") if mask_parts else None
        nn = torch.full((total,), -9, dtype=torch.int32, device="cuda")
        d2 = torch.zeros((total,), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = self.L.lc_gpu_knearest_batch(self.ws, x.data_ptr(), arr, len(frames),
                                          None if m is None else m.data_ptr(), nn.data_ptr(),
                                          d2.data_ptr(), 1)
        assert rc == 0, _capi.gpu_error()
        return nn.cpu().numpy(), d2.cpu().numpy()

    def stats(self):
        buf = (ctypes.c_longlong * 16)()
        ms = ctypes.c_double()
        self.L.lc_gpu_stats(self.ws, buf, 16, ctypes.byref(ms))
        return list(buf), ms.value


def assert_same(got, want, label=""):
    gn, gd = got
    wn, wd = want
    gn = np.asarray(gn).reshape(wn.shape)
    gd = np.asarray(gd).reshape(wd.shape)
    if not np.array_equal(gn, wn):
        bad = np.argwhere((gn != wn).any(axis=1)).ravel()
        i = int(bad[0])
        raise AssertionError(f"{label}: {bad.size} rows differ; row {i}: got {gn[i].tolist()} "
                             f"want {wn[i].tolist()} (d2 got {gd[i].tolist()} want {wd[i].tolist()})")
    # exact: the FP64 distances follow the reference expression bit for bit
    same = (gd == wd) | (np.isnan(gd) & np.isnan(wd))
    if not same.all():
        fin = ~np.isnan(wd)
        rel = np.max(np.abs(gd[fin] - wd[fin]) / np.maximum(np.abs(wd[fin]), 1e-300))
        raise AssertionError(f"{label}: dist2 differs, max rel err {rel:.3e}")
