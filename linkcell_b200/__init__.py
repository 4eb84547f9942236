"""Periodic linked-cell k-nearest search on NVIDIA B200 (sm_100a).

Drop-in for the reference Python entry ``linkcell.knearest``
(HaoZeke/linkcell v0.3.3, python/src/lib.rs:321-412, python/src/gpu.rs):
same signature, accepted shapes, error types and messages, and results
identical to the reference CPU walk. Every search runs on the GPU through
``liblinkcell_b200.so``: CUDA inputs stay on the device and give CUDA
outputs; host inputs are copied to the device and the outputs come back as
host arrays. There is no CPU fallback.

Arrays are anything with ``__dlpack__`` (numpy, torch, ...).
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np

from . import _capi
from ._capi import LcCell, LcFrame

__version__ = "0.3.3"
__all__ = ["__version__", "gpu_available", "knearest", "knearest_batch", "Workspace",
           "MODE_PLAIN_F64", "MODE_FAST_F32", "MODE_LEARNED", "MODE_REPLAY"]

MODE_PLAIN_F64 = 0
MODE_FAST_F32 = 1
MODE_LEARNED = 2
MODE_REPLAY = 3

_XYZ_SHAPE_MSG = "xyz must be float64 shape (n, 3), (n_frames, n, 3), or (n*3,)"
_CELL_SHAPE_MSG = ("cell must be float64 shape (3,) ortho, (3, 3) lattice rows, "
                   "or (4, 3) rows plus origin")
_KDLCPU, _KDLCUDA = 1, 2


def gpu_available() -> bool:
    """True when a CUDA device is usable (reference python/src/lib.rs:414-417)."""
    return bool(_capi.load().lc_gpu_available())


def _device_of(obj):
    """(is_cuda, device_index) from the DLPack device of obj."""
    try:
        import torch
        if isinstance(obj, torch.Tensor):
            return obj.is_cuda, (obj.device.index if obj.is_cuda else -1)
    except ImportError:  # pragma: no cover
        pass
    if hasattr(obj, "__dlpack_device__"):
        dev_type, dev_id = obj.__dlpack_device__()
        return int(dev_type) == _KDLCUDA, int(dev_id)
    return False, -1


def _host_array(obj, dtype=None):
    if isinstance(obj, np.ndarray):
        a = obj
    elif hasattr(obj, "__dlpack__"):
        try:
            a = np.from_dlpack(obj)
        except (TypeError, RuntimeError, BufferError):
            a = np.asarray(obj)
    else:
        a = np.asarray(obj)
    if dtype is not None and a.dtype != dtype:
        raise ValueError(f"expected {np.dtype(dtype).name}")
    return np.ascontiguousarray(a)


def _xyz_dims(shape):
    """(n, n_frames) for (n,3), (F,n,3) or (3n,) (python/src/lib.rs:213-233)."""
    if len(shape) == 2 and shape[1] == 3 and shape[0] > 0:
        return int(shape[0]), 1
    if len(shape) == 3 and shape[2] == 3 and shape[0] > 0 and shape[1] > 0:
        return int(shape[1]), int(shape[0])
    if len(shape) == 1 and shape[0] > 0 and shape[0] % 3 == 0:
        return int(shape[0]) // 3, 1
    raise ValueError(_XYZ_SHAPE_MSG)


def _cell_struct(cell_arr: np.ndarray) -> LcCell:
    """lc_cell from (3,), (3,3) or (4,3) doubles (python/src/lib.rs:235-308)."""
    d = cell_arr.reshape(-1)
    if cell_arr.shape == (3,):
        vals = [d[0], 0, 0, 0, d[1], 0, 0, 0, d[2], 0, 0, 0]
    elif cell_arr.shape == (3, 3):
        vals = list(d[:9]) + [0, 0, 0]
    elif cell_arr.shape == (4, 3):
        vals = list(d[:12])
    else:
        raise ValueError(_CELL_SHAPE_MSG)
    return LcCell(*[float(v) for v in vals])


def _cell_n(shape) -> int:
    if tuple(shape) == (3,):
        return 3
    if tuple(shape) == (3, 3):
        return 9
    if tuple(shape) == (4, 3):
        return 12
    if len(shape) == 1 and shape[0] in (3, 9, 12):
        return int(shape[0])
    raise ValueError(_CELL_SHAPE_MSG)


def _bool_mask_i32(m: np.ndarray, n: int) -> np.ndarray:
    """Host mask of n int32 or float64 entries as 0/1 int32 (python/src/lib.rs:188-211)."""
    if m.size != n:
        raise ValueError("mask length must be n")
    if m.dtype == np.int32:
        return np.ascontiguousarray((m.reshape(-1) != 0).astype(np.int32))
    if m.dtype == np.float64:
        return np.ascontiguousarray((m.reshape(-1) != 0.0).astype(np.int32))
    raise ValueError("mask must be int32 or float64")


class Workspace:
    """One device workspace (grow-only buffers, one CUDA stream).

    Wraps ``lc_gpu_workspace``. ``mode`` selects the walk; every mode gives
    identical results, and the learned walk (the default) is the fastest.
    """

    def __init__(self, mode: int = MODE_LEARNED):
        L = _capi.load()
        self._L = L
        self._ws = L.lc_gpu_workspace_new()
        if not self._ws:
            raise RuntimeError(_capi.gpu_error())
        self.mode = mode

    def __del__(self):
        ws = getattr(self, "_ws", None)
        if ws:
            self._L.lc_gpu_workspace_free(ws)
            self._ws = None

    @property
    def mode(self) -> int:
        return int(self._L.lc_gpu_get_mode(self._ws))

    @mode.setter
    def mode(self, m: int):
        if self._L.lc_gpu_set_mode(self._ws, int(m)) != 0:
            raise ValueError(_capi.gpu_error())

    def use_stream(self, stream) -> None:
        """Enqueue on a CUDA stream (handle or torch stream); None restores the own stream.

        Handle 0 (torch's default stream) maps to the CUDA legacy default
        stream, so the search stays ordered after torch's pending work.
        """
        if stream is None:
            self._L.lc_gpu_set_stream(self._ws, None)
            return
        h = int(getattr(stream, "cuda_stream", stream))
        self._L.lc_gpu_set_stream(self._ws, ctypes.c_void_p(h if h else 1))

    def set_stats(self, on: bool = True) -> None:
        """Count walk statistics in the learned mode's warp walk (off by
        default; they cost about 3 % of that walk)."""
        self._L.lc_gpu_set_stats(self._ws, 1 if on else 0)

    def stats(self) -> dict:
        buf = (ctypes.c_longlong * 16)()
        ms = ctypes.c_double()
        self._L.lc_gpu_stats(self._ws, buf, 16, ctypes.byref(ms))
        names = ["pairs", "inserts", "replays", "shells", "pruned", "reranks", "prop_under",
                 "prop_over", "prop_exact", "revisited", "fallback"]
        out = {name: int(buf[i]) for i, name in enumerate(names)}
        out["device_ms"] = ms.value
        return out

    @property
    def handle(self):
        return self._ws


_tls = threading.local()


def _workspace_for(device_index: int) -> Workspace:
    cache = getattr(_tls, "ws", None)
    if cache is None:
        cache = _tls.ws = {}
    ws = cache.get(device_index)
    if ws is None:
        import torch
        with torch.cuda.device(device_index):
            ws = Workspace()
        cache[device_index] = ws
    return ws


def _raise_from_lib(msg: str):
    if msg in ("singular or non-positive cell", "bad cell", "k must be at least 1",
               "mask length must be n"):
        raise ValueError(msg)
    raise RuntimeError(msg)


def knearest(xyz, cell, k, mask=None, cell_hint=None, *, workspace: Workspace | None = None,
             sync: bool = True):
    """Periodic linked-cell k-nearest search.

    xyz: float64 (n, 3), (n_frames, n, 3) or (n*3,). cell: float64 (3,)
    ortho lengths, (3, 3) lattice rows or (4, 3) rows plus origin, on any
    device. mask: optional, n entries (int32 or float64 on the host; int32
    on the device of a CUDA xyz), nonzero keeps a point. cell_hint: target
    cell edge, default 3.0.

    Returns (indices, dist2): int32 with -1 in unused slots and float64 with
    NaN there, shaped (n, k) or (n_frames, n, k). CUDA xyz gives torch CUDA
    tensors (enqueued on torch's current stream; ``sync=False`` skips the
    final stream wait), host xyz gives numpy arrays.
    """
    k = int(k)
    if k == 0:
        raise ValueError("k must be at least 1")
    if k < 0:
        raise OverflowError("can't convert negative int to unsigned")
    hint = 0.0 if cell_hint is None else float(cell_hint)
    L = _capi.load()
    is_cuda, dev = _device_of(xyz)
    if is_cuda:
        return _knearest_cuda(L, xyz, cell, k, mask, hint, dev, workspace, sync)
    cell_cuda, _ = _device_of(cell)
    cell_arr = _host_array(cell if not cell_cuda else cell.cpu(), np.float64) \
        if not cell_cuda else _host_array(cell.cpu(), np.float64)
    cs = _cell_struct(cell_arr)
    x = _host_array(xyz)
    if x.dtype != np.float64:
        raise ValueError(_XYZ_SHAPE_MSG)
    n, frames = _xyz_dims(x.shape)
    m = None
    if mask is not None:
        m = _bool_mask_i32(_host_array(mask), n)
    shape = (n, k) if frames == 1 else (frames, n, k)
    nn = np.empty(shape, dtype=np.int32)
    d2 = np.empty(shape, dtype=np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    rc = L.lc_knearest_many(x.ctypes.data_as(dp), n, frames, ctypes.byref(cs), k,
                            None if m is None else m.ctypes.data_as(ip), hint,
                            nn.ctypes.data_as(ip), d2.ctypes.data_as(dp))
    if rc != 0:
        _raise_from_lib(_capi.cpu_error())
    return nn, d2


def _knearest_cuda(L, xyz, cell, k, mask, hint, dev, workspace, sync):
    import torch
    x = xyz if isinstance(xyz, torch.Tensor) else torch.from_dlpack(xyz)
    if x.dtype != torch.float64:
        raise ValueError(_XYZ_SHAPE_MSG)
    x = x.contiguous()
    n, frames = _xyz_dims(tuple(x.shape))
    mptr = None
    mt = None
    if mask is not None:
        mt = mask if isinstance(mask, torch.Tensor) else torch.from_dlpack(mask)
        if not mt.is_cuda or mt.device.index != dev:
            raise ValueError("mask must be on the same CUDA device")
        if mt.numel() != n:
            raise ValueError("mask length must be n")
        if mt.dtype != torch.int32:
            mt = (mt != 0).to(torch.int32)
        mt = mt.contiguous()
        mptr = mt.data_ptr()
    ws = workspace if workspace is not None else _workspace_for(dev)
    shape = (n, k) if frames == 1 else (frames, n, k)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream()
        ws.use_stream(stream)
        nn = torch.empty(shape, dtype=torch.int32, device=x.device)
        d2 = torch.empty(shape, dtype=torch.float64, device=x.device)
        cell_cuda, cdev = _device_of(cell)
        if cell_cuda:
            ct = cell if isinstance(cell, torch.Tensor) else torch.from_dlpack(cell)
            if cdev != dev:
                raise ValueError("cell and xyz must sit on the same CUDA device")
            cn = _cell_n(tuple(ct.shape))
            ct = ct.to(torch.float64).contiguous()
            rc = L.lc_gpu_knearest_many_dcell(ws.handle, x.data_ptr(), n, frames, ct.data_ptr(),
                                              cn, k, mptr, hint, nn.data_ptr(), d2.data_ptr(),
                                              1 if sync else 0)
        else:
            cs = _cell_struct(_host_array(cell, np.float64))
            rc = L.lc_gpu_knearest_many(ws.handle, x.data_ptr(), n, frames, ctypes.byref(cs), k,
                                        mptr, hint, nn.data_ptr(), d2.data_ptr(), 1 if sync else 0)
        msg = _capi.gpu_error() if rc != 0 else None
        ws.use_stream(None)
    if rc != 0:
        _raise_from_lib(msg)
    return nn, d2


def knearest_batch(xyz, frames, mask=None, *, workspace: Workspace | None = None,
                   sync: bool = True):
    """Heterogeneous batch (extension): frames with their own cell, n, k and mask.

    xyz: float64 (sum n_f, 3), a CUDA tensor (lc_gpu_knearest_batch, CUDA
    outputs on torch's current stream) or host memory (lc_knearest_batch,
    numpy outputs). frames: list of dicts with keys n, k, cell ((3,), (3,3)
    or (4,3) host doubles), optional cell_hint and mask_offset. Returns flat
    (indices, dist2) of sum n_f * k_f entries; frame f starts at sum over
    g < f of n_g * k_g.
    """
    L = _capi.load()
    arr = (LcFrame * len(frames))()
    total = 0
    for f, fr in enumerate(frames):
        arr[f].n = int(fr["n"])
        arr[f].k = int(fr["k"])
        arr[f].cell = _cell_struct(np.asarray(fr["cell"], dtype=np.float64))
        arr[f].cell_hint = float(fr.get("cell_hint", 0.0) or 0.0)
        arr[f].mask_offset = int(fr.get("mask_offset", -1))
        total += arr[f].n * arr[f].k
    cuda_in, _ = _device_of(xyz)
    if not cuda_in:
        x = np.ascontiguousarray(_host_array(xyz), dtype=np.float64)
        m = None if mask is None else np.ascontiguousarray((_host_array(mask) != 0).astype(np.int32))
        nn = np.empty(total, dtype=np.int32)
        d2 = np.empty(total, dtype=np.float64)
        rc = L.lc_knearest_batch(x.ctypes.data, arr, len(frames),
                                 None if m is None else m.ctypes.data, nn.ctypes.data,
                                 d2.ctypes.data)
        if rc != 0:
            _raise_from_lib(_capi.cpu_error())
        return nn, d2
    import torch
    x = xyz if isinstance(xyz, torch.Tensor) else torch.from_dlpack(xyz)
    x = x.contiguous()
    if x.dtype != torch.float64:
        raise ValueError("xyz must be float64")
    dev = x.device.index
    ws = workspace if workspace is not None else _workspace_for(dev)
    with torch.cuda.device(dev):
        ws.use_stream(torch.cuda.current_stream())
        nn = torch.empty(total, dtype=torch.int32, device=x.device)
        d2 = torch.empty(total, dtype=torch.float64, device=x.device)
        mptr = None
        if mask is not None:
            mask = mask.to(torch.int32).contiguous()
            mptr = mask.data_ptr()
        rc = L.lc_gpu_knearest_batch(ws.handle, x.data_ptr(), arr, len(frames), mptr,
                                     nn.data_ptr(), d2.data_ptr(), 1 if sync else 0)
        msg = _capi.gpu_error() if rc != 0 else None
        ws.use_stream(None)
    if rc != 0:
        _raise_from_lib(msg)
    return nn, d2
