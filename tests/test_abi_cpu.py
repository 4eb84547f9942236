"""The product C ABI without a GPU: it loads, exports every declared symbol,
and its argument checks give the reference's messages in the reference's
order (src/capi.rs:195-227, tests/abi.rs). No compute call is made."""

import ctypes
import os
import re
import threading

import numpy as np
import pytest

from conftest import ROOT, has_gpu


def _declared_symbols():
    names = set()
    for hdr in ("linkcell.h", "linkcell_gpu.h"):
        text = open(os.path.join(ROOT, "include", hdr)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(lc_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    names.discard("lc_cell_ortho")  # static inline in the header
    return sorted(names)


def test_exports_every_declared_symbol(lib):
    from linkcell_b200 import _capi
    declared = _declared_symbols()
    assert len(declared) >= 22
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_capi.EXPORTS)


def test_version(lib):
    assert lib.lc_version() == b"0.3.3"


def _cell(lx=10.0, ly=10.0, lz=10.0):
    from linkcell_b200 import LcCell
    return LcCell(lx, 0, 0, 0, ly, 0, 0, 0, lz, 0, 0, 0)


def _call(lib, xyz, n, k, mask=None, hint=0.0, cell=None, out=None):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.full(max(1, n * k if n * k < 10**6 else 1), -7, dtype=np.int32) if out is None else out
    c = _cell() if cell is None else cell
    mp = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32).ctypes.data_as(
        ctypes.POINTER(ctypes.c_int))
    rc = lib.lc_knearest(xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n,
                         ctypes.byref(c), k, mp, hint,
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return rc, out


def test_error_order_and_messages(lib):
    rc, _ = _call(lib, np.zeros(3), 0, 1)
    assert rc != 0 and lib.lc_last_error() == b"no points"
    rc, _ = _call(lib, np.zeros(3), 1, 0)
    assert rc != 0 and lib.lc_last_error() == b"k must be at least 1"
    # tests/abi.rs:308-320: n = isize::MAX / 3 + 1
    rc, _ = _call(lib, np.zeros(3), (2**63 - 1) // 3 + 1, 1)
    assert rc != 0 and lib.lc_last_error() == b"n * k overflows"
    from linkcell_b200 import LcCell
    bad = LcCell(1, 0, 0, 2, 0, 0, 0, 0, 1, 0, 0, 0)
    rc, _ = _call(lib, np.zeros(6), 2, 1, cell=bad)
    assert rc != 0 and lib.lc_last_error() == b"singular or non-positive cell"
    rc, _ = _call(lib, np.random.default_rng(1).random(12) * 10, 4, 1, hint=1e-9)
    assert rc != 0 and lib.lc_last_error() == b"linked-cell mesh is too fine"


def test_null_pointer(lib):
    c = _cell()
    out = np.zeros(2, dtype=np.int32)
    rc = lib.lc_knearest(None, 2, ctypes.byref(c), 1, None, 0.0,
                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert rc != 0 and lib.lc_last_error() == b"null pointer"
    assert lib.lc_gpu_knearest_many(None, None, 2, 1, None, 1, None, 0.0, None, None, 1) == 1
    assert lib.lc_gpu_last_error() == b"null pointer"


def test_all_masked_needs_no_mesh(lib):
    """src/knearest.rs:370-375: all-masked input succeeds with -1 rows even when
    the mesh would be too fine; nothing runs on a device."""
    out = np.full(6, 5, dtype=np.int32)
    rc, out = _call(lib, np.zeros(9), 3, 2, mask=[0, 0, 0], hint=1e-9, out=out)
    assert rc == 0 and lib.lc_last_error() is None
    assert (out == -1).all()


def test_version_leaves_error_slot(lib):
    """tests/abi.rs:289-306."""
    _call(lib, np.zeros(3), 0, 1)
    before = lib.lc_last_error()
    lib.lc_version()
    assert lib.lc_last_error() == before == b"no points"


def test_error_slots_are_thread_local(lib):
    """tests/abi.rs:264-287."""
    seen = {}

    def a():
        _call(lib, np.zeros(3), 0, 1)
        seen["a"] = lib.lc_last_error()

    def b():
        _call(lib, np.zeros(3), 1, 0)
        seen["b"] = lib.lc_last_error()

    ta, tb = threading.Thread(target=a), threading.Thread(target=b)
    ta.start(); tb.start(); ta.join(); tb.join()
    assert seen == {"a": b"no points", "b": b"k must be at least 1"}


@pytest.mark.skipif(has_gpu(), reason="checks the no-device message")
def test_no_device_fails_loudly(lib):
    rc, _ = _call(lib, np.array([0.0, 0, 0, 1, 0, 0]), 2, 1)
    assert rc != 0 and lib.lc_last_error() == b"no CUDA device available"
    assert lib.lc_gpu_available() == 0
    assert lib.lc_gpu_workspace_new() is None
    assert lib.lc_gpu_last_error() == b"CUDA driver or nvrtc not loaded"


def test_struct_layout():
    from linkcell_b200 import LcCell, LcFrame
    assert ctypes.sizeof(LcCell) == 12 * 8
    assert ctypes.sizeof(LcFrame) == 8 + 8 + 96 + 8 + 8


def test_host_batch_argument_checks(lib):
    """lc_knearest_batch validates every frame before it needs a device."""
    from linkcell_b200 import LcCell, LcFrame
    L = lib
    xyz = np.zeros((4, 3))
    out = np.zeros(64, dtype=np.int32)

    def call(frames, mask=None):
        arr = (LcFrame * len(frames))(*frames)
        return L.lc_knearest_batch(xyz.ctypes.data, arr, len(frames),
                                   None if mask is None else mask.ctypes.data, out.ctypes.data,
                                   None)

    box = LcCell(10.0, 0, 0, 0, 10.0, 0, 0, 0, 10.0, 0, 0, 0)
    flat = LcCell(10.0, 0, 0, 20.0, 0, 0, 0, 0, 10.0, 0, 0, 0)  # a and b parallel
    good = LcFrame(2, 2, box, 0.0, -1)
    assert call([good, LcFrame(0, 2, box, 0.0, -1)]) == 1
    assert L.lc_last_error() == b"no points"
    assert call([good, LcFrame(2, 0, box, 0.0, -1)]) == 1
    assert L.lc_last_error() == b"k must be at least 1"
    assert call([good, LcFrame(2, 2, box, 0.0, 0)]) == 1  # masked frame, no mask
    assert L.lc_last_error() == b"null pointer"
    assert call([good, LcFrame(2, 2, flat, 0.0, -1)]) == 1
    assert L.lc_last_error() == b"singular or non-positive cell"
    assert call([]) == 1
    assert L.lc_last_error() == b"no points"
    if not has_gpu():
        assert call([good, good]) == 1
        assert L.lc_last_error() == b"no CUDA device available"
