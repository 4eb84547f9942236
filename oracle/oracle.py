"""ctypes view of the CPU oracle (test infrastructure, not product code).

The oracle restates the reference CPU walk (HaoZeke/linkcell v0.3.3,
src/cell.rs + src/knearest.rs + src/capi.rs) in C++; see linkcell_oracle.cpp.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblinkcell_oracle.so")


class OrcCell(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("ax", "ay", "az", "bx", "by", "bz", "cx", "cy", "cz", "ox", "oy", "oz")]


def build() -> str:
    """Compile the oracle library with its Makefile (g++ -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        llp = ctypes.POINTER(ctypes.c_longlong)
        cp = ctypes.POINTER(OrcCell)
        sz = ctypes.c_size_t
        L.orc_knearest_many.argtypes = [dp, sz, sz, cp, sz, ip, ctypes.c_double, ip, dp, ctypes.c_int]
        L.orc_knearest_many.restype = ctypes.c_int
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_knearest_brute.argtypes = [dp, sz, cp, sz, ip, ip, dp]
        L.orc_knearest_mic27.argtypes = [dp, sz, cp, sz, ip, ip, dp]
        L.orc_cell_info.argtypes = [cp, ctypes.c_double, dp, dp, dp, ip]
        L.orc_fold_bin.argtypes = [dp, sz, cp, ip, ctypes.c_double, dp, ip]
        L.orc_walk_stats.argtypes = [dp, sz, cp, sz, ip, ctypes.c_double, ip, llp, ctypes.c_int]
        L.orc_time_sample.argtypes = [dp, sz, cp, sz, ip, ctypes.c_double, sz, sz, sz, ctypes.c_int,
                                      dp, dp, llp, llp]
        L.orc_knearest_subset.argtypes = [dp, sz, cp, sz, ip, ctypes.c_double, llp, sz, ip, dp,
                                          ctypes.c_int, llp]
        L.orc_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def make_cell(cell) -> OrcCell:
    """Cell from (3,) ortho lengths, (3,3) lattice rows or (4,3) rows + origin."""
    c = np.asarray(cell, dtype=np.float64)
    if c.shape == (3,):
        rows = np.diag(c)
        origin = np.zeros(3)
    elif c.shape == (3, 3):
        rows, origin = c, np.zeros(3)
    elif c.shape == (4, 3):
        rows, origin = c[:3], c[3]
    else:
        raise ValueError("cell must be (3,), (3,3) or (4,3)")
    vals = list(rows.reshape(-1)) + list(origin)
    return OrcCell(*[float(v) for v in vals])


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class OracleError(RuntimeError):
    pass


def last_error() -> str | None:
    m = lib().orc_last_error()
    return None if m is None else m.decode()


def knearest(xyz, cell, k, mask=None, cell_hint=0.0, n_frames=1, threads=0):
    """Reference walk. Returns (indices int32, dist2 float64) shaped (F*n, k)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0] // n_frames
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    nn = np.empty((n * n_frames, k), dtype=np.int32)
    d2 = np.empty((n * n_frames, k), dtype=np.float64)
    oc = make_cell(cell)
    rc = lib().orc_knearest_many(_dptr(xyz), n, n_frames, ctypes.byref(oc), k, _iptr(m),
                                 float(cell_hint or 0.0), _iptr(nn), _dptr(d2), threads)
    if rc != 0:
        raise OracleError(last_error())
    return nn, d2


def _brute(fn, xyz, cell, k, mask=None):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    nn = np.empty((n, k), dtype=np.int32)
    d2 = np.empty((n, k), dtype=np.float64)
    oc = make_cell(cell)
    rc = fn(_dptr(xyz), n, ctypes.byref(oc), k, _iptr(m), _iptr(nn), _dptr(d2))
    if rc != 0:
        raise OracleError(last_error())
    return nn, d2


def brute(xyz, cell, k, mask=None):
    """knearest_brute (src/knearest.rs:508-541)."""
    return _brute(lib().orc_knearest_brute, xyz, cell, k, mask)


def mic27(xyz, cell, k, mask=None):
    """oracle_knearest (tests/agree.rs:186-210)."""
    return _brute(lib().orc_knearest_mic27, xyz, cell, k, mask)


def cell_info(cell, cell_hint=0.0):
    info = np.zeros(5)
    h = np.zeros(9)
    hinv = np.zeros(9)
    grid = np.zeros(4, dtype=np.int32)
    oc = make_cell(cell)
    rc = lib().orc_cell_info(ctypes.byref(oc), float(cell_hint), _dptr(info), _dptr(h), _dptr(hinv),
                             _iptr(grid))
    return rc, dict(widths=info[:3].copy(), cell_min=float(info[3]), ortho=bool(info[4]),
                    h=h, hinv=hinv, nx=int(grid[0]), ny=int(grid[1]), nz=int(grid[2]),
                    max_reach=int(grid[3]))


def fold_bin(xyz, cell, mask=None, cell_hint=0.0):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    folded = np.empty((n, 3))
    cid = np.empty(n, dtype=np.int32)
    oc = make_cell(cell)
    rc = lib().orc_fold_bin(_dptr(xyz), n, ctypes.byref(oc), _iptr(m), float(cell_hint),
                            _dptr(folded), _iptr(cid))
    if rc != 0:
        raise OracleError(last_error())
    return folded, cid


def walk_stats(xyz, cell, k, mask=None, cell_hint=0.0, threads=0):
    """Per-source stop reach and heap-push counts of the reference walk."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    reach = np.empty(n, dtype=np.int32)
    visits = np.empty(n, dtype=np.int64)
    oc = make_cell(cell)
    rc = lib().orc_walk_stats(_dptr(xyz), n, ctypes.byref(oc), k, _iptr(m), float(cell_hint),
                              _iptr(reach), visits.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)),
                              threads)
    if rc != 0:
        raise OracleError(last_error())
    return reach, visits


def time_sample(xyz, cell, k, mask=None, cell_hint=0.0, first=0, stride=1, count=None, threads=0):
    """Times the reference fold/bin over all points plus the walk of a sample."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    if count is None:
        count = n
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    prep = ctypes.c_double()
    walk = ctypes.c_double()
    walked = ctypes.c_longlong()
    chk = ctypes.c_longlong()
    oc = make_cell(cell)
    rc = lib().orc_time_sample(_dptr(xyz), n, ctypes.byref(oc), k, _iptr(m), float(cell_hint),
                               first, stride, count, threads, ctypes.byref(prep), ctypes.byref(walk),
                               ctypes.byref(walked), ctypes.byref(chk))
    if rc != 0:
        raise OracleError(last_error())
    return dict(prep_s=prep.value, walk_s=walk.value, walked=walked.value, checksum=chk.value)


def knearest_subset(xyz, cell, k, sources, mask=None, cell_hint=0.0, threads=0,
                    with_visits=False):
    """Reference rows for the given source indices only: (len(sources), k).
    with_visits also returns each source's heap pushes (the candidate pairs
    the reference walk evaluates for it)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = xyz.shape[0]
    src = np.ascontiguousarray(sources, dtype=np.int64)
    m = None if mask is None else np.ascontiguousarray(mask, dtype=np.int32)
    nn = np.empty((src.size, k), dtype=np.int32)
    d2 = np.empty((src.size, k), dtype=np.float64)
    visits = np.zeros(src.size, dtype=np.int64) if with_visits else None
    oc = make_cell(cell)
    llp = ctypes.POINTER(ctypes.c_longlong)
    rc = lib().orc_knearest_subset(_dptr(xyz), n, ctypes.byref(oc), k, _iptr(m), float(cell_hint),
                                   src.ctypes.data_as(llp), src.size, _iptr(nn), _dptr(d2),
                                   threads, None if visits is None else visits.ctypes.data_as(llp))
    if rc != 0:
        raise OracleError(last_error())
    return (nn, d2, visits) if with_visits else (nn, d2)
