"""ctypes binding of liblinkcell_b200.so (the C ABI of include/linkcell*.h).

The library must exist (``python -m linkcell_b200.build``); importing the
package without it raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblinkcell_b200.so")


class LcCell(ctypes.Structure):
    """struct lc_cell: rows a, b, c and the origin."""

    _fields_ = [(n, ctypes.c_double) for n in
                ("ax", "ay", "az", "bx", "by", "bz", "cx", "cy", "cz", "ox", "oy", "oz")]


class LcFrame(ctypes.Structure):
    """struct lc_frame of lc_gpu_knearest_batch."""

    _fields_ = [("n", ctypes.c_size_t), ("k", ctypes.c_size_t), ("cell", LcCell),
                ("cell_hint", ctypes.c_double), ("mask_offset", ctypes.c_longlong)]


# Every symbol include/linkcell.h and include/linkcell_gpu.h declare.
EXPORTS = (
    "lc_knearest", "lc_knearest_d2", "lc_knearest_many", "lc_last_error", "lc_version",
    "lc_gpu_available", "lc_gpu_last_error", "lc_gpu_workspace_new", "lc_gpu_workspace_free",
    "lc_gpu_knearest", "lc_gpu_knearest_many", "lc_gpu_knearest_many_dcell", "lc_gpu_queue",
    "lc_gpu_wait", "lc_gpu_alloc", "lc_gpu_free", "lc_gpu_fill_i32", "lc_gpu_memcpy",
    "lc_gpu_set_mode", "lc_gpu_get_mode", "lc_gpu_set_proposal", "lc_gpu_set_tpp",
    "lc_gpu_get_tpp", "lc_gpu_set_graph", "lc_gpu_graph_captures", "lc_gpu_set_stream", "lc_gpu_stats",
    "lc_gpu_set_stats", "lc_gpu_set_scan_limit",
    "lc_gpu_phase_times", "lc_gpu_phase_times4", "lc_gpu_neighbors_within", "lc_gpu_set_model", "lc_gpu_log_shells", "lc_gpu_training_rows",
    "lc_gpu_proposals",
    "lc_gpu_mlp_params", "lc_gpu_mlp_scratch_floats", "lc_gpu_mlp_forward", "lc_gpu_mlp_grad",
    "lc_gpu_mlp_adam",
    "lc_gpu_knearest_batch", "lc_gpu_knearest_noalloc", "lc_knearest_batch",
    "lc_gpu_knearest_shard", "lc_gpu_set_walk_shape", "lc_gpu_walk_shape",
)

_lib = None


def load():
    """Load the library and declare every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m linkcell_b200.build` "
            "(the search has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    vp = ctypes.c_void_p
    sz = ctypes.c_size_t
    cp = ctypes.POINTER(LcCell)
    d = ctypes.c_double
    i = ctypes.c_int
    L.lc_knearest.argtypes = [dp, sz, cp, sz, ip, d, ip]
    L.lc_knearest_d2.argtypes = [dp, sz, cp, sz, ip, d, ip, dp]
    L.lc_knearest_many.argtypes = [dp, sz, sz, cp, sz, ip, d, ip, dp]
    for f in ("lc_knearest", "lc_knearest_d2", "lc_knearest_many"):
        getattr(L, f).restype = i
    L.lc_last_error.restype = ctypes.c_char_p
    L.lc_version.restype = ctypes.c_char_p
    L.lc_gpu_available.restype = i
    L.lc_gpu_last_error.restype = ctypes.c_char_p
    L.lc_gpu_workspace_new.restype = vp
    L.lc_gpu_workspace_free.argtypes = [vp]
    L.lc_gpu_knearest.argtypes = [vp, vp, sz, cp, sz, vp, d, vp, vp]
    L.lc_gpu_knearest_many.argtypes = [vp, vp, sz, sz, cp, sz, vp, d, vp, vp, i]
    L.lc_gpu_knearest_many_dcell.argtypes = [vp, vp, sz, sz, vp, i, sz, vp, d, vp, vp, i]
    L.lc_gpu_queue.argtypes = [vp]
    L.lc_gpu_queue.restype = vp
    L.lc_gpu_wait.argtypes = [vp]
    L.lc_gpu_alloc.argtypes = [ctypes.POINTER(vp), sz]
    L.lc_gpu_free.argtypes = [vp]
    L.lc_gpu_fill_i32.argtypes = [vp, i, sz]
    L.lc_gpu_memcpy.argtypes = [vp, vp, sz, i]
    L.lc_gpu_set_mode.argtypes = [vp, i]
    L.lc_gpu_get_mode.argtypes = [vp]
    L.lc_gpu_set_proposal.argtypes = [vp, i]
    L.lc_gpu_set_tpp.argtypes = [vp, i]
    L.lc_gpu_get_tpp.argtypes = [vp]
    L.lc_gpu_set_walk_shape.argtypes = [vp, i, i]
    L.lc_gpu_walk_shape.argtypes = [vp, ip, ip, i]
    L.lc_gpu_set_graph.argtypes = [vp, i]
    L.lc_gpu_graph_captures.argtypes = [vp]
    L.lc_gpu_set_stats.argtypes = [vp, i]
    L.lc_gpu_set_scan_limit.argtypes = [vp, i, ctypes.c_longlong]
    L.lc_gpu_set_stream.argtypes = [vp, vp]
    L.lc_gpu_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), i, dp]
    L.lc_gpu_phase_times.argtypes = [vp, dp, dp, dp]
    L.lc_gpu_phase_times4.argtypes = [vp, dp, dp, dp, dp]
    L.lc_gpu_neighbors_within.argtypes = [vp, vp, vp, sz, sz, ctypes.c_double, vp, vp, vp, sz,
                                          ctypes.POINTER(sz)]
    fp = ctypes.POINTER(ctypes.c_float)
    ll = ctypes.c_longlong
    L.lc_gpu_set_model.argtypes = [vp, fp, sz, ctypes.c_float]
    L.lc_gpu_log_shells.argtypes = [vp, i]
    L.lc_gpu_training_rows.argtypes = [vp, vp, vp, ll, ll, ll]
    L.lc_gpu_training_rows.restype = ll
    L.lc_gpu_proposals.argtypes = [vp, vp, ll, ll, ll]
    L.lc_gpu_proposals.restype = ll
    L.lc_gpu_mlp_params.restype = i
    L.lc_gpu_mlp_scratch_floats.argtypes = [i]
    L.lc_gpu_mlp_scratch_floats.restype = sz
    L.lc_gpu_mlp_forward.argtypes = [vp, vp, i, vp, vp, vp]
    L.lc_gpu_mlp_grad.argtypes = [vp, vp, vp, i, vp, vp, vp, vp]
    L.lc_gpu_mlp_adam.argtypes = [vp, vp, vp, vp, i, ctypes.c_float, vp]
    L.lc_gpu_knearest_batch.argtypes = [vp, vp, ctypes.POINTER(LcFrame), sz, vp, vp, vp, i]
    L.lc_knearest_batch.argtypes = [vp, ctypes.POINTER(LcFrame), sz, vp, vp, vp]
    L.lc_gpu_knearest_noalloc.argtypes = [vp, sz, cp, sz, vp, d, vp, vp, vp, i]
    L.lc_gpu_knearest_shard.argtypes = [vp, vp, sz, sz, cp, sz, vp, d, i, i, vp, vp, vp, i]
    _lib = L
    return L


def cpu_error() -> str:
    m = load().lc_last_error()
    return m.decode() if m else "linkcell: knearest failed"


def gpu_error() -> str:
    m = load().lc_gpu_last_error()
    return m.decode() if m else "gpu knearest failed"
