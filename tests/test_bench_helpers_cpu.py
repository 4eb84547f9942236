"""bench.py helpers that need no GPU: the cell edge of the gpulite baseline
and the workload names."""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    sys.path.insert(0, ROOT)
    import bench
    return bench


def _cells(cell, edge):
    """The reference mesh of a cell at a given edge (src/knearest.rs:42-48,377-397)."""
    h = np.asarray(cell, dtype=np.float64)
    a, b, c = h
    det = abs(float(np.dot(a, np.cross(b, c))))
    widths = [det / np.linalg.norm(np.cross(b, c)), det / np.linalg.norm(np.cross(c, a)),
              det / np.linalg.norm(np.cross(a, b))]
    edge = min(edge, *widths)
    return int(np.prod([max(1, int(np.floor(w / edge))) for w in widths]))


def test_gpulite_hint_is_the_finest_mesh_under_the_cap():
    B = _bench()
    from linkcell_b200 import workloads as W
    for L in (120.0, 260.0, 435.65):
        cell = W.sheared_rows(L)
        edge = B.gpulite_hint(cell)
        assert _cells(cell, edge) <= B.GPULITE_CELLS
        if edge > 3.0:
            assert _cells(cell, round(edge - 0.05, 2)) > B.GPULITE_CELLS


def test_workload_names():
    B = _bench()
    assert B.workload_name(4_000_000, 32) == "bimodal_triclinic_4M_k32"
    assert B.workload_name(1_000_000, 32) == "bimodal_triclinic_n1000000_k32"
    assert B.workload_name(4_000_000, 64) == "bimodal_triclinic_n4000000_k64"
