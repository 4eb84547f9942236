"""Seeded synthetic workloads of the k-nearest benchmarks.

No public dataset is involved: every input is generated here, seeded, from
the shapes, sizes and densities the benchmark configurations state.

- ``uniform_ortho``: N points i.i.d. uniform in an orthorhombic box.
- ``fcc_triclinic``: 1M FCC sites (a = 3.6) with Gaussian jitter, mapped
  into a sheared cell, 10 % shifted by integer lattice vectors, Bernoulli
  mask (k = 16).
- ``bimodal_triclinic``: 4M points in the same cell shape with a dense half
  (0.1 / unit^3) and a sparse half (0.005), 1 % of points exactly on bin
  faces and 0.5 % exact duplicates (k = 32, or 64 for the learned config).
- ``frames_batch``: many small frames with their own sheared cells,
  densities, k and masks.
"""

from __future__ import annotations

import math

import numpy as np


def sheared_rows(L: float) -> np.ndarray:
    """Rows a, b, c of the benchmark cell: a=(L,0,0), b=(0.3L,0.95L,0), c=(0.1L,0.2L,0.97L)."""
    return np.array([[L, 0.0, 0.0], [0.3 * L, 0.95 * L, 0.0], [0.1 * L, 0.2 * L, 0.97 * L]])


def widths_of(rows: np.ndarray) -> np.ndarray:
    a, b, c = rows
    det = abs(np.linalg.det(rows))
    return np.array([det / np.linalg.norm(np.cross(b, c)), det / np.linalg.norm(np.cross(c, a)),
                     det / np.linalg.norm(np.cross(a, b))])


def bins_of(rows: np.ndarray, edge: float = 3.0) -> np.ndarray:
    w = widths_of(rows)
    edge = min(edge, *w)
    return np.maximum(1, np.floor(w / edge)).astype(np.int64)


def uniform_ortho(n: int = 4096, box: float = 20.0, seed: int = 0):
    """C0: n uniform points in an orthorhombic box; k=12, hint 3.0."""
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, box, size=(n, 3))
    return dict(xyz=xyz, cell=np.array([box, box, box], dtype=np.float64), k=12, mask=None,
                cell_hint=3.0, name=f"uniform_ortho_n{n}")


def fcc_triclinic(n: int = 1_000_000, seed: int = 1, k: int = 16):
    """C1: FCC lattice (a=3.6), sigma 0.15 jitter, sheared cell at density 0.085."""
    rng = np.random.default_rng(seed)
    a0 = 3.6
    m = int(math.ceil((n / 4) ** (1.0 / 3.0)))
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1)
    sites = (g.reshape(-1, 1, 3) + base.reshape(1, 4, 3)).reshape(-1, 3) * a0
    keep = rng.permutation(sites.shape[0])[:n]
    sites = sites[keep] + rng.normal(0.0, 0.15, size=(n, 3))
    frac = sites / (m * a0)
    L = (n / (0.085 * 0.9215)) ** (1.0 / 3.0)
    rows = sheared_rows(L)
    xyz = frac @ rows
    shifted = rng.random(n) < 0.10
    shifts = rng.integers(-2, 3, size=(int(shifted.sum()), 3))
    xyz[shifted] += shifts @ rows
    mask = (rng.random(n) < 0.9).astype(np.int32)
    return dict(xyz=np.ascontiguousarray(xyz), cell=rows, k=k, mask=mask, cell_hint=3.0,
                name=f"fcc_triclinic_n{n}")


def bimodal_triclinic(n: int = 4_000_000, seed: int = 2, k: int = 32, dense: float = 0.1,
                      sparse: float = 0.005, face_frac: float = 0.01, dup_frac: float = 0.005):
    """C2 / C4: bimodal density in the sheared cell, face points and exact duplicates."""
    rng = np.random.default_rng(seed)
    mean = 0.5 * (dense + sparse)
    L = (n / (mean * 0.9215)) ** (1.0 / 3.0)
    rows = sheared_rows(L)
    n_dense = int(round(n * dense / (dense + sparse)))
    frac = rng.random((n, 3))
    frac[:n_dense, 0] *= 0.5
    frac[n_dense:, 0] = 0.5 + 0.5 * frac[n_dense:, 0]
    perm = rng.permutation(n)
    frac = frac[perm]
    nb = bins_of(rows)
    n_face = int(n * face_frac)
    idx = rng.choice(n, size=n_face, replace=False)
    axis = rng.integers(0, 3, size=n_face)
    for ax in range(3):
        sel = idx[axis == ax]
        frac[sel, ax] = rng.integers(0, nb[ax], size=sel.size) / float(nb[ax])
    xyz = frac @ rows
    n_dup = int(n * dup_frac)
    dst = rng.choice(n, size=n_dup, replace=False)
    src = rng.integers(0, n, size=n_dup)
    xyz[dst] = xyz[src]
    return dict(xyz=np.ascontiguousarray(xyz), cell=rows, k=k, mask=None, cell_hint=3.0,
                name=f"bimodal_triclinic_n{n}_k{k}")


def frames_batch(n_frames: int = 256, seed: int = 3, n_min: int = 1000, n_max: int = 200_000):
    """C3: frames with their own sheared cells, densities, k and masks.

    N is drawn log-uniform; the edges are then scaled to hold N at the drawn
    density, clamped to [20, 120], and N re-derived from the clamped volume.
    """
    rng = np.random.default_rng(seed)
    frames = []
    for _ in range(n_frames):
        n_want = math.exp(rng.uniform(math.log(n_min), math.log(n_max)))
        dens = rng.uniform(0.05, 0.12)
        ratio = rng.uniform(20.0, 120.0, size=3)
        s1, s2, s3 = rng.uniform(-0.4, 0.4, size=3)
        unit = np.array([[ratio[0], 0, 0], [s1 * ratio[1], ratio[1], 0],
                         [s2 * ratio[2], s3 * ratio[2], ratio[2]]])
        vol = abs(np.linalg.det(unit))
        scale = ((n_want / dens) / vol) ** (1.0 / 3.0)
        edges = np.clip(ratio * scale, 20.0, 120.0)
        rows = np.array([[edges[0], 0, 0], [s1 * edges[1], edges[1], 0],
                         [s2 * edges[2], s3 * edges[2], edges[2]]])
        n = int(max(2, round(abs(np.linalg.det(rows)) * dens)))
        k = int(rng.choice([4, 8, 16, 32]))
        frac = rng.random((n, 3))
        xyz = frac @ rows
        mask = (rng.random(n) < 0.95).astype(np.int32)
        frames.append(dict(xyz=np.ascontiguousarray(xyz), cell=rows, k=k, mask=mask,
                           cell_hint=3.0, n=n))
    return frames


def lcg_fracs(seed: int, count: int) -> np.ndarray:
    """The fixture generator of the reference tests (tests/agree.rs:144-147):
    s = s * 6364136223846793005 + 1 (mod 2^64), frac = (s >> 11) / 2^53."""
    out = np.empty(count)
    s = seed
    for t in range(count):
        s = (s * 6364136223846793005 + 1) % (1 << 64)
        out[t] = (s >> 11) / float(1 << 53)
    return out
