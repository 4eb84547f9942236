"""Seeded random sweep of the device path against the oracle.

Each case draws a cell (orthorhombic or sheared, with an origin), a point
count, k (sometimes above the point count), a cell hint, points inside and
far outside the cell with exact duplicates and points on bin faces, an
optional mask (sometimes all zero), one to three frames, a walk mode, a
walk design and, for the learned mode, the shipped network or a fixed
shell proposal. Every row must equal the oracle's: indices, tie order, -1
padding and dist2 bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from gpu_helpers import DeviceRunner, assert_same

pytestmark = pytest.mark.gpu

CASES = 480


def _case(seed):
    rng = np.random.default_rng(1000 + seed)
    lengths = rng.uniform(4.0, 40.0, size=3)
    if rng.random() < 0.35:
        rows = np.diag(lengths)
    else:
        s = rng.uniform(-0.45, 0.45, size=3)
        rows = np.array([[lengths[0], 0.0, 0.0],
                         [s[0] * lengths[1], lengths[1], 0.0],
                         [s[1] * lengths[2], s[2] * lengths[2], lengths[2]]])
    origin = rng.uniform(-50.0, 50.0, size=3) if rng.random() < 0.3 else np.zeros(3)
    cell = np.vstack([rows, origin])
    n = int(np.exp(rng.uniform(0.0, np.log(5000.0))))
    # k past the point count (padding) only on small frames: above 256 every
    # source takes the literal replay, whose cost grows with n k
    k = int(rng.integers(1, 81)) if (n > 64 or rng.random() < 0.7) else int(n + rng.integers(0, 5))
    hint = 0.0 if rng.random() < 0.3 else float(rng.uniform(0.7, 9.0))
    frames = int(rng.integers(1, 4))
    frac = rng.random((frames * n, 3))
    faces = rng.random(frames * n) < 0.05
    frac[faces] = np.round(frac[faces] * 8.0) / 8.0  # exactly on bin faces of many meshes
    xyz = frac @ rows + origin
    far = rng.random(frames * n) < 0.1
    xyz[far] += rng.integers(-4, 5, size=(int(far.sum()), 3)) @ rows
    dup = np.flatnonzero(rng.random(frames * n) < 0.03)
    if dup.size and n > 1:
        xyz[dup] = xyz[rng.integers(0, frames * n, size=dup.size)]
    mask = None
    u = rng.random()
    if u < 0.25:
        mask = (rng.random(n) < rng.uniform(0.3, 0.95)).astype(np.int32)
    elif u < 0.28:
        mask = np.zeros(n, dtype=np.int32)
    mode = int(rng.integers(0, 4))
    tpp = 32 if rng.random() < 0.5 else 1
    shell = int(rng.integers(1, 7)) if (mode == 2 and rng.random() < 0.4) else 0
    return dict(cell=cell, n=n, k=k, hint=hint, frames=frames, xyz=xyz, mask=mask, mode=mode,
                tpp=tpp, shell=shell)


@pytest.fixture(scope="module")
def fuzz_runner(gpu):
    r = DeviceRunner()
    yield r
    r.close()


@pytest.mark.parametrize("block", range(8))
def test_random_sweep(fuzz_runner, oracle_mod, block):
    r = fuzz_runner
    per = CASES // 8
    for seed in range(block * per, (block + 1) * per):
        c = _case(seed)
        want = oracle_mod.knearest(c["xyz"], c["cell"], c["k"], mask=c["mask"],
                                   cell_hint=c["hint"], n_frames=c["frames"])
        r.set_mode(c["mode"])
        r.set_tpp(c["tpp"])
        r.set_proposal(c["shell"])
        r.set_stats(seed % 2 == 1)  # both builds of the warp walk: counting and not
        got = r.run(c["xyz"], c["cell"], c["k"], mask=c["mask"], hint=c["hint"],
                    n_frames=c["frames"])
        label = (f"seed {seed}: n={c['n']} k={c['k']} frames={c['frames']} hint={c['hint']:.2f} "
                 f"mode={c['mode']} tpp={c['tpp']} shell={c['shell']} "
                 f"mask={'none' if c['mask'] is None else int(c['mask'].sum())}")
        assert_same(got, want, label)


def _frame(rng):
    """One frame of a heterogeneous batch: its own cell, n, k, hint, mask."""
    lengths = rng.uniform(5.0, 30.0, size=3)
    s = rng.uniform(-0.4, 0.4, size=3) * (rng.random() < 0.6)
    rows = np.array([[lengths[0], 0.0, 0.0],
                     [s[0] * lengths[1], lengths[1], 0.0],
                     [s[1] * lengths[2], s[2] * lengths[2], lengths[2]]])
    n = int(np.exp(rng.uniform(0.0, np.log(3000.0))))
    k = int(rng.integers(1, 65))
    xyz = rng.random((n, 3)) @ rows + rng.integers(-2, 3, size=(n, 3)) @ rows
    mask = (rng.random(n) < 0.9).astype(np.int32) if rng.random() < 0.4 else None
    hint = float(rng.uniform(1.0, 6.0)) if rng.random() < 0.7 else 0.0
    return dict(xyz=xyz, cell=rows, k=k, mask=mask, cell_hint=hint)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_random_batches(fuzz_runner, oracle_mod, mode):
    """lc_gpu_knearest_batch with random heterogeneous frames."""
    r = fuzz_runner
    r.set_mode(mode)
    r.set_tpp(0)
    r.set_proposal(0)
    for b in range(12):
        rng = np.random.default_rng(5000 + 100 * mode + b)
        frames = [_frame(rng) for _ in range(int(rng.integers(1, 7)))]
        nn, d2 = r.batch(frames)
        off = 0
        for i, f in enumerate(frames):
            n, k = len(f["xyz"]), f["k"]
            want = oracle_mod.knearest(f["xyz"], f["cell"], k, mask=f["mask"],
                                       cell_hint=f["cell_hint"])
            got = (nn[off:off + n * k].reshape(n, k), d2[off:off + n * k].reshape(n, k))
            assert_same(got, want, f"batch {b} mode {mode} frame {i}")
            off += n * k


def test_random_device_cells(fuzz_runner, oracle_mod):
    """lc_gpu_knearest_many_dcell (the cell planned on the device) on random
    cells in each of its layouts."""
    import torch
    r = fuzz_runner
    r.set_tpp(0)
    r.set_proposal(0)
    for seed in range(36):
        rng = np.random.default_rng(7000 + seed)
        c = _case(seed + 10_000)
        if c["k"] > 256:
            continue
        rows, origin = c["cell"][:3], c["cell"][3]
        cell_n = [3, 9, 12][seed % 3]
        if cell_n == 3:
            rows = np.diag(np.diag(rows))
            origin = np.zeros(3)
            vals = np.diag(rows)
        elif cell_n == 9:
            origin = np.zeros(3)
            vals = rows.reshape(-1)
        else:
            vals = np.concatenate([rows.reshape(-1), origin])
        n, frames, k = c["n"], c["frames"], c["k"]
        xyz = rng.random((frames * n, 3)) @ rows + origin
        xyz += rng.integers(-2, 3, size=(frames * n, 3)) @ rows
        want = oracle_mod.knearest(xyz, np.vstack([rows, origin]), k, mask=c["mask"],
                                   cell_hint=c["hint"], n_frames=frames)
        r.set_mode(c["mode"])
        x = torch.as_tensor(xyz, device="cuda")
        cd = torch.as_tensor(np.array(vals, dtype=np.float64), device="cuda")
        m = None if c["mask"] is None else torch.as_tensor(c["mask"], device="cuda")
        nn = torch.full((frames * n, k), -9, dtype=torch.int32, device="cuda")
        d2 = torch.zeros((frames * n, k), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = r.L.lc_gpu_knearest_many_dcell(r.ws, x.data_ptr(), n, frames, cd.data_ptr(), cell_n,
                                            k, None if m is None else m.data_ptr(), c["hint"],
                                            nn.data_ptr(), d2.data_ptr(), 1)
        assert rc == 0, seed
        assert_same((nn.cpu().numpy(), d2.cpu().numpy()), want, f"dcell seed {seed} cell_n {cell_n}")
