"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Indices must match exactly (tie order, masks, -1 padding) and dist2 must be
bit-identical to the reference expression (stronger than the 1e-12
relative bound). Every walk mode is checked.
"""

import numpy as np
import pytest

from gpu_helpers import DeviceRunner, assert_same, host_abi

pytestmark = pytest.mark.gpu

MODES = [0, 1, 2, 3]
HEX = [[10.0, 0.0, 0.0], [5.0, 8.660254037844386, 0.0], [0.0, 0.0, 10.0]]
TRI = [[10.0, 0.0, 0.0], [3.0, 9.0, 0.0], [1.0, 2.0, 8.0]]


@pytest.fixture(scope="module", params=[32, 1], ids=["team", "thread"])
def runner(gpu, request):
    """Both walk designs: a warp per source and a thread per source."""
    r = DeviceRunner()
    r.set_tpp(request.param)
    yield r
    r.close()


def _oracle(O, xyz, cell, k, mask=None, hint=0.0, n_frames=1):
    return O.knearest(xyz, cell, k, mask=mask, cell_hint=hint, n_frames=n_frames)


def test_reference_kats_all_paths(runner, oracle_mod, kats):
    """Every known-answer case of the reference suite, through the host ABI
    and the device ABI in every mode."""
    for cs in kats["cases"]:
        want = _oracle(oracle_mod, cs["xyz"], cs["cell"], cs["k"], cs["mask"], cs["cell_hint"])
        assert_same(host_abi(cs["xyz"], cs["cell"], cs["k"], cs["mask"], cs["cell_hint"]), want,
                    f"host {cs['name']}")
        for mode in MODES:
            runner.set_mode(mode)
            got = runner.run(cs["xyz"], cs["cell"], cs["k"], cs["mask"], cs["cell_hint"])
            assert_same(got, want, f"device mode {mode} {cs['name']}")
        if cs["expect_nn"] is not None:
            nn, _ = got
            for i, row in enumerate(cs["expect_nn"]):
                if row is not None:
                    assert nn[i].tolist() == row, cs["name"]
    runner.set_mode(0)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("cell,n,k,hint", [
    ([20.0, 20.0, 20.0], 4096, 12, 3.0),
    ([20.0, 18.0, 22.0], 1000, 1, 0.0),
    ([15.0, 15.0, 15.0], 700, 33, 2.0),
    (HEX, 900, 8, 2.0),
    (TRI, 1500, 17, 0.0),
    ([[30.0, 0, 0], [9.0, 28.5, 0], [3.0, 6.0, 29.1]], 3000, 32, 3.0),
    ([[30.0, 0, 0], [9.0, 28.5, 0], [3.0, 6.0, 29.1]], 1200, 64, 3.0),
])
def test_random_cells(runner, oracle_mod, mode, cell, n, k, hint):
    rng = np.random.default_rng(n * 31 + k)
    frac = rng.random((n, 3))
    rows = np.diag(cell) if np.asarray(cell).shape == (3,) else np.asarray(cell)
    xyz = frac @ rows + rng.integers(-3, 4, size=(n, 3)) @ rows  # points outside the cell too
    want = _oracle(oracle_mod, xyz, cell, k, hint=hint)
    runner.set_mode(mode)
    assert_same(runner.run(xyz, cell, k, hint=hint), want, f"mode {mode}")


@pytest.mark.parametrize("mode", MODES)
def test_masks(runner, oracle_mod, mode):
    rng = np.random.default_rng(7)
    xyz = rng.random((2500, 3)) * 17.0
    runner.set_mode(mode)
    for p in (0.7, 0.05):
        mask = (rng.random(2500) < p).astype(np.int32)
        want = _oracle(oracle_mod, xyz, [17.0, 17.0, 17.0], 10, mask)
        assert_same(runner.run(xyz, [17.0, 17.0, 17.0], 10, mask), want, f"p={p}")
    one = np.zeros(2500, dtype=np.int32)
    one[123] = 1
    want = _oracle(oracle_mod, xyz, [17.0, 17.0, 17.0], 4, one)
    assert_same(runner.run(xyz, [17.0, 17.0, 17.0], 4, one), want, "single active")
    none = np.zeros(2500, dtype=np.int32)
    want = _oracle(oracle_mod, xyz, [17.0, 17.0, 17.0], 4, none)
    assert_same(runner.run(xyz, [17.0, 17.0, 17.0], 4, none), want, "all masked")


@pytest.mark.parametrize("mode", MODES)
def test_duplicates_and_lattice_ties(runner, oracle_mod, mode):
    """Exact duplicates (dist2 == 0 kept, as on the CPU) and a cubic lattice
    where most k-th distances tie: the tie order must follow the reference
    heap exactly."""
    runner.set_mode(mode)
    rng = np.random.default_rng(11)
    xyz = rng.random((3000, 3)) * 16.0
    dst = rng.choice(3000, 300, replace=False)
    xyz[dst] = xyz[rng.integers(0, 3000, 300)]
    for k in (1, 5, 16):
        want = _oracle(oracle_mod, xyz, [16.0, 16.0, 16.0], k)
        assert_same(runner.run(xyz, [16.0, 16.0, 16.0], k), want, f"dups k={k}")
    # examples/knn_hot.rs:15-26: cubic lattice in a 50^3 box, hint 3.0
    nside = 16
    a = 50.0 / nside
    g = np.stack(np.meshgrid(np.arange(nside), np.arange(nside), np.arange(nside),
                             indexing="ij"), -1).reshape(-1, 3)[:, ::-1] * a
    for k in (4, 7, 19):
        want = _oracle(oracle_mod, g, [50.0, 50.0, 50.0], k, hint=3.0)
        assert_same(runner.run(g, [50.0, 50.0, 50.0], k, hint=3.0), want, f"lattice k={k}")


@pytest.mark.parametrize("mode", MODES)
def test_small_boxes_revisit_images(runner, oracle_mod, mode):
    """Meshes of 1-3 cells per axis: one cell is visited under several lattice
    shifts and the per-index minimum must win."""
    runner.set_mode(mode)
    rng = np.random.default_rng(5)
    for cell, n, k, hint in (([5.0, 5.0, 5.0], 20, 10, 3.0), ([7.0, 4.0, 9.0], 40, 39, 2.0),
                             (HEX, 30, 12, 4.0), (TRI, 25, 30, 0.0), ([3.0, 3.0, 3.0], 2, 3, 0.0)):
        rows = np.diag(cell) if np.asarray(cell).shape == (3,) else np.asarray(cell)
        xyz = rng.random((n, 3)) @ rows
        want = _oracle(oracle_mod, xyz, cell, k, hint=hint)
        assert_same(runner.run(xyz, cell, k, hint=hint), want, f"{cell} n={n} k={k}")


@pytest.mark.parametrize("mode", MODES)
def test_many_frames_share_cell_and_mask(runner, oracle_mod, mode):
    runner.set_mode(mode)
    rng = np.random.default_rng(3)
    n, F = 800, 3
    xyz = rng.random((F * n, 3)) * 12.0
    mask = (rng.random(n) < 0.8).astype(np.int32)
    want = _oracle(oracle_mod, xyz, [12.0, 12.0, 12.0], 6, mask, n_frames=F)
    assert_same(runner.run(xyz, [12.0, 12.0, 12.0], 6, mask, n_frames=F), want, "frames")
    assert_same(host_abi(xyz, [12.0, 12.0, 12.0], 6, mask, n_frames=F), want, "frames host")


@pytest.mark.parametrize("mode", MODES)
def test_lattice_ties_large_k(runner, oracle_mod, mode):
    """k of 100 and 200 on a cubic lattice with duplicates: the k-th values tie,
    so sources go through the literal warp replay with 4 and 8 heap slots per
    lane (k up to 128 and 256)."""
    runner.set_mode(mode)
    runner.set_stats(True)
    nside = 12
    a = 30.0 / nside
    g = np.stack(np.meshgrid(np.arange(nside), np.arange(nside), np.arange(nside),
                             indexing="ij"), -1).reshape(-1, 3)[:, ::-1] * a
    rng = np.random.default_rng(5)
    dup = g[rng.choice(len(g), 40, replace=False)]
    xyz = np.ascontiguousarray(np.concatenate([g, dup]), dtype=np.float64)
    try:
        for k in (100, 200):
            want = _oracle(oracle_mod, xyz, [30.0, 30.0, 30.0], k, hint=3.0)
            assert_same(runner.run(xyz, [30.0, 30.0, 30.0], k, hint=3.0), want,
                        f"lattice k={k} mode {mode}")
        cnt, _ = runner.stats()
        assert mode == 3 or cnt[2] > 0  # ties sent to the replay
    finally:
        runner.set_stats(False)
        runner.set_mode(0)


def test_large_k_and_replay_all(runner, oracle_mod):
    """k above the shared-memory heap (exact sequential walk for every source)."""
    rng = np.random.default_rng(2)
    xyz = rng.random((600, 3)) * 9.0
    for k in (257, 400):
        want = _oracle(oracle_mod, xyz, [9.0, 9.0, 9.0], k)
        assert_same(runner.run(xyz, [9.0, 9.0, 9.0], k), want, f"k={k}")


def test_nonfinite_points(runner, oracle_mod):
    """NaN coordinates: the whole frame takes the literal replay of the
    reference heap, whose comparisons treat NaN exactly like the Rust code."""
    rng = np.random.default_rng(4)
    xyz = rng.random((200, 3)) * 8.0
    xyz[17, 1] = np.nan
    xyz[40] = np.inf
    want = _oracle(oracle_mod, xyz, [8.0, 8.0, 8.0], 5)
    assert_same(runner.run(xyz, [8.0, 8.0, 8.0], 5), want, "nan")


def test_origin_and_far_images(runner, oracle_mod):
    rng = np.random.default_rng(8)
    cell = np.array([[20.0, 0, 0], [4.0, 19.0, 0], [-3.0, 2.0, 21.0], [-5.0, 7.5, 100.0]])
    xyz = rng.random((2000, 3)) * 40.0 - 1000.0
    want = _oracle(oracle_mod, xyz, cell, 9)
    assert_same(runner.run(xyz, cell, 9), want, "origin")


def test_face_points(runner, oracle_mod):
    """Points placed exactly on bin faces before the cell map (bimodal
    workload construction)."""
    from linkcell_b200 import workloads as W
    w = W.bimodal_triclinic(n=60000, seed=21, k=32, face_frac=0.2, dup_frac=0.01)
    for mode in MODES:
        runner.set_mode(mode)
        want = _oracle(oracle_mod, w["xyz"], w["cell"], 32, hint=3.0)
        assert_same(runner.run(w["xyz"], w["cell"], 32, hint=3.0), want, f"mode {mode}")


def test_batch_heterogeneous_frames(runner, oracle_mod):
    from linkcell_b200 import workloads as W
    frames = W.frames_batch(n_frames=12, seed=13, n_min=50, n_max=3000)
    runner.set_mode(0)
    nn, d2 = runner.batch(frames)
    off = 0
    for i, f in enumerate(frames):
        n, k = len(f["xyz"]), f["k"]
        want = _oracle(oracle_mod, f["xyz"], f["cell"], k, f["mask"], f["cell_hint"])
        got = (nn[off:off + n * k].reshape(n, k), d2[off:off + n * k].reshape(n, k))
        assert_same(got, want, f"frame {i}")
        off += n * k


def test_async_wait_and_reuse(runner, oracle_mod):
    rng = np.random.default_rng(1)
    for n in (5000, 300, 8000):  # grow, shrink, grow
        xyz = rng.random((n, 3)) * 25.0
        want = _oracle(oracle_mod, xyz, [25.0, 25.0, 25.0], 8)
        assert_same(runner.run(xyz, [25.0, 25.0, 25.0], 8, wait=0), want, f"n={n}")


@pytest.mark.parametrize("shell", [1, 2, 3, 6])
def test_learned_walk_any_proposal_is_exact(runner, oracle_mod, shell):
    """The learned walk opens the proposed shell with its stop bound as the
    filter; short proposals restart, long ones over-visit; results never
    change."""
    from linkcell_b200 import workloads as W
    w = W.bimodal_triclinic(n=80000, seed=31, k=32)
    want = _oracle(oracle_mod, w["xyz"], w["cell"], 32, hint=3.0)
    runner.set_mode(2)
    runner.set_proposal(shell)
    runner.set_stats(True)  # the warp walk counts only on request
    try:
        assert_same(runner.run(w["xyz"], w["cell"], 32, hint=3.0), want, f"proposal {shell}")
        cnt, _ = runner.stats()
        under, over, exact = cnt[6], cnt[7], cnt[8]
        assert under + over + exact > 0
        if shell == 1:
            assert under > 0
    finally:
        runner.set_stats(False)
        runner.set_proposal(0)
        runner.set_mode(0)


@pytest.mark.parametrize("k", [1, 17, 48, 64])
@pytest.mark.parametrize("shell", [2, 4])
def test_learned_walk_k_up_to_64(runner, oracle_mod, k, shell):
    """The cube select walk serves k up to 64 (S buffer of 128); smaller and
    larger k, any proposal, same rows as the reference."""
    from linkcell_b200 import workloads as W
    w = W.bimodal_triclinic(n=40000, seed=57 + k, k=k)
    want = _oracle(oracle_mod, w["xyz"], w["cell"], k, hint=3.0)
    runner.set_mode(2)
    runner.set_proposal(shell)
    try:
        assert_same(runner.run(w["xyz"], w["cell"], k, hint=3.0), want, f"k={k} proposal {shell}")
    finally:
        runner.set_proposal(0)
        runner.set_mode(0)


def test_fp32_counters_show_filtering(runner, oracle_mod):
    from linkcell_b200 import workloads as W
    w = W.bimodal_triclinic(n=100000, seed=41, k=16)
    runner.set_mode(1)
    runner.run(w["xyz"], w["cell"], 16, hint=3.0)
    cnt, ms = runner.stats()
    pairs, reranks, pruned = cnt[0], cnt[5], cnt[4]
    assert reranks < pairs and pruned > 0 and ms > 0
    runner.set_mode(0)
