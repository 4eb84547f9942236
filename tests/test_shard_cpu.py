"""The search split across ranks (linkcell_b200.shard) on CPU: two and three
gloo ranks, each holding the same input. The device share is replaced by a
stand-in built from the oracle's rows, cut the way the device cuts them
(contiguous ranges of the cell-sorted sources; masked rows owned by rank 0;
every other row left as garbage), so that the test exercises the split,
the ownership and the all-reduce combine. The combined rows must equal the
one-rank search bit for bit on every rank."""

from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CELL = [[24.0, 0.0, 0.0], [5.0, 23.0, 0.0], [2.0, 4.0, 22.0]]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    rng = np.random.default_rng(21)
    xyz = rng.random((1500, 3)) @ np.asarray(CELL)
    mask = (rng.random(1500) < 0.85).astype(np.int32)
    return xyz, mask


def _oracle_share(xyz, cell, k, mask, cell_hint, *, rank, world):
    """Rows of this rank's contiguous range of cell-sorted active sources,
    garbage elsewhere (as the device leaves another rank's rows)."""
    import torch
    from oracle import oracle as O
    O.build()
    want_nn, want_d2 = O.knearest(xyz, cell, k, mask=mask, cell_hint=cell_hint)
    _, cid = O.fold_bin(xyz, cell, mask=mask, cell_hint=cell_hint)
    active = np.flatnonzero(mask != 0)
    order = active[np.argsort(cid[active], kind="stable")]
    cuts = [len(order) * r // world for r in range(world + 1)]
    mine = order[cuts[rank]:cuts[rank + 1]]
    owned = np.zeros(len(xyz), dtype=np.int32)
    owned[mine] = 1
    if rank == 0:
        owned[mask == 0] = 1
    nn = np.full(want_nn.shape, 777 + rank, dtype=np.int32)
    d2 = np.full(want_d2.shape, 3.5 + rank)
    nn[owned != 0] = want_nn[owned != 0]
    d2[owned != 0] = want_d2[owned != 0]
    return torch.as_tensor(nn), torch.as_tensor(d2), torch.as_tensor(owned)


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from linkcell_b200 import shard
        xyz, mask = _inputs()
        nn, d2 = shard.knearest_sharded(xyz, CELL, 9, mask, 3.0, search=_oracle_share)
        q.put((rank, nn.numpy().tobytes(), d2.numpy().tobytes()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_split_search_combines_to_the_one_rank_rows(world):
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    O.build()
    xyz, mask = _inputs()
    want_nn, want_d2 = O.knearest(xyz, CELL, 9, mask=mask, cell_hint=3.0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, nn_b, d2_b in got:
        nn = np.frombuffer(nn_b, dtype=np.int32).reshape(want_nn.shape)
        d2 = np.frombuffer(d2_b, dtype=np.float64).reshape(want_d2.shape)
        assert np.array_equal(nn, want_nn), f"rank {rank}: indices differ"
        same = (d2 == want_d2) | (np.isnan(d2) & np.isnan(want_d2))
        assert same.all(), f"rank {rank}: dist2 differs"


def test_one_process_is_the_whole_search():
    sys.path.insert(0, ROOT)
    from linkcell_b200 import shard
    from oracle import oracle as O
    O.build()
    xyz, mask = _inputs()
    nn, d2 = shard.knearest_sharded(xyz, CELL, 5, mask, 3.0, search=_oracle_share)
    want = O.knearest(xyz, CELL, 5, mask=mask, cell_hint=3.0)
    assert np.array_equal(nn.numpy(), want[0])
    assert ((d2.numpy() == want[1]) | (np.isnan(d2.numpy()) & np.isnan(want[1]))).all()
