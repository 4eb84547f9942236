"""The shell-proposal network on the GPU: forward, gradient and Adam kernels
against the CPU reference (oracle/mlp_ref.py); training lowers the loss; the
learned walk with the shipped network stays exact and does less work than
the walk without it."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _trainer(params, batch):
    from linkcell_b200.learn import Trainer
    return Trainer(params, batch=batch)


def test_forward_and_gradient_match_cpu(gpu):
    import torch
    from linkcell_b200.learn import init_params
    from oracle import mlp_ref as M
    rng = np.random.default_rng(1)
    p = init_params(5)
    p[M.N_HID * M.N_IN:M.N_HID * M.N_IN + M.N_HID] = rng.normal(0, 0.1, M.N_HID)  # biases
    for B in (1, 37, 300):
        X = rng.random((B, M.N_IN)).astype(np.float32) * 2.0
        y = rng.integers(0, M.N_OUT, B).astype(np.int32)
        t = _trainer(p, B)
        Xd, yd = torch.as_tensor(X, device="cuda"), torch.as_tensor(y, device="cuda")
        probs = t.probs(Xd).cpu().numpy()
        ref = M.forward(p, X)
        assert np.max(np.abs(probs - ref["probs"])) < 2e-5
        g, loss = t.grad(Xd, yd)
        lref, gref = M.loss_and_grad(p, X, y)
        g = g.cpu().numpy()
        rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
        assert rel < 1e-4, rel
        assert abs(float(loss.item()) - lref) < 1e-4 * max(1.0, abs(lref))


def test_adam_matches_cpu(gpu):
    import torch
    from linkcell_b200.learn import init_params
    from oracle import mlp_ref as M
    rng = np.random.default_rng(2)
    p = init_params(7)
    X = rng.random((64, M.N_IN)).astype(np.float32)
    y = rng.integers(0, M.N_OUT, 64).astype(np.int32)
    t = _trainer(p, 64)
    Xd, yd = torch.as_tensor(X, device="cuda"), torch.as_tensor(y, device="cuda")
    pc, m, v = p.astype(np.float64), np.zeros(p.size), np.zeros(p.size)
    for step in range(1, 4):
        g, _ = t.grad(Xd, yd)  # the Adam kernel is checked on the GPU's own gradient
        pc, m, v = M.adam(pc, g.cpu().numpy().astype(np.float64), m, v, step, 1e-3)
        t.adam_step(lr=1e-3)
        assert np.max(np.abs(t.params() - pc)) < 1e-6


def test_training_lowers_loss(gpu):
    from linkcell_b200 import learn
    X, y = learn.collect(runs=6, n=30000, rows_per_run=1500, log=lambda *a: None)
    assert X.shape[0] > 5000 and int(y.min()) >= 0 and int(y.max()) <= 7
    t0 = learn.Trainer(learn.init_params(0), batch=1024)
    _, l0 = t0.grad(X[:1024].contiguous(), y[:1024].contiguous())
    l0 = float(l0.item())
    t, (Xv, yv) = learn.train(X, y, epochs=4, batch=1024, log=lambda *a: None)
    _, l1 = t.grad(Xv[:1024].contiguous(), yv[:1024].contiguous())
    assert float(l1.item()) < 0.7 * l0


def test_learned_walk_with_network_is_exact_and_saves_work(gpu, oracle_mod):
    """The shipped network's proposals keep every index exact and cut the
    walk's work against the FP32 walk without proposals (same GPU, same
    inputs): fewer candidate distances and FP64 reranks."""
    import os
    from gpu_helpers import DeviceRunner, assert_same
    from linkcell_b200 import learn, workloads as W
    if not os.path.exists(learn.MODEL_PATH):
        pytest.skip("no trained network shipped")
    w = W.bimodal_triclinic(n=150000, seed=77, k=32)
    want = oracle_mod.knearest(w["xyz"], w["cell"], 32, cell_hint=3.0)
    r = DeviceRunner()
    r.set_stats(True)  # counters of the learned warp walk are collected on request
    try:
        r.set_mode(1)
        assert_same(r.run(w["xyz"], w["cell"], 32, hint=3.0), want, "fast")
        fast, _ = r.stats()
        learn.attach(r.ws)
        r.set_mode(2)
        assert_same(r.run(w["xyz"], w["cell"], 32, hint=3.0), want, "learned")
        lrn, _ = r.stats()
    finally:
        r.close()
    proposals = lrn[6] + lrn[7] + lrn[8]
    assert proposals > 0.9 * 150000
    assert lrn[6] < 0.05 * proposals  # short proposals (restarts) stay rare
    assert lrn[5] < fast[5]  # fewer FP64 reranks


@pytest.mark.parametrize("n,rows,stride,seed", [(60000, 3000, 20, 5), (2500, 2500, 1, 9)])
def test_tensor_core_proposals_match_cpu_network(gpu, n, rows, stride, seed):
    """The walk's proposals (tensor-core inference, FP16) agree with the CPU
    reference network on the same features for nearly every source; a
    disagreement only moves work, never the result. The second case is a
    mesh of a few cells per axis: a tile's halo wraps the box more than once
    and most tiles are partly outside the mesh."""
    import ctypes
    import os
    import torch
    from linkcell_b200 import _capi, _cell_struct, learn, workloads as W
    from oracle import mlp_ref as M
    if not os.path.exists(learn.MODEL_PATH):
        pytest.skip("no trained network shipped")
    params, tau, _ = learn.load()
    L = _capi.load()
    w = W.bimodal_triclinic(n=n, seed=seed, k=32)
    ws = L.lc_gpu_workspace_new()
    try:
        learn.attach(ws)
        assert L.lc_gpu_set_mode(ws, 2) == 0 and L.lc_gpu_log_shells(ws, 1) == 0
        x = torch.as_tensor(w["xyz"], device="cuda")
        nn = torch.empty((n, 32), dtype=torch.int32, device="cuda")
        cell = _cell_struct(np.asarray(w["cell"]))
        torch.cuda.synchronize()
        assert L.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), 32, None, 3.0,
                                      nn.data_ptr(), None, 1) == 0, _capi.gpu_error()
        X = torch.empty((rows, 126), dtype=torch.float32, device="cuda")
        y = torch.empty((rows,), dtype=torch.int32, device="cuda")
        got = L.lc_gpu_training_rows(ws, ctypes.c_void_p(X.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                     rows, stride, 0)
        prop = np.empty(rows, dtype=np.int8)
        got2 = L.lc_gpu_proposals(ws, prop.ctypes.data_as(ctypes.c_void_p), rows, stride, 0)
    finally:
        L.lc_gpu_workspace_free(ws)
    assert got == got2 > min(1000, rows // 2)
    probs = M.forward(params.astype(np.float64), X[:got].cpu().numpy())["probs"]
    cum = np.cumsum(probs, axis=1)
    want = np.argmax(cum >= tau, axis=1) + 1
    want[want >= 8] = 0
    want[~(cum >= tau).any(axis=1)] = 0
    agree = np.mean(want == prop[:got])
    assert agree > 0.99, agree
