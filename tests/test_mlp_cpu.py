"""The CPU reference of the shell-proposal MLP against finite differences,
and the saved network file format (no GPU)."""

import os

import numpy as np

from conftest import ROOT


def test_reference_gradient_matches_finite_differences():
    from oracle import mlp_ref as M
    from linkcell_b200.learn import init_params
    rng = np.random.default_rng(0)
    p = init_params(3).astype(np.float64)
    X = rng.random((9, M.N_IN))
    y = rng.integers(0, M.N_OUT, 9)
    _, g = M.loss_and_grad(p, X, y)
    idx = rng.choice(p.size, 40, replace=False)
    for i in idx:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, X, y)[0] - M.loss_and_grad(pm, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_model_file_roundtrip(tmp_path):
    from linkcell_b200 import learn
    p = learn.init_params(1)
    path = os.path.join(tmp_path, "m.f32")
    learn.save(p, 0.85, path, "meta text")
    q, tau, meta = learn.load(path)
    assert np.array_equal(p, q) and abs(tau - 0.85) < 1e-7 and meta == "meta text"


def test_shipped_model_loads():
    from linkcell_b200 import learn
    if not os.path.exists(learn.MODEL_PATH):
        return
    p, tau, meta = learn.load()
    assert p.size == learn.n_params() and 0 < tau <= 1 and np.isfinite(p).all()
