"""Training of the shell-proposal network on the GPU.

Data: (features, settled shell) pairs logged by the plain FP64 walk on
seeded bimodal triclinic frames (dense half 0.1 / unit^3, sparse half
0.005, the benchmark cell shape), one run per seed, k cycling through
16, 32, 64. Features are log(1 + occupancy) of the 5x5x5 cells around a
source's home cell plus k / 64; the label is the settled shell (the reach
at which the walk stopped) minus one, capped at 7.

Training: mini-batch Adam on the mean softmax cross-entropy, with the
library's own forward, backward and Adam kernels (lc_gpu_mlp_*); torch only
provides device buffers.

Usage: python -m linkcell_b200.learn [--runs 200] [--n 100000] [--epochs 12]
"""

from __future__ import annotations

import argparse
import ctypes
import os
import struct
import time

import numpy as np

from . import _capi
from . import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_PATH = os.path.join(HERE, "data", "shell_mlp.f32")
MAGIC = b"LCMLP001"
N_IN, N_HID, N_OUT = 126, 64, 8


def n_params() -> int:
    return N_HID * N_IN + N_HID + N_HID * N_HID + N_HID + N_OUT * N_HID + N_OUT


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation, biases zero."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2.0 / N_IN), (N_HID, N_IN)), np.zeros(N_HID),
             rng.normal(0, np.sqrt(2.0 / N_HID), (N_HID, N_HID)), np.zeros(N_HID),
             rng.normal(0, np.sqrt(1.0 / N_HID), (N_OUT, N_HID)), np.zeros(N_OUT)]
    return np.concatenate([p.reshape(-1) for p in parts]).astype(np.float32)


def save(params: np.ndarray, tau: float, path: str = MODEL_PATH, meta: str = "") -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as fh:
        fh.write(MAGIC)
        fh.write(struct.pack("<if", params.size, float(tau)))
        m = meta.encode()
        fh.write(struct.pack("<i", len(m)))
        fh.write(m)
        fh.write(params.astype(np.float32).tobytes())


def load(path: str = MODEL_PATH):
    """(params float32, tau, meta) of a saved network."""
    with open(path, "rb") as fh:
        if fh.read(8) != MAGIC:
            raise ValueError(f"{path}: not a shell-proposal model")
        n, tau = struct.unpack("<if", fh.read(8))
        (ml,) = struct.unpack("<i", fh.read(4))
        meta = fh.read(ml).decode()
        params = np.frombuffer(fh.read(4 * n), dtype=np.float32).copy()
    if params.size != n_params():
        raise ValueError(f"{path}: {params.size} parameters, expected {n_params()}")
    return params, tau, meta


def attach(workspace_handle, path: str = MODEL_PATH, tau: float | None = None) -> None:
    """Load the saved network into a workspace (lc_gpu_set_model)."""
    L = _capi.load()
    params, saved_tau, _ = load(path)
    rc = L.lc_gpu_set_model(workspace_handle, params.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                            params.size, float(tau if tau is not None else saved_tau))
    if rc != 0:
        raise RuntimeError(_capi.gpu_error())


def collect(runs: int = 200, n: int = 100_000, rows_per_run: int = 2000, seed0: int = 100,
            ks=(16, 32, 64), log=print):
    """Logged plain walks -> (X [rows, 126] float32, y [rows] int32) on the GPU."""
    import torch
    L = _capi.load()
    ws = L.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    assert L.lc_gpu_set_mode(ws, 0) == 0
    assert L.lc_gpu_log_shells(ws, 1) == 0
    X = torch.empty((runs * rows_per_run, N_IN), dtype=torch.float32, device="cuda")
    y = torch.empty((runs * rows_per_run,), dtype=torch.int32, device="cuda")
    from . import _cell_struct
    filled = 0
    t0 = time.time()
    for r in range(runs):
        k = ks[r % len(ks)]
        w = W.bimodal_triclinic(n=n, seed=seed0 + r, k=k)
        xd = torch.as_tensor(w["xyz"], device="cuda")
        nn = torch.empty((n, k), dtype=torch.int32, device="cuda")
        cell = _cell_struct(np.asarray(w["cell"]))
        torch.cuda.synchronize()
        rc = L.lc_gpu_knearest_many(ws, xd.data_ptr(), n, 1, ctypes.byref(cell), k, None, 3.0,
                                    nn.data_ptr(), None, 1)
        assert rc == 0, _capi.gpu_error()
        stride = max(1, n // rows_per_run)
        got = L.lc_gpu_training_rows(ws, ctypes.c_void_p(X[filled:].data_ptr()),
                                     ctypes.c_void_p(y[filled:].data_ptr()),
                                     rows_per_run, stride, r % stride)
        assert got >= 0, _capi.gpu_error()
        filled += int(got)
    L.lc_gpu_workspace_free(ws)
    log(f"collected {filled} rows from {runs} runs in {time.time() - t0:.1f} s")
    return X[:filled], y[:filled]


class Trainer:
    """Adam on the library's MLP kernels; parameters live on the device."""

    def __init__(self, params: np.ndarray, batch: int = 4096, lr: float = 2e-3):
        import torch
        self.torch = torch
        self.L = _capi.load()
        self.p = torch.as_tensor(params, device="cuda").contiguous()
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.batch = batch
        self.lr = lr
        self.step = 0
        self.scratch = torch.empty(int(self.L.lc_gpu_mlp_scratch_floats(batch)),
                                   dtype=torch.float32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or 1)

    def grad(self, X, y):
        rc = self.L.lc_gpu_mlp_grad(self.p.data_ptr(), X.data_ptr(), y.data_ptr(), X.shape[0],
                                    self.g.data_ptr(), self.loss.data_ptr(), self.scratch.data_ptr(),
                                    self.stream)
        assert rc == 0, _capi.gpu_error()
        return self.g, self.loss

    def adam_step(self, lr=None):
        """One Adam step with the gradient currently in self.g."""
        self.step += 1
        rc = self.L.lc_gpu_mlp_adam(self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                    self.v.data_ptr(), self.step, float(lr or self.lr), self.stream)
        assert rc == 0, _capi.gpu_error()

    def train_step(self, X, y, lr=None):
        self.grad(X, y)
        self.adam_step(lr)

    def probs(self, X):
        torch = self.torch
        out = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device="cuda")
        scratch = torch.empty(int(self.L.lc_gpu_mlp_scratch_floats(X.shape[0])),
                              dtype=torch.float32, device="cuda")
        rc = self.L.lc_gpu_mlp_forward(self.p.data_ptr(), X.data_ptr(), X.shape[0], out.data_ptr(),
                                       scratch.data_ptr(), self.stream)
        assert rc == 0, _capi.gpu_error()
        return out

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy()


def train(X, y, epochs: int = 12, batch: int = 4096, lr: float = 2e-3, seed: int = 0, log=print):
    import torch
    gen = torch.Generator(device="cuda").manual_seed(seed)
    rows = X.shape[0]
    n_val = max(batch, rows // 10)
    perm = torch.randperm(rows, device="cuda", generator=gen)
    val, tr = perm[:n_val], perm[n_val:]
    t = Trainer(init_params(seed), batch=batch, lr=lr)
    steps_per_epoch = max(1, tr.numel() // batch)
    for ep in range(epochs):
        order = tr[torch.randperm(tr.numel(), device="cuda", generator=gen)]
        lr_ep = lr * (0.5 ** (ep // 4))
        for s in range(steps_per_epoch):
            idx = order[s * batch:(s + 1) * batch]
            t.train_step(X[idx].contiguous(), y[idx].contiguous(), lr=lr_ep)
        pv = t.probs(X[val].contiguous())
        acc = float((pv.argmax(1).to(torch.int32) == y[val]).float().mean())
        nll = float(-torch.log(pv[torch.arange(n_val, device="cuda"), y[val].long()] + 1e-12).mean())
        log(f"epoch {ep + 1}: val accuracy {acc:.4f} val nll {nll:.4f}")
    return t, (X[val], y[val])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=200)
    ap.add_argument("--n", type=int, default=100_000)
    ap.add_argument("--rows-per-run", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--tau", type=float, default=0.95)
    ap.add_argument("--out", default=MODEL_PATH)
    a = ap.parse_args()
    X, y = collect(a.runs, a.n, a.rows_per_run)
    t, _ = train(X, y, epochs=a.epochs)
    meta = (f"runs={a.runs} n={a.n} rows={X.shape[0]} ks=16,32,64 seeds=100..{99 + a.runs} "
            f"epochs={a.epochs}")
    save(t.params(), a.tau, a.out, meta)
    print(f"saved {a.out}")


if __name__ == "__main__":
    main()
