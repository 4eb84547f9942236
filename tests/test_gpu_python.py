"""The Python entry on a GPU, mirroring the reference's
tests/python/test_knearest.py and test_knearest_cuda.py."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(xyz, cell, k, **kw):
    import linkcell_b200 as L
    nn, d2 = L.knearest(xyz, cell, k, **kw)
    return np.from_dlpack(nn), np.from_dlpack(d2)


def test_periodic_image_host(gpu):
    xyz = np.ascontiguousarray([[0.2, 0.0, 0.0], [9.4, 0.0, 0.0]], dtype=np.float64)
    nn, d2 = _pair(xyz, np.array([10.0, 10.0, 10.0]), 1)
    assert nn.shape == (2, 1) and d2.shape == (2, 1)
    assert nn[:, 0].tolist() == [1, 0]
    assert abs(d2[0, 0] - 0.64) < 1e-12 and abs(d2[1, 0] - 0.64) < 1e-12


def test_lattice_rows_and_mask(gpu):
    xyz = np.ascontiguousarray([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]], dtype=np.float64)
    nn, d2 = _pair(xyz, np.eye(3) * 10.0, 1)
    assert nn[0, 0] == 1 and abs(d2[0, 0] - 1.0) < 1e-12
    xyz = np.ascontiguousarray([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1.0, 0]], dtype=np.float64)
    nn, _ = _pair(xyz, np.array([10.0, 10.0, 10.0]), 1, mask=np.array([1, 0, 1], dtype=np.int32))
    assert nn[:, 0].tolist() == [2, -1, 0]
    nn, _ = _pair(xyz, np.array([10.0, 10.0, 10.0]), 1, mask=np.array([1.0, 0.0, 1.0]))
    assert nn[:, 0].tolist() == [2, -1, 0]


def test_batched_frames_host(gpu):
    frame = np.ascontiguousarray([[0.2, 0.0, 0.0], [9.4, 0.0, 0.0]], dtype=np.float64)
    nn, d2 = _pair(np.stack([frame, frame]), np.array([10.0, 10.0, 10.0]), 1)
    assert nn.shape == (2, 2, 1)
    assert nn[0, 0, 0] == 1 and nn[1, 1, 0] == 0
    assert abs(d2[0, 0, 0] - 0.64) < 1e-12


def test_torch_cuda_paths(gpu):
    import torch
    import linkcell_b200 as L
    xyz_h = np.ascontiguousarray([[0.2, 0.0, 0.0], [9.4, 0.0, 0.0]], dtype=np.float64)
    cell_h = np.ascontiguousarray([10.0, 10.0, 10.0], dtype=np.float64)
    xyz_d = torch.from_numpy(xyz_h).cuda()
    # CUDA xyz, host cell
    nn, d2 = L.knearest(xyz_d, cell_h, 1)
    out, out_d2 = torch.from_dlpack(nn), torch.from_dlpack(d2)
    assert out.device.type == "cuda" and out_d2.device.type == "cuda"
    assert out.shape == (2, 1) and int(out[0, 0]) == 1
    assert abs(float(out_d2[0, 0]) - 0.64) < 1e-12
    # CUDA xyz, CUDA cell (cell inverted from device doubles)
    nn, d2 = L.knearest(xyz_d, torch.from_numpy(cell_h).cuda(), 1)
    assert int(torch.from_dlpack(nn)[0, 0]) == 1
    assert abs(float(torch.from_dlpack(d2)[0, 0]) - 0.64) < 1e-12
    # host xyz, CUDA cell
    nn, d2 = L.knearest(xyz_h, torch.from_numpy(cell_h).cuda(), 1)
    assert int(np.from_dlpack(nn)[0, 0]) == 1
    # batched CUDA
    xb = torch.from_numpy(np.stack([xyz_h, xyz_h])).cuda()
    nn, d2 = L.knearest(xb, cell_h, 1)
    assert tuple(nn.shape) == (2, 2, 1) and int(nn[0, 0, 0]) == 1
    assert abs(float(d2[1, 1, 0]) - 0.64) < 1e-12
    # CUDA mask
    x3 = torch.tensor([[0.0, 0, 0], [1.0, 0, 0], [0.0, 1.0, 0]], dtype=torch.float64,
                      device="cuda")
    nn, _ = L.knearest(x3, cell_h, 1, mask=torch.tensor([1, 0, 1], dtype=torch.int32,
                                                          device="cuda"))
    assert nn[:, 0].tolist() == [2, -1, 0]


def test_cuda_matches_oracle_on_default_stream_work(gpu, oracle_mod):
    """Inputs produced by pending torch work on the default stream are seen in
    order (the search enqueues on torch's current stream)."""
    import torch
    import linkcell_b200 as L
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand((20000, 3), dtype=torch.float64, device="cuda", generator=g) * 30.0
    x = x * 1.0  # pending kernels when knearest is called
    nn, d2 = L.knearest(x, np.array([30.0, 30.0, 30.0]), 9)
    want = oracle_mod.knearest(x.cpu().numpy(), [30.0, 30.0, 30.0], 9)
    assert np.array_equal(nn.cpu().numpy(), want[0])
    assert np.array_equal(d2.cpu().numpy(), want[1], equal_nan=True)


def test_errors_on_gpu(gpu):
    import torch
    import linkcell_b200 as L
    with pytest.raises(ValueError, match="k must"):
        L.knearest(torch.zeros((2, 3), dtype=torch.float64, device="cuda"),
                   np.array([10.0, 10.0, 10.0]), 0)
    with pytest.raises(RuntimeError, match="too many cells"):
        L.knearest(torch.rand((4, 3), dtype=torch.float64, device="cuda"),
                   np.array([10.0, 10.0, 10.0]), 1, cell_hint=1e-9)
    with pytest.raises(RuntimeError, match="linked-cell mesh is too fine"):
        L.knearest(np.random.default_rng(0).random((4, 3)), np.array([10.0, 10.0, 10.0]), 1,
                   cell_hint=1e-9)


def test_knearest_batch_host_and_cuda(gpu, oracle_mod):
    """linkcell_b200.knearest_batch: host arrays give numpy rows (lc_knearest_batch),
    CUDA tensors give CUDA rows (lc_gpu_knearest_batch), both the oracle's."""
    import torch
    import linkcell_b200 as L
    from linkcell_b200 import workloads as W
    frames = W.frames_batch(n_frames=5, seed=23, n_min=200, n_max=4000)
    xyz = np.concatenate([f["xyz"] for f in frames]).astype(np.float64)
    mask = np.concatenate([f["mask"] for f in frames]).astype(np.int32)
    spec, off = [], 0
    for f in frames:
        spec.append(dict(n=len(f["xyz"]), k=f["k"], cell=f["cell"], cell_hint=f["cell_hint"],
                         mask_offset=off))
        off += len(f["xyz"])
    nn_h, d2_h = L.knearest_batch(xyz, spec, mask)
    nn_c, d2_c = L.knearest_batch(torch.as_tensor(xyz, device="cuda"), spec,
                                  torch.as_tensor(mask, device="cuda"))
    assert isinstance(nn_h, np.ndarray) and nn_c.is_cuda
    assert np.array_equal(nn_h, nn_c.cpu().numpy())
    assert np.array_equal(d2_h.view(np.int64), d2_c.cpu().numpy().view(np.int64))
    pos = 0
    for i, f in enumerate(frames):
        n, k = len(f["xyz"]), f["k"]
        want = oracle_mod.knearest(f["xyz"], f["cell"], k, mask=f["mask"],
                                   cell_hint=f["cell_hint"])
        assert np.array_equal(nn_h[pos:pos + n * k].reshape(n, k), want[0]), f"frame {i}"
        pos += n * k
