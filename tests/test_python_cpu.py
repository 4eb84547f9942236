"""Python entry without a GPU: the argument handling of linkcell.knearest
(python/src/lib.rs:188-412) that happens before any device work, mirrored
from tests/python/test_knearest.py."""

import numpy as np
import pytest

from conftest import has_gpu


def test_version_and_available(lib):
    import linkcell_b200 as L
    assert L.__version__ == "0.3.3"
    assert isinstance(L.gpu_available(), bool)


def test_k_zero():
    import linkcell_b200 as L
    with pytest.raises(ValueError, match="k must"):
        L.knearest(np.zeros((2, 3)), np.array([10.0, 10.0, 10.0]), 0)


def test_bad_shapes(lib):
    import linkcell_b200 as L
    cell = np.array([10.0, 10.0, 10.0])
    with pytest.raises(ValueError, match="xyz must be float64"):
        L.knearest(np.zeros((2, 4)), cell, 1)
    with pytest.raises(ValueError, match="xyz must be float64"):
        L.knearest(np.zeros((2, 3), dtype=np.float32), cell, 1)
    with pytest.raises(ValueError, match="cell must be float64"):
        L.knearest(np.zeros((2, 3)), np.zeros(4), 1)
    with pytest.raises(ValueError, match="mask length must be n"):
        L.knearest(np.zeros((2, 3)), cell, 1, mask=np.ones(3, dtype=np.int32))
    with pytest.raises(ValueError, match="mask must be int32 or float64"):
        L.knearest(np.zeros((2, 3)), cell, 1, mask=np.ones(2, dtype=np.int64))


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_host_call_without_device_raises(lib):
    import linkcell_b200 as L
    with pytest.raises(RuntimeError, match="no CUDA device"):
        L.knearest(np.array([[0.2, 0, 0], [9.4, 0, 0]]), np.array([10.0, 10.0, 10.0]), 1)
