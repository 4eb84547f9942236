"""Pins the CPU oracle against the reference's own known answers.

The oracle (oracle/linkcell_oracle.cpp) restates the reference walk; these
tests check it against the literal expectations and agreement properties of
the reference test suite, stored in tests/golden/reference_kats.json
(generated by tests/golden/make_golden.py with file:line citations).
"""

import numpy as np
import pytest


def almost(a, b):
    # tests/agree.rs:6-8
    return abs(a - b) <= 1e-12 * (1.0 + max(abs(a), abs(b)))


def _cases(kats):
    return kats["cases"]


def test_literal_expectations(oracle_mod, kats):
    for cs in _cases(kats):
        if cs["expect_nn"] is None and cs["expect_d2"] is None:
            continue
        nn, d2 = oracle_mod.knearest(cs["xyz"], cs["cell"], cs["k"], mask=cs["mask"],
                                     cell_hint=cs["cell_hint"])
        if cs["expect_nn"] is not None:
            for i, row in enumerate(cs["expect_nn"]):
                if row is not None:
                    assert nn[i].tolist() == row, (cs["name"], cs["source"], i)
        if cs["expect_d2"] is not None:
            for i, row in enumerate(cs["expect_d2"]):
                if row is not None:
                    for a, b in zip(d2[i], row):
                        assert almost(a, b), (cs["name"], cs["source"], i, a, b)


def test_walk_equals_brute_and_27_image(oracle_mod, kats):
    """tests/agree.rs:60-82,109-132,230-254,256-379: walk == brute == 27-image."""
    for cs in _cases(kats):
        nn, d2 = oracle_mod.knearest(cs["xyz"], cs["cell"], cs["k"], mask=cs["mask"],
                                     cell_hint=cs["cell_hint"])
        bn, bd = oracle_mod.brute(cs["xyz"], cs["cell"], cs["k"], cs["mask"])
        mn = np.array(cs["mic27_nn"], dtype=np.int32)
        md = np.array([[np.nan if v is None else v for v in row] for row in cs["mic27_d2"]])
        assert np.array_equal(nn, mn), (cs["name"], cs["source"])
        assert np.array_equal(nn, bn), (cs["name"], cs["source"])
        for got, want in ((d2, md), (d2, bd)):
            ok = np.isnan(want) == np.isnan(got)
            assert ok.all(), cs["name"]
            fin = ~np.isnan(want)
            assert all(almost(a, b) for a, b in zip(got[fin], want[fin])), cs["name"]


def test_wrap_cases_see_the_image(oracle_mod, kats):
    """tests/agree.rs:370-377: first neighbour across the boundary, dist2 < 1."""
    for cs in _cases(kats):
        if cs["source"] != "tests/agree.rs:256-379":
            continue
        nn, d2 = oracle_mod.knearest(cs["xyz"], cs["cell"], cs["k"], cell_hint=2.0)
        assert d2[0, 0] < 1.0, cs["name"]
        if len(cs["xyz"]) == 3 and cs["k"] == 1:
            assert nn[0, 0] == 1, cs["name"]


def test_error_messages(oracle_mod):
    """src/error.rs:24-36 through src/capi.rs:195-227; tests/abi.rs:121-320."""
    O = oracle_mod
    with pytest.raises(O.OracleError, match="^no points$"):
        O.knearest(np.zeros((0, 3)), [10, 10, 10], 1)
    with pytest.raises(O.OracleError, match="^k must be at least 1$"):
        _zero_k(O)
    with pytest.raises(O.OracleError, match="^singular or non-positive cell$"):
        O.knearest(np.zeros((2, 3)), [[1, 0, 0], [2, 0, 0], [0, 0, 1]], 1)
    with pytest.raises(O.OracleError, match="^singular or non-positive cell$"):
        O.knearest(np.zeros((2, 3)), [0.0, 1.0, 1.0], 1)
    with pytest.raises(O.OracleError, match="^linked-cell mesh is too fine$"):
        O.knearest(np.random.default_rng(0).random((4, 3)) * 10, [10, 10, 10], 1, cell_hint=1e-9)


def _zero_k(O):
    import ctypes
    xyz = np.zeros((1, 3))
    nn = np.zeros(1, dtype=np.int32)
    oc = O.make_cell([10, 10, 10])
    rc = O.lib().orc_knearest_many(O._dptr(xyz), 1, 1, ctypes.byref(oc), 0, None, 0.0,
                                   O._iptr(nn), None, 1)
    if rc != 0:
        raise O.OracleError(O.last_error())


def test_all_masked_skips_the_mesh(oracle_mod):
    """src/knearest.rs:370-375: an all-masked search returns before sizing the mesh."""
    nn, d2 = oracle_mod.knearest(np.zeros((3, 3)), [10, 10, 10], 2, mask=[0, 0, 0], cell_hint=1e-9)
    assert (nn == -1).all() and np.isnan(d2).all()


def test_cell_unit(oracle_mod):
    """src/cell.rs:391-422: ortho flag, sheared cell not ortho, widths."""
    rc, info = oracle_mod.cell_info([10.0, 11.0, 12.0])
    assert rc == 0 and info["ortho"]
    assert info["widths"].tolist() == [10.0, 11.0, 12.0]
    rc, info = oracle_mod.cell_info([[10, 0, 0], [5, 8.66, 0], [0, 0, 10]])
    assert rc == 0 and not info["ortho"]


def test_parallel_equals_serial(oracle_mod):
    from linkcell_b200 import workloads as W
    w = W.uniform_ortho(3000, 15.0, seed=5)
    a = oracle_mod.knearest(w["xyz"], w["cell"], 7, cell_hint=2.0, threads=1)
    b = oracle_mod.knearest(w["xyz"], w["cell"], 7, cell_hint=2.0, threads=8)
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(a[1], b[1], equal_nan=True)


def test_subset_matches_full(oracle_mod):
    from linkcell_b200 import workloads as W
    w = W.uniform_ortho(2000, 14.0, seed=9)
    full = oracle_mod.knearest(w["xyz"], w["cell"], 5)
    src = np.array([0, 7, 1999, 512])
    sub = oracle_mod.knearest_subset(w["xyz"], w["cell"], 5, src)
    assert np.array_equal(sub[0], full[0][src])
    assert np.array_equal(sub[1], full[1][src], equal_nan=True)
