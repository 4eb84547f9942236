"""Writes tests/golden/reference_kats.json: the known-answer cases of the
reference test suite (HaoZeke/linkcell v0.3.3), restated as data.

Each case carries the reference file:line it comes from, its inputs, and
either the literal expected values the reference asserts ("expect") or the
statement that the reference asserts agreement with its brute-force
checkers ("agree": knearest == knearest_brute == 27-image oracle). For the
agreement cases the expected rows are computed here by the 27-image checker
restated in oracle/ (tests/agree.rs:161-210), which shares no code path with
the linked-cell walk.

Run from the repository root: python tests/golden/make_golden.py
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from linkcell_b200.workloads import lcg_fracs  # noqa: E402
from oracle import oracle as O  # noqa: E402

HEX = [[10.0, 0.0, 0.0], [5.0, 8.660254037844386, 0.0], [0.0, 0.0, 10.0]]
TRI = [[10.0, 0.0, 0.0], [3.0, 9.0, 0.0], [1.0, 2.0, 8.0]]
ORTHO10 = [10.0, 10.0, 10.0]


def kat(name, src, xyz, cell, k, expect_nn=None, expect_d2=None, mask=None, hint=0.0, rows=None):
    return dict(name=name, source=src, xyz=xyz, cell=cell, k=k, mask=mask, cell_hint=hint,
                expect_nn=expect_nn, expect_d2=expect_d2, rows=rows)


def literal_cases():
    c = []
    # src/lib.rs:55-66 and tests/agree.rs:39-47 (hint 2.0), tests/abi.rs:322-343
    c.append(kat("periodic_image", "src/lib.rs:55-66", [[0.2, 0, 0], [9.4, 0, 0]], ORTHO10, 1,
                 expect_nn=[[1], [0]], expect_d2=[[0.64], [0.64]]))
    c.append(kat("periodic_image_hint2", "tests/agree.rs:39-47", [[0.2, 0, 0], [9.4, 0, 0]], ORTHO10,
                 1, expect_nn=[[1], [0]], expect_d2=[[0.64], [0.64]], hint=2.0))
    # src/lib.rs:72-84: one bin, two images of the source
    c.append(kat("same_bin_two_images", "src/lib.rs:72-84", [[0.1, 0, 0], [1.0, 0, 0], [9.8, 0, 0]],
                 ORTHO10, 2, expect_nn=[[2, 1], None, None], expect_d2=[[0.09, 0.81], None, None],
                 hint=10.0))
    # src/lib.rs:88-99, tests/agree.rs:511-518
    c.append(kat("packed_row_major", "src/lib.rs:88-99", [[0, 0, 0], [1, 0, 0]], ORTHO10, 2,
                 expect_nn=[[1, -1], [0, -1]]))
    # src/knearest.rs:321-334, tests/agree.rs:49-58
    c.append(kat("mask_rows", "src/knearest.rs:321-334", [[0, 0, 0], [1, 0, 0], [0, 1, 0]], ORTHO10,
                 1, mask=[1, 0, 1], expect_nn=[[2], [-1], [0]]))
    # tests/agree.rs:29-37
    c.append(kat("two_points_k1", "tests/agree.rs:29-37", [[0, 0, 0], [1, 0, 0]], ORTHO10, 1,
                 expect_nn=[[1], [0]], expect_d2=[[1.0], None], hint=2.0))
    # tests/agree.rs:95-107: hex prism image shorter than the Cartesian vector
    c.append(kat("hex_image", "tests/agree.rs:95-107", [[0.2, 0.1, 1.0], [9.7, 0.1, 1.0]], HEX, 1,
                 expect_nn=[[1], None], hint=2.0))
    # tests/agree.rs:549-558
    c.append(kat("corner_wrap", "tests/agree.rs:549-558",
                 [[0.1, 0.1, 0.1], [9.8, 9.8, 9.8], [5.0, 5.0, 5.0]], ORTHO10, 1,
                 expect_nn=[[1], None, None], hint=2.0))
    # tests/agree.rs:520-530
    c.append(kat("into_d2_image", "tests/agree.rs:520-530", [[0.2, 0, 0], [9.4, 0, 0]], ORTHO10, 1,
                 expect_nn=[[1], [0]], expect_d2=[[0.64], [0.64]]))
    # tests/abi.rs:157-193 (C ABI equals the safe API on this input)
    c.append(kat("abi_packed_k3", "tests/abi.rs:157-193",
                 [[0, 0, 0], [1, 0, 0], [0, 1.5, 0], [0, 0, 2.0], [9.7, 0.2, 0.1]], ORTHO10, 3))
    # tests/abi.rs:195-240 and tests/agree.rs:461-481 (null mask == all ones)
    c.append(kat("mask_none_k2", "tests/abi.rs:195-240",
                 [[0, 0, 0], [1.2, 0, 0], [0, 1.4, 0], [0, 0, 1.6]], ORTHO10, 2))
    c.append(kat("mask_none_k3", "tests/agree.rs:461-481",
                 [[0, 0, 0], [1.2, 0, 0], [0, 1.4, 0], [0, 0, 1.6], [2, 2, 2]], ORTHO10, 3))
    # tests/agree.rs:431-459: packed layout for k in {1,2,3,5}
    for k in (1, 2, 3, 5):
        c.append(kat(f"packed_layout_k{k}", "tests/agree.rs:431-459",
                     [[0, 0, 0], [1, 0, 0], [0, 2, 0], [0, 0, 3]], ORTHO10, k))
    return c


def agree_cases():
    """Inputs of the reference's walk == brute == 27-image tests."""
    c = []
    # tests/agree.rs:60-82: ortho 12x11x13, N=64, LCG seed 1, k=4, hint 2.5
    f = lcg_fracs(1, 64 * 3).reshape(64, 3) * np.array([12.0, 11.0, 13.0])
    c.append(kat("random_ortho_64", "tests/agree.rs:60-82", f.tolist(), [12.0, 11.0, 13.0], 4,
                 hint=2.5))
    # tests/agree.rs:109-132: hex prism, N=48, seed 7, k=4, hint 2.0
    u = lcg_fracs(7, 48 * 3).reshape(48, 3)
    xyz = np.stack([10.0 * u[:, 0] + 5.0 * u[:, 1], 8.660254037844386 * u[:, 1], 10.0 * u[:, 2]], 1)
    c.append(kat("sheared_hex_48", "tests/agree.rs:109-132", xyz.tolist(), HEX, 4, hint=2.0))
    # tests/gpu_agree.cpp:69-99: triclinic N=48 seed 7 k=4 (default hint)
    xyz = np.stack([10.0 * u[:, 0] + 3.0 * u[:, 1] + 1.0 * u[:, 2], 9.0 * u[:, 1] + 2.0 * u[:, 2],
                    8.0 * u[:, 2]], 1)
    c.append(kat("gpu_agree_triclinic_48", "tests/gpu_agree.cpp:69-99", xyz.tolist(), TRI, 4))
    c.append(kat("gpu_agree_ortho_face", "tests/gpu_agree.cpp:86-90",
                 [[0.2, 1.0, 1.0], [9.7, 1.0, 1.0]], ORTHO10, 1))
    c.append(kat("gpu_agree_hex_face", "tests/gpu_agree.cpp:92-97",
                 [[0.2, 0.1, 1.0], [9.7, 0.1, 1.0]], HEX, 1))
    # tests/agree.rs:230-254: small-n matrix on hex and triclinic cells
    matrix = [("n=5 k=1", 5, 1, 1, 2.0), ("n=5 k=4", 5, 4, 1, 2.0), ("n=8 k=1", 8, 1, 11, 0.0),
              ("n=8 k=4", 8, 4, 11, 2.0), ("n=12 k=1", 12, 1, 3, 1.5), ("n=12 k=4", 12, 4, 3, 0.0)]
    for cname, rows in (("hex", HEX), ("triclinic", TRI)):
        R = np.array(rows)
        for label, n, k, seed, hint in matrix:
            fr = lcg_fracs(seed, n * 3).reshape(n, 3)
            xyz = fr @ R  # Cell::cartesian with zero origin (tests/agree.rs:149-159)
            c.append(kat(f"{cname} {label} seed={seed}", "tests/agree.rs:230-254", xyz.tolist(),
                         rows, k, hint=hint))
    # tests/agree.rs:256-379: face / edge / corner wrap cases, hint 2.0
    wraps = [
        ("ortho-face-x k=1", ORTHO10, [[0.12, 5, 5], [9.79, 5, 5], [5, 5, 5]], 1),
        ("ortho-face-y k=1", ORTHO10, [[5, 0.12, 5], [5, 9.79, 5], [5, 5, 5]], 1),
        ("ortho-face-z k=1", ORTHO10, [[5, 5, 0.12], [5, 5, 9.79], [5, 5, 5]], 1),
        ("ortho-edge-xy k=1", ORTHO10, [[0.12, 0.11, 5], [9.80, 9.81, 5], [5, 5, 5]], 1),
        ("ortho-corner k=1", ORTHO10, [[0.11, 0.12, 0.13], [9.82, 9.81, 9.80], [5, 5, 5]], 1),
        ("ortho-faces k=4", ORTHO10, [[0.10, 5, 5], [9.85, 5, 5], [5, 0.11, 5], [5, 9.84, 5],
                                      [5, 5, 0.12], [5, 5, 9.83], [5, 5, 5]], 4),
        ("ortho-same-bin two images k=2", ORTHO10, [[0.1, 0, 0], [1.0, 0, 0], [9.8, 0, 0]], 2),
        ("hex-face-a k=1", HEX, [[0.20, 0.10, 5], [9.70, 0.10, 5], [5, 4, 5]], 1),
        ("hex-corner k=1", HEX, [[0.25, 0.20, 0.25], [14.75, 8.46, 9.75], [5, 4.3, 5]], 1),
        ("hex-faces k=4", HEX, [[0.20, 0.15, 5], [9.70, 0.15, 5], [5.2, 0.20, 5], [7.7, 8.40, 5],
                                [5, 4.3, 0.20], [5, 4.3, 9.75], [5, 4.3, 5]], 4),
        ("triclinic-face-a k=1", TRI, [[0.20, 0.20, 4], [9.75, 0.20, 4], [6, 5, 4]], 1),
        ("triclinic-corner k=1", TRI, [[0.20, 0.20, 0.20], [13.80, 10.80, 7.80], [7, 5.5, 4]], 1),
        ("triclinic-wrap k=4", TRI, [[0.18, 0.15, 0.20], [13.82, 10.78, 7.79], [9.80, 0.25, 0.30],
                                     [0.25, 8.80, 0.22], [0.22, 0.30, 7.75], [7, 5.5, 4]], 4),
    ]
    for name, cell, xyz, k in wraps:
        c.append(kat(name, "tests/agree.rs:256-379", [[float(v) for v in p] for p in xyz], cell, k,
                     hint=2.0))
    return c


def main():
    cases = literal_cases() + agree_cases()
    for cs in cases:
        nn, d2 = O.mic27(cs["xyz"], cs["cell"], cs["k"], cs["mask"])
        cs["mic27_nn"] = nn.tolist()
        cs["mic27_d2"] = [[None if np.isnan(v) else float(v) for v in row] for row in d2]
    errors = [
        # src/error.rs:24-36 via src/capi.rs:195-227; tests/abi.rs:121-144,242-262,308-320
        dict(name="empty", source="tests/abi.rs:121-144", n=0, k=1, expect="no points"),
        dict(name="zero_k", source="tests/abi.rs:242-262", n=1, k=0, expect="k must be at least 1"),
        dict(name="overflow", source="tests/abi.rs:308-320", n=(2**63 - 1) // 3 + 1, k=1,
             expect="n * k overflows"),
    ]
    out = dict(reference="HaoZeke/linkcell v0.3.3", generator="tests/golden/make_golden.py",
               cases=cases, errors=errors)
    path = os.path.join(ROOT, "tests", "golden", "reference_kats.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print(f"wrote {len(cases)} cases to {path}")


if __name__ == "__main__":
    main()
