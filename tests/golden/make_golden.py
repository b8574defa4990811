"""Regenerate tests/golden/*.json.

reference_tests.json holds the known answers of the reference's own unit tests
for this path, read as text from the reference tree (sample/test/...):
  - FilterTest          test-optimization/test_filter.cpp:63-124
  - FilterHelmholtzTest test-optimization/test_filter.cpp:126-175
  - MMASolverTest.toy   test-optimization/test_opt_solver.cpp:17-73
  - BmatrixTest.cubic8  test-basis/test_bmatrix.cpp:123-146
oracle_trajectory.json is a short OC and MMA design trajectory of the CPU
restatement (oracle/) on small cantilevers, committed so that a change of the
oracle itself shows up as a test failure.

Usage: python tests/golden/make_golden.py [/path/to/reference]
(default: the environment variable ICARAT_REFERENCE, else /root/reference)
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _read(ref, rel):
    with open(os.path.join(ref, rel)) as f:
        return f.read()


def reference_known_answers(ref):
    filt = _read(ref, "sample/test/test-optimization/test_filter.cpp")
    block = filt[filt.index("TEST(FilterTest, filter)"):filt.index("TEST(FilterHelmholtzTest")]
    radius = float(re.search(r"double radius = ([0-9.]+);", block).group(1))
    answer = [float(v) for _, v in sorted(
        (int(i), v) for i, v in re.findall(r"answer\[(\d)\] = ([0-9.]+);", block))]
    dfds = [float(v) for _, v in sorted(
        (int(i), v) for i, v in re.findall(r"dfds\[(\d)\] = ([0-9.e-]+);", block))]
    s_dens = [float(v) for _, v in sorted(
        (int(i), v) for i, v in re.findall(r"\bs\[(\d)\] = ([0-9.e-]+);", block))]
    norm_tol = float(re.search(r"EXPECT_LT\(norm, ([0-9.e-]+)\);", block).group(1))
    beta_hi = float(re.search(r"double beta = ([0-9.]+);", block).group(1))
    lo_hi = re.search(r"EXPECT_LT\(s_thre\[0\], ([0-9.]+)\);\s*EXPECT_GT\(s_thre\[1\], ([0-9.]+)\);",
                      block)
    der_tol = float(re.findall(r"EXPECT_LT\(norm, ([0-9.e-]+)\);", block)[-1])

    mma = _read(ref, "sample/test/test-optimization/test_opt_solver.cpp")
    mblock = mma[mma.index("TEST(MMASolverTest, toy)"):mma.index("TEST(GCMMASolverTest")]
    nm = re.search(r"int n = (\d+), m = (\d+);", mblock)
    x0 = [float(v) for v in re.search(r"vector<double> s\(\{([^}]*)\}\)", mblock).group(1).split(",")]
    move = float(re.search(r"SetMoveLimit\(([0-9.]+)\)", mblock).group(1))
    osc = float(re.search(r"SetOscillation\(([0-9.]+)\)", mblock).group(1))
    asym = [float(v) for v in re.search(r"SetAsymptotes\(([^)]*)\)", mblock).group(1).split(",")]
    iters = int(re.search(r"for\(int k = 0; k < (\d+); k\+\+\)", mblock).group(1))
    obj_lt = float(re.search(r"EXPECT_LT\(objective, ([0-9.]+)\);", mblock).group(1))
    g_lt = float(re.search(r"EXPECT_LT\(abs\(constraints\[0\]\), ([0-9.e-]+)\);", mblock).group(1))
    smax = float(re.search(r"smax = vector<double>\(n, ([0-9.]+)\)", mblock).group(1))

    hblock = filt[filt.index("TEST(FilterHelmholtzTest"):]
    hblock = hblock[:hblock.index("\n}\n") + 3]
    h_radius = float(re.search(r"double radius = ([0-9.]+);", hblock).group(1))
    h_answer = [float(v) for _, v in sorted(
        (int(i), v) for i, v in re.findall(r"answer\[(\d)\] = ([0-9.]+);", hblock))]
    h_s = [float(v) for _, v in sorted(
        (int(i), v) for i, v in re.findall(r"\bs\[(\d)\] = ([0-9.e-]+);", hblock))]
    h_tol = float(re.search(r"EXPECT_LT\(norm, ([0-9.e-]+)\);", hblock).group(1))

    bm = _read(ref, "sample/test/test-basis/test_bmatrix.cpp")
    bblock = bm[bm.index("TEST(BmatrixTest, cubic8)"):bm.index("TEST(BmatrixTest, cubic20)")]
    vol_tol = float(re.search(r"EXPECT_LT\(abs\(volume - 1.0\), ([0-9.e-]+)\);", bblock).group(1))

    return {
        "filter_2x2": {
            "source": "sample/test/test-optimization/test_filter.cpp:63-124",
            "radius": radius, "centroids": [[0.5, 0.5, 0.0], [1.5, 0.5, 0.0],
                                            [0.5, 1.5, 0.0], [1.5, 1.5, 0.0]],
            "design_s_sens": [0.5] * 4, "dfds": dfds, "design_s": s_dens,
            "answer": answer, "norm2_tol": norm_tol,
            "threshold_beta": beta_hi, "threshold_lo_below": float(lo_hi.group(1)),
            "threshold_hi_above": float(lo_hi.group(2)),
            "derivative_beta1_norm2_tol": der_tol,
        },
        "mma_toy": {
            "source": "sample/test/test-optimization/test_opt_solver.cpp:17-73",
            "n": int(nm.group(1)), "m": int(nm.group(2)), "x0": x0, "xmin": 0.0,
            "xmax": smax, "move": move, "albefa": osc, "asymptotes": asym,
            "iterations": iters, "objective_lt": obj_lt, "constraint_abs_lt": g_lt,
        },
        "helmholtz_2x2": {
            "source": "sample/test/test-optimization/test_filter.cpp:126-175",
            "mesh": "2 x 2 unit quad4 (as a 2 x 2 x 1 hexa8 slab: z-independent data give "
                    "the same nodal system scaled by the layer)",
            "radius": h_radius, "design_s": h_s, "answer": h_answer,
            "answer_sens": h_answer, "norm2_tol": h_tol,
        },
        "hexa8_volume": {
            "source": "sample/test/test-basis/test_bmatrix.cpp:123-146",
            "volume": 1.0, "tol": vol_tol,
        },
    }


def oracle_trajectory():
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    out = {}
    for name, (nx, ny, nz, method, R, steps) in {
            "oc_8x4x4": (8, 4, 4, "oc", 1.5, 6),
            "mma_8x4x4": (8, 4, 4, "mma", 2.5, 6)}.items():
        P = O.Problem(nx, ny, nz)
        F = O.Filter(P, R)
        L = O.Loop(P, F, method=method, x0=0.3, move=0.2 if method == "mma" else 0.15,
                   cg_tol=1e-12)
        comp = []
        for _ in range(steps):
            L.step()
            comp.append(L.scalars()["compliance"])
        out[name] = {"grid": [nx, ny, nz], "method": method, "radius": R, "x0": 0.3,
                     "cg_rtol": 1e-12, "compliance": comp,
                     "x_final": L.get("x").tolist()}
    return out


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ICARAT_REFERENCE",
                                                               "/root/reference")
    with open(os.path.join(HERE, "reference_tests.json"), "w") as f:
        json.dump(reference_known_answers(ref), f, indent=1)
    with open(os.path.join(HERE, "oracle_trajectory.json"), "w") as f:
        json.dump(oracle_trajectory(), f)
    print("written")
