"""The C++ sample driver (icarat2_b200/examples/opt_cantilever.cpp), written
against include/icarat_b200.hpp in the shape of the reference's sample mains,
reproduces the oracle's design trajectory (compliance <= 1e-10 relative)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "icarat2_b200", "examples", "opt_cantilever")


@pytest.mark.parametrize("method,R,solver", [("mma", 2.5, "MG_CG"), ("oc", 1.5, "Eigen_CG")])
def test_cpp_driver_trajectory(oracle, method, R, solver):
    if not os.path.exists(EXE):
        from icarat2_b200 import build
        build.build()
    nx, ny, nz, steps = 16, 8, 8, 6
    out = subprocess.run([EXE, str(nx), str(ny), str(nz), str(steps), str(R), method, solver],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    comp = [float(l.split()[2]) for l in out.stdout.splitlines() if l.startswith("step")]
    assert len(comp) == steps
    P = oracle.Problem(nx, ny, nz)
    F = oracle.Filter(P, R)
    L = oracle.Loop(P, F, method=method, x0=0.3, move=0.2 if method == "mma" else 0.15,
                    cg_tol=1e-12)
    ref = []
    for _ in range(steps):
        L.step()
        ref.append(L.scalars()["compliance"])
    assert np.allclose(comp, ref, rtol=1e-10, atol=0)


def test_cpp_driver_rejects_unknown_solver():
    if not os.path.exists(EXE):
        from icarat2_b200 import build
        build.build()
    out = subprocess.run([EXE, "4", "2", "2", "1", "1.5", "mma", "No_Such_Solver"],
                         capture_output=True, text=True, timeout=120)
    assert out.returncode == 2 and "Solver type name is wrong" in out.stdout


def test_cpp_driver_direct_solver_names(oracle):
    """the reference's direct solver names ("Eigen_LDLT", opt_mma_Helmholtz.cpp:99)
    run multigrid-PCG to 1e-12: the trajectory matches the oracle's loop"""
    if not os.path.exists(EXE):
        from icarat2_b200 import build
        build.build()
    nx, ny, nz, steps = 16, 8, 8, 3
    for name in ("Eigen_LDLT", "Eigen_SparseLU", "Eigen_ICCG"):
        out = subprocess.run([EXE, str(nx), str(ny), str(nz), str(steps), "1.5", "mma", name],
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stdout + out.stderr
        comp = [float(l.split()[2]) for l in out.stdout.splitlines() if l.startswith("step")]
        P = oracle.Problem(nx, ny, nz)
        L = oracle.Loop(P, oracle.Filter(P, 1.5), method="mma", x0=0.3, move=0.2,
                        cg_tol=1e-12)
        ref = []
        for _ in range(steps):
            L.step()
            ref.append(L.scalars()["compliance"])
        assert np.allclose(comp, ref, rtol=1e-9, atol=0)


@pytest.mark.parametrize("method", ["mma", "oc"])
def test_cpp_helmholtz_driver_trajectory(oracle, method):
    """examples/opt_mma_helmholtz.cpp (the opt_mma_Helmholtz.cpp loop through
    FilterHelmholtz of include/icarat_b200.hpp) against the oracle's loop with
    the Helmholtz filter (MMA, threshold; both Helmholtz CGs at the reference's
    1e-10, elasticity CG at 1e-12): compliance <= 1e-7 relative."""
    exe = os.path.join(ROOT, "icarat2_b200", "examples", "opt_mma_helmholtz")
    if not os.path.exists(exe):
        from icarat2_b200 import build
        build.build()
    nx, ny, nz, steps, R = 16, 8, 8, 4, 2.0
    out = subprocess.run([exe, str(nx), str(ny), str(nz), str(steps), str(R), "MG_CG", method],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    comp = [float(l.split()[2]) for l in out.stdout.splitlines() if l.startswith("step")]
    assert len(comp) == steps
    P = oracle.Problem(nx, ny, nz)
    L = oracle.Loop(P, None, method=method, x0=0.3, move=0.2 if method == "mma" else 0.15,
                    use_threshold=True, cg_tol=1e-12, helmholtz_R=R)
    ref = []
    for _ in range(steps):
        L.step()
        ref.append(L.scalars()["compliance"])
    assert np.allclose(comp, ref, rtol=1e-7, atol=0)


def test_cpp_multi_load_driver(oracle):
    """examples/opt_multi_load.cpp (the opt_multi_load.cpp loop through the C
    ABI: 3 load cases, design / non-design IDs, Helmholtz filter, MMA) against
    oracle.CaseLoop: compliance sums <= 1e-7 relative over 3 iterations."""
    exe = os.path.join(ROOT, "icarat2_b200", "examples", "opt_multi_load")
    if not os.path.exists(exe):
        from icarat2_b200 import build
        build.build()
    nx, ny, nz, steps, R = 16, 8, 8, 3, 2.0
    out = subprocess.run([exe, str(nx), str(ny), str(nz), str(steps), str(R)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    comp = [float(l.split()[2]) for l in out.stdout.splitlines() if l.startswith("step")]
    assert len(comp) == steps
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, ny), (0, nz)))]
    cases = [[((0, 0, -1.0), ((nx, nx), (ny // 2, ny // 2), (0, 0)))],
             [((0, -1.0, 0), ((nx, nx), (ny, ny), (nz, nz)))],
             [((0, 0, 1.0), ((nx, nx), (0, 0), (nz, nz)))]]
    Ps = [oracle.Problem(nx, ny, nz, dirichlet=d, loads=c) for c in cases]
    e = np.arange(nx * ny * nz)
    M = oracle.CaseLoop(Ps, None, helmholtz_R=R, design_ids=e[e % nx < nx - 2],
                        nondesign_ids=e[e % nx >= nx - 2])
    ref = [M.step()[0] for _ in range(steps)]
    assert np.allclose(comp, ref, rtol=1e-7, atol=0)
