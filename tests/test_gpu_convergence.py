"""The sample drivers' stopping rule, Optimize::isConvergence(1e-5, 50)
(src/optimization/opt_base.hpp:28-43, called at opt_macro_oc.cpp:137): the
device loop (icarat_loop_is_convergence) and the C++ sample driver over
include/icarat_b200.hpp stop at the same design iteration as the oracle's
loop with the restated test, on a 16x8x8 OC cantilever (R = 1.5, move 0.15;
solves to rtol 1e-12, compliance within 1e-10 of the oracle every step)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "icarat2_b200", "examples", "opt_cantilever")
CAP = 600


@pytest.fixture(scope="module")
def oracle_stop(oracle):
    nx, ny, nz = 16, 8, 8
    P = oracle.Problem(nx, ny, nz)
    L = oracle.Loop(P, oracle.Filter(P, 1.5), method="oc", x0=0.3, move=0.15, cg_tol=1e-12)
    conv, comp, k = oracle.Convergence(), [], 0
    state = 1
    while state == 1 and k < CAP:
        k += 1
        L.step()
        comp.append(L.scalars()["compliance"])
        state = conv.is_convergence(comp[-1], k, 1e-5, 50)
    assert state == 0, "the oracle loop did not converge within %d steps" % CAP
    return k, comp


def test_device_loop_stops_with_the_oracle(gpu, oracle_stop):
    k_ref, comp = oracle_stop
    G = gpu.Context(16, 8, 8)
    G.loop_init(0.3, method="oc", filter_radius=1.5, move=0.15,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3))
    state, k = 1, 0
    while state == 1 and k < CAP:
        k += 1
        info = G.loop_step()
        assert abs(info.compliance - comp[k - 1]) <= 1e-10 * comp[k - 1]
        state = G.loop_is_convergence(1e-5, 50)
    assert state == 0 and k == k_ref and k > 50


def test_cpp_driver_stops_with_the_oracle(oracle_stop):
    if not os.path.exists(EXE):
        from icarat2_b200 import build
        build.build()
    k_ref, comp = oracle_stop
    out = subprocess.run([EXE, "16", "8", "8", str(CAP), "1.5", "oc", "MG_CG"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.splitlines()
    steps = [float(l.split()[2]) for l in lines if l.startswith("step")]
    assert ("converged %d" % k_ref) in lines
    assert len(steps) == k_ref
    assert np.allclose(steps, comp, rtol=1e-10, atol=0)


def test_convergence_needs_a_step(gpu):
    G = gpu.Context(4, 2, 2)
    G.loop_init(0.3, method="oc", filter_radius=1.5)
    with pytest.raises(gpu.IcaratError) as e:
        G.loop_is_convergence()
    assert e.value.status == gpu.ERR_STATE
