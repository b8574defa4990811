"""Design trajectories of the timed configurations against the oracle loop.

Config 1 exactly (sample/algorithm/opt-macro-oc/opt_macro_oc.cpp:83-172 on
the 32x16x16 cantilever: OC move 0.15, radius filter R = 1.5, uniform start
0.3, solves to the reference default rtol 1e-10, 50 iterations), against the
oracle's loop with its Jacobi-PCG ("Eigen_CG") at the same rtol:
  - Jacobi-PCG on the GPU (the reference's solver): the same CG iteration
    count every step, compliance, constraint and dc/drho within 1e-10
    relative every step (measured about 1e-12); the design x within 1e-9:
    the two sides round differently (summation order), and the OC updates
    carry those 1e-12 differences forward, about 1e-11 per step (measured
    4e-10 after 50 steps);
  - MG-PCG (4 levels) on the GPU: a different Krylov path to the same
    tolerance, so each solve may differ from the oracle's by the solver
    error allowed at rtol 1e-10: compliance and dc/drho within 1e-10
    (measured 3e-11), the design within 1e-8 after 50 steps (measured 4e-9).

The bench's headline settings (MMA move 0.2, R = 2.5, 4-level MG-PCG to
rtol 1e-8 started from the previous design's solution, the coarse factor of
the previous design reused while this design's is computed on a second
stream) over 10 iterations on 64x32x32, against the oracle loop solved to
1e-12 (the exact trajectory to about 1e-11).  A solver stopped at rtol 1e-8
is allowed the error that tolerance permits; the bound is calibrated by the
reference's own solver: the oracle loop with Jacobi-PCG stopped at the same
rtol 1e-8.  The GPU's largest deviation from the exact trajectory over the
10 steps, in compliance, constraint, dc/drho and x, must be at most 4 times
the oracle's own rtol-1e-8 deviation (plus 1e-12): the GPU solve at 1e-8 is
as accurate as the reference's at 1e-8 (measured on 48x24x24: 0.2x, 0.9x,
1.0x and 0.95x of it).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def oracle_run(oracle, P, R, method, move, tol, steps):
    L = oracle.Loop(P, oracle.Filter(P, R), method=method, x0=0.3, move=move, cg_tol=tol)
    rows = []
    for _ in range(steps):
        L.step()
        s = L.scalars()
        rows.append(dict(c=s["compliance"], g=s["constraint"], it=s["cg_iters"],
                         x=L.get("x").copy(), dfds=L.get("dfds").copy()))
    return rows


@pytest.fixture(scope="module")
def config1(oracle):
    P = oracle.Problem(32, 16, 16)
    return oracle_run(oracle, P, 1.5, "oc", 0.15, 1e-10, 50)


@pytest.mark.parametrize("solver,x_tol", [("jacobi", 1e-9), ("mg", 1e-8)])
def test_config1_oc_trajectory(gpu, config1, solver, x_tol):
    m = gpu.JACOBI_PCG if solver == "jacobi" else gpu.MG_PCG
    G = gpu.Context(32, 16, 16)
    G.loop_init(0.3, method="oc", filter_radius=1.5, move=0.15,
                solve=gpu.solve_opts(m, rtol=1e-10, mg_levels=4))
    for k, r in enumerate(config1):
        info = G.loop_step()
        assert info.status == gpu.OK
        assert abs(info.compliance - r["c"]) <= 1e-10 * r["c"], k
        assert abs(info.constraint - r["g"]) <= 1e-10 * abs(r["g"]), k
        assert rel(G.loop_get("dfds"), r["dfds"]) <= 1e-10, k
        assert rel(G.loop_get("x"), r["x"]) <= x_tol, k
        if solver == "jacobi":
            # the oracle's OpenMP dot products sum in an order that depends on
            # the host's thread count, so near rtol 1e-10 its iteration count
            # can move by a few out of ~400 from one machine to the next
            assert abs(info.cg_iterations - r["it"]) <= max(1, 0.01 * r["it"]), k


def test_headline_settings_trajectory(oracle, gpu):
    nx, ny, nz, steps = 64, 32, 32, 10
    P = oracle.Problem(nx, ny, nz)
    exact = oracle_run(oracle, P, 2.5, "mma", 0.2, 1e-12, steps)
    ref8 = oracle_run(oracle, P, 2.5, "mma", 0.2, 1e-8, steps)
    G = gpu.Context(nx, ny, nz)
    G.loop_init(0.3, method="mma", filter_radius=2.5, move=0.2,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-8, mg_levels=4, warm_start=1,
                                     coarse_lag=1))
    dev_gpu = dict(c=0.0, g=0.0, x=0.0, dfds=0.0)
    dev_ref = dict(c=0.0, g=0.0, x=0.0, dfds=0.0)
    for k in range(steps):
        info = G.loop_step()
        assert info.status == gpu.OK and info.cg_rel_residual < 1e-8
        e, o = exact[k], ref8[k]
        got = dict(c=info.compliance, g=info.constraint, x=G.loop_get("x"),
                   dfds=G.loop_get("dfds"))
        for key, dev in ((dev_gpu, got), (dev_ref, o)):
            key["c"] = max(key["c"], abs(dev["c"] - e["c"]) / e["c"])
            key["g"] = max(key["g"], abs(dev["g"] - e["g"]))
            key["x"] = max(key["x"], rel(dev["x"], e["x"]))
            key["dfds"] = max(key["dfds"], rel(dev["dfds"], e["dfds"]))
    print("deviation from the exact trajectory: GPU %s, oracle at rtol 1e-8 %s"
          % (dev_gpu, dev_ref))
    for k in dev_gpu:
        assert dev_gpu[k] <= 4.0 * dev_ref[k] + 1e-12, k
