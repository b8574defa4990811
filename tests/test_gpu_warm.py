"""FP64 CG warm start (icarat_solve_opts.warm_start with JACOBI_PCG / MG_PCG):
the solve begins from the context's previous solution and keeps the stop test
||r|| < rtol ||b||, so it returns the cold solve's solution to the tolerance
in fewer iterations; through the loop (one solution per load case) the design
trajectories stay those of the oracle.

Tolerances: solutions <= 1e-8 relative at rtol 1e-12; trajectories as the
loop parity tests (compliance 1e-9, design 1e-8)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("method", ["jacobi", "mg"])
def test_warm_solve_matches_cold(gpu, method):
    m = {"jacobi": gpu.JACOBI_PCG, "mg": gpu.MG_PCG}[method]
    nx, ny, nz = 24, 12, 12
    rng = np.random.default_rng(4)
    rho = rng.uniform(0.2, 1.0, nx * ny * nz)
    rho2 = np.clip(rho * rng.uniform(0.95, 1.05, rho.size), 0.01, 1.0)
    cold, warm = gpu.Context(nx, ny, nz), gpu.Context(nx, ny, nz)
    ow = gpu.solve_opts(m, 1e-12, 20000, 3, warm_start=1)
    oc = gpu.solve_opts(m, 1e-12, 20000, 3)
    warm.set_design(rho)
    warm.solve(ow)  # nothing held yet: a cold start
    warm.set_design(rho2)
    uw, iw = warm.solve(ow)
    cold.set_design(rho2)
    uc, ic = cold.solve(oc)
    assert iw.status == 0 and ic.status == 0
    assert rel(uw, uc) <= 1e-8
    assert iw.iterations < ic.iterations
    # the held solution is the next solve's start: no iteration when it
    # already meets the tolerance.  CG stops on its recurrence residual, so
    # the true residual of the solution it returned can sit just above rtol;
    # then a few iterations bring it below.
    f = warm.fext()
    r_true = np.linalg.norm(f - warm.apply_K(uw)) / np.linalg.norm(f)
    u3, i3 = warm.solve(ow)
    assert i3.status == 0 and rel(u3, uw) <= 1e-10
    if r_true < 0.99e-12:
        assert i3.iterations == 0 and np.array_equal(u3, uw)
    elif r_true > 1.01e-12:
        assert 1 <= i3.iterations < ic.iterations // 10, (r_true, i3.iterations)


def test_warm_loop_and_multi_load_track_oracle(oracle, gpu):
    nx, ny, nz = 16, 8, 8
    P, G = oracle.Problem(nx, ny, nz), gpu.Context(nx, ny, nz)
    L = oracle.Loop(P, oracle.Filter(P, 1.5), method="mma", x0=0.3, move=0.2, cg_tol=1e-12)
    G.loop_init(0.3, method="mma", filter_radius=1.5, move=0.2,
                solve=gpu.solve_opts(gpu.MG_PCG, 1e-12, 10000, 3, warm_start=1))
    its = []
    for _ in range(5):
        L.step()
        info = G.loop_step()
        s = L.scalars()
        its.append(info.cg_iterations)
        assert abs(info.compliance - s["compliance"]) <= 1e-9 * s["compliance"]
    assert rel(G.loop_get("x"), L.get("x")) <= 1e-8
    # multi-load: each case warm-starts from its own last solution
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, ny), (0, nz)))]
    cases = [[((0, 0, -1.0), ((nx, nx), (ny // 2, ny // 2), (0, 0)))],
             [((0, -1.0, 0), ((nx, nx), (ny, ny), (nz, nz)))]]
    F = []
    for lo in cases:
        c = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
        F.append(c.fext())
        c.close()
    G = gpu.Context(nx, ny, nz, dirichlet=d, loads=cases[0])
    G.loop_init(0.3, method="mma", filter_radius=1.5, move=0.2, use_threshold=True,
                solve=gpu.solve_opts(gpu.MG_PCG, 1e-12, 10000, 3, warm_start=1))
    G.set_load_cases(np.array(F))
    Ps = [oracle.Problem(nx, ny, nz, dirichlet=d, loads=lo) for lo in cases]
    M = oracle.CaseLoop(Ps, oracle.Filter(Ps[0], 1.5))
    for _ in range(4):
        comp, const, _ = M.step()
        info = G.loop_step()
        assert abs(info.compliance - comp) <= 1e-9 * comp
    assert rel(G.loop_get("x"), M.x) <= 1e-8
