"""Mixed-precision solver (FP32 multigrid-PCG refined by FP64 residuals).

The solver has no reference counterpart; it is checked against the FP64 paths:
  - displacements against the CPU oracle (FP64, rtol 1e-12) at small sizes:
    <= 1e-6 relative (the tolerance stated for the mixed path);
  - at larger sizes against the library's own FP64 multigrid-PCG solve
    (rtol 1e-12): compliance and compliance sensitivities <= 1e-6 relative;
  - the reported residual is an FP64 residual f - K u, recomputed here
    through the FP64 operator.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def mixed(gpu, rtol, **kw):
    return gpu.solve_opts(gpu.MIXED_IR, rtol=rtol, mg_levels=kw.pop("mg_levels", 3), **kw)


def test_mixed_matches_oracle(oracle, gpu):
    P, G = oracle.Problem(16, 8, 8), gpu.Context(16, 8, 8)
    rho = np.random.default_rng(31).uniform(0.1, 0.5, P.nelx)
    val_ref, _, _ = P.solve(rho, tol=1e-12)
    G.set_design(rho)
    val, info = G.solve(mixed(gpu, 1e-10))
    assert info.status == gpu.OK and info.rel_residual < 1e-10
    assert info.refreshes >= 1
    assert rel(val, val_ref) <= 1e-6
    f = G.fext()
    assert np.linalg.norm(f - G.apply_K(val)) < 1e-10 * np.linalg.norm(f) * 1.001


@pytest.mark.parametrize("rtol", [1e-6, 1e-8])
def test_mixed_compliance_and_sensitivity_vs_fp64(gpu, rtol):
    """64x32x32, densities U[0.1, 0.5] (the mixed-precision workload's
    distribution), filter-free sensitivities."""
    G = gpu.Context(64, 32, 32)
    rho = np.random.default_rng(32).uniform(0.1, 0.5, G.nelx)
    G.set_design(rho)
    u64, i64 = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=4))
    c64 = G.compliance()
    dc64, _ = G.sensitivity(1.0)
    u32, i32 = G.solve(mixed(gpu, rtol, mg_levels=4))
    assert i32.status == gpu.OK and i32.rel_residual < rtol
    c32 = G.compliance()
    dc32, _ = G.sensitivity(1.0)
    assert abs(c32 - c64) <= 1e-6 * abs(c64)
    assert rel(dc32, dc64) <= 1e-6
    # iterations of the FP32 loop stay close to the FP64 solver's
    ref = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=rtol, mg_levels=4))[1]
    assert i32.iterations <= ref.iterations + 3


def test_mixed_high_contrast(gpu):
    """Solid/void design (E contrast ~5e8): the FP64 residual reaches 1e-6
    (by the FP32 iteration, or by the FP64 MG-PCG finish after it stalls)."""
    G = gpu.Context(32, 16, 16)
    rng = np.random.default_rng(33)
    rho = np.where(rng.uniform(size=G.nelx) < 0.5, 1.0, 1e-3)
    G.set_design(rho)
    u64, _ = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-10, mg_levels=3))
    u, info = G.solve(mixed(gpu, 1e-6))
    assert info.status in (gpu.OK, gpu.WARN_STAGNATION)
    assert info.rel_residual < 1e-6
    f = G.fext()
    assert np.linalg.norm(f - G.apply_K(u)) < 1.001e-6 * np.linalg.norm(f)


def test_mixed_iteration_cap(gpu):
    G = gpu.Context(16, 8, 8)
    G.set_design(np.full(G.nelx, 0.3))
    u, info = G.solve(mixed(gpu, 1e-14, maxit=3, refresh=1e-6))
    # the cap forces a last FP64 refresh that folds the correction into u
    assert info.status == gpu.WARN_MAXITER and info.iterations == 4
    assert info.refreshes >= 1 and np.abs(u).max() > 0
    assert info.rel_residual < 1.0


def test_mixed_zero_rhs(gpu):
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, 4), (0, 4)))]
    G = gpu.Context(8, 4, 4, dirichlet=d, loads=[])
    G.set_design(np.full(G.nelx, 0.5))
    u, info = G.solve(mixed(gpu, 1e-8, mg_levels=2))
    assert info.status == gpu.OK and info.iterations == 0 and not u.any()


def test_mixed_bad_refresh_is_rejected(gpu):
    G = gpu.Context(8, 4, 4)
    G.set_design(np.full(G.nelx, 0.5))
    with pytest.raises(gpu.IcaratError) as e:
        G.solve(mixed(gpu, 1e-8, mg_levels=2, refresh=1.5))
    assert e.value.status == gpu.ERR_ARG


def test_mixed_reused_graph_and_rhs(gpu):
    """The captured iteration graph is reused across designs and right-hand
    sides; each solve still matches a fresh FP64 solve."""
    G = gpu.Context(32, 16, 16)
    rng = np.random.default_rng(34)
    for k in range(3):
        G.set_design(rng.uniform(0.1, 0.5, G.nelx))
        f = rng.standard_normal(G.numeq)
        u64, _ = G.solve_rhs(f, gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3))
        u32, info = G.solve_rhs(f, mixed(gpu, 1e-9))
        assert info.status == gpu.OK
        assert rel(u32, u64) <= 1e-6


def test_mixed_design_loop(oracle, gpu):
    """MMA design loop with the mixed solver: compliance and constraint track
    the FP64 oracle loop to 1e-6 over 6 steps."""
    P, G = oracle.Problem(16, 8, 8), gpu.Context(16, 8, 8)
    F = oracle.Filter(P, 2.5)
    L = oracle.Loop(P, F, method="mma", x0=0.3, move=0.2, cg_tol=1e-12)
    G.loop_init(0.3, method="mma", filter_radius=2.5, move=0.2,
                solve=mixed(gpu, 1e-10))
    for _ in range(6):
        L.step()
        info = G.loop_step()
        s = L.scalars()
        assert info.status == gpu.OK
        assert abs(info.compliance - s["compliance"]) <= 1e-6 * s["compliance"]
        assert abs(info.constraint - s["constraint"]) <= 1e-6 * max(1.0, abs(s["constraint"]))
    assert rel(G.loop_get("x"), L.get("x")) <= 1e-6


def test_mixed_warm_start(gpu):
    """Starting from the previous solution: a solve of the same system ends at
    once, and the next design of a loop needs fewer iterations than from 0."""
    G = gpu.Context(32, 16, 16)
    rng = np.random.default_rng(35)
    rho = rng.uniform(0.1, 0.5, G.nelx)
    G.set_design(rho)
    u0, i0 = G.solve(mixed(gpu, 1e-8))
    u1, i1 = G.solve(mixed(gpu, 1e-8, warm_start=1))
    assert i1.status == gpu.OK and i1.iterations == 0 and rel(u1, u0) == 0.0
    rho2 = np.clip(rho * (1.0 + 0.05 * rng.standard_normal(G.nelx)), 0.05, 1.0)
    G.set_design(rho2)
    ucold, icold = G.solve(mixed(gpu, 1e-8))
    G.set_design(rho)
    G.solve(mixed(gpu, 1e-8))
    G.set_design(rho2)
    uwarm, iwarm = G.solve(mixed(gpu, 1e-8, warm_start=1))
    assert iwarm.status == gpu.OK and iwarm.rel_residual < 1e-8
    assert iwarm.iterations < icold.iterations
    assert rel(uwarm, ucold) <= 1e-6


def test_mixed_floating_islands(gpu):
    """Thresholded noise smoothed along x only: solid streaks floating in a
    1e-9 void, an operator whose condition the FP32 iteration cannot follow.
    The FP64 residual is recomputed at least every 50 iterations, and an FP32
    iteration that stalls far above the tolerance is finished by FP64
    MG-PCG, so the solve still meets rtol (checked with the FP64 operator)
    instead of drifting or ending with a non-finite value."""
    G = gpu.Context(64, 32, 32)
    rng = np.random.default_rng(5)
    x = np.convolve(rng.standard_normal(G.nelx), np.ones(9) / 9.0, mode="same")
    rho = np.where(x >= np.quantile(x, 0.65), 1.0, 1e-3)
    G.set_design(rho)
    u, info = G.solve(mixed(gpu, 1e-8))
    assert info.status == gpu.OK, (info.status, info.iterations, info.rel_residual)
    f = G.fext()
    assert np.linalg.norm(f - G.apply_K(u)) < 1.01e-8 * np.linalg.norm(f)
