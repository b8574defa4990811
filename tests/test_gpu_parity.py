"""Parity of the sm_100a library (through its C ABI) with the CPU oracle.

Tolerances (stated per test):
  - DOF map, loads, element matrix, filter sums: bit-exact;
  - K u: max |diff| <= 1e-14 max |y| (FP64, different summation order);
  - solves: both sides to rtol 1e-12, solution <= 1e-8 relative, compliance
    <= 1e-10 relative;
  - one-step sensitivity / OC / MMA: <= 1e-12 relative;
  - design trajectories (N iterations, rtol 1e-12): compliance, x <= 1e-10.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_tests.json")))


def pair(oracle, gpu, nx, ny, nz, **kw):
    return oracle.Problem(nx, ny, nz, **kw), gpu.Context(nx, ny, nz, **kw)


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


# ------------------------------------------------------------------ setup data
@pytest.mark.parametrize("grid", [(4, 2, 2), (7, 3, 5), (32, 16, 16)])
def test_dof_map_and_loads_bit_exact(oracle, gpu, grid):
    P, G = pair(oracle, gpu, *grid)
    assert np.array_equal(P.dof(), G.dof_map())
    assert G.numeq == P.numeq and G.numnp == P.numnp and G.nelx == P.nelx
    assert np.array_equal(P.fext(), G.fext())


def test_dof_map_partial_flags_and_values(oracle, gpu):
    d = [((1, 0, 1), (0.0, 0.5, 0.0), ((0, 0), (0, 2), (0, 2))),
         ((0, 1, 0), (0.0, 0.0, 0.25), ((3, 3), (1, 1), (0, 0)))]
    loads = [((0.0, 0.0, -1.0), ((3, 3), (2, 2), (2, 2)))]
    P, G = pair(oracle, gpu, 3, 2, 2, dirichlet=d, loads=loads)
    assert np.array_equal(P.dof(), G.dof_map())
    assert np.array_equal(P.fext(), G.fext())


def test_element_matrix_bit_exact(oracle, gpu):
    P, G = pair(oracle, gpu, 3, 2, 2)
    a, va = P.ke0()
    b, vb = G.element_stiffness()
    assert np.array_equal(a, b) and va == vb


DIST_LOADS = [
    ("xmax face", (7.0, 3.0, 5.0), ((0.0, 0.0, -1.0), ((7, 7), (0, 3), (0, 5)))),
    ("zmin face", (7.0, 3.0, 5.0), ((0.0, 0.5, -1.0), ((0, 7), (0, 3), (0, 0)))),
    ("zmax face", (7.0, 3.0, 5.0), ((1.0, 0.0, 0.0), ((0, 7), (0, 3), (5, 5)))),
    ("ymin patch", (7.0, 3.0, 5.0), ((0.0, 0.0, -2.0), ((2, 5), (0, 0), (1, 4)))),
    ("ymax face", (7.0, 3.0, 5.0), ((0.0, -1.0, 0.0), ((0, 7), (3, 3), (0, 5)))),
    ("thick box", (7.0, 3.0, 5.0), ((0.3, -0.2, 1.0), ((1, 4.5), (0, 2), (0, 2.5)))),
    ("xmax stretched", (3.5, 3.0, 7.5), ((0.0, 0.0, -1.0), ((3.5, 3.5), (0, 3), (0, 7.5)))),
]


@pytest.mark.parametrize("name,lengths,load", DIST_LOADS, ids=[d[0] for d in DIST_LOADS])
def test_distributed_loads_bit_exact(oracle, gpu, name, lengths, load):
    """distributed Neumann boxes (generateLoadMain, SurfaceLoad) followed by a
    point load, on a 7 x 3 x 5 box"""
    lx, ly, lz = lengths
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, ly), (0, lz)))]
    loads = [load, ((0.0, 0.0, -1.0), ((lx, lx), (1.2, 1.2), (0, 0)))]
    P, G = pair(oracle, gpu, 7, 3, 5, lx=lx, ly=ly, lz=lz, dirichlet=d, loads=loads)
    assert np.array_equal(P.fext(), G.fext())
    assert np.count_nonzero(G.fext()) > 4


# ------------------------------------------------------------------ K u
@pytest.mark.parametrize("grid", [(4, 2, 2), (9, 5, 6), (24, 12, 12)])
def test_apply_K_matches_csr(oracle, gpu, grid):
    P, G = pair(oracle, gpu, *grid)
    rng = np.random.default_rng(11)
    rho = rng.uniform(0.01, 1.0, P.nelx)
    u = rng.standard_normal(P.numeq)
    P.assemble(rho)
    G.set_design(rho)
    y_ref = P.apply_K(u)
    y = G.apply_K(u)
    assert rel(y, y_ref) <= 1e-14


def test_apply_K_symmetry_and_rigid_modes_large(gpu):
    """Size-independent properties at 128x64x64 (no Dirichlet): v.Ku = u.Kv
    and K annihilates the six rigid-body modes."""
    G = gpu.Context(128, 64, 64, dirichlet=[], loads=[])
    rng = np.random.default_rng(4)
    G.set_design(rng.uniform(0.01, 1.0, G.nelx))
    u = rng.standard_normal(G.numeq)
    v = rng.standard_normal(G.numeq)
    Ku, Kv = G.apply_K(u), G.apply_K(v)
    assert abs(v @ Ku - u @ Kv) <= 1e-12 * abs(v @ Ku)
    n = np.arange(G.numnp)
    X = np.stack([n % 129, (n // 129) % 65, n // (129 * 65)], 1).astype(float)
    scale = np.abs(Ku).max()
    for d in range(3):
        t = np.zeros((G.numnp, 3))
        t[:, d] = 1.0
        assert np.abs(G.apply_K(t.ravel())).max() <= 1e-12 * scale
    r = np.zeros((G.numnp, 3))
    r[:, 0], r[:, 1] = -X[:, 1], X[:, 0]
    assert np.abs(G.apply_K(r.ravel())).max() <= 1e-11 * scale * 128


# ------------------------------------------------------------------ solves
def test_solve_before_design_is_an_error(gpu):
    G = gpu.Context(4, 2, 2)
    with pytest.raises(gpu.IcaratError) as e:
        G.solve()
    assert e.value.status == gpu.ERR_STATE


@pytest.mark.parametrize("grid", [(8, 4, 4), (16, 8, 8)])
def test_jacobi_pcg_matches_oracle(oracle, gpu, grid):
    P, G = pair(oracle, gpu, *grid)
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.05, 1.0, P.nelx)
    val_ref, it_ref, _ = P.solve(rho, tol=1e-12)
    G.set_design(rho)
    val, info = G.solve(gpu.solve_opts(gpu.JACOBI_PCG, rtol=1e-12))
    assert info.status == gpu.OK
    assert abs(info.iterations - it_ref) <= max(2, it_ref // 50)
    assert rel(val, val_ref) <= 1e-8
    assert abs(G.compliance() - P.compliance(val_ref)) <= 1e-10 * P.compliance(val_ref)


def test_jacobi_pcg_default_tolerance_semantics(oracle, gpu):
    """Reference defaults rtol 1e-10, zero initial guess: same iteration count."""
    P, G = pair(oracle, gpu, 32, 16, 16)
    rho = np.full(P.nelx, 0.3)
    val_ref, it_ref, rr_ref = P.solve(rho)
    G.set_design(rho)
    la = gpu.LinearAnalysis(G)
    val = la.solve("Eigen_CG")
    assert abs(la.info.iterations - it_ref) <= 2
    assert la.info.rel_residual < 1e-10
    assert rel(val, val_ref) <= 1e-7


@pytest.mark.parametrize("levels", [2, 3, 4])
def test_mg_pcg_matches_oracle(oracle, gpu, levels):
    P, G = pair(oracle, gpu, 16, 8, 8)
    rng = np.random.default_rng(8)
    rho = rng.uniform(0.001, 1.0, P.nelx)
    val_ref, it_ref, _ = P.solve(rho, tol=1e-12)
    G.set_design(rho)
    val, info = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=levels))
    assert info.status == gpu.OK
    assert info.iterations < it_ref
    assert rel(val, val_ref) <= 1e-8


def test_mg_pcg_high_contrast_large(gpu):
    """128x64x64 random solid/void design (E contrast 5e8): MG-PCG reaches the
    recursive rtol 1e-8 (the stop rule of CG.cpp:105-108), and the true
    residual f - K u, evaluated in FP64 with displacements up to 1e6 times
    the solid ones, is within the attainable accuracy (1e-6 relative)."""
    G = gpu.Context(128, 64, 64)
    rng = np.random.default_rng(9)
    rho = np.where(rng.uniform(size=G.nelx) < 0.4, 1.0, 1e-3)
    G.set_design(rho)
    val, info = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-8, mg_levels=4))
    assert info.status == gpu.OK and info.rel_residual < 1e-8
    f = G.fext()
    r = f - G.apply_K(val)
    assert np.linalg.norm(r) <= 1e-6 * np.linalg.norm(f)


def test_mg_pcg_true_residual_moderate_contrast(gpu):
    G = gpu.Context(64, 32, 32)
    rng = np.random.default_rng(10)
    G.set_design(rng.uniform(0.2, 1.0, G.nelx))
    val, info = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-10, mg_levels=4))
    f = G.fext()
    assert np.linalg.norm(f - G.apply_K(val)) <= 2e-10 * np.linalg.norm(f)


def test_solve_maxit_warning(gpu):
    G = gpu.Context(16, 8, 8)
    G.set_design(np.full(G.nelx, 0.3))
    val, info = G.solve(gpu.solve_opts(gpu.JACOBI_PCG, rtol=1e-14, maxit=5))
    assert info.status == gpu.WARN_MAXITER and info.iterations == 6


def test_nan_design_is_reported(gpu):
    G = gpu.Context(8, 4, 4)
    rho = np.full(G.nelx, 0.5)
    rho[3] = np.nan
    G.set_design(rho)
    with pytest.raises(gpu.IcaratError) as e:
        G.solve()
    assert e.value.status == gpu.ERR_NAN


def test_prescribed_displacement_rhs(oracle, gpu):
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, 4), (0, 4))),
         ((0, 0, 1), (0.0, 0.0, -0.01), ((8, 8), (0, 4), (0, 4)))]
    P, G = pair(oracle, gpu, 8, 4, 4, dirichlet=d, loads=[])
    rho = np.full(P.nelx, 0.6)
    val_ref, _, _ = P.solve(rho, tol=1e-12)
    G.set_design(rho)
    val, info = G.solve(gpu.solve_opts(rtol=1e-12))
    assert rel(val, val_ref) <= 1e-8
    assert np.allclose(G.node_values(), P.node_values(val_ref), rtol=1e-8, atol=1e-15)


# ------------------------------------------------------------------ sensitivities
def test_node_values_and_sensitivity(oracle, gpu):
    P, G = pair(oracle, gpu, 12, 6, 6)
    rng = np.random.default_rng(12)
    rho = rng.uniform(0.05, 1.0, P.nelx)
    G.set_design(rho)
    val, _ = G.solve(gpu.solve_opts(rtol=1e-12))
    nv = G.node_values()
    assert np.array_equal(nv, P.node_values(val))
    dfds, dgds = G.sensitivity(0.5)
    rdf, rdg = P.sensitivity(rho, nv, 0.5)
    assert rel(dfds, rdf) <= 1e-12
    assert np.array_equal(dgds, rdg)


# ------------------------------------------------------------------ filter
def test_filter_known_answers(gpu):
    """FilterTest (test_filter.cpp:63-124) on a 2x2x1 voxel box, R = 2."""
    g = GOLD["filter_2x2"]
    G = gpu.Context(2, 2, 1)
    F = gpu.Filter(G, g["radius"])
    ans = np.array(g["answer"])
    with pytest.raises(gpu.IcaratError) as e:  # transposed before forward
        F.densityFilter(g["dfds"], True)
    assert e.value.status == gpu.ERR_STATE
    s_new = F.densityFilter(g["design_s"], False)
    assert ((s_new - ans) ** 2).sum() < g["norm2_tol"]
    d_new = F.densityFilter(g["dfds"], True)
    assert ((d_new - ans) ** 2).sum() < g["norm2_tol"]
    sf = F.sensitivityFilter(g["design_s_sens"], g["dfds"])
    assert ((sf - ans) ** 2).sum() < g["norm2_tol"]
    thr = F.threshold(s_new, g["threshold_beta"], 0.5)
    assert thr[0] < g["threshold_lo_below"] and thr[1] > g["threshold_hi_above"]
    der = F.thresholdDerivative(s_new, 1.0, 0.5)
    assert ((der - 1.0) ** 2).sum() < g["derivative_beta1_norm2_tol"]


@pytest.mark.parametrize("R", [1.0, 1.5, 2.5, 3.0])
def test_filter_bit_exact(oracle, gpu, R):
    P, G = pair(oracle, gpu, 13, 7, 6)
    F = oracle.Filter(P, R)
    G.filter_setup(R)
    rng = np.random.default_rng(int(R * 10))
    x = rng.uniform(0.0, 1.0, P.nelx)
    assert np.array_equal(G.density_filter(x), F.density_filter(x))
    g = rng.standard_normal(P.nelx)
    assert np.array_equal(G.density_filter(g, True), F.density_filter(g, True))
    s = rng.uniform(0.1, 1.0, P.nelx)
    a = G.sensitivity_filter(s, g)
    b = F.sensitivity_filter(s, g, np.full(P.nelx, P.ke0()[1]))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("R", [1.5, 2.5])
def test_transposed_filter_bit_exact_wide_range(oracle, gpu, R):
    """The transposed filter divides every term by its weight sum in the
    reference's order; the GPU divides through a correctly rounded reciprocal
    with one FMA correction (Markstein) and must still give the reference's
    quotients exactly: 16 k elements, inputs of both signs spread over 16
    decades, about a million divisions."""
    P, G = pair(oracle, gpu, 40, 20, 20)
    F = oracle.Filter(P, R)
    G.filter_setup(R)
    rng = np.random.default_rng(int(R * 100))
    x = rng.uniform(0.0, 1.0, P.nelx)
    assert np.array_equal(G.density_filter(x), F.density_filter(x))
    g = rng.standard_normal(P.nelx) * 10.0 ** rng.uniform(-8.0, 8.0, P.nelx)
    assert np.array_equal(G.density_filter(g, True), F.density_filter(g, True))


def test_threshold_matches(oracle, gpu):
    G = gpu.Context(10, 5, 5)
    x = np.random.default_rng(2).uniform(0, 1, G.nelx)
    for beta in (1.0, 4.0, 16.0):
        assert rel(G.threshold(x, beta, 0.5), oracle.threshold(x, beta, 0.5)) < 1e-14
        assert rel(G.threshold_derivative(x, beta, 0.5),
                   oracle.threshold_derivative(x, beta, 0.5)) < 1e-13


def test_filter_of_constant_large(gpu):
    G = gpu.Context(256, 128, 128, dirichlet=[], loads=[])
    G.filter_setup(3.0)
    x = np.full(G.nelx, 0.37)
    assert np.abs(G.density_filter(x) - 0.37).max() < 1e-15


# ------------------------------------------------------------------ OC / MMA
@pytest.mark.parametrize("use_thr", [False, True])
def test_oc_update_matches_oracle(oracle, gpu, use_thr):
    P, G = pair(oracle, gpu, 12, 6, 6)
    F = oracle.Filter(P, 1.5)
    G.filter_setup(1.5)
    rng = np.random.default_rng(21)
    x = rng.uniform(0.2, 0.6, P.nelx)
    df = -rng.uniform(0.1, 3.0, P.nelx)
    dg = np.ones(P.nelx)
    V0 = 0.4 * P.nelx
    xmin, xmax = np.full(P.nelx, 1e-4), np.ones(P.nelx)
    beta = 2.0

    def vol(xk):
        f = F.density_filter(xk)
        return (oracle.threshold(f, beta, 0.5) if use_thr else f).sum()

    a, sa = oracle.oc_update(x, df, V0, dg, xmin, xmax, vol)
    b, sb = G.oc_update(x, df, V0, dg, xmin, xmax, use_threshold=use_thr, beta=beta)
    assert sa == sb
    assert rel(b, a) <= 1e-12


def test_mma_toy_known_answer_on_gpu(oracle, gpu):
    """MMASolverTest.toy (test_opt_solver.cpp:17-73) through the GPU MMA,
    step by step against the oracle (which is bit-identical to the reference)."""
    g = GOLD["mma_toy"]
    n, m = g["n"], g["m"]
    G = gpu.MMASolver(n, m)
    O = oracle.MMA(n, m)
    for M in (G,):
        M.SetMoveLimit(g["move"])
        M.SetOscillation(g["albefa"])
        M.SetAsymptotes(*g["asymptotes"])
    O.set_move_limit(g["move"])
    O.set_oscillation(g["albefa"])
    O.set_asymptotes(*g["asymptotes"])
    s = np.array(g["x0"])
    so = s.copy()
    smin, smax = np.full(n, g["xmin"]), np.full(n, g["xmax"])
    for _ in range(g["iterations"]):
        obj = (s ** 2).sum()
        c = np.array([((s - [5, 2, 1]) ** 2).sum() - 9, ((s - [3, 4, 3]) ** 2).sum() - 9])
        dc = np.zeros(n * m)
        dc[0::2], dc[1::2] = 2 * (s - [5, 2, 1]), 2 * (s - [3, 4, 3])
        co = np.array([((so - [5, 2, 1]) ** 2).sum() - 9, ((so - [3, 4, 3]) ** 2).sum() - 9])
        dco = np.zeros(n * m)
        dco[0::2], dco[1::2] = 2 * (so - [5, 2, 1]), 2 * (so - [3, 4, 3])
        G.Update(s, 2 * s, c, dc, smin, smax)
        so = O.update(so, 2 * so, co, dco, smin, smax)
        assert rel(s, so) <= 1e-12
    assert obj < g["objective_lt"]
    assert np.all(np.abs(c) < g["constraint_abs_lt"])


def test_mma_large_n_matches_oracle(oracle, gpu):
    rng = np.random.default_rng(31)
    n = 50000
    G = gpu.MMASolver(n, 1)
    O = oracle.MMA(n, 1)
    G.SetMoveLimit(0.2)
    O.set_move_limit(0.2)
    x = rng.uniform(0.1, 0.9, n)
    xg, xo = x.copy(), x.copy()
    for _ in range(4):
        df = -rng.uniform(0.1, 2.0, n)
        dg = np.full(n, 1.0 / n)
        g = np.array([xo.mean() - 0.5])
        G.Update(xg, df, g, dg, np.full(n, 1e-4), np.ones(n))
        xo = O.update(xo, df, g, dg, np.full(n, 1e-4), np.ones(n))
        assert rel(xg, xo) <= 1e-12
        xg = xo.copy()  # re-align so rounding does not compound


# ------------------------------------------------------------------ design loop
@pytest.mark.parametrize("method,R,grid,steps", [("oc", 1.5, (16, 8, 8), 8),
                                                 ("mma", 2.5, (16, 8, 8), 8)])
def test_design_trajectory(oracle, gpu, method, R, grid, steps):
    P, G = pair(oracle, gpu, *grid)
    F = oracle.Filter(P, R)
    move = 0.2 if method == "mma" else 0.15
    L = oracle.Loop(P, F, method=method, x0=0.3, move=move, cg_tol=1e-12)
    G.loop_init(0.3, method=method, filter_radius=R, move=move,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3))
    for _ in range(steps):
        L.step()
        info = G.loop_step()
        s = L.scalars()
        assert abs(info.compliance - s["compliance"]) <= 1e-10 * s["compliance"]
        assert abs(info.constraint - s["constraint"]) <= 1e-10 * max(1.0, abs(s["constraint"]))
    assert rel(G.loop_get("x"), L.get("x")) <= 1e-10
    assert rel(G.loop_get("dfds"), L.get("dfds")) <= 1e-9
