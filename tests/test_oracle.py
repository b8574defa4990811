"""Pinning of the CPU oracle (oracle/) against the reference's own known
answers, the reference's own MMA/OC code compiled from its sources
(oracle/_ref), and independent closed forms.  CPU only."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_tests.json")))
TRAJ = json.load(open(os.path.join(HERE, "golden", "oracle_trajectory.json")))


# ---------------------------------------------------------------- filter
def test_filter_known_answers(oracle):
    """FilterTest (test_filter.cpp:63-124): 2x2 mesh, R = 2."""
    g = GOLD["filter_2x2"]
    F = oracle.Filter(centroids=np.array(g["centroids"]), radius=g["radius"])
    ans = np.array(g["answer"])
    out = F.sensitivity_filter(g["design_s_sens"], g["dfds"], np.ones(4))
    assert ((out - ans) ** 2).sum() < g["norm2_tol"]
    s_new = F.density_filter(g["design_s"], False)
    assert ((s_new - ans) ** 2).sum() < g["norm2_tol"]
    d_new = F.density_filter(g["dfds"], True)
    assert ((d_new - ans) ** 2).sum() < g["norm2_tol"]
    thr = oracle.threshold(s_new, g["threshold_beta"], 0.5)
    assert thr[0] < g["threshold_lo_below"] and thr[1] > g["threshold_hi_above"]
    der = oracle.threshold_derivative(s_new, 1.0, 0.5)
    assert ((der - 1.0) ** 2).sum() < g["derivative_beta1_norm2_tol"]


def test_filter_hexa_equals_quad(oracle):
    """The distance filter is dimension-agnostic: 2x2x1 hexa8, R = 2."""
    g = GOLD["filter_2x2"]
    P = oracle.Problem(2, 2, 1)
    F = oracle.Filter(P, g["radius"], faithful=True)
    out = F.density_filter(g["design_s"], False)
    assert ((out - np.array(g["answer"])) ** 2).sum() < g["norm2_tol"]


def test_filter_transposed_needs_forward(oracle):
    P = oracle.Problem(3, 2, 2)
    F = oracle.Filter(P, 1.5)
    with pytest.raises(RuntimeError):
        F.density_filter(np.ones(P.nelx), True)


@pytest.mark.parametrize("R", [1.0, 1.5, 2.5, 3.0])
def test_filter_bucketed_lists_equal_faithful(oracle, R):
    """Grid-bucketed neighbour lists == the O(N^2) preNeighbour lists."""
    P = oracle.Problem(7, 5, 4)
    a = oracle.Filter(P, R, faithful=True).lists()
    b = oracle.Filter(P, R, faithful=False).lists()
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_filter_stencil_sizes(oracle):
    """Interior stencil sizes 19 / 81 / 123 at R = 1.5 / 2.5 / 3."""
    P = oracle.Problem(9, 9, 9)
    centre = 4 + 4 * 9 + 4 * 81
    for R, n in [(1.5, 19), (2.5, 81), (3.0, 123)]:
        ptr, _, _ = oracle.Filter(P, R).lists()
        assert ptr[centre + 1] - ptr[centre] == n


# ---------------------------------------------------------------- MMA / OC
def _mma_toy(cls):
    g = GOLD["mma_toy"]
    n, m = g["n"], g["m"]
    mma = cls(n, m)
    mma.set_move_limit(g["move"])
    mma.set_oscillation(g["albefa"])
    mma.set_asymptotes(*g["asymptotes"])
    s = np.array(g["x0"])
    smin = np.full(n, g["xmin"])
    smax = np.full(n, g["xmax"])
    hist = []
    for _ in range(g["iterations"]):
        obj = (s ** 2).sum()
        dobj = 2 * s
        c = np.array([((s - [5, 2, 1]) ** 2).sum() - 9, ((s - [3, 4, 3]) ** 2).sum() - 9])
        dc = np.zeros(n * m)
        dc[0::2] = 2 * (s - [5, 2, 1])
        dc[1::2] = 2 * (s - [3, 4, 3])
        s = mma.update(s, dobj, c, dc, smin, smax)
        hist.append(s.copy())
    return obj, c, np.array(hist)


def test_mma_toy_known_answer(oracle):
    """MMASolverTest.toy (test_opt_solver.cpp:17-73)."""
    g = GOLD["mma_toy"]
    obj, c, _ = _mma_toy(oracle.MMA)
    assert obj < g["objective_lt"]
    assert np.all(np.abs(c) < g["constraint_abs_lt"])


def test_mma_toy_matches_reference_code(oracle):
    """The restatement is bit-identical to the reference MMASolver.cpp."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    _, _, a = _mma_toy(oracle.MMA)
    _, _, b = _mma_toy(oracle.RefMMA)
    assert np.array_equal(a, b)


def test_mma_large_matches_reference_code(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    rng = np.random.default_rng(3)
    n = 2000
    ours, ref = oracle.MMA(n, 1), oracle.RefMMA(n, 1)
    for M in (ours, ref):
        M.set_move_limit(0.2)
    x = rng.uniform(0.1, 0.9, n)
    xa, xb = x.copy(), x.copy()
    for it in range(4):
        df = -rng.uniform(0.1, 2.0, n)
        dg = np.full(n, 1.0 / n)
        g = np.array([xa.mean() - 0.5])
        xa = ours.update(xa, df, g, dg, np.full(n, 1e-4), np.ones(n))
        xb = ref.update(xb, df, g, dg, np.full(n, 1e-4), np.ones(n))
        assert np.array_equal(xa, xb)


def test_oc_matches_reference_code(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    P = oracle.Problem(6, 4, 3)
    F = oracle.Filter(P, 1.5)
    rng = np.random.default_rng(5)
    x = rng.uniform(0.2, 0.6, P.nelx)
    df = -rng.uniform(0.1, 3.0, P.nelx)
    dg = np.ones(P.nelx)
    V0 = 0.4 * P.nelx

    def vol(xk):
        return F.density_filter(xk).sum()

    a, _ = oracle.oc_update(x, df, V0, dg, np.full(P.nelx, 1e-4), np.ones(P.nelx), vol)
    b = oracle.ref_oc_update(x, df, V0, dg, np.full(P.nelx, 1e-4), np.ones(P.nelx), vol)
    assert np.array_equal(a, b)


# ---------------------------------------------------------------- element
def test_hexa8_unit_cube_volume(oracle):
    """BmatrixTest.cubic8 (test_bmatrix.cpp:123-146)."""
    g = GOLD["hexa8_volume"]
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                  [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    _, vol = oracle.hexa8_ke(X)
    assert abs(vol - g["volume"]) < g["tol"]


def _ke_gauss3(E=1.0, nu=0.3):
    """Independent integration: 3-point Gauss per axis, numpy einsum."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    pts, wts = np.polynomial.legendre.leggauss(3)
    loc = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                    [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]])
    K = np.zeros((24, 24))
    for a, wa in zip(pts, wts):
        for b, wb in zip(pts, wts):
            for c, wc in zip(pts, wts):
                r = np.array([a, b, c])
                s = 2 * loc - 1
                # physical coordinates x = (1 + r) / 2 on a unit cube, so
                # dN/dx = 2 dN/dr with N_a = prod_d (1 + s_d r_d) / 2
                dN = np.zeros((3, 8))
                for d in range(3):
                    others = [e for e in range(3) if e != d]
                    dN[d] = s[:, d] * np.prod(0.5 * (1 + s[:, others] * r[others]), axis=1)
                B = np.zeros((6, 24))
                B[0, 0::3], B[1, 1::3], B[2, 2::3] = dN
                B[3, 0::3], B[3, 1::3] = dN[1], dN[0]
                B[4, 1::3], B[4, 2::3] = dN[2], dN[1]
                B[5, 0::3], B[5, 2::3] = dN[2], dN[0]
                K += wa * wb * wc * 0.125 * B.T @ D @ B
    return K


def test_ke0_independent_integration(oracle):
    P = oracle.Problem(2, 2, 2)
    ke, vol = P.ke0()
    ref = _ke_gauss3()
    assert np.abs(ke - ref).max() < 1e-14 * np.abs(ref).max()
    assert abs(vol - 1.0) < 1e-14


def test_ke0_rigid_body_null_space(oracle):
    ke, _ = oracle.Problem(2, 2, 2).ke0()
    X = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                  [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], float)
    modes = []
    for d in range(3):
        t = np.zeros((8, 3))
        t[:, d] = 1
        modes.append(t.ravel())
    for (a, b) in [(0, 1), (1, 2), (0, 2)]:
        r = np.zeros((8, 3))
        r[:, a], r[:, b] = -X[:, b], X[:, a]
        modes.append(r.ravel())
    for m in modes:
        assert np.abs(ke @ m).max() < 1e-14
    ev = np.linalg.eigvalsh(0.5 * (ke + ke.T))
    assert (ev > 1e-10).sum() == 18


# ---------------------------------------------------------------- mesh / DOF
@pytest.mark.parametrize("grid,numeq", [((32, 16, 16), 27744), ((64, 32, 32), 209088)])
def test_dof_counts(oracle, grid, numeq):
    P = oracle.Problem(*grid)
    assert P.numeq == numeq
    assert P.neq == 3 * (grid[0] + 1) * (grid[1] + 1) * (grid[2] + 1)


def test_dof_numbering_rules(oracle):
    """countDOF: free components node-major, constrained after; partial flags."""
    d = [((1, 0, 1), (0.0, 0.5, 0.0), ((0, 0), (0, 2), (0, 2))),
         ((0, 1, 0), (0.0, 0.0, 0.25), ((3, 3), (1, 1), (0, 0)))]
    loads = [((0.0, 0.0, -1.0), ((3, 3), (2, 2), (2, 2))),
             ((1.0, 0.0, 0.0), ((3, 3), (2, 2), (2, 2)))]
    P = oracle.Problem(3, 2, 2, dirichlet=d, loads=loads)
    dof = P.dof()
    xyz = P.xyz()
    free = dof < P.numeq
    # free numbers ascend node-major; constrained ones ascend after numeq
    assert np.array_equal(dof[free], np.arange(P.numeq))
    assert np.array_equal(np.sort(dof[~free]), np.arange(P.numeq, P.neq))
    assert np.array_equal(dof[~free], np.arange(P.numeq, P.neq))
    on_face = xyz[:, 0] == 0
    assert np.all(~free[on_face][:, 0]) and np.all(free[on_face][:, 1])
    f = P.fext()
    n_load = np.where((xyz == [3, 2, 2]).all(axis=1))[0][0]
    assert f[dof[n_load, 2]] == -1.0 and f[dof[n_load, 0]] == 1.0
    assert np.count_nonzero(f) == 2


# ---------------------------------------------------------------- K, solve
def _scipy_K(P, design_s):
    ke, _ = P.ke0()
    conn = P.conn()
    dof = P.dof()
    E = (1 - design_s ** P.penal) * P.E1 + design_s ** P.penal * P.E2
    edof = dof[conn].reshape(-1, 24)
    rows = np.repeat(edof, 24, axis=1).ravel()
    cols = np.tile(edof, (1, 24)).ravel()
    vals = (E[:, None, None] * ke[None]).ravel()
    keep = (rows < P.numeq) & (cols < P.numeq)
    return sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(P.numeq, P.numeq))


def test_csr_matches_scipy_assembly(oracle):
    P = oracle.Problem(5, 4, 3)
    rng = np.random.default_rng(0)
    rho = rng.uniform(0.05, 1.0, P.nelx)
    P.assemble(rho)
    rp, col, val = P.csr()
    A = sp.csr_matrix((val, col, rp), shape=(P.numeq, P.numeq))
    B = _scipy_K(P, rho)
    assert abs(A - B).max() < 1e-15 * abs(B).max()
    u = rng.standard_normal(P.numeq)
    assert np.abs(P.apply_K(u) - B @ u).max() < 1e-13 * np.abs(B @ u).max()


def test_pcg_matches_direct_solve(oracle):
    P = oracle.Problem(8, 4, 4)
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.1, 1.0, P.nelx)
    val, it, rr = P.solve(rho, tol=1e-13)
    B = _scipy_K(P, rho)
    ref = spla.spsolve(B.tocsc(), P.fext())
    assert rr < 1e-13
    assert np.abs(val - ref).max() < 1e-9 * np.abs(ref).max()
    assert abs(P.compliance(val) - P.fext() @ ref) < 1e-11 * abs(P.fext() @ ref)


def test_sensitivity_finite_difference(oracle):
    """dc/drho against central differences (fdm.cpp style, delta = 1e-7)."""
    P = oracle.Problem(4, 2, 2)
    rng = np.random.default_rng(2)
    rho = rng.uniform(0.3, 0.9, P.nelx)
    val, _, _ = P.solve(rho, tol=1e-14)
    dfds, dgds = P.sensitivity(rho, P.node_values(val))
    assert np.allclose(dgds, 1.0)
    for e in [0, 5, 11, P.nelx - 1]:
        h = 1e-7
        rp, rm = rho.copy(), rho.copy()
        rp[e] += h
        rm[e] -= h
        cp = P.compliance(P.solve(rp, tol=1e-14)[0])
        cm = P.compliance(P.solve(rm, tol=1e-14)[0])
        fd = (cp - cm) / (2 * h)
        assert abs(fd - dfds[e]) < 1e-5 * abs(dfds[e])


def test_node_value_truncation(oracle):
    P = oracle.Problem(2, 1, 1)
    val = np.zeros(P.numeq)
    val[0], val[1], val[2] = 5e-16, -2e-15, 0.25
    nv = P.node_values(val)
    dof = P.dof()
    flat = nv.ravel()[np.argsort(dof.ravel())][:P.numeq]
    assert flat[0] == 0.0 and flat[1] == -2e-15 and flat[2] == 0.25


# ---------------------------------------------------------------- loop
@pytest.mark.parametrize("name", ["oc_8x4x4", "mma_8x4x4"])
def test_oracle_trajectory_fixture(oracle, name):
    t = TRAJ[name]
    P = oracle.Problem(*t["grid"])
    F = oracle.Filter(P, t["radius"])
    L = oracle.Loop(P, F, method=t["method"], x0=t["x0"],
                    move=0.2 if t["method"] == "mma" else 0.15, cg_tol=t["cg_rtol"])
    comp = []
    for _ in range(len(t["compliance"])):
        L.step()
        comp.append(L.scalars()["compliance"])
    assert np.allclose(comp, t["compliance"], rtol=1e-12, atol=0)
    assert np.allclose(L.get("x"), t["x_final"], rtol=1e-10, atol=1e-12)


def test_oc_volume_constraint_met(oracle):
    P = oracle.Problem(16, 8, 8)
    F = oracle.Filter(P, 1.5)
    L = oracle.Loop(P, F, method="oc", x0=0.3)
    for _ in range(5):
        L.step()
    x = L.get("x")
    assert abs(F.density_filter(x).sum() - 0.3 * P.nelx) < 1e-3 * P.nelx


def test_helmholtz_filter_known_answers(oracle):
    # FilterHelmholtzTest (test_filter.cpp:126-175): 2 x 2 unit quad4, R = 2,
    # density and sensitivity calls; as a 2 x 2 x 1 hexa8 slab
    g = GOLD["helmholtz_2x2"]
    s = np.array(g["design_s"])
    out, _ = oracle.helmholtz_filter(2, 2, 1, g["radius"], s)
    sens, _ = oracle.helmholtz_filter(2, 2, 1, g["radius"], s, is_sens=True)
    assert ((out - np.array(g["answer"])) ** 2).sum() < g["norm2_tol"]
    assert ((sens - np.array(g["answer_sens"])) ** 2).sum() < g["norm2_tol"]


def test_helmholtz_filter_properties(oracle):
    # a constant design passes through (the PDE filter preserves constants);
    # the map is symmetric (its sensitivity call is the same linear map);
    # a finer solve changes nothing beyond its tolerance
    nx, ny, nz, R = 6, 4, 3, 1.7
    n = nx * ny * nz
    c, _ = oracle.helmholtz_filter(nx, ny, nz, R, np.full(n, 0.37))
    assert np.abs(c - 0.37).max() < 1e-12
    rng = np.random.default_rng(3)
    x, y = rng.random(n), rng.random(n)
    Hx, _ = oracle.helmholtz_filter(nx, ny, nz, R, x)
    Hy, _ = oracle.helmholtz_filter(nx, ny, nz, R, y, is_sens=True)
    assert abs(Hx @ y - x @ Hy) < 1e-12 * abs(Hx @ y)
    # stretched elements (lx != nx) keep both properties
    c2, _ = oracle.helmholtz_filter(nx, ny, nz, R, np.full(n, 0.5), lx=2.0 * nx)
    assert np.abs(c2 - 0.5).max() < 1e-12


def test_helmholtz_loop_oracle(oracle):
    # the loop with the Helmholtz filter (opt_macro_oc.cpp:73-74): step 1
    # filters the start design with the same map as helmholtz_filter, and
    # OC (Helmholtz volume functor) and MMA steps run and lower compliance
    nx, ny, nz, R = 8, 4, 4, 1.5
    for method in ("oc", "mma"):
        P = oracle.Problem(nx, ny, nz)
        L = oracle.Loop(P, None, method=method, x0=0.3, use_threshold=True,
                        cg_tol=1e-12, helmholtz_R=R)
        L.step()
        ref, _ = oracle.helmholtz_filter(nx, ny, nz, R, np.full(P.nelx, 0.3), tol=1e-10)
        assert np.abs(L.get("xfil") - ref).max() < 1e-12
        c1 = L.scalars()["compliance"]
        for _ in range(3):
            L.step()
        assert L.scalars()["compliance"] < c1


def test_case_loop_matches_c_loop(oracle):
    # the composed multi-case loop with one case and no domains is the C
    # loop (MMA, threshold on and off)
    nx, ny, nz = 8, 4, 4
    for thr in (False, True):
        P = oracle.Problem(nx, ny, nz)
        F = oracle.Filter(P, 1.5)
        L = oracle.Loop(P, F, method="mma", x0=0.3, move=0.2, use_threshold=thr, cg_tol=1e-12)
        P2 = oracle.Problem(nx, ny, nz)
        F2 = oracle.Filter(P2, 1.5)
        M = oracle.CaseLoop([P2], F2, use_threshold=thr)
        for _ in range(3):
            L.step()
            comp, const, _ = M.step()
            s = L.scalars()
            assert abs(comp - s["compliance"]) <= 1e-12 * s["compliance"]
            assert abs(const - s["constraint"]) <= 1e-12
        assert np.abs(M.x - L.get("x")).max() <= 1e-12


def test_case_loop_domains_and_cases(oracle):
    # zeroed sensitivities stay zero on the non-design IDs, and two load
    # cases give the sum of the two single-case compliances on step 1
    nx, ny, nz = 8, 4, 4
    loads = [[((0.0, 0.0, -1.0), ((nx, nx), (2, 2), (0, 0)))],
             [((0.0, -1.0, 0.0), ((nx, nx), (4, 4), (4, 4)))]]
    dirich = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, ny), (0, nz)))]
    Ps = [oracle.Problem(nx, ny, nz, dirichlet=dirich, loads=l) for l in loads]
    nd = np.arange(0, 32)
    M = oracle.CaseLoop(Ps, oracle.Filter(Ps[0], 1.5), nondesign_ids=nd,
                        design_ids=np.arange(32, Ps[0].nelx))
    comp, _, _ = M.step()
    assert not M.dfds[nd].any() and not M.dgds[nd].any()
    singles = []
    for l in loads:
        P = oracle.Problem(nx, ny, nz, dirichlet=dirich, loads=l)
        singles.append(oracle.CaseLoop([P], oracle.Filter(P, 1.5)).step()[0])
    assert abs(comp - sum(singles)) <= 1e-12 * comp


def test_distributed_load_totals(oracle):
    # a traction on a whole free face sums to traction x area (Gauss rule
    # exact for the bilinear face); a z-max box goes to the x-min faces of
    # the top elements as SurfaceLoad::judgeLine picks them
    nx, ny, nz = 6, 4, 3
    free = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, 0), (0, 0)))]  # one corner node
    P = oracle.Problem(nx, ny, nz, lx=3.0, ly=2.0, lz=6.0, dirichlet=free,
                       loads=[((0.0, 0.0, -2.0), ((3, 3), (0, 2), (0, 6)))])
    assert abs(P.fext().sum() + 2.0 * 2.0 * 6.0) < 1e-12
    P = oracle.Problem(nx, ny, nz, dirichlet=free,
                       loads=[((0.0, 0.0, 1.0), ((0, nx), (0, ny), (nz, nz)))])
    f = P.fext()
    assert abs(f.sum() - nx * ny * 1.0) < 1e-12  # 24 unit x-min faces of the top layer
    # the x-min face of a top element spans z = nz - 1 .. nz: the layer below
    # the loaded face receives half of the load
    d, z = P.dof(), P.xyz()[:, 2]
    below = [d[n, 2] for n in range(P.numnp) if z[n] == nz - 1 and d[n, 2] < P.numeq]
    assert abs(f[below].sum() - nx * ny * 0.5) < 1e-12
