"""Helmholtz PDE filter (FilterHelmholtz, src/optimization/filter_helm.hpp)
on the GPU, through the C ABI, against the oracle and the reference's test.

Tolerances:
  - the reference's FilterHelmholtzTest answers: squared-norm error < 1e-10
    at the default CG tolerance (1e-10), as the reference test checks;
  - against the oracle: both CGs to ||r|| < 1e-12 ||F||, filtered values
    <= 1e-9 relative to max |out| (FP64, different summation order), CG
    iteration counts within 2;
  - constants pass through to 1e-8; the density and sensitivity calls are
    the same symmetric map: |x.H(y) - H(x).y| <= 1e-9 |H(x).y|.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_tests.json")))


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def test_helmholtz_known_answers(gpu):
    """FilterHelmholtzTest (test_filter.cpp:126-175): 2 x 2 unit quad4, R = 2,
    on a 2 x 2 x 1 voxel slab (z-independent data give the same nodal system
    scaled by the layer thickness)."""
    g = GOLD["helmholtz_2x2"]
    G = gpu.Context(2, 2, 1, dirichlet=[], loads=[])
    F = gpu.FilterHelmholtz(G, g["radius"])
    out = F.densityFilter(g["design_s"], "Eigen_CG", 0, False)
    assert ((out - np.array(g["answer"])) ** 2).sum() < g["norm2_tol"]
    assert F.info.status == 0 and F.info.rel_residual < 1e-10
    sens = F.densityFilter(g["design_s"], "Eigen_CG", 0, True)
    assert ((sens - np.array(g["answer_sens"])) ** 2).sum() < g["norm2_tol"]
    with pytest.raises(gpu.IcaratError) as e:
        F.densityFilter(g["design_s"], "No_Such_Solver")
    assert e.value.status == gpu.ERR_UNSUPPORTED


CASES = [
    (2, 2, 1, 2.0, None),
    (1, 1, 1, 1.0, None),
    (5, 3, 4, 1.7, None),
    (13, 7, 6, 2.5, None),
    (4, 3, 2, 1.3, (8.0, 3.0, 1.0)),  # stretched voxels 2 x 1 x 0.5
    (20, 10, 10, 3.0, None),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("is_sens", [False, True])
def test_helmholtz_matches_oracle(oracle, gpu, case, is_sens):
    nx, ny, nz, R, box = case
    lx, ly, lz = box if box else (nx, ny, nz)
    G = gpu.Context(nx, ny, nz, lx=lx, ly=ly, lz=lz, dirichlet=[], loads=[])
    G.helmholtz_setup(R)
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz)
    x = rng.uniform(1e-3, 1.0, G.nelx) if not is_sens else rng.standard_normal(G.nelx)
    a, info = G.helmholtz_filter(x, is_sens, rtol=1e-12)
    b, its = oracle.helmholtz_filter(nx, ny, nz, R, x, is_sens=is_sens, tol=1e-12,
                                     lx=lx, ly=ly, lz=lz)
    assert info.status == 0 and info.rel_residual < 1e-12
    assert rel(a, b) <= 1e-9
    assert abs(info.iterations - its) <= 2


def test_helmholtz_properties_large(gpu):
    nx, ny, nz, R = 96, 48, 48, 3.0
    G = gpu.Context(nx, ny, nz, dirichlet=[], loads=[])
    G.helmholtz_setup(R)
    c, info = G.helmholtz_filter(np.full(G.nelx, 0.37), rtol=1e-12)
    assert info.status == 0
    assert np.abs(c - 0.37).max() < 1e-8
    rng = np.random.default_rng(5)
    x, y = rng.random(G.nelx), rng.random(G.nelx)
    Hx, _ = G.helmholtz_filter(x, rtol=1e-12)
    Hy, _ = G.helmholtz_filter(y, True, rtol=1e-12)
    assert abs(Hx @ y - x @ Hy) <= 1e-9 * abs(Hx @ y)
    # linearity
    Hxy, _ = G.helmholtz_filter(2.0 * x - 0.5 * y, rtol=1e-12)
    Hy_d, _ = G.helmholtz_filter(y, rtol=1e-12)
    assert rel(Hxy, 2.0 * Hx - 0.5 * Hy_d) <= 1e-9


def test_helmholtz_zero_input_and_cap(gpu):
    G = gpu.Context(6, 4, 3, dirichlet=[], loads=[])
    G.helmholtz_setup(2.0)
    z, info = G.helmholtz_filter(np.zeros(G.nelx))
    assert info.iterations == 0 and info.status == 0 and not z.any()
    x = np.random.default_rng(1).random(G.nelx)
    _, info = G.helmholtz_filter(x, rtol=1e-14, maxit=2)
    assert info.status == gpu.WARN_MAXITER and info.iterations == 3


def test_helmholtz_state_and_arguments(gpu):
    G = gpu.Context(4, 2, 2, dirichlet=[], loads=[])
    with pytest.raises(gpu.IcaratError) as e:
        G.helmholtz_filter(np.ones(G.nelx))
    assert e.value.status == gpu.ERR_STATE
    with pytest.raises(gpu.IcaratError) as e:
        G.helmholtz_setup(-1.0)
    assert e.value.status == gpu.ERR_ARG
    G.helmholtz_setup(1.5)
    with pytest.raises(gpu.IcaratError) as e:
        G.helmholtz_filter(np.ones(G.nelx), rtol=float("nan"))
    assert e.value.status == gpu.ERR_ARG
    # a second setup replaces the first
    G.helmholtz_setup(2.5)
    G.helmholtz_filter(np.ones(G.nelx))


def test_helmholtz_dev_matches_host_and_leaves_solve_alone(gpu):
    import torch

    G = gpu.Context(16, 8, 8)
    rho = np.random.default_rng(3).uniform(0.2, 1.0, G.nelx)
    G.set_design(rho)
    u0, _ = G.solve(gpu.solve_opts(gpu.JACOBI_PCG, 1e-10, 5000))
    G.helmholtz_setup(2.0)
    h, info_h = G.helmholtz_filter(rho, rtol=1e-12)
    xd = torch.tensor(rho, dtype=torch.float64, device="cuda")
    od = torch.empty_like(xd)
    info_d = G.helmholtz_filter_dev(xd.data_ptr(), od.data_ptr(), rtol=1e-12)
    torch.cuda.synchronize()
    assert np.array_equal(od.cpu().numpy(), h)
    assert info_d.iterations == info_h.iterations
    with pytest.raises(gpu.IcaratError):
        G.helmholtz_filter_dev(xd.data_ptr(), xd.data_ptr())
    u1, _ = G.solve(gpu.solve_opts(gpu.JACOBI_PCG, 1e-10, 5000))
    assert np.array_equal(u0, u1)


@pytest.mark.parametrize("method,R,thr", [("mma", 2.0, True), ("oc", 1.0, True),
                                          ("mma", 1.5, False)])
def test_helmholtz_loop_matches_oracle(oracle, gpu, method, R, thr):
    """opt_mma_Helmholtz.cpp:86-170 (MMA) and opt_macro_oc.cpp:83-172 (OC,
    Helmholtz filter inside the volume functor): 3 design iterations on both
    sides, elasticity CG to 1e-12, Helmholtz CG to the reference's 1e-10 on
    both sides, so values agree to 1e-7 relative."""
    nx, ny, nz = 12, 6, 6
    P, G = oracle.Problem(nx, ny, nz), gpu.Context(nx, ny, nz)
    move = 0.2 if method == "mma" else 0.15
    L = oracle.Loop(P, None, method=method, x0=0.3, move=move, use_threshold=thr,
                    cg_tol=1e-12, helmholtz_R=R)
    G.loop_init(0.3, method=method, filter_radius=R, move=move, use_threshold=thr,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2), filter="helmholtz")
    for _ in range(3):
        L.step()
        info = G.loop_step()
        s = L.scalars()
        assert info.status in (0, 1)
        assert abs(info.compliance - s["compliance"]) <= 1e-7 * s["compliance"]
        assert abs(info.constraint - s["constraint"]) <= 1e-7 * max(1.0, abs(s["constraint"]))
    for which in ("xfil", "x", "dfds", "dgds"):
        assert rel(G.loop_get(which), L.get(which)) <= 1e-6, which


@pytest.mark.parametrize("use_thr", [False, True])
def test_oc_update_with_helmholtz_functor(oracle, gpu, use_thr):
    """OC::UpdateVariables with the volume functor of opt_macro_oc.cpp:153-164
    over the Helmholtz filter (icarat_oc_update, filter_kind 1) against the
    oracle's OC with that functor built from its Helmholtz restatement (both
    filters' CGs at the reference's 1e-10): same bisection steps, x to 1e-8."""
    nx, ny, nz, R = 10, 5, 5, 1.0
    G = gpu.Context(nx, ny, nz)
    G.helmholtz_setup(R)
    rng = np.random.default_rng(31)
    n = G.nelx
    x = rng.uniform(0.2, 0.6, n)
    dfdx = -rng.uniform(0.1, 2.0, n)
    dgdx = np.full(n, 1.0)
    xmin, xmax = np.full(n, 1e-4), np.ones(n)
    vol = G.element_stiffness()[1]
    beta, T = 2.0, 0.5
    g0 = 0.35 * n * vol

    def volume(xk):
        f, _ = oracle.helmholtz_filter(nx, ny, nz, R, xk, tol=1e-10)
        t = oracle.threshold(f, beta, T) if use_thr else f
        return float(np.sum(t * vol))

    ref, steps_ref = oracle.oc_update(x, dfdx, g0, dgdx, xmin, xmax, volume)
    got, steps = G.oc_update(x, dfdx, g0, dgdx, xmin, xmax, use_threshold=use_thr, beta=beta,
                             T=T, filter="helmholtz")
    assert steps == steps_ref
    assert np.abs(got - ref).max() <= 1e-8
    with pytest.raises(gpu.IcaratError) as e:
        gpu.Context(4, 2, 2).oc_update(x[:16], dfdx[:16], 1.0, dgdx[:16], xmin[:16],
                                       xmax[:16], filter="helmholtz")
    assert e.value.status == gpu.ERR_STATE
