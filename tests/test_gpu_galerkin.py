"""Galerkin coarse operators of the multigrid (ICARAT_COARSE_GALERKIN).

* Every coarse level's operator, as the V-cycle applies it
  (icarat_mg_level_apply), equals D P^T A P D of the level above computed by
  the CPU checker oracle/galerkin.py from the oracle's CSR stiffness, to
  1e-12 relative, on a random and on a thresholded solid / void design.
* The coarsest dense solve of the Galerkin hierarchy meets 1e-10.
* MG-PCG and the mixed-precision solver with Galerkin coarse operators meet
  their tolerance on solid / void designs (the residual recomputed with the
  oracle's CSR stiffness), give the compliance of a direct solve of the
  oracle's system to 100 rtol, and need fewer iterations than with the rediscretised coarse operators,
  which is what the option is for.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import galerkin as GL

pytestmark = pytest.mark.gpu


def solid_void(nelx, rng, frac=0.45):
    """thresholded smoothed noise: densities 1 (solid) and 1e-3 (void)"""
    x = rng.standard_normal(nelx)
    x = np.convolve(x, np.ones(9) / 9.0, mode="same")
    t = np.quantile(x, 1.0 - frac)
    return np.where(x >= t, 1.0, 1e-3)


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("design", ["random", "solid_void"])
def test_levels_match_galerkin_product(oracle, gpu, design):
    nx, ny, nz, levels = 16, 8, 8, 3
    P = oracle.Problem(nx, ny, nz)
    G = gpu.Context(nx, ny, nz)
    rng = np.random.default_rng(21)
    rho = rng.uniform(0.02, 1.0, P.nelx) if design == "random" else solid_void(P.nelx, rng)
    P.assemble(rho)
    G.set_design(rho)
    H = GL.hierarchy(P, levels)
    o = gpu.solve_opts(gpu.MG_PCG, mg_levels=levels, coarse_op=gpu.COARSE_GALERKIN)
    for l in range(1, levels):
        A, fixed = H[l]
        x = rng.standard_normal(A.shape[0])
        x[fixed.T.ravel()] = 0.0
        y = G.mg_level_apply(l, x, o)
        assert rel(y, A @ x) <= 1e-12, (l, rel(y, A @ x))


def test_galerkin_coarsest_dense_solve(gpu):
    G = gpu.Context(32, 16, 16)
    G.set_design(np.random.default_rng(4).uniform(0.3, 1.0, G.nelx))
    o = gpu.solve_opts(gpu.MG_PCG, mg_levels=3, coarse_op=gpu.COARSE_GALERKIN)
    G.mg_level_apply(2, np.zeros(3 * 9 * 5 * 5), o)  # builds the Galerkin hierarchy
    r, n = G.coarse_check(3)
    assert n > 0 and r <= 1e-10, (r, n)


@pytest.mark.parametrize("method,rtol", [("MG_PCG", 1e-10), ("MIXED_IR", 1e-8)])
def test_solve_on_solid_void_designs(oracle, gpu, method, rtol):
    nx, ny, nz = 32, 16, 16
    P = oracle.Problem(nx, ny, nz)
    G = gpu.Context(nx, ny, nz)
    rho = solid_void(P.nelx, np.random.default_rng(8))
    P.assemble(rho)
    G.set_design(rho)
    m = getattr(gpu, method)
    f = P.fext()
    rp, col, val = P.csr()
    K = sp.csr_matrix((val, col, rp), shape=(P.numeq, P.numeq))
    u_ref = spla.spsolve(K.tocsc(), f)
    its = {}
    for name, cop in (("galerkin", gpu.COARSE_GALERKIN), ("rediscretised", gpu.COARSE_REDISCRETISED)):
        o = gpu.solve_opts(m, rtol=rtol, maxit=5000, mg_levels=3, coarse_op=cop)
        u, info = G.solve(o)
        assert info.status == gpu.OK, (name, info.status)
        its[name] = info.iterations
        if name == "galerkin":
            r = f - P.apply_K(u)
            assert np.linalg.norm(r) <= 1.5 * rtol * np.linalg.norm(f)
            c, c_ref = float(f @ u), float(f @ u_ref)
            assert abs(c - c_ref) <= 100 * rtol * abs(c_ref), (c, c_ref)
    assert its["galerkin"] < its["rediscretised"], its
