"""FP64 element-by-element K u on the FP64 tensor cores (DMMA).

The operator is exact FP64 arithmetic in a different summation order than
the node stencil, so the two agree to a few units in the last place of the
largest entry: max |y_tc - y_node| <= 1e-13 max |y_node|.  Grids cover the
tile edges (31 x 7 owned nodes per tile), several node-layer chunks along z,
uneven sizes and constrained faces; the solvers are checked against the
node-stencil runs of the same problem."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_inf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("grid", [(4, 2, 2), (16, 8, 8), (30, 6, 5), (31, 7, 12), (33, 9, 20),
                                  (64, 32, 32), (40, 20, 100), (7, 50, 9)])
def test_tc_fp64_matches_node_stencil(gpu, grid):
    nx, ny, nz = grid
    G = gpu.Context(nx, ny, nz)
    rng = np.random.default_rng(nx * 10000 + ny * 100 + nz)
    G.set_design(rng.uniform(0.01, 1.0, G.nelx))
    u = rng.standard_normal(G.numeq)
    y_node = G.apply_K_op(u, gpu.OP_FP64)
    y_tc = G.apply_K_op(u, gpu.OP_TC_FP64)
    assert rel_inf(y_tc, y_node) <= 1e-13


def test_apply_follows_the_solver_choice(gpu):
    # after a solve with fp64_tc=1, icarat_apply_K on 64x32x32 (70k nodes)
    # takes the tensor-core path; the result equals the node stencil's to
    # rounding either way
    G = gpu.Context(64, 32, 32)
    rng = np.random.default_rng(5)
    G.set_design(rng.uniform(0.05, 1.0, G.nelx))
    u = rng.standard_normal(G.numeq)
    y_node = G.apply_K_op(u, gpu.OP_FP64)
    assert rel_inf(G.apply_K(u), y_node) <= 1e-13
    G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-3, fp64_tc=1), want_val=False)
    assert rel_inf(G.apply_K(u), y_node) <= 1e-13


@pytest.mark.parametrize("method", ["mg", "jacobi"])
def test_solvers_on_tc_fp64_match_node_stencil(gpu, method):
    nx, ny, nz = 64, 32, 32
    G = gpu.Context(nx, ny, nz)
    rng = np.random.default_rng(6)
    G.set_design(rng.uniform(0.1, 1.0, G.nelx))
    m = gpu.MG_PCG if method == "mg" else gpu.JACOBI_PCG
    rtol = 1e-9 if method == "mg" else 1e-6
    u_tc, i_tc = G.solve(gpu.solve_opts(m, rtol=rtol, mg_levels=4, fp64_tc=1))
    u_nd, i_nd = G.solve(gpu.solve_opts(m, rtol=rtol, mg_levels=4, fp64_tc=-1))
    assert i_tc.status == gpu.OK and i_nd.status == gpu.OK
    assert abs(i_tc.iterations - i_nd.iterations) <= 2
    assert rel_inf(u_tc, u_nd) <= 100 * rtol
    f = G.fext()
    r = f - G.apply_K_op(u_tc, gpu.OP_FP64)
    assert np.linalg.norm(r) <= 1.001 * rtol * np.linalg.norm(f)


def test_fp64_tc_option_range(gpu):
    G = gpu.Context(8, 4, 4)
    G.set_design(np.full(G.nelx, 0.5))
    with pytest.raises(gpu.IcaratError) as e:
        G.solve(gpu.solve_opts(gpu.MG_PCG, mg_levels=2, fp64_tc=2))
    assert e.value.status == gpu.ERR_ARG


def test_tc_fp64_timing(gpu):
    G = gpu.Context(64, 32, 32)
    G.set_design(np.full(G.nelx, 0.5))
    assert G.time_operator(5, gpu.OP_TC_FP64) > 0.0
