"""Stiffness operators by precision: the FP32 CUDA-core stencil and the
tcgen05 element-by-element operator (BF16 hi/lo split, FP32 accumulation),
each against the FP64 operator on the same design and displacement.

Tolerances (max |y - y64| / max |y64|), from the arithmetic of each form:
  - FP32 stencil: 1e-6 (FP32 rounding of Ke0, E, u and the sums);
  - tensor cores, 3 BF16 products: 5e-5 (about 16 significant bits per
    product, FP32 accumulation);
  - tensor cores, 1 BF16 product: 1e-2 (8 significant bits).
Grids include sizes that are not multiples of the 31 x 7 node tile and
single-layer z chunks.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {1: 1e-6, 2: 5e-5, 3: 1e-2}


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("grid", [(2, 1, 1), (8, 4, 4), (31, 7, 3), (33, 17, 9), (64, 32, 32),
                                  (63, 9, 40)])
@pytest.mark.parametrize("op", [1, 2, 3])
def test_operator_matches_fp64(gpu, grid, op):
    G = gpu.Context(*grid)
    rng = np.random.default_rng(sum(grid) + op)
    G.set_design(rng.uniform(0.05, 1.0, G.nelx))
    u = rng.standard_normal(G.numeq)
    y64 = G.apply_K(u)
    y = G.apply_K_op(u, op)
    assert rel(y, y64) <= TOL[op]


def test_operator_energy_on_solution_and_void_design(gpu):
    """Displacements that solve K u = f on a solid/void design (SIMP contrast
    ~1e9): K u nearly cancels to the point load, so the error is measured in
    energy, |u . (y - y64)| / (u . y64).  Rounding u itself to FP32 (shared
    by both operators; the void displacements are huge) dominates: about
    2e-4 for each, bound 5e-4.  Without the tensor-core operator's removal
    of each element's translation before the BF16 split this error was
    6e-3."""
    G = gpu.Context(48, 24, 24)
    rng = np.random.default_rng(7)
    rho = np.where(rng.uniform(size=G.nelx) < 0.5, 1.0, 1e-3)
    G.set_design(rho)
    u, _ = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-10, mg_levels=3))
    y64 = G.apply_K(u)
    energy = u @ y64
    e_tc = abs(u @ (G.apply_K_op(u, gpu.OP_TC_BF16X3) - y64)) / energy
    e_32 = abs(u @ (G.apply_K_op(u, gpu.OP_FP32) - y64)) / energy
    print("relative energy error: tensor cores %.3g, FP32 %.3g" % (e_tc, e_32))
    assert e_tc <= 5e-4
    assert e_32 <= 5e-4


def test_unknown_operator_is_rejected(gpu):
    G = gpu.Context(8, 4, 4)
    G.set_design(np.full(G.nelx, 0.5))
    with pytest.raises(gpu.IcaratError) as e:
        G.apply_K_op(np.zeros(G.numeq), 7)
    assert e.value.status == gpu.ERR_ARG


def test_operator_timing_entry(gpu):
    G = gpu.Context(32, 16, 16)
    G.set_design(np.full(G.nelx, 0.5))
    for op in (0, 1, 2, 3):
        assert G.time_operator(3, op) > 0.0


@pytest.mark.parametrize("fine_op,krylov_op", [(1, 1), (2, 1), (3, 1), (2, 2)])
def test_mixed_solver_operator_choices(gpu, fine_op, krylov_op):
    """Every operator choice converges to the FP64 residual target; only the
    iteration count depends on it."""
    G = gpu.Context(32, 16, 16)
    G.set_design(np.random.default_rng(5).uniform(0.1, 0.5, G.nelx))
    u64, _ = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3))
    u, info = G.solve(gpu.solve_opts(gpu.MIXED_IR, rtol=1e-8, mg_levels=3, maxit=1000,
                                     fine_op=fine_op, krylov_op=krylov_op))
    assert info.status == gpu.OK and info.rel_residual < 1e-8
    assert rel(u, u64) <= 1e-6


def test_mixed_solver_rejects_fp64_operator_choice(gpu):
    G = gpu.Context(8, 4, 4)
    G.set_design(np.full(G.nelx, 0.5))
    with pytest.raises(gpu.IcaratError) as e:
        G.solve(gpu.solve_opts(gpu.MIXED_IR, rtol=1e-8, mg_levels=2, fine_op=9))
    assert e.value.status == gpu.ERR_ARG


@pytest.mark.parametrize("grid", [(8, 4, 4), (31, 7, 3), (33, 17, 9), (64, 32, 32)])
def test_every_operator_matches_oracle_csr(oracle, gpu, grid):
    """Each operator of icarat_apply_K_op against the oracle's assembled CSR
    K_ff (triplet assembly of the reference, oracle/icarat_oracle.c), not
    only against the GPU's own FP64 stencil.  Tolerances as above; both FP64
    forms (node stencil, FP64 tensor cores) <= 1e-14."""
    P, G = oracle.Problem(*grid), gpu.Context(*grid)
    rng = np.random.default_rng(sum(grid))
    rho = rng.uniform(0.05, 1.0, P.nelx)
    P.assemble(rho)
    G.set_design(rho)
    u = rng.standard_normal(P.numeq)
    y = P.apply_K(u)
    tol = {gpu.OP_FP64: 1e-14, gpu.OP_TC_FP64: 1e-14, **TOL}
    for op, t in tol.items():
        assert rel(G.apply_K_op(u, op), y) <= t, op
