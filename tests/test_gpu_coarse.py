"""Coarsest-level dense solve of the multigrid (banded Cholesky, register
64 x 64 diagonal blocks, recursive triangular inverse on the FP64 tensor
cores): K_c x = b solved through the dense inverse factor and checked with
the coarsest level's own stencil, ||b - K_c x|| <= 1e-10 ||b|| (moduli in
[0.027, 1], so the coarse operators are well enough conditioned for that
bound), on grids whose longest axis is x, y or z, of 1 to 61 diagonal
blocks, with clamped faces on different sides."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid,levels", [
    ((32, 16, 16), 2),   # 16x8x8 coarsest: 3,888 unknowns, 61 blocks
    ((16, 8, 8), 2),     # 8x4x4: 594 unknowns
    ((24, 12, 12), 3),   # 6x3x3
    ((8, 16, 32), 2),    # z longest
    ((12, 40, 8), 2),    # y longest, uneven
    ((4, 4, 4), 2),      # one block
])
def test_coarse_dense_solve(gpu, grid, levels):
    nx, ny, nz = grid
    G = gpu.Context(nx, ny, nz)
    G.set_design(np.random.default_rng(sum(grid)).uniform(0.3, 1.0, G.nelx))
    rel, n = G.coarse_check(levels)
    assert n > 0
    assert rel <= 1e-10, (rel, n)


def test_coarse_dense_solve_other_supports(gpu):
    # clamped bottom face (z = 0) instead of the left face, load on top
    nx, ny, nz = 32, 16, 16
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0.0, nx), (0.0, ny), (0.0, 0.0)))]
    lo = [((0.0, 0.0, -1.0), ((nx / 2, nx / 2), (ny / 2, ny / 2), (nz, nz)))]
    G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
    G.set_design(np.random.default_rng(3).uniform(0.3, 1.0, G.nelx))
    rel, n = G.coarse_check(2)
    assert n == 3 * 17 * 9 * 8
    assert rel <= 1e-10
