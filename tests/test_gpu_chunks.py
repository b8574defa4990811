"""Iterations past convergence change nothing.

The solvers replay graph chunks of iterations and read the stop flag between
chunks, so a chunk can hold iterations after the one that converged: their
CG kernels and (through the solve's stop flag) their V-cycle kernels return
at entry.  A solve replayed one iteration per chunk and the same solve in
chunks of 7 must therefore stop at the same iteration with bit-identical
solutions, for every solver and coarse-operator variant.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [
    ("MG_PCG", {}),
    ("MG_PCG", {"coarse_op": "COARSE_GALERKIN"}),
    ("MIXED_IR", {}),
    ("MIXED_IR", {"fine_op": "OP_FP32"}),
    ("JACOBI_PCG", {}),
]


@pytest.mark.parametrize("method,extra", CASES,
                         ids=["mg", "mg_galerkin", "mixed_tc", "mixed_fp32", "jacobi"])
def test_chunk_size_does_not_change_the_solve(gpu, method, extra):
    G = gpu.Context(32, 16, 16)
    G.set_design(np.random.default_rng(12).uniform(0.05, 1.0, G.nelx))
    kw = {k: getattr(gpu, v) for k, v in extra.items()}
    m = getattr(gpu, method)
    rtol = 1e-6 if method == "MIXED_IR" else 1e-8
    out = []
    chunk = 1
    for _ in range(2):
        o = gpu.solve_opts(m, rtol=rtol, maxit=5000, mg_levels=3, chunk=chunk, **kw)
        u, info = G.solve(o)
        assert info.status == gpu.OK, (chunk, info.status)
        out.append((np.array(u, copy=True), info.iterations))
        chunk = info.iterations + 3  # one chunk, three iterations past convergence
    (u1, it1), (u2, it2) = out
    assert it1 == it2, (it1, it2)
    assert np.array_equal(u1, u2)
