"""The CPU checker of the Galerkin coarse operators (oracle/galerkin.py):
its fine operator is the oracle's CSR stiffness, its coarse operators are
symmetric, annihilate the rigid translations on an unconstrained box (the
trilinear prolongation reproduces constants), and constrain the components
the coincident fine nodes constrain."""
import numpy as np

from oracle import galerkin as GL
from oracle import oracle as O


def test_full_operator_is_the_csr_stiffness():
    P = O.Problem(4, 2, 2)
    rng = np.random.default_rng(3)
    rho = rng.uniform(0.05, 1.0, P.nelx)
    P.assemble(rho)
    A, fixed = GL.full_operator(P)
    dof = P.dof()
    u = rng.standard_normal(P.numeq)
    x = np.zeros(3 * P.numnp)
    free = dof < P.numeq
    nodes, comps = np.nonzero(free)
    x[comps * P.numnp + nodes] = u[dof[nodes, comps]]
    y = A @ x
    ref = P.apply_K(u)
    got = y[comps * P.numnp + nodes][np.argsort(dof[nodes, comps])]
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
    assert np.all(fixed == ~free)


def test_coarse_operators_symmetric_and_translation_free():
    P = O.Problem(8, 4, 4, dirichlet=[], loads=[])
    rng = np.random.default_rng(5)
    P.assemble(rng.uniform(0.05, 1.0, P.nelx))
    H = GL.hierarchy(P, 3)
    for l, (A, fixed) in enumerate(H):
        assert not fixed.any()
        d = abs(A - A.T).max()
        assert d <= 1e-14 * abs(A).max()
        n = A.shape[0] // 3
        for c in range(3):
            t = np.zeros(3 * n)
            t[c * n:(c + 1) * n] = 1.0
            assert np.abs(A @ t).max() <= 1e-12 * abs(A).max()


def test_coarse_constraints_follow_the_coincident_node():
    P = O.Problem(8, 4, 4)  # cantilever: x = 0 face fixed
    P.assemble(np.full(P.nelx, 0.5))
    H = GL.hierarchy(P, 3)
    for l, (A, fixed) in enumerate(H):
        NX = 8 // 2 ** l + 1
        i = np.arange(fixed.shape[0]) % NX
        assert np.all(fixed[i == 0]) and not fixed[i > 0].any()
        rows = np.flatnonzero(fixed.T.ravel())
        assert abs(A[rows]).max() == 0.0
