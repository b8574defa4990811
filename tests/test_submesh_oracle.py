"""The CPU restatement of the [mesh] selection path (oracle/submesh.py),
pinned to the C restatement of the box path: with one selection box covering
the whole box it must give the C oracle's DOF map and loads bit for bit, its
K u to 1e-15, its sensitivities to 1e-13 and its OC / MMA design loops to
1e-12; on an L-bracket it keeps the node and element counts of the union of
two boxes, and a box that cuts elements is refused like modifyMesh's "error
in mesh_icarat"."""
import numpy as np
import pytest


def lbracket(n=12, t=4, nz=4):
    boxes = [((0, n), (0, t), (0, nz)), ((0, t), (0, n), (0, nz))]
    dirichlet = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, t), (n, n), (0, nz)))]
    loads = [((0.0, -1.0, 0.0), ((n, n), (t / 2, t / 2), (nz / 2, nz / 2)))]
    return boxes, dirichlet, loads


def test_full_box_selection_is_the_box_path(oracle):
    from oracle import submesh as S
    nx, ny, nz = 6, 3, 4
    d, l = oracle.cantilever_bc(nx, ny, nz)
    P = oracle.Problem(nx, ny, nz)
    Q = S.SelProblem(nx, ny, nz, [((0, nx), (0, ny), (0, nz))], d, l)
    assert np.array_equal(Q.dof, P.dof().reshape(-1, 3)) and Q.numeq == P.numeq
    assert np.array_equal(Q.fext, P.fext())
    rng = np.random.default_rng(0)
    rho = rng.uniform(0.1, 1.0, P.nelx)
    P.assemble(rho)
    u = rng.standard_normal(P.numeq)
    y = P.apply_K(u)
    assert np.abs(Q.K(rho) @ u - y).max() <= 1e-15 * np.abs(y).max()
    val, _, _ = P.solve(rho, tol=1e-14)
    a = P.sensitivity(rho, P.node_values(val))
    b = Q.sensitivity(rho, Q.node_values(val))
    assert np.abs(a[0] - b[0]).max() <= 1e-13 * np.abs(a[0]).max()
    assert np.array_equal(a[1], b[1])
    for method, move in (("mma", 0.2), ("oc", 0.15)):
        L = oracle.Loop(P, oracle.Filter(P, 1.5), method=method, x0=0.3, move=move,
                        cg_tol=1e-14)
        M = S.SelLoop(Q, 1.5, method=method)
        for _ in range(3):
            L.step()
            M.step()
            c = L.scalars()["compliance"]
            assert abs(c - M.compliance) <= 1e-12 * c
        assert np.abs(L.get("x") - M.x).max() <= 1e-12


def test_lbracket_counts_and_numbering():
    from oracle import submesh as S
    boxes, d, l = lbracket()
    Q = S.SelProblem(12, 12, 4, boxes, d, l)
    assert Q.nelx == 12 * 4 * 4 * 2 - 4 * 4 * 4
    assert Q.numnp == 13 * 5 * 5 * 2 - 5 * 5 * 5
    assert np.all(np.diff(Q.node_ids) > 0) and np.all(np.diff(Q.elem_ids) > 0)
    # the clamped face: 5 x 5 nodes, all three components constrained
    assert Q.numeq == 3 * (Q.numnp - 25)
    assert Q.fext.sum() == -1.0


def test_cutting_box_is_refused():
    from oracle import submesh as S
    with pytest.raises(ValueError):
        S.SelProblem(6, 3, 3, [((0, 2.5), (0, 3), (0, 3))], [], [])
