"""[mesh] selection (MeshIcarat::modifyMesh, src/io/mesh_icarat.hpp:636-755)
on the GPU, through the C ABI, against the CPU restatement oracle/submesh.py
on an L-bracket (the shape of sample/algorithm/opt-macro-gcmma/lbracket.toml):

  - sizes, kept ids, DOF map and loads: bit-exact;
  - K u: max |diff| <= 1e-14 max |y|;
  - Jacobi- and MG-PCG to rtol 1e-12 against a direct solve: solution
    <= 1e-8, compliance <= 1e-10 relative;
  - radius filter, both directions: bit-exact (neighbours among the kept
    elements only, in ascending id);
  - sensitivities (same displacements): <= 1e-11 relative (numpy sums
    u_e^T Ke0 u_e in another order than the kernel);
  - OC and MMA design loops over 5 iterations: compliance <= 1e-10,
    design <= 1e-10.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, T, NZ = 12, 4, 4


def lbracket():
    boxes = [((0, N), (0, T), (0, NZ)), ((0, T), (0, N), (0, NZ))]
    dirichlet = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, T), (N, N), (0, NZ)))]
    loads = [((0.0, -1.0, 0.0), ((N, N), (T / 2, T / 2), (NZ / 2, NZ / 2)))]
    return boxes, dirichlet, loads


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def pair(gpu):
    from oracle import submesh as S
    boxes, d, l = lbracket()
    Q = S.SelProblem(N, N, NZ, boxes, d, l)
    G = gpu.Context(N, N, NZ, dirichlet=d, loads=l, selection=boxes)
    return Q, G


def test_mesh_dofs_and_loads_bit_exact(pair):
    Q, G = pair
    assert (G.numnp, G.nelx, G.numeq, G.neq) == (Q.numnp, Q.nelx, Q.numeq, 3 * Q.numnp)
    nodes, elems = G.selection_ids()
    assert np.array_equal(nodes, Q.node_ids) and np.array_equal(elems, Q.elem_ids)
    assert np.array_equal(G.dof_map(), Q.dof)
    assert np.array_equal(G.fext(), Q.fext)


def test_stiffness_and_solves(pair, gpu):
    Q, G = pair
    rng = np.random.default_rng(5)
    rho = rng.uniform(0.05, 1.0, Q.nelx)
    G.set_design(rho)
    u = rng.standard_normal(Q.numeq)
    y = Q.K(rho) @ u
    assert rel(G.apply_K(u), y) <= 1e-14
    ref = Q.solve(rho)
    cref = Q.compliance(ref)
    for m, lev in ((gpu.JACOBI_PCG, 1), (gpu.MG_PCG, 3)):
        val, info = G.solve(gpu.solve_opts(m, rtol=1e-12, mg_levels=lev))
        assert info.status == gpu.OK
        assert rel(val, ref) <= 1e-8
        assert abs(G.compliance() - cref) <= 1e-10 * cref
    nv = G.node_values()
    assert np.allclose(nv, Q.node_values(val), rtol=1e-8, atol=1e-14 * np.abs(nv).max())
    dfds, dgds = G.sensitivity(0.5)
    rd, rg = Q.sensitivity(rho, nv, 0.5)
    assert rel(dfds, rd) <= 1e-11
    assert np.array_equal(dgds, rg)


@pytest.mark.parametrize("R", [1.5, 2.5])
def test_filter_bit_exact(pair, oracle, R):
    Q, G = pair
    F = oracle.Filter(centroids=Q.centroids, radius=R)
    G.filter_setup(R)
    x = np.random.default_rng(int(R * 10)).uniform(0.0, 1.0, Q.nelx)
    assert np.array_equal(G.density_filter(x), F.density_filter(x))
    g = np.random.default_rng(3).standard_normal(Q.nelx)
    assert np.array_equal(G.density_filter(g, is_sens=True), F.density_filter(g, True))


@pytest.mark.parametrize("method", ["oc", "mma"])
def test_design_loop(gpu, method):
    from oracle import submesh as S
    boxes, d, l = lbracket()
    Q = S.SelProblem(N, N, NZ, boxes, d, l)
    G = gpu.Context(N, N, NZ, dirichlet=d, loads=l, selection=boxes)
    move = 0.2 if method == "mma" else 0.15
    L = S.SelLoop(Q, 1.5, method=method, move=move)
    G.loop_init(0.3, method=method, filter_radius=1.5, move=move,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3))
    for _ in range(5):
        L.step()
        info = G.loop_step()
        assert info.status == gpu.OK
        assert abs(info.compliance - L.compliance) <= 1e-10 * L.compliance
        assert abs(info.constraint - L.constraint) <= 1e-10 * max(1.0, abs(L.constraint))
    assert rel(G.loop_get("x"), L.x) <= 1e-10
    assert rel(G.loop_get("dfds"), L.dfds) <= 1e-9


def test_refusals(gpu):
    # a box that cuts elements: a kept element would lose a node
    with pytest.raises(gpu.IcaratError) as e:
        gpu.Context(6, 3, 3, selection=[((0, 2.5), (0, 3), (0, 3))])
    assert e.value.status == gpu.ERR_ARG and "mesh_icarat" in str(e.value)
    boxes, d, l = lbracket()
    G = gpu.Context(N, N, NZ, dirichlet=d, loads=l, selection=boxes)
    with pytest.raises(gpu.IcaratError) as e:
        G.helmholtz_setup(1.5)
    assert e.value.status == gpu.ERR_UNSUPPORTED


def test_box_context_ids_are_identity(gpu):
    G = gpu.Context(4, 2, 2)
    nodes, elems = G.selection_ids()
    assert np.array_equal(nodes, np.arange(G.numnp)) and np.array_equal(elems, np.arange(G.nelx))
