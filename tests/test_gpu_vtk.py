"""Element von Mises stress and VTK output of a solved context (through the
C ABI) against the oracle: Mises (Elastic::makeMisesStress restated in the
oracle) to 1e-8 relative with both solves at rtol 1e-12; the file written
from the context equals the reference's format (oracle.vtk_ascii) filled
with the context's own node values, design and Mises, byte for byte."""
import numpy as np
import pytest

from test_vtk import parse_binary

pytestmark = pytest.mark.gpu


def test_mises_matches_oracle(oracle, gpu):
    nx, ny, nz = 12, 6, 6
    P, G = oracle.Problem(nx, ny, nz), gpu.Context(nx, ny, nz)
    rho = np.random.default_rng(8).uniform(0.05, 1.0, P.nelx)
    val, _, _ = P.solve(rho, tol=1e-12)
    ref = oracle.mises(P, rho, P.node_values(val))
    G.set_design(rho)
    G.solve(gpu.solve_opts(gpu.JACOBI_PCG, 1e-12, 20000), want_val=False)
    m = G.mises()
    assert np.abs(m - ref).max() <= 1e-8 * np.abs(ref).max()


def test_write_vtk_from_context(oracle, gpu, tmp_path):
    nx, ny, nz = 6, 3, 3
    G = gpu.Context(nx, ny, nz)
    with pytest.raises(gpu.IcaratError) as e:
        G.write_vtk(str(tmp_path / "x.vtk"))
    assert e.value.status == gpu.ERR_STATE
    rho = np.random.default_rng(2).uniform(0.1, 1.0, G.nelx)
    G.set_design(rho)
    G.solve(gpu.solve_opts(gpu.JACOBI_PCG, 1e-10, 5000), want_val=False)
    nv, m = G.node_values(), G.mises()
    a = tmp_path / "a.vtk"
    G.write_vtk(str(a))
    assert a.read_bytes() == oracle.vtk_ascii(nx, ny, nz, nv, rho, m)
    b = tmp_path / "b.vtk"
    G.write_vtk(str(b), binary=True)
    r = parse_binary(b.read_bytes(), nx, ny, nz)
    assert np.array_equal(r["disp"], nv.reshape(-1, 3).astype(np.float32))
    assert np.array_equal(r["density"], rho.astype(np.float32))
    assert np.array_equal(r["mises"], m.astype(np.float32))
