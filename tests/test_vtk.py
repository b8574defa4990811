"""The VTK writer of the library on host arrays (icarat_write_vtk_arrays, no
GPU work) against the reference's format restated in the oracle
(oracle.vtk_ascii, after src/io/export_vtk.hpp), and the oracle's Mises
restatement against a closed form.  ASCII: byte for byte; BINARY: the same
sections, big-endian float32 / int32 values equal to the inputs rounded to
float32."""
import numpy as np


def parse_binary(data, nx, ny, nz):
    numnp, nelx = (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
    out = {}
    p = 0

    def line():
        nonlocal p
        q = data.index(b"\n", p)
        s = data[p:q].decode()
        p = q + 1
        return s

    assert [line() for _ in range(4)] == ["# vtk DataFile Version 4.1", "vtk output", "BINARY",
                                          "DATASET UNSTRUCTURED_GRID"]
    assert line() == "" and line() == "POINTS\t%d\tfloat" % numnp
    out["points"] = np.frombuffer(data[p:p + 12 * numnp], ">f4").reshape(-1, 3)
    p += 12 * numnp
    assert line() == "" and line() == "" and line() == "CELLS %d\t%d" % (nelx, 9 * nelx)
    out["cells"] = np.frombuffer(data[p:p + 36 * nelx], ">i4").reshape(-1, 9)
    p += 36 * nelx
    assert line() == "" and line() == "" and line() == "CELL_TYPES\t%d" % nelx
    out["types"] = np.frombuffer(data[p:p + 4 * nelx], ">i4")
    p += 4 * nelx
    assert line() == "" and line() == "" and line() == "POINT_DATA\t%d" % numnp
    assert line() == "VECTORS displacement float"
    out["disp"] = np.frombuffer(data[p:p + 12 * numnp], ">f4").reshape(-1, 3)
    p += 12 * numnp
    assert line() == "" and line() == "" and line() == "CELL_DATA\t%d" % nelx
    for name in ("density", "mises"):
        assert line() == "SCALARS %s float" % name and line() == "LOOKUP_TABLE default"
        out[name] = np.frombuffer(data[p:p + 4 * nelx], ">f4")
        p += 4 * nelx
        assert line() == ""
    assert p == len(data)
    return out


def test_vtk_ascii_bytes_and_binary(oracle, gpu, tmp_path):
    nx, ny, nz = 4, 3, 2
    numnp, nelx = (nx + 1) * (ny + 1) * (nz + 1), nx * ny * nz
    rng = np.random.default_rng(4)
    nv = rng.standard_normal((numnp, 3)) * 10.0 ** rng.integers(-8, 3, (numnp, 3))
    nv[0] = 0.0
    nv[1, 1] = -0.0
    dens, mis = rng.random(nelx), rng.random(nelx) * 1e4
    for box in (None, (7.5, 3.0, 0.4)):
        lx, ly, lz = box if box else (None, None, None)
        a = tmp_path / "a.vtk"
        gpu.write_vtk_arrays(str(a), nx, ny, nz, nv, dens, mis, lx=lx, ly=ly, lz=lz)
        assert a.read_bytes() == oracle.vtk_ascii(nx, ny, nz, nv, dens, mis, lx=lx, ly=ly, lz=lz)
    # fields may be left out
    gpu.write_vtk_arrays(str(a), nx, ny, nz, density=dens)
    assert a.read_bytes() == oracle.vtk_ascii(nx, ny, nz, density=dens)
    b = tmp_path / "b.vtk"
    gpu.write_vtk_arrays(str(b), nx, ny, nz, nv, dens, mis, binary=True)
    r = parse_binary(b.read_bytes(), nx, ny, nz)
    xyz = np.stack(np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1),
                               indexing="ij"), -1).transpose(2, 1, 0, 3).reshape(-1, 3)
    assert np.array_equal(r["points"], xyz.astype(np.float32))
    assert np.array_equal(r["cells"][:, 0], np.full(nelx, 8))
    assert r["cells"][0, 1:].tolist() == [0, 1, 6, 5, 20, 21, 26, 25]
    assert np.array_equal(r["types"], np.full(nelx, 12))
    assert np.array_equal(r["disp"], nv.astype(np.float32))
    assert np.array_equal(r["density"], dens.astype(np.float32))
    assert np.array_equal(r["mises"], mis.astype(np.float32))


def test_vtk_writer_errors(gpu, tmp_path):
    import pytest
    with pytest.raises(gpu.IcaratError) as e:
        gpu.write_vtk_arrays(str(tmp_path / "no_dir" / "x.vtk"), 2, 2, 2)
    assert e.value.status == gpu.ERR_ARG
    with pytest.raises(ValueError):
        gpu.write_vtk_arrays(str(tmp_path / "x.vtk"), 2, 2, 2, density=np.zeros(3))


def test_oracle_mises_closed_form(oracle):
    # u = eps x (a uniform strain): sigma = E D eps everywhere
    nx, ny, nz = 3, 2, 2
    P = oracle.Problem(nx, ny, nz)
    eps = np.array([1e-3, -2e-4, 5e-4, 3e-4, -1e-4, 2e-4])  # xx yy zz gxy gyz gzx
    G = np.array([[eps[0], eps[3] / 2, eps[5] / 2], [eps[3] / 2, eps[1], eps[4] / 2],
                  [eps[5] / 2, eps[4] / 2, eps[2]]])
    nv = P.xyz() @ G.T
    rho = np.full(P.nelx, 0.7)
    m = oracle.mises(P, rho, nv)
    nu = P.nu
    E = (1 - 0.7 ** 3) * P.E1 + 0.7 ** 3 * P.E2
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    tr = eps[:3].sum()
    s = np.array([lam * tr + 2 * mu * eps[0], lam * tr + 2 * mu * eps[1],
                  lam * tr + 2 * mu * eps[2], mu * eps[3], mu * eps[4], mu * eps[5]])
    ref = np.sqrt(s[0] ** 2 + s[1] ** 2 + s[2] ** 2 - s[0] * s[1] - s[1] * s[2] - s[2] * s[0]
                  + 3 * (s[3] ** 2 + s[4] ** 2 + s[5] ** 2))
    assert np.abs(m - ref).max() <= 1e-12 * ref
