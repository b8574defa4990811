"""The oracle's ray-parity voxeliser (restating the library's voxel.cu)
against closed shapes with known insides, and the STL reader.  Voxel
centres closer to a surface than its faceting error are not compared."""
import numpy as np

import voxel_shapes as S


def centres(dims, origin, pitch):
    nx, ny, nz = dims
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([origin[0] + (i.ravel() + 0.5) * pitch[0],
                     origin[1] + (j.ravel() + 0.5) * pitch[1],
                     origin[2] + (k.ravel() + 0.5) * pitch[2]], 1)


def test_box_and_sphere(oracle):
    dims, org, pit = (12, 10, 9), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    P = centres(dims, org, pit)
    m = oracle.voxelize(S.box((2.3, 1.7, 0.6), (9.4, 8.2, 7.1)), dims, org, pit)
    ref = np.all((P > (2.3, 1.7, 0.6)) & (P < (9.4, 8.2, 7.1)), 1)
    assert np.array_equal(m.astype(bool), ref)
    c, R = np.array([6.1, 4.9, 4.3]), 3.7
    m = oracle.voxelize(S.icosphere(c, R, 3), dims, org, pit)
    d = np.linalg.norm(P - c, axis=1)
    sure = np.abs(d - R) > 0.02 * R  # facets of level 3 lie within 1.3 % of R
    assert np.array_equal(m.astype(bool)[sure], (d < R)[sure])
    assert m.sum() > 100


def test_torus_four_crossings(oracle):
    dims, org, pit = (24, 24, 8), (-6.0, -6.0, -2.0), (0.5, 0.5, 0.5)
    P = centres(dims, org, pit)
    R, r = 3.5, 1.4
    m = oracle.voxelize(S.torus((0, 0, 0), R, r, 96, 48), dims, org, pit)
    q = np.sqrt((np.hypot(P[:, 0], P[:, 1]) - R) ** 2 + P[:, 2] ** 2)
    sure = np.abs(q - r) > 0.05
    assert np.array_equal(m.astype(bool)[sure], (q < r)[sure])


def test_shared_edges_and_vertices_on_column_centres(oracle):
    # an octahedron whose vertices and projected edges pass exactly through
    # column centres: each centre inside the projection is counted once on
    # the upper and once on the lower sheet
    dims, org, pit = (9, 9, 9), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0)
    P = centres(dims, org, pit)
    c, r = np.array([4.5, 4.5, 4.5]), 3.0
    m = oracle.voxelize(S.octahedron(c, r), dims, org, pit)
    l1 = np.abs(P - c).sum(1)
    sure = np.abs(l1 - r) > 1e-9
    assert np.array_equal(m.astype(bool)[sure], (l1 < r)[sure])
    # columns through the projected vertices and edges have crossings at
    # distinct heights, so their inside centres are found
    assert m.reshape(9, 9, 9)[4, 4, :].sum() == 5


def test_read_stl_binary_and_ascii(gpu, tmp_path):
    tri = S.icosphere((1.0, 2.0, 3.0), 2.0, 1)
    S.write_stl_binary(tmp_path / "b.stl", tri)
    S.write_stl_ascii(tmp_path / "a.stl", tri)
    assert np.array_equal(gpu.read_stl(str(tmp_path / "b.stl")),
                          tri.astype(np.float32).astype(np.float64))
    assert np.array_equal(gpu.read_stl(str(tmp_path / "a.stl")), tri)
