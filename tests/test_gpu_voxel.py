"""GPU voxeliser (icarat_voxelize) against the oracle's restatement, mask for
mask, on shapes with one to four crossings per column and with vertices and
edges on column centres; the STL path of scripts/stl_to_vtk_voxel.py end to
end; a voxelised design domain driving the loop's non-design IDs."""
import numpy as np
import pytest

import voxel_shapes as S

pytestmark = pytest.mark.gpu

SHAPES = [
    ("box", lambda: S.box((2.3, 1.7, 0.6), (9.4, 8.2, 7.1)), (12, 10, 9), (0, 0, 0), (1, 1, 1)),
    ("sphere", lambda: S.icosphere((6.1, 4.9, 4.3), 3.7, 3), (12, 10, 9), (0, 0, 0), (1, 1, 1)),
    ("torus", lambda: S.torus((0, 0, 0), 3.5, 1.4, 96, 48), (24, 24, 8), (-6, -6, -2),
     (0.5, 0.5, 0.5)),
    ("octahedron", lambda: S.octahedron((4.5, 4.5, 4.5), 3.0), (9, 9, 9), (0, 0, 0),
     (1, 1, 1)),
    ("fine sphere", lambda: S.icosphere((0.1, -0.2, 0.05), 1.0, 5), (64, 48, 40),
     (-1.1, -1.3, -1.0), (2.2 / 64, 2.2 / 48, 2.1 / 40)),
]


@pytest.mark.parametrize("name,make,dims,org,pit", SHAPES, ids=[s[0] for s in SHAPES])
def test_voxelize_matches_oracle(oracle, gpu, name, make, dims, org, pit):
    tri = make()
    m = gpu.voxelize(tri, dims, np.array(org, float), np.array(pit, float))
    ref = oracle.voxelize(tri, dims, org, pit)
    assert np.array_equal(m, ref)
    assert 0 < m.sum() < m.size


def test_voxelize_stl_file_and_domain(gpu, tmp_path):
    tri = S.torus((0, 0, 0), 3.0, 1.2, 64, 32)
    S.write_stl_binary(tmp_path / "t.stl", tri)
    for cubic in (False, True):
        mask, dims, lo, pitch = gpu.voxelize_stl(str(tmp_path / "t.stl"), 32, cubic=cubic)
        assert dims == (32, 32, 32) and mask.size == 32 ** 3
        assert (np.allclose(pitch, pitch[0]) if cubic else np.allclose(pitch[:2], 8.4 / 32))
        assert 0 < mask.sum() < mask.size
    # the voxelised shape as the design domain of a short loop: outside
    # voxels are non-design and keep zero sensitivities
    mask, dims, lo, pitch = gpu.voxelize_stl(str(tmp_path / "t.stl"), 16)
    G = gpu.Context(16, 16, 16, lx=16 * pitch[0], ly=16 * pitch[1], lz=16 * pitch[2])
    d, nd = gpu.design_nondesign_ids(G.nelx, np.nonzero(mask == 0)[0])
    G.loop_init(np.where(mask == 1, 0.5, 1e-4), method="mma", filter_radius=1.5 * pitch[0])
    G.loop_set_domains(d, nd)
    for _ in range(2):
        info = G.loop_step()
        assert info.status in (0, 1)
    assert not G.loop_get("dfds")[nd].any()


def test_voxelize_errors(gpu):
    with pytest.raises(gpu.IcaratError) as e:
        gpu.voxelize(np.full((1, 9), np.nan), (2, 2, 2), np.zeros(3), np.ones(3))
    assert e.value.status == gpu.ERR_ARG
    with pytest.raises(gpu.IcaratError) as e:
        gpu.voxelize(S.box((0, 0, 0), (1, 1, 1)), (2, 2, 2), np.zeros(3), np.zeros(3))
    assert e.value.status == gpu.ERR_ARG
