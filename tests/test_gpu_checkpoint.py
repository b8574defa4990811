"""Checkpoint / resume of the device loop (icarat_loop_save / icarat_loop_load):
a run interrupted after 3 design iterations and resumed on a new context
repeats the uninterrupted run's later iterations exactly (compliance,
constraint, design, convergence test), for OC and for MMA with warm-started
solves; snapshots of another mesh and files that are not snapshots are
refused with ICARAT_ERR_ARG."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = (16, 8, 8)


def make(gpu, method):
    G = gpu.Context(*GRID)
    G.loop_init(0.3, method=method, filter_radius=1.5, move=0.2 if method == "mma" else 0.15,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3, warm_start=1))
    return G


@pytest.mark.parametrize("method", ["oc", "mma"])
def test_resumed_run_repeats_the_uninterrupted_one(gpu, tmp_path, method):
    A = make(gpu, method)
    full = []
    for _ in range(6):
        info = A.loop_step()
        full.append((info.compliance, info.constraint, A.loop_is_convergence(1e-2, 4)))
    B = make(gpu, method)
    for _ in range(3):
        B.loop_step()
        B.loop_is_convergence(1e-2, 4)
    path = str(tmp_path / "loop.snap")
    B.loop_save(path)
    B.close()
    R = gpu.Context(*GRID)
    R.loop_load(path)
    for k in range(3, 6):
        info = R.loop_step()
        assert info.step == k + 1
        assert (info.compliance, info.constraint) == full[k][:2]
        assert R.loop_is_convergence(1e-2, 4) == full[k][2]
    assert np.array_equal(R.loop_get("x"), A.loop_get("x"))


def test_snapshot_refusals(gpu, tmp_path):
    A = make(gpu, "mma")
    A.loop_step()
    path = str(tmp_path / "a.snap")
    A.loop_save(path)
    other = gpu.Context(8, 4, 4)
    with pytest.raises(gpu.IcaratError) as e:
        other.loop_load(path)
    assert e.value.status == gpu.ERR_ARG
    junk = tmp_path / "junk.snap"
    junk.write_bytes(b"not a snapshot" * 10)
    with pytest.raises(gpu.IcaratError) as e:
        A.loop_load(str(junk))
    assert e.value.status == gpu.ERR_ARG
