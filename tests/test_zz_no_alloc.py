"""icarat_solve_noalloc: the solve for callers that cannot allocate device
memory when they call the solver (for example a host application that
reserved the whole GPU for its own memory pool).  Called through the C ABI,
twice in a row on the same buffers, it must reproduce the existing solve
(icarat_solve_rhs, Jacobi-PCG) to 1e-12 relative with the same iteration
count, leave the device's free memory unchanged from its first call on a new
context on, and refuse grids beyond ICARAT_NOALLOC_MAX_DOFS and options it
does not run.  The test allocates its own device buffers (with torch) before
it measures; the entry point allocates none.
Collected last so that a stop-at-first-failure run has run everything else.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_DOFS = 131072  # ICARAT_NOALLOC_MAX_DOFS in include/icarat_gpu.h


def test_noalloc_matches_existing_solve_twice(gpu):
    import torch
    G = gpu.Context(32, 16, 16)
    assert G.neq <= MAX_DOFS
    rng = np.random.default_rng(17)
    G.set_design(rng.uniform(0.05, 1.0, G.nelx))
    f = G.fext() + 0.01 * rng.standard_normal(G.numeq)
    opts = gpu.solve_opts(gpu.JACOBI_PCG, rtol=1e-10, maxit=10000)
    ref, ref_info = G.solve_rhs(f, opts)
    assert ref_info.status == gpu.OK
    d_f = torch.tensor(f, dtype=torch.float64, device="cuda")
    for _ in range(2):
        d_u = torch.full((G.numeq,), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        info = G.solve_noalloc(d_f.data_ptr(), d_u.data_ptr(), opts)
        torch.cuda.synchronize()
        u = d_u.cpu().numpy()
        assert info.status == gpu.OK
        assert info.iterations == ref_info.iterations
        assert np.abs(u - ref).max() <= 1e-12 * np.abs(ref).max()


def test_noalloc_first_call_leaves_free_memory_unchanged(gpu):
    """On a context that has only been created and given a design, the first
    two calls change the device's free memory by nothing (cudaMemGetInfo)."""
    import torch
    G = gpu.Context(24, 12, 12)
    G.set_design(np.full(G.nelx, 0.4))
    d_f = torch.tensor(G.fext(), dtype=torch.float64, device="cuda")
    d_u = torch.zeros(G.numeq, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    infos = [G.solve_noalloc(d_f.data_ptr(), d_u.data_ptr()) for _ in range(2)]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert all(i.status == gpu.OK for i in infos)
    assert free1 == free0, (free0, free1)


def test_noalloc_rejects_grids_beyond_the_buffer(gpu):
    import torch
    G = gpu.Context(48, 32, 32)  # 3 * 49 * 33 * 33 = 160083 DOFs > limit
    assert G.neq > MAX_DOFS
    G.set_design(np.full(G.nelx, 0.3))
    d = torch.zeros(G.numeq, dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.IcaratError) as e:
        G.solve_noalloc(d.data_ptr(), d.data_ptr())
    assert e.value.status == gpu.ERR_ARG
    assert "ICARAT_NOALLOC_MAX_DOFS" in str(e.value)


@pytest.mark.parametrize("kw", [dict(fp64_tc=1), dict(warm_start=1)])
def test_noalloc_rejects_options_it_does_not_run(gpu, kw):
    import torch
    G = gpu.Context(8, 4, 4)
    G.set_design(np.full(G.nelx, 0.3))
    d = torch.zeros(G.numeq, dtype=torch.float64, device="cuda")
    with pytest.raises(gpu.IcaratError) as e:
        G.solve_noalloc(d.data_ptr(), d.data_ptr(), gpu.solve_opts(gpu.JACOBI_PCG, **kw))
    assert e.value.status == gpu.ERR_UNSUPPORTED
