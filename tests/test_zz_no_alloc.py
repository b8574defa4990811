"""icarat_solve_noalloc: the solve for callers that cannot allocate device
memory when they call the solver (for example a host application that
reserved the whole GPU for its own memory pool).  Called through the C ABI,
twice in a row on the same buffers, it must reproduce the existing solve
(icarat_solve_rhs, Jacobi-PCG) to 1e-12 relative with the same iteration
count, and it must refuse grids beyond ICARAT_NOALLOC_MAX_DOFS.  The test
allocates its own device buffers (with torch); the entry point allocates none.
Collected last so that a stop-at-first-failure run has run everything else.
"""
import ctypes as C

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
