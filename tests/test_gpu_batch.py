"""Batched solver (one persistent launch over many designs of uneven size,
or every design's own mixed-precision multigrid solve, interleaved).

Every member is checked against the library's FP64 multigrid-PCG solve of the
same design on its own context (rtol 1e-12): displacements <= 1e-6 relative
(the tolerance stated for the FP32-operator paths), and the reported FP64
residual recomputed through the FP64 operator.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(16, 8, 8), (24, 12, 12), (8, 4, 4), (32, 16, 16), (16, 8, 8)]


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def problems(gpu, sizes, seed):
    rng = np.random.default_rng(seed)
    out = []
    for nx, ny, nz in sizes:
        node = (nx, int(rng.integers(0, ny + 1)), int(rng.integers(0, nz + 1)))
        out.append((nx, ny, nz) + gpu.cantilever_bc(nx, ny, nz, load_node=node))
    return out


def reference(gpu, pr, rho, levels):
    nx, ny, nz, d, lo = pr
    G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
    G.set_design(rho)
    u, _ = G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=levels))
    return u


def test_batch_matches_individual_solves(gpu):
    prs = problems(gpu, SIZES, 1)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(2)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    infos = B.solve(B.opts(rtol=1e-9))
    for i, pr in enumerate(prs):
        assert infos[i].status == gpu.OK and infos[i].rel_residual < 1e-9
        assert infos[i].refreshes >= 1
        u = B.solution(i)
        assert rel(u, reference(gpu, pr, rhos[i], 2)) <= 1e-6
        f = B[i].fext()
        assert np.linalg.norm(f - B[i].apply_K(u)) < 1.001e-9 * np.linalg.norm(f)


def test_batch_reuse_with_new_designs_and_compliance(gpu):
    prs = problems(gpu, [(16, 8, 8), (32, 16, 16)], 3)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(4)
    for rep in range(3):
        rhos = [rng.uniform(0.05, 1.0, B[i].nelx) for i in range(len(B))]
        for i, r in enumerate(rhos):
            B[i].set_design(r)
        infos = B.solve(B.opts(rtol=1e-10))
        for i, pr in enumerate(prs):
            assert infos[i].status == gpu.OK
            nx, ny, nz, d, lo = pr
            G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
            G.set_design(rhos[i])
            G.solve(gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2), want_val=False)
            assert abs(B[i].compliance() - G.compliance()) <= 1e-8 * G.compliance()


def test_batch_iteration_cap(gpu):
    B = gpu.Batch(problems(gpu, [(16, 8, 8), (8, 4, 4)], 5))
    for i in range(len(B)):
        B[i].set_design(np.full(B[i].nelx, 0.4))
    infos = B.solve(B.opts(rtol=1e-14, maxit=5))
    for inf in infos:
        assert inf.status == gpu.WARN_MAXITER and inf.iterations == 5


def test_batch_member_without_load(gpu):
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, 8), (0, 8)))]
    prs = [(16, 8, 8, d, []), (16, 8, 8) + gpu.cantilever_bc(16, 8, 8)]
    B = gpu.Batch(prs)
    for i in range(2):
        B[i].set_design(np.full(B[i].nelx, 0.5))
    infos = B.solve(B.opts(rtol=1e-8))
    assert infos[0].status == gpu.OK and infos[0].iterations == 0
    assert not B.solution(0).any()
    assert infos[1].status == gpu.OK and infos[1].iterations > 0


def test_batch_autotune(gpu):
    prs = problems(gpu, SIZES, 6)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(7)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    tile, bpsm, ms = B.autotune()
    assert tile in (128, 256, 512, 1024) and bpsm >= 1 and ms > 0
    infos = B.solve(B.opts(rtol=1e-9))
    for i, pr in enumerate(prs):
        assert infos[i].status == gpu.OK
        assert rel(B.solution(i), reference(gpu, pr, rhos[i], 2)) <= 1e-6


@pytest.mark.parametrize("tile,bpsm", [(32, 1), (128, 2), (1024, 0)])
def test_batch_explicit_shapes(gpu, tile, bpsm):
    prs = problems(gpu, [(24, 12, 12), (8, 4, 4)], 8)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(9)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    infos = B.solve(B.opts(rtol=1e-9, tile=tile, blocks_per_sm=bpsm))
    for i, pr in enumerate(prs):
        assert infos[i].status == gpu.OK
        assert rel(B.solution(i), reference(gpu, pr, rhos[i], 2)) <= 1e-6


def test_batch_design_loop_tracks_individual_loops(gpu):
    prs = problems(gpu, [(16, 8, 8), (24, 12, 12)], 10)
    B = gpu.Batch(prs)
    solo = []
    for i, (nx, ny, nz, d, lo) in enumerate(prs):
        B[i].loop_init(0.3, method="mma", filter_radius=1.5, move=0.2)
        G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
        G.loop_init(0.3, method="mma", filter_radius=1.5, move=0.2,
                    solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2))
        solo.append(G)
    for _ in range(3):
        infos = B.loop_step(B.opts(rtol=1e-10))
        for i, G in enumerate(solo):
            ref = G.loop_step()
            assert infos[i].status == gpu.OK
            assert abs(infos[i].compliance - ref.compliance) <= 1e-6 * ref.compliance
    for i, G in enumerate(solo):
        assert rel(B[i].loop_get("x"), G.loop_get("x")) <= 1e-6


def test_batch_rejects_mixed_element_sizes(gpu):
    d, lo = gpu.cantilever_bc(8, 4, 4)
    prs = [(8, 4, 4, 8.0, 4.0, 4.0, d, lo), (8, 4, 4, 16.0, 4.0, 4.0, d, lo)]
    with pytest.raises(gpu.IcaratError) as e:
        gpu.Batch(prs)
    assert e.value.status == gpu.ERR_UNSUPPORTED


# ---- interleaved per-design mixed-precision multigrid (method MIXED_IR) ----

def test_batch_concurrent_mg_matches_individual_solves(gpu):
    prs = problems(gpu, SIZES, 11)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(12)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    jac = B.solve(B.opts(rtol=1e-9))
    infos = B.solve(B.opts(rtol=1e-9, method=gpu.MIXED_IR))
    for i, pr in enumerate(prs):
        assert infos[i].status == gpu.OK and infos[i].rel_residual < 1e-9
        assert infos[i].refreshes >= 1
        # multigrid needs far fewer iterations than the Jacobi launch
        assert infos[i].iterations < jac[i].iterations
        u = B.solution(i)
        assert rel(u, reference(gpu, pr, rhos[i], 2)) <= 1e-6
        f = B[i].fext()
        assert np.linalg.norm(f - B[i].apply_K(u)) < 1.001e-9 * np.linalg.norm(f)


def test_batch_concurrent_mg_levels_and_chunk(gpu):
    # 32x16x16 takes 4 levels, 24x12x12 and 8x4x4 only 3
    prs = problems(gpu, [(32, 16, 16), (24, 12, 12), (8, 4, 4)], 13)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(14)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    for chunk in (1, 3):
        infos = B.solve(B.opts(rtol=1e-10, method=gpu.MIXED_IR, mg_levels=4, chunk=chunk))
        for i, pr in enumerate(prs):
            assert infos[i].status == gpu.OK
            assert rel(B.solution(i), reference(gpu, pr, rhos[i], 2)) <= 1e-6


def test_batch_concurrent_warm_start(gpu):
    prs = problems(gpu, [(16, 8, 8), (32, 16, 16)], 15)
    B = gpu.Batch(prs)
    for i in range(len(B)):
        B[i].set_design(np.full(B[i].nelx, 0.4))
    o = B.opts(rtol=1e-9, method=gpu.MIXED_IR, warm_start=True)
    cold = B.solve(o)  # nothing solved yet: starts from 0
    warm = B.solve(o)  # same designs: starts at the solution
    for c, w in zip(cold, warm):
        assert c.status == gpu.OK and c.iterations > 0
        assert w.status == gpu.OK and w.iterations == 0


def test_batch_concurrent_iteration_cap_and_empty_load(gpu):
    d = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, 8), (0, 8)))]
    prs = [(16, 8, 8, d, []), (16, 8, 8) + gpu.cantilever_bc(16, 8, 8)]
    B = gpu.Batch(prs)
    for i in range(2):
        B[i].set_design(np.full(B[i].nelx, 0.5))
    infos = B.solve(B.opts(rtol=1e-14, maxit=3, refresh=1e-6, method=gpu.MIXED_IR))
    assert infos[0].status == gpu.OK and infos[0].iterations == 0
    assert not B.solution(0).any()
    # the mixed solver's cap: the iteration past maxit is the final refresh
    assert infos[1].status == gpu.WARN_MAXITER and infos[1].iterations == 4


def test_batch_concurrent_design_loop_tracks_individual_loops(gpu):
    prs = problems(gpu, [(16, 8, 8), (24, 12, 12), (32, 16, 16)], 16)
    B = gpu.Batch(prs)
    solo = []
    for i, (nx, ny, nz, d, lo) in enumerate(prs):
        B[i].loop_init(0.3, method="mma", filter_radius=1.5, move=0.2)
        G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
        G.loop_init(0.3, method="mma", filter_radius=1.5, move=0.2,
                    solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2))
        solo.append(G)
    o = B.opts(rtol=1e-10, method=gpu.MIXED_IR, warm_start=True)
    for _ in range(3):
        infos = B.loop_step(o)
        for i, G in enumerate(solo):
            ref = G.loop_step()
            assert infos[i].status == gpu.OK
            assert abs(infos[i].compliance - ref.compliance) <= 1e-6 * ref.compliance
    for i, G in enumerate(solo):
        assert rel(B[i].loop_get("x"), G.loop_get("x")) <= 1e-6


def test_batch_rejects_unknown_method(gpu):
    B = gpu.Batch(problems(gpu, [(8, 4, 4)], 17))
    B[0].set_design(np.full(B[0].nelx, 0.5))
    for o in (B.opts(method=7), B.opts(method=gpu.MIXED_IR, mg_levels=1),
              B.opts(method=gpu.MIXED_IR, chunk=-1)):
        with pytest.raises(gpu.IcaratError) as e:
            B.solve(o)
        assert e.value.status == gpu.ERR_ARG


def test_batch_design_loop_with_helmholtz_filter(gpu):
    """members looping with the Helmholtz filter (opt_mma_Helmholtz.cpp) in
    the interleaved batch mode track standalone loops to 1e-6"""
    prs = problems(gpu, [(16, 8, 8), (24, 12, 12)], 18)
    B = gpu.Batch(prs)
    solo = []
    for i, (nx, ny, nz, d, lo) in enumerate(prs):
        B[i].loop_init(0.3, method="mma", filter_radius=2.0, move=0.2, use_threshold=True,
                       filter="helmholtz")
        G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
        G.loop_init(0.3, method="mma", filter_radius=2.0, move=0.2, use_threshold=True,
                    solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2),
                    filter="helmholtz")
        solo.append(G)
    o = B.opts(rtol=1e-10, method=gpu.MIXED_IR, warm_start=True)
    for _ in range(3):
        infos = B.loop_step(o)
        for i, G in enumerate(solo):
            ref = G.loop_step()
            assert infos[i].status == gpu.OK
            assert abs(infos[i].compliance - ref.compliance) <= 1e-6 * ref.compliance
    for i, G in enumerate(solo):
        assert rel(B[i].loop_get("x"), G.loop_get("x")) <= 1e-6


# ---- one persistent multigrid-PCG launch over all designs (method MG_PCG) ----

MG_SIZES = [(16, 8, 8), (24, 12, 12), (32, 16, 16), (8, 8, 8), (16, 8, 8), (40, 16, 8)]


def test_batch_persistent_mg_matches_individual_solves(gpu):
    """uneven grids, one launch: every design meets rtol in FP64 and matches
    its own FP64 MG-PCG solve to 1e-6; far fewer iterations than the
    persistent Jacobi launch"""
    prs = problems(gpu, MG_SIZES, 21)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(22)
    rhos = [rng.uniform(0.05, 1.0, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    infos = B.solve(B.opts(rtol=1e-9, method=gpu.MG_PCG, mg_levels=4))
    jac = B.solve(B.opts(rtol=1e-9))
    for i, pr in enumerate(prs):
        assert infos[i].status == gpu.OK and infos[i].rel_residual < 1e-9, (i, infos[i].status)
        assert infos[i].iterations * 3 < jac[i].iterations
    infos = B.solve(B.opts(rtol=1e-9, method=gpu.MG_PCG, mg_levels=4))
    for i, pr in enumerate(prs):
        u = B.solution(i)
        assert rel(u, reference(gpu, pr, rhos[i], 2)) <= 1e-6
        f = B[i].fext()
        assert np.linalg.norm(f - B[i].apply_K(u)) < 1.001e-9 * np.linalg.norm(f)


def test_batch_persistent_mg_warm_start_cap_and_autotune(gpu):
    prs = problems(gpu, [(16, 8, 8), (32, 16, 16), (8, 4, 4)], 23)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(24)
    rhos = [rng.uniform(0.1, 0.9, B[i].nelx) for i in range(len(B))]
    for i, r in enumerate(rhos):
        B[i].set_design(r)
    tile, bpsm, ms = B.autotune_mg(3)
    assert tile in (128, 256, 512, 1024) and bpsm >= 1 and ms > 0
    cold = B.solve(B.opts(rtol=1e-10, method=gpu.MG_PCG, mg_levels=3))
    for i, r in enumerate(rhos):
        B[i].set_design(np.clip(r * 1.02, 0.0, 1.0))
    warm = B.solve(B.opts(rtol=1e-10, method=gpu.MG_PCG, mg_levels=3, warm_start=True))
    for i, pr in enumerate(prs):
        assert cold[i].status == gpu.OK and warm[i].status == gpu.OK
        assert warm[i].iterations <= cold[i].iterations
        ref = reference(gpu, pr, np.clip(rhos[i] * 1.02, 0.0, 1.0), 2)
        assert rel(B.solution(i), ref) <= 1e-6
    capped = B.solve(B.opts(rtol=1e-14, maxit=2, method=gpu.MG_PCG, mg_levels=3))
    assert all(c.status == gpu.WARN_MAXITER and c.iterations == 2 for c in capped)


def test_batch_persistent_mg_design_loop_tracks_individual_loops(gpu):
    prs = problems(gpu, [(16, 8, 8), (24, 12, 12)], 25)
    B = gpu.Batch(prs)
    solo = []
    for i, (nx, ny, nz, d, lo) in enumerate(prs):
        B[i].loop_init(0.3, method="mma", filter_radius=1.5, move=0.2)
        G = gpu.Context(nx, ny, nz, dirichlet=d, loads=lo)
        G.loop_init(0.3, method="mma", filter_radius=1.5, move=0.2,
                    solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=2))
        solo.append(G)
    o = B.opts(rtol=1e-10, method=gpu.MG_PCG, mg_levels=3, warm_start=True)
    for _ in range(4):
        infos = B.loop_step(o)
        for i, G in enumerate(solo):
            ref = G.loop_step()
            assert infos[i].status == gpu.OK
            assert abs(infos[i].compliance - ref.compliance) <= 1e-6 * ref.compliance
    for i, G in enumerate(solo):
        assert rel(B[i].loop_get("x"), G.loop_get("x")) <= 1e-6


@pytest.mark.parametrize("method", ["MG_PCG", "MIXED_IR"])
def test_batch_floating_islands_finish_in_fp64(gpu, method):
    """A design of solid streaks floating in a 1e-9 void beside an ordinary
    one: a design whose FP32 iteration stalls is finished by FP64 MG-PCG, so
    every design of the batch meets rtol.  Checked again with the context's
    FP64 K u, whose rounding, with island displacements of 1e6, is itself
    about 1e-8 of ||f||: to 10 rtol."""
    prs = problems(gpu, [(32, 16, 16), (32, 16, 16)], 41)
    B = gpu.Batch(prs)
    rng = np.random.default_rng(5)
    x = np.convolve(rng.standard_normal(B[0].nelx), np.ones(9) / 9.0, mode="same")
    B[0].set_design(np.where(x >= np.quantile(x, 0.65), 1.0, 1e-3))
    B[1].set_design(rng.uniform(0.1, 0.6, B[1].nelx))
    infos = B.solve(B.opts(rtol=1e-8, method=getattr(gpu, method), mg_levels=3))
    for i in range(2):
        assert infos[i].status == gpu.OK, (i, infos[i].status, infos[i].rel_residual)
        u, f = B.solution(i), B[i].fext()
        assert np.linalg.norm(f - B[i].apply_K(u)) < 1e-7 * np.linalg.norm(f)
