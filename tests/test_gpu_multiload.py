"""Multi-load loops and design / non-design domains on the GPU against the
oracle's composed loop (oracle.CaseLoop), through the C ABI.

Reference loops: sample/software/opt-multi-load/opt_multi_load.cpp:100-200
(several load cases per design iteration, Helmholtz filter, design IDs) and
sample/algorithm/opt-macro-mma-nondesign/opt_macro_mma_nondesign.cpp:90-178
(non-design boxes, radius filter).

Tolerances: elasticity CG to 1e-12 on both sides; with the radius filter the
compliance and constraint agree to 1e-9 and the designs to 1e-8 over 4 MMA
iterations; with the Helmholtz filter (its CG at the reference's 1e-10 on
both sides) to 1e-7 and 1e-6.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, NY, NZ = 16, 8, 8
DIRICH = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, NY), (0, NZ)))]
CASES = [
    [((0.0, 0.0, -1.0), ((NX, NX), (NY // 2, NY // 2), (0, 0)))],
    [((0.0, -1.0, 0.0), ((NX, NX), (NY, NY), (NZ, NZ)))],
    [((0.0, 0.0, 1.0), ((NX, NX), (0, 0), (NZ, NZ)))],
]


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


def fext_cases(gpu, cases):
    F = []
    for loads in cases:
        c = gpu.Context(NX, NY, NZ, dirichlet=DIRICH, loads=loads)
        F.append(c.fext())
        c.close()
    return np.array(F)


def run_pair(oracle, gpu, cases, filt, R, x0, design_ids, nondesign_ids, steps, tol_c,
             tol_x):
    G = gpu.Context(NX, NY, NZ, dirichlet=DIRICH, loads=cases[0])
    G.loop_init(x0, method="mma", filter_radius=R, move=0.2, use_threshold=True,
                solve=gpu.solve_opts(gpu.MG_PCG, rtol=1e-12, mg_levels=3), filter=filt)
    if len(cases) > 1:
        G.set_load_cases(fext_cases(gpu, cases))
    if design_ids is not None or len(nondesign_ids):
        G.loop_set_domains(design_ids, nondesign_ids)
    Ps = [oracle.Problem(NX, NY, NZ, dirichlet=DIRICH, loads=l) for l in cases]
    if filt == "helmholtz":
        M = oracle.CaseLoop(Ps, None, helmholtz_R=R, x0=x0, design_ids=design_ids,
                            nondesign_ids=nondesign_ids)
    else:
        M = oracle.CaseLoop(Ps, oracle.Filter(Ps[0], R), x0=x0, design_ids=design_ids,
                            nondesign_ids=nondesign_ids)
    for _ in range(steps):
        comp, const, its = M.step()
        info = G.loop_step()
        assert info.status in (0, 1)
        assert abs(info.compliance - comp) <= tol_c * comp
        assert abs(info.constraint - const) <= tol_c * max(1.0, abs(const))
    assert rel(G.loop_get("x"), M.x) <= tol_x
    d = G.loop_get("dfds")
    assert rel(d, M.dfds) <= tol_x
    if len(nondesign_ids):
        assert not d[nondesign_ids].any() and not G.loop_get("dgds")[nondesign_ids].any()
    return G


def test_multi_load_radius(oracle, gpu):
    G = run_pair(oracle, gpu, CASES, "radius", 1.5, 0.3, None, (), 4, 1e-9, 1e-8)
    G.set_load_cases(None)  # back to the context's own load
    G.loop_step()


def test_nondesign_boxes_single_load(oracle, gpu):
    # two boxes as in the sample's toml: solid near the load, void inside;
    # with two boxes every element counts in the volume (the reference's
    # per-box design list), which nondesign_boxes reproduces
    boxes = [(1.0, ((12.0, 16.0), (2.0, 6.0), (0.0, 3.0))),
             (1.0e-4, ((3.0, 6.0), (2.0, 6.0), (2.0, 6.0)))]
    x0, d, nd = gpu.nondesign_boxes(NX, NY, NZ, boxes, 0.35)
    assert len(d) == NX * NY * NZ and len(nd) > 0
    run_pair(oracle, gpu, CASES[:1], "radius", 1.5, x0, d, nd, 4, 1e-9, 1e-8)


def test_multi_load_helmholtz_with_domains(oracle, gpu):
    # opt_multi_load.cpp: Helmholtz filter, non-design IDs from a list
    # (non_design_domain.hpp: design = all minus them)
    nd_ids = np.arange(NX - 2, NX * NY * NZ, NX)  # two columns of elements at the loaded end
    nd_ids = np.unique(np.concatenate([nd_ids, nd_ids + 1]))
    d, nd = gpu.design_nondesign_ids(NX * NY * NZ, nd_ids)
    run_pair(oracle, gpu, CASES, "helmholtz", 2.0, 0.3, d, nd, 3, 1e-7, 1e-6)


def test_cases_and_domains_arguments(gpu):
    G = gpu.Context(NX, NY, NZ, dirichlet=DIRICH, loads=CASES[0])
    with pytest.raises(ValueError):
        G.set_load_cases(np.zeros((2, G.numeq + 1)))
    with pytest.raises(gpu.IcaratError) as e:
        G.loop_set_domains(None, [0])
    assert e.value.status == gpu.ERR_STATE  # before loop_init
    G.loop_init(0.3, method="oc", filter_radius=1.5)
    with pytest.raises(gpu.IcaratError) as e:
        G.loop_set_domains([G.nelx], [])
    assert e.value.status == gpu.ERR_ARG
    G.set_load_cases(fext_cases(gpu, CASES[:2]))
    with pytest.raises(gpu.IcaratError) as e:
        G.loop_step()  # OC takes one load case
    assert e.value.status == gpu.ERR_UNSUPPORTED
    B = gpu.Batch([(NX, NY, NZ, DIRICH, CASES[0])])
    B[0].loop_init(0.3, method="mma", filter_radius=1.5)
    B[0].set_load_cases(fext_cases(gpu, CASES[:2]))
    with pytest.raises(gpu.IcaratError) as e:
        B.loop_step()  # batch members take one load case each
    assert e.value.status == gpu.ERR_UNSUPPORTED
    B.close()
