"""Profiling drivers: run exactly one piece of work between cudaProfilerStart
and cudaProfilerStop, so that an external profiler started with
`--profile-from-start off` (ncu) captures that piece and nothing of the
set-up.

    python -m icarat2_b200.profile_cases solve 128x64x64 mg 4 1e-8
        one K u = f solve of the cantilever (densities U[0.1, 0.5], seed 0),
        after a warm-up solve and a design change (so the per-design
        multigrid set-up is inside the captured region);
        methods: jacobi, mg, mixed; an optional 6th argument "galerkin"
        selects Galerkin coarse operators
    python -m icarat2_b200.profile_cases operator 256x128x128 2 3
        `reps` launches of K u with operator 0 FP64, 1 FP32, 2 tensor cores
        BF16x3, 3 tensor cores BF16, 4 FP64 tensor cores (after one warm-up
        launch)
    python -m icarat2_b200.profile_cases headline 5
        one design iteration of the bench's headline loop (128x64x64,
        uniform start density 0.3, filter radius 2.5, MMA move 0.2, 4-level
        MG-PCG to 1e-8 with the coarse factor reused and the solve started
        from the previous design's solution) after `warm` warm-up iterations
    python -m icarat2_b200.profile_cases net 256x128x128
        one inference of the U-net (random weights, seed 1) on the load of
        the cantilever, after one warm-up inference
    python -m icarat2_b200.profile_cases loop 256x128x128 mixed 6 1e-6 3
        one design iteration of the MMA loop (densities U[0.1, 0.5], seed 0,
        filter radius 3, move 0.2) after `warm` warm-up iterations; methods
        mg, mixed (warm-started), jacobi
    python -m icarat2_b200.profile_cases ocloop 128x64x64 1.5 5
        one design iteration of the OC loop of opt_macro_oc.cpp (uniform
        start 0.3, radius filter R, move 0.15, 4-level MG-PCG to 1e-8 with
        the coarse factor reused and warm starts) after `warm` warm-up
        iterations: filter, sensitivity and the OC bisection kernel
    python -m icarat2_b200.profile_cases batch 8 64x32x32 1e-6
        one batched multigrid-PCG solve (the persistent launch, 4 levels) of
        `n` cantilevers of the grid (densities U[0.1, 0.6], seed 3) after
        two warm-up solves
    python -m icarat2_b200.profile_cases helm 256x128x128 2.0
        one Helmholtz PDE filter call (design U[0, 1], seed 0, CG to 1e-10)
        after one warm-up call
"""
import ctypes as C
import sys

import numpy as np

import icarat2_b200 as gpu


def _profiler():
    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            return C.CDLL(name)
        except OSError:
            continue
    raise OSError("libcudart not found")


def _grid(s):
    return tuple(int(v) for v in s.split("x"))


def solve(grid, method, levels, rtol, coarse="rediscretised"):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz)
    rho = np.random.default_rng(0).uniform(0.1, 0.5, G.nelx)
    G.set_design(rho)
    m = {"jacobi": gpu.JACOBI_PCG, "mg": gpu.MG_PCG, "mixed": gpu.MIXED_IR}[method]
    cop = gpu.COARSE_GALERKIN if coarse == "galerkin" else gpu.COARSE_REDISCRETISED
    o = gpu.solve_opts(m, rtol=float(rtol), mg_levels=int(levels), coarse_op=cop)
    G.solve(o, want_val=False)
    G.set_design(rho * 1.01)
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    _, info = G.solve(o, want_val=False)
    rt.cudaProfilerStop()
    print("iterations %d rel_residual %.3g status %d" % (info.iterations, info.rel_residual,
                                                         info.status))


def operator(grid, op, reps):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz)
    G.set_design(np.random.default_rng(1).uniform(0.1, 0.5, G.nelx))
    rt = _profiler()
    rt.cudaProfilerStart()
    ms = G.time_operator(int(reps), int(op))
    rt.cudaProfilerStop()
    print("ms per launch %.4f" % ms)


def loop(grid, method, levels, rtol, warm):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz)
    rho = np.random.default_rng(0).uniform(0.1, 0.5, G.nelx)
    m = {"jacobi": gpu.JACOBI_PCG, "mg": gpu.MG_PCG, "mixed": gpu.MIXED_IR}[method]
    o = gpu.solve_opts(m, rtol=float(rtol), mg_levels=int(levels),
                       warm_start=1 if method == "mixed" else 0)
    G.loop_init(rho, method="mma", filter_radius=3.0, move=0.2, solve=o)
    for _ in range(int(warm)):
        G.loop_step()
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    info = G.loop_step()
    G.synchronize()
    rt.cudaProfilerStop()
    print("cg iterations %d compliance %.6g status %d" % (info.cg_iterations, info.compliance,
                                                         info.status))


def headline(warm):
    G = gpu.Context(128, 64, 64)
    o = gpu.solve_opts(gpu.MG_PCG, rtol=1e-8, mg_levels=4, coarse_lag=1, warm_start=1)
    G.loop_init(0.3, method="mma", filter_radius=2.5, move=0.2, solve=o)
    for _ in range(int(warm)):
        G.loop_step()
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    info = G.loop_step()
    G.synchronize()
    rt.cudaProfilerStop()
    print("cg iterations %d compliance %.6g status %d" % (info.cg_iterations, info.compliance,
                                                         info.status))


def ocloop(grid, radius, warm):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz)
    o = gpu.solve_opts(gpu.MG_PCG, rtol=1e-8, mg_levels=4, coarse_lag=1, warm_start=1)
    G.loop_init(0.3, method="oc", filter_radius=float(radius), move=0.15, solve=o)
    for _ in range(int(warm)):
        G.loop_step()
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    info = G.loop_step()
    G.synchronize()
    rt.cudaProfilerStop()
    print("cg iterations %d compliance %.6g oc steps %d status %d" % (
        info.cg_iterations, info.compliance, info.update_steps, info.status))


def net(grid):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz)
    G.set_design(np.full(G.nelx, 0.5))
    N = gpu.Net(seed=1)
    f = G.fext()
    N.infer(G, f)
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    u = N.infer(G, f)
    G.synchronize()
    rt.cudaProfilerStop()
    print("|u| %.6g" % float(np.linalg.norm(u)))


def helm(grid, radius):
    nx, ny, nz = _grid(grid)
    G = gpu.Context(nx, ny, nz, dirichlet=[], loads=[])
    G.helmholtz_setup(float(radius))
    x = np.random.default_rng(0).uniform(0.0, 1.0, G.nelx)
    G.helmholtz_filter(x)
    G.synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    out, info = G.helmholtz_filter(x)
    G.synchronize()
    rt.cudaProfilerStop()
    print("cg iterations %d rel_residual %.3g sum %.12g" % (info.iterations,
                                                           info.rel_residual, out.sum()))


def batch(n, grid, rtol):
    nx, ny, nz = _grid(grid)
    bc = gpu.cantilever_bc(nx, ny, nz)
    B = gpu.Batch([(nx, ny, nz) + tuple(bc)] * int(n))
    rng = np.random.default_rng(3)
    for i in range(int(n)):
        B[i].set_design(rng.uniform(0.1, 0.6, B[i].nelx))
    o = B.opts(rtol=float(rtol), method=gpu.MG_PCG, mg_levels=4)
    for _ in range(2):
        B.solve(o)
    B[0].synchronize()
    rt = _profiler()
    rt.cudaProfilerStart()
    inf = B.solve(o)
    rt.cudaProfilerStop()
    print("iterations %d status %s" % (max(x.iterations for x in inf),
                                       sorted({x.status for x in inf})))


def main(argv):
    if len(argv) >= 5 and argv[0] == "solve":
        solve(*argv[1:6])
    elif len(argv) >= 4 and argv[0] == "batch":
        batch(*argv[1:4])
    elif len(argv) >= 6 and argv[0] == "loop":
        loop(*argv[1:6])
    elif len(argv) >= 4 and argv[0] == "ocloop":
        ocloop(*argv[1:4])
    elif len(argv) >= 2 and argv[0] == "headline":
        headline(argv[1])
    elif len(argv) >= 3 and argv[0] == "helm":
        helm(argv[1], argv[2])
    elif len(argv) >= 2 and argv[0] == "net":
        net(argv[1])
    elif len(argv) >= 4 and argv[0] == "operator":
        operator(*argv[1:4])
    else:
        sys.stderr.write(__doc__)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
