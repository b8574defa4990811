#!/usr/bin/env python
"""Design iterations per second of the SIMP compliance loop on one B200.

Workload (one "step" = one design iteration): the 3-D cantilever at
128x64x64 hexa8 voxels (524,288 elements, 1,622,400 free DOFs), E0 = 1,
Emin = 1e-9, nu = 0.3, p = 3, uniform start 0.3, radius filter R = 2.5,
MMA update with move 0.2 and the volume constraint of the sample drivers,
FP64 K u inside 4-level geometric-multigrid PCG to relative residual 1e-8.
A step is filter -> solve -> compliance/volume -> sensitivity -> filter^T ->
MMA, exactly the loop body of the reference sample drivers.

  value : device-resident loop (icarat_loop_step), CUDA events on the
          library's stream, L2 flushed between steps (excluded from timing)
  e2e   : the same step through the reference-facing host-pointer calls
          (filter, set_design, solve, sensitivity, filter^T, MMASolver::Update)
          with every host<->device copy inside the timed region, the host
          buffers in pinned memory
  --impl reference : the CPU restatement of the reference path (oracle/,
          Jacobi-PCG as the reference "Eigen_CG" solver) on the host's physical
          cores, full design iterations of the same trajectory window

Multi-GPU (torchrun): every rank optimises its own replica (independent
designs, no data-path collective); value = all ranks' design iterations /
max-over-ranks time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "design-iter/s"
WORKLOAD = "SIMP cantilever 128x64x64 hexa8, MMA move 0.2, R=2.5, FP64 MG-PCG (4 levels) rtol 1e-8"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--grid", default="128x64x64")
    p.add_argument("--radius", type=float, default=2.5)
    p.add_argument("--levels", type=int, default=4)
    p.add_argument("--coarse-lag", type=int, default=1,
                   help="1: reuse the previous design's coarsest factor while this "
                        "design's is computed on a second stream")
    p.add_argument("--smooth", type=int, default=2)
    p.add_argument("--warm-start", type=int, default=1,
                   help="headline FP64 MG-PCG starts from the previous design's solution "
                        "(stop test unchanged: ||r|| < rtol ||b||)")
    p.add_argument("--rtol", type=float, default=1e-8)
    p.add_argument("--cpu-sample", action="store_true",
                   help="internal: time one full CPU design iteration and print it")
    p.add_argument("--ref-budget", type=float, default=120.0,
                   help="reference arm: seconds of timed design iterations at most "
                        "(fewer timed steps than requested when they do not fit)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--alt-levels", type=int, default=5,
                   help="also time the loop with this many multigrid levels (0: skip)")
    p.add_argument("--mixed-grid", default="256x128x128",
                   help="grid of the mixed-precision section ('' skips it)")
    p.add_argument("--mixed-levels", type=int, default=6)
    p.add_argument("--mixed-steps", type=int, default=5)
    p.add_argument("--batch-steps", type=int, default=3,
                   help="design iterations of the 80-design batch section (0: skip)")
    p.add_argument("--batch-rtol", type=float, default=1e-6)
    p.add_argument("--learned-grid", default="96x48x48",
                   help="grid of the learned-preconditioner section ('' skips it)")
    p.add_argument("--learned-train", type=int, default=64,
                   help="training samples generated by the plain solver")
    p.add_argument("--learned-epochs", type=int, default=3)
    p.add_argument("--helm-grid", default="256x128x128",
                   help="Helmholtz PDE filter measurement grid ('' skips it)")
    p.add_argument("--helm-radius", type=float, default=2.0,
                   help="Helmholtz filter radius (element lengths)")
    p.add_argument("--helm-sample", default="128x64x64",
                   help="grid of the oracle's timed Helmholtz call")
    p.add_argument("--multi-load", type=int, default=1,
                   help="measure the 3-case multi-load loop (0 skips it)")
    p.add_argument("--multi-steps", type=int, default=20,
                   help="timed design iterations of each multi-load run (the "
                        "iteration growth along the trajectory is the point)")
    p.add_argument("--cpu-helm", action="store_true",
                   help="(internal) time the oracle's Helmholtz filter and exit")
    p.add_argument("--cpu-config1", action="store_true",
                   help="(internal) time the oracle's 50-iteration OC run of the "
                        "32x16x16 cantilever and exit")
    p.add_argument("--config1", type=int, default=1,
                   help="time the 32x16x16 OC run (50 iterations, rtol 1e-10) on the GPU "
                        "and on the CPU restatement (0 skips it)")
    return p.parse_args()


def grid_of(a):
    nx, ny, nz = (int(v) for v in a.grid.split("x"))
    return nx, ny, nz


def config(a, extra=None):
    nx, ny, nz = grid_of(a)
    c = {"workload": "SIMP cantilever %s hexa8, MMA move 0.2, R=%g, FP64, %s rtol %g" % (
             a.grid, a.radius, "MG-PCG (%d levels)" % a.levels if a.impl == "ours"
             else "Jacobi-PCG", a.rtol),
         "grid": [nx, ny, nz], "elements": nx * ny * nz,
         "free_dofs": 3 * (nx + 1) * (ny + 1) * (nz + 1) - 3 * (ny + 1) * (nz + 1),
         "update": "MMA", "move": 0.2, "filter_radius": a.radius, "volfrac": 0.3,
         "solver": "MG-PCG" if a.impl == "ours" else "Jacobi-PCG (Eigen_CG semantics)",
         "mg_levels": a.levels, "rtol": a.rtol}
    if a.impl == "ours":
        c["coarse_factor"] = ("previous design's, this design's computed on a second stream "
                              "during the solve" if a.coarse_lag else "this design's")
        c["initial_guess"] = ("the previous design's solution (stop test ||r|| < rtol ||b||)"
                              if a.warm_start else "zero")
    if extra:
        c.update(extra)
    return c


# --------------------------------------------------------------------- CPU arm
def host_cpu():
    """(physical cores this process may use, CPU model name) from lscpu."""
    model, pairs = "unknown", set()
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                model = ln.split(":", 1)[1].strip()
        par = subprocess.run(["lscpu", "-p=CPU,CORE,SOCKET"], capture_output=True,
                             text=True).stdout
        allowed = os.sched_getaffinity(0)
        for ln in par.splitlines():
            if ln.startswith("#"):
                continue
            cpu, core, sock = ln.split(",")[:3]
            if int(cpu) in allowed:
                pairs.add((core, sock))
    except (OSError, ValueError):
        pass
    cores = len(pairs) if pairs else (os.cpu_count() or 1)
    return cores, model


def cpu_design_iteration(a, cg_maxit, threads):
    """One first-design iteration of the oracle; returns timings (s) and CG its."""
    from oracle import oracle as O
    O.lib.or_set_threads(threads)
    nx, ny, nz = grid_of(a)
    P = O.Problem(nx, ny, nz)
    F = O.Filter(P, a.radius)
    L = O.Loop(P, F, method="mma", x0=0.3, move=0.2, cg_tol=a.rtol, cg_maxit=cg_maxit)
    t0 = time.perf_counter()
    L.step()
    t = time.perf_counter() - t0
    s = L.scalars()
    return t, s


def reference_arm(a):
    """The CPU restatement of the reference path, timed in full: W warm-up and
    then timed design iterations of one trajectory (the GPU arm's window),
    every solve uncapped to rtol.  The number of timed iterations is cut to
    what fits a wall-clock budget (--ref-budget seconds for the timed part)
    and reported as "steps"."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    cores, model = host_cpu()
    O.lib.or_set_threads(cores)
    nx, ny, nz = grid_of(a)
    t_setup = time.perf_counter()
    P = O.Problem(nx, ny, nz)
    F = O.Filter(P, a.radius)
    L = O.Loop(P, F, method="mma", x0=0.3, move=0.2, cg_tol=a.rtol, cg_maxit=100000)
    t_setup = time.perf_counter() - t_setup
    warm = []
    for _ in range(a.warmup):
        t0 = time.perf_counter()
        L.step()
        warm.append(time.perf_counter() - t0)
    times, iters = [], []
    t_begin = time.perf_counter()
    for k in range(a.steps):
        t0 = time.perf_counter()
        L.step()
        times.append(time.perf_counter() - t0)
        iters.append(L.scalars()["cg_iters"])
        spent = time.perf_counter() - t_begin
        if k + 1 < a.steps and spent + spent / (k + 1) > a.ref_budget:
            break
    ms = 1000.0 * sum(times) / len(times)
    value = 1000.0 / ms
    sample = ("design iterations %d-%d of the workload's trajectory on the CPU "
              "restatement (oracle/, OpenMP, %d threads = physical cores of %s): "
              "filter, CSR assembly, Jacobi-PCG to rtol %g uncapped (reference "
              "Eigen_CG semantics; %s iterations), sensitivity, filter^T, MMA; %d "
              "warm-up iterations first (%.1f s), %d of %d requested timed iterations "
              "within the %g s budget; setup (mesh, CSR pattern, filter lists) %.1f s "
              "not timed" % (a.warmup + 1, a.warmup + len(times), cores, model, a.rtol,
                             "/".join(str(i) for i in iters), a.warmup, sum(warm),
                             len(times), a.steps, a.ref_budget, t_setup))
    line = {"metric": METRIC, "value": value, "unit": "design-iter/s", "impl": "reference",
            "n_gpus": a.gpus, "steps": len(times), "steps_requested": a.steps,
            "warmup": a.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": config(a),
            "host_cpu": {"model": model, "physical_cores": cores},
            "cpu_baseline": {"value": value, "unit": "design-iter/s", "cores": cores,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "design-iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_helm(a):
    """The oracle's Helmholtz filter (assembly, Jacobi-PCG to 1e-10, readout)
    on the sample grid, one call, one thread."""
    from oracle import oracle as O

    nx, ny, nz = (int(v) for v in a.helm_sample.split("x"))
    x = np.random.default_rng(0).uniform(0.0, 1.0, nx * ny * nz)
    t0 = time.perf_counter()
    _, its = O.helmholtz_filter(nx, ny, nz, a.helm_radius, x, tol=1e-10, maxit=10000)
    t = time.perf_counter() - t0
    print(json.dumps({"t": t, "iters": its, "threads": 1, "grid": a.helm_sample}), flush=True)
    return 0


CONFIG1 = dict(grid=(32, 16, 16), radius=1.5, move=0.15, x0=0.3, rtol=1e-10, steps=50)


def cpu_config1(a):
    """The 32x16x16 OC run of opt_macro_oc.cpp (50 iterations, Jacobi-PCG to
    1e-10 as Eigen_CG) on the CPU restatement, physical cores; setup excluded."""
    from oracle import oracle as O
    cores, model = host_cpu()
    O.lib.or_set_threads(cores)
    c = CONFIG1
    P = O.Problem(*c["grid"])
    L = O.Loop(P, O.Filter(P, c["radius"]), method="oc", x0=c["x0"], move=c["move"],
               cg_tol=c["rtol"])
    t0 = time.perf_counter()
    comp = []
    for _ in range(c["steps"]):
        L.step()
        comp.append(L.scalars()["compliance"])
    t = time.perf_counter() - t0
    print(json.dumps({"t": t, "threads": cores, "model": model, "compliance": comp,
                      "x": L.get("x").tolist()}), flush=True)
    return 0


def config1_section(a, G, torch, dev):
    """The reference's own configuration on the GPU: the 32x16x16 OC run of
    opt_macro_oc.cpp (R = 1.5, move 0.15, start 0.3, rtol 1e-10, 50
    iterations) with Jacobi-PCG (the reference's solver) and with MG-PCG,
    CUDA events around all 50 iterations, against the CPU restatement's run of
    the same 50 iterations; the trajectories' largest differences from the
    CPU run are reported beside the rates."""
    c = CONFIG1
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--cpu-config1"],
                       capture_output=True, text=True)
    cpu = json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else None
    out = {"workload": "opt_macro_oc.cpp run: 32x16x16, OC move 0.15, R = 1.5, start 0.3, "
                       "rtol 1e-10, 50 iterations", "steps": c["steps"]}
    for name, meth in (("gpu_jacobi_pcg", G.JACOBI_PCG), ("gpu_mg_pcg", G.MG_PCG)):
        C = G.Context(*c["grid"], device=dev.index)
        C.loop_init(c["x0"], method="oc", filter_radius=c["radius"], move=c["move"],
                    solve=G.solve_opts(meth, c["rtol"], 10000, 4, a.smooth))
        s = torch.cuda.ExternalStream(C.stream_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        comp = [C.loop_step().compliance for _ in range(c["steps"])]
        e1.record(s)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        row = {"value": 1000.0 * c["steps"] / ms, "unit": "design-iter/s",
               "ms_per_step": ms / c["steps"], "compliance_last": comp[-1]}
        if cpu:
            row["max_rel_compliance_diff_vs_cpu"] = max(
                abs(x - y) / y for x, y in zip(comp, cpu["compliance"]))
            row["max_abs_design_diff_vs_cpu"] = float(
                np.abs(C.loop_get("x") - np.array(cpu["x"])).max())
        out[name] = row
        C.close()
    if cpu:
        out["cpu_port"] = {"value": c["steps"] / cpu["t"], "unit": "design-iter/s",
                           "s_total": cpu["t"], "cores": cpu["threads"], "model": cpu["model"],
                           "kind": "port"}
    return out


def cpu_sample(a):
    threads, _ = host_cpu()
    t, s = cpu_design_iteration(a, 100000, threads)
    print(json.dumps({"t": t, "cg_iters": s["cg_iters"], "threads": threads}), flush=True)
    return 0


# --------------------------------------------------------------------- GPU arm
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id):
        self.bus = bus_id  # PCI bus number of this process's GPU (int) or None
        self.rows = []
        self.proc = None

    def _mine(self, field):
        # nvidia-smi pci.bus_id looks like 00000000:1B:00.0
        try:
            return self.bus is not None and int(field.split(":")[1], 16) == int(self.bus)
        except (IndexError, ValueError):
            return False

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        mine = [r for r in rows if self._mine(r[0])]
        rows = mine or rows
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows)}


def fp64_peak_tflops(torch, dev):
    """Measured FP64 dense peak (cuBLAS DGEMM 8192^3, best of 5)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def traffic_from_profiles(grid):
    """dram bytes per launch of the stencil kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_cg_spmv_%s.txt" % grid)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def mixed_section(a, G, torch, dev, flush, world, dist):
    """256x128x128 cantilever, densities U[0.1, 0.5] (seed 0), R = 3, MMA:
    design iterations per second of the mixed-precision loop (FP32 multigrid
    PCG with the tcgen05 BF16 smoother, FP64 residual refresh) against the
    plain FP64 multigrid-PCG loop (FP64 tensor-core operator on the finest
    level) at the same residual, compliance and dc error of one solve
    against an FP64 solve at rtol 1e-12, and K u GDOF/s of every operator
    on the same design."""
    from icarat2_b200.replicas import job_rate
    nx, ny, nz = (int(v) for v in a.mixed_grid.split("x"))
    nelx, nd = nx * ny * nz, 3 * (nx + 1) * (ny + 1) * (nz + 1)
    rho0 = np.random.default_rng(0).uniform(0.1, 0.5, nelx)
    levels = a.mixed_levels
    out = {"grid": [nx, ny, nz], "mg_levels": levels, "filter_radius": 3.0,
           "update": "MMA move 0.2", "rho0": "U[0.1, 0.5] seed 0"}

    def loop_rate(method, rtol, warm=0, lag=0):
        c = G.Context(nx, ny, nz, device=dev.index)
        c.loop_init(rho0, method="mma", filter_radius=3.0, move=0.2,
                    solve=G.solve_opts(method, rtol, 10000, levels, a.smooth,
                                       warm_start=warm, coarse_lag=lag))
        s = torch.cuda.ExternalStream(c.stream_ptr(), device=dev)
        for _ in range(a.warmup):
            c.loop_step()
        torch.cuda.synchronize()
        ms, its = 0.0, []
        for _ in range(a.mixed_steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            its.append(c.loop_step().cg_iterations)
            e1.record(s)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            with torch.cuda.stream(s):
                flush.zero_()
        torch.cuda.synchronize()
        value, ms = job_rate(ms, a.mixed_steps, world, dist, dev)
        c.close()
        return {"value": value, "unit": "design-iter/s", "ms_per_step": ms / a.mixed_steps,
                "cg_iterations_per_step": its}

    for rtol in (1e-6, 1e-8):
        m = loop_rate(G.MIXED_IR, rtol)
        w = loop_rate(G.MIXED_IR, rtol, warm=1)
        p = loop_rate(G.MG_PCG, rtol)
        pw = loop_rate(G.MG_PCG, rtol, warm=1)
        out["rtol_%g" % rtol] = {"mixed": m, "mixed_warm_start": w, "fp64_mg_pcg": p,
                                 "fp64_mg_pcg_warm_start": pw,
                                 "speedup_mixed_vs_fp64": m["value"] / p["value"],
                                 "speedup_mixed_warm_vs_fp64": w["value"] / p["value"],
                                 "speedup_mixed_warm_vs_fp64_warm": w["value"] / pw["value"]}
        if rtol == 1e-6:
            # both solvers with warm starts and the coarsest factor reused
            # from the previous design (computed beside the solve)
            wl = loop_rate(G.MIXED_IR, rtol, warm=1, lag=1)
            pwl = loop_rate(G.MG_PCG, rtol, warm=1, lag=1)
            out["rtol_%g" % rtol].update({
                "mixed_warm_lag": wl, "fp64_mg_pcg_warm_lag": pwl,
                "speedup_mixed_warm_lag_vs_fp64": wl["value"] / p["value"],
                "speedup_mixed_warm_lag_vs_fp64_warm_lag": wl["value"] / pwl["value"]})
    # accuracy of one solve on the first design against FP64 at rtol 1e-12
    c = G.Context(nx, ny, nz, device=dev.index)
    c.filter_setup(3.0)
    c.set_design(c.density_filter(rho0, False))
    c.solve(G.solve_opts(G.MG_PCG, 1e-12, 10000, levels, a.smooth), want_val=False)
    c64 = c.compliance()
    dc64, _ = c.sensitivity(1.0)
    for rtol in (1e-6, 1e-8):
        _, info = c.solve(G.solve_opts(G.MIXED_IR, rtol, 10000, levels, a.smooth),
                          want_val=False)
        dc, _ = c.sensitivity(1.0)
        out["rtol_%g" % rtol]["compliance_rel_err"] = abs(c.compliance() - c64) / abs(c64)
        out["rtol_%g" % rtol]["dc_max_rel_err"] = float(np.abs(dc - dc64).max() /
                                                        np.abs(dc64).max())
        out["rtol_%g" % rtol]["fp64_residual"] = info.rel_residual
    # K u throughput of every operator on this design
    ku = {}
    for name, op in (("fp64", G.OP_FP64), ("tc_fp64", G.OP_TC_FP64), ("fp32", G.OP_FP32),
                     ("tc_bf16x3", G.OP_TC_BF16X3), ("tc_bf16", G.OP_TC_BF16)):
        ms_op = c.time_operator(20, op)
        ku[name] = {"ms": ms_op, "gdof_s": nd / (ms_op * 1e-3) / 1e9}
    out["ku"] = ku
    # the tensor-core kernel against HBM: algorithmic bytes of a K u with
    # FP32 u, y and E
    bytes32 = 8.0 * nd + 4.0 * nelx
    for name in ("tc_bf16x3", "tc_bf16"):
        ms_tc = ku[name]["ms"]
        out["roofline_" + name] = {"bound": "hbm", "achieved": bytes32 / (ms_tc * 1e-3) / 1e9,
                                   "unit": "GB/s", "bytes_per_launch": bytes32}
    # the FP64 tensor-core operator against the measured DGEMM rate
    flops = 1152.0 * nelx
    out["roofline_tc_fp64"] = {"bound": "fp64 tensor", "achieved":
                               flops / (ku["tc_fp64"]["ms"] * 1e-3) / 1e12, "unit": "TFLOP/s",
                               "flops_per_launch": flops}
    c.close()
    return out


def helmholtz_section(a, G, torch, dev, flush, world, dist):
    """Helmholtz PDE filter (densityFilter of FilterHelmholtz) of a U[0, 1]
    design (seed 0) on the helm grid, CG to the reference's 1e-10: device
    call, host-pointer call, the CG iteration's bytes against HBM and the
    oracle's call on a smaller grid."""
    from icarat2_b200.replicas import job_rate

    nx, ny, nz = (int(v) for v in a.helm_grid.split("x"))
    c = G.Context(nx, ny, nz, dirichlet=[], loads=[], device=dev.index)
    c.helmholtz_setup(a.helm_radius)
    nelx, numnp = c.nelx, c.numnp
    x = np.random.default_rng(0).uniform(0.0, 1.0, nelx)
    xd = torch.tensor(x, dtype=torch.float64, device=dev)
    od = torch.empty_like(xd)
    st = torch.cuda.ExternalStream(c.stream_ptr(), device=dev)
    for _ in range(a.warmup):
        c.helmholtz_filter_dev(xd.data_ptr(), od.data_ptr())
    torch.cuda.synchronize()
    l0 = G.kernel_launches()
    ms, its = 0.0, []
    for _ in range(a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its.append(c.helmholtz_filter_dev(xd.data_ptr(), od.data_ptr()).iterations)
        e1.record(st)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        with torch.cuda.stream(st):
            flush.zero_()
        torch.cuda.synchronize()
    launches = G.kernel_launches() - l0
    value, total = job_rate(ms, a.steps, world, dist, dev)
    ms_call = total / a.steps
    it = sum(its) / len(its)
    # per node and CG iteration: K p (read p, write Ap: 16 B), the Jacobi
    # update (read x p r Ap, write x r: 48 B; the diagonal comes from the node
    # class), p = D^-1 r + beta p (read r p, write p: 24 B); per call:
    # right-hand side, CG start and readout
    bytes_call = numnp * (88.0 * it + 8 + 48 + 8) + 16.0 * nelx
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    gbs = bytes_call / (ms_call * 1e-3) / 1e9
    # host-pointer call: pinned input and output, copies inside the events
    xh = torch.empty(nelx, dtype=torch.float64, pin_memory=True).numpy()
    oh = torch.empty(nelx, dtype=torch.float64, pin_memory=True).numpy()
    xh[:] = x
    e_ms = 0.0
    for k in range(a.warmup + a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        c.helmholtz_filter(xh, out=oh)
        e1.record(st)
        e1.synchronize()
        if k >= a.warmup:
            e_ms += e0.elapsed_time(e1)
        with torch.cuda.stream(st):
            flush.zero_()
        torch.cuda.synchronize()
    e2e_v = job_rate(e_ms, a.steps, world, dist, dev)[0]
    ok = bool(np.allclose(oh, od.cpu().numpy(), rtol=0, atol=1e-12))
    c.close()
    # the MMA loop of opt_mma_Helmholtz.cpp (Helmholtz filter R = 2 elements,
    # threshold, move 0.2) on the headline grid and solver
    gx, gy, gz = grid_of(a)
    cl = G.Context(gx, gy, gz, device=dev.index)
    cl.loop_init(0.3, method="mma", filter_radius=2.0, move=0.2, use_threshold=True,
                 solve=G.solve_opts(G.MG_PCG, a.rtol, 10000, a.levels, a.smooth,
                                    coarse_lag=a.coarse_lag, warm_start=a.warm_start),
                 filter="helmholtz")
    sl = torch.cuda.ExternalStream(cl.stream_ptr(), device=dev)
    for _ in range(a.warmup):
        cl.loop_step()
    torch.cuda.synchronize()
    l_ms = 0.0
    for _ in range(a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(sl)
        cl.loop_step()
        e1.record(sl)
        e1.synchronize()
        l_ms += e0.elapsed_time(e1)
        with torch.cuda.stream(sl):
            flush.zero_()
        torch.cuda.synchronize()
    loop_v, loop_total = job_rate(l_ms, a.steps, world, dist, dev)
    cl.close()
    out = {"grid": a.helm_grid, "radius": a.helm_radius, "rtol": 1e-10,
           "value": value, "unit": "filter-calls/s", "ms_per_call": ms_call,
           "cg_iterations": its, "gpu_launches_per_call": launches / a.steps,
           "e2e": {"value": e2e_v, "unit": "filter-calls/s", "h2d_bytes_per_step": 8 * nelx,
                   "d2h_bytes_per_step": 8 * nelx, "host_memory": "pinned",
                   "matches_device_call": ok},
           "roofline": {"bound": "hbm", "kernel": "Jacobi-PCG iteration (k_helm_spmv, "
                        "k_helm_update, k_helm_pupdate) + rhs/readout",
                        "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                        "bytes_per_call": bytes_call},
           "mma_loop": {"grid": a.grid, "value": loop_v, "unit": "design-iter/s",
                        "ms_per_step": loop_total / a.steps,
                        "workload": "opt_mma_Helmholtz loop: Helmholtz filter R = 2, "
                                    "threshold, MMA move 0.2, MG-PCG %g" % a.rtol}}
    if not a.no_cpu_baseline and world == 1:
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--cpu-helm",
                            "--helm-sample", a.helm_sample, "--helm-radius",
                            str(a.helm_radius)], capture_output=True, text=True)
        if r.returncode == 0:
            cl = json.loads(r.stdout.strip().splitlines()[-1])
            sx, sy, sz = (int(v) for v in a.helm_sample.split("x"))
            s_np = (sx + 1) * (sy + 1) * (sz + 1)
            rate = s_np * cl["iters"] / cl["t"]  # node-iterations/s
            out["cpu_baseline"] = {
                "value": rate / (numnp * it), "unit": "filter-calls/s", "cores": 1,
                "kind": "port",
                "sample": "oracle Helmholtz filter (assembly, Jacobi-PCG to 1e-10, readout) "
                          "on %s: %.3f s, %d iterations; scaled to the measured grid by "
                          "node-iterations" % (a.helm_sample, cl["t"], cl["iters"])}
    return out


def multi_load_section(a, G, torch, dev, flush, world, dist, coarse_op=0):
    """The opt_multi_load loop on the headline grid: 3 point-load cases (tip
    down, tip sideways at the top edge, tip up at the far edge), Helmholtz
    filter R = 2, threshold, MMA move 0.2, the headline solver per case
    (coarse_op: its coarse multigrid operators), a.multi_steps timed steps."""
    from icarat2_b200.replicas import job_rate

    nx, ny, nz = grid_of(a)
    dirich = [((1, 1, 1), (0.0, 0.0, 0.0), ((0, 0), (0, ny), (0, nz)))]
    cases = [[((0.0, 0.0, -1.0), ((nx, nx), (ny // 2, ny // 2), (0, 0)))],
             [((0.0, -1.0, 0.0), ((nx, nx), (ny, ny), (nz, nz)))],
             [((0.0, 0.0, 1.0), ((nx, nx), (0, 0), (nz, nz)))]]
    F = []
    for loads in cases:
        c = G.Context(nx, ny, nz, dirichlet=dirich, loads=loads, device=dev.index)
        F.append(c.fext())
        c.close()
    c = G.Context(nx, ny, nz, dirichlet=dirich, loads=cases[0], device=dev.index)
    c.loop_init(0.3, method="mma", filter_radius=2.0, move=0.2, use_threshold=True,
                solve=G.solve_opts(G.MG_PCG, a.rtol, 10000, a.levels, a.smooth,
                                   coarse_lag=a.coarse_lag, warm_start=a.warm_start,
                                   coarse_op=coarse_op),
                filter="helmholtz")
    c.set_load_cases(np.array(F))
    st = torch.cuda.ExternalStream(c.stream_ptr(), device=dev)
    for _ in range(a.warmup):
        c.loop_step()
    torch.cuda.synchronize()
    ms, its = 0.0, []
    for _ in range(a.multi_steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        its.append(c.loop_step().cg_iterations)
        e1.record(st)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        with torch.cuda.stream(st):
            flush.zero_()
        torch.cuda.synchronize()
    v, total = job_rate(ms, a.multi_steps, world, dist, dev)
    c.close()
    return {"grid": a.grid, "load_cases": len(cases), "value": v, "unit": "design-iter/s",
            "ms_per_step": total / a.multi_steps, "steps": a.multi_steps,
            "cg_iterations_per_step": its,
            "coarse_operators": "Galerkin" if coarse_op else "rediscretised",
            "workload": "opt_multi_load loop: 3 load cases, Helmholtz filter R = 2, "
                        "threshold, MMA move 0.2, MG-PCG %g per case" % a.rtol}


def voxel_section(a, G, dev):
    """STL -> voxel design domain: a UV sphere of 2 x 256 x 128 triangles
    voxelised on a 256^3 grid over its bounding box, host arrays in and out
    (one blocking call, wall clock over 5 calls after a warm-up)."""
    nu, nv = 256, 128
    u = np.linspace(0, 2 * np.pi, nu, endpoint=False)
    w = np.linspace(0, np.pi, nv + 1)
    P = np.stack([np.outer(np.sin(w), np.cos(u)), np.outer(np.sin(w), np.sin(u)),
                  np.outer(np.cos(w), np.ones(nu))], -1)  # (nv+1, nu, 3)
    a00, a01 = P[:-1, :], np.roll(P[:-1, :], -1, axis=1)
    a10, a11 = P[1:, :], np.roll(P[1:, :], -1, axis=1)
    tri = np.concatenate([np.concatenate([a00, a10, a11], -1).reshape(-1, 9),
                          np.concatenate([a00, a11, a01], -1).reshape(-1, 9)])
    G.voxelize_stl(tri, 64, device=dev.index)
    ts = []
    for _ in range(5):
        t0 = time.perf_counter()
        mask, dims, lo, pitch = G.voxelize_stl(tri, 256, device=dev.index)
        ts.append(time.perf_counter() - t0)
    return {"triangles": int(tri.shape[0]), "grid": "256^3", "ms_per_call": 1e3 * min(ts),
            "inside_fraction": float(mask.mean()),
            "timing": "host wall clock of the blocking call (triangles in, 16.8 MB mask out)"}


def batch_problems(G, seed=1):
    """64 cantilevers 64x32x32 and 16 of nx in {32, 48, 64, 80, 96} (2:1:1,
    cycled); load node uniform over the right-face nodes, volume fraction
    U[0.2, 0.5] (the uniform start density), filter radius U[1.5, 3.0]."""
    rng = np.random.default_rng(seed)
    sizes = [(64, 32, 32)] * 64 + [(n, n // 2, n // 2) for n in [32, 48, 64, 80, 96] * 4][:16]
    out = []
    for nx, ny, nz in sizes:
        node = (nx, int(rng.integers(0, ny + 1)), int(rng.integers(0, nz + 1)))
        out.append({"grid": (nx, ny, nz), "bc": G.cantilever_bc(nx, ny, nz, load_node=node),
                    "volfrac": float(rng.uniform(0.2, 0.5)),
                    "radius": float(rng.uniform(1.5, 3.0))})
    return out


def batch_section(a, G, torch, dev):
    """Design iterations per second of the batch: one batched solve per step
    as ONE persistent multigrid-PCG launch over all 80 designs (every
    design's own 4-level hierarchy, FP32 V-cycles, FP64 refresh and stop
    test, warm starts, CUDA graph, autotuned shape), and the interleaved
    per-design mixed multigrid mode, against the same designs stepped one by
    one with each context's own FP64 multigrid-PCG (4 levels) at the same
    rtol."""
    probs = batch_problems(G)
    B = G.Batch([p["grid"] + tuple(p["bc"]) for p in probs], device=dev.index)
    rtol = a.batch_rtol
    for i, p in enumerate(probs):
        B[i].loop_init(p["volfrac"], method="mma", filter_radius=p["radius"], move=0.2,
                       solve=G.solve_opts(G.MG_PCG, rtol, 10000, 4, a.smooth))
    opts = B.opts(rtol=rtol, method=G.MG_PCG, mg_levels=4, warm_start=True)
    B.loop_step(opts)  # first step: V0, hierarchies, graph
    tile, bpsm, ms_it = B.autotune_mg(4)
    for _ in range(max(1, a.warmup - 1)):
        B.loop_step(opts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    its = []
    for _ in range(a.batch_steps):
        infos = B.loop_step(opts)
        its.append(int(np.mean([x.cg_iterations for x in infos])))
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    # solve-only: one batched solve of the current designs from zero
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    sinfo = B.solve(B.opts(rtol=rtol, method=G.MG_PCG, mg_levels=4))
    torch.cuda.synchronize()
    t_solve = time.perf_counter() - t1
    # every design's own mixed-precision multigrid-PCG (FP32 operator and
    # V-cycle, FP64 refresh), the designs interleaved on their own streams,
    # each solve warm-started from the design's previous displacement
    copts = B.opts(rtol=rtol, method=G.MIXED_IR, mg_levels=4, warm_start=True)
    B.loop_step(copts)  # graphs of every design
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    cits = []
    for _ in range(a.batch_steps):
        infos = B.loop_step(copts)
        cits.append(int(np.mean([x.cg_iterations for x in infos])))
    torch.cuda.synchronize()
    t_conc = time.perf_counter() - t3
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    csinfo = B.solve(B.opts(rtol=rtol, method=G.MIXED_IR, mg_levels=4))
    torch.cuda.synchronize()
    t_csolve = time.perf_counter() - t4
    # the same designs stepped one at a time with their own FP64 MG-PCG
    for i in range(len(B)):
        B[i].loop_step()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    for _ in range(a.batch_steps):
        for i in range(len(B)):
            B[i].loop_step()
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t2
    n = len(B)
    nodes = sum((p["grid"][0] + 1) * (p["grid"][1] + 1) * (p["grid"][2] + 1) for p in probs)
    out = {"designs": n, "grids": "64 x 64x32x32 + 16 of 32..96 (2:1:1)", "rtol": rtol,
           "update": "MMA move 0.2", "tuned_tile": tile, "tuned_ctas_per_sm": bpsm,
           "tuned_ms_per_iteration": ms_it, "nodes": nodes,
           "batched": {"value": n * a.batch_steps / t_batch, "unit": "design-iter/s",
                       "solver": "one persistent multigrid-PCG launch for all designs "
                                 "(FP32 V-cycles, FP64 refresh), warm starts, CUDA graph",
                       "mean_cg_iterations_per_step": its,
                       "timing": "host wall clock around whole batch steps (synchronised)"},
           "concurrent_mixed_mg": {"value": n * a.batch_steps / t_conc,
                                   "unit": "design-iter/s",
                                   "mean_cg_iterations_per_step": cits,
                                   "solve_only_cold_ms": 1000.0 * t_csolve,
                                   "solve_only_max_iterations":
                                       max(x.iterations for x in csinfo),
                                   "timing": "host wall clock around whole batch steps"},
           "one_by_one_fp64_mg_pcg": {"value": n * a.batch_steps / t_seq,
                                      "unit": "design-iter/s"},
           "batched_solve_only_cold_ms": 1000.0 * t_solve,
           "batched_solve_max_iterations": max(x.iterations for x in sinfo),
           "statuses": sorted({x.status for x in sinfo})}
    out["speedup_batched_vs_one_by_one"] = out["batched"]["value"] / \
        out["one_by_one_fp64_mg_pcg"]["value"]
    out["speedup_concurrent_vs_one_by_one"] = out["concurrent_mixed_mg"]["value"] / \
        out["one_by_one_fp64_mg_pcg"]["value"]
    B.close()
    return out


def smooth_field(rng, nx, ny, nz, passes=3):
    a = rng.standard_normal((nz, ny, nx))
    for _ in range(passes):
        b = np.zeros_like(a)
        for ax in range(3):
            b += np.roll(a, 1, ax) + np.roll(a, -1, ax)
        a = (a + b) / 7.0
    return (a - a.mean()) / a.std()


def learned_samples(G, nx, ny, nz, n, seed, levels):
    """Designs of one family (smooth base density in [0.15, 0.9], 10 %
    smooth perturbations) with a unit load at a random right-face node;
    solutions by the plain FP64 MG-PCG (rtol 1e-10)."""
    base = np.clip(0.5 + 0.25 * smooth_field(np.random.default_rng(30), nx, ny, nz), 0.15, 0.9)
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        node = (nx, int(rng.integers(0, ny + 1)), int(rng.integers(0, nz + 1)))
        d, lo = G.cantilever_bc(nx, ny, nz, load_node=node)
        c = G.Context(nx, ny, nz, dirichlet=d, loads=lo)
        rho = np.clip(base * (1.0 + 0.1 * smooth_field(rng, nx, ny, nz)), 0.1, 1.0).ravel()
        c.set_design(rho)
        u, _ = c.solve(G.solve_opts(G.MG_PCG, 1e-10, 10000, levels, 2))
        out.append((c, rho, c.fext(), u))
    return out


def learned_section(a, G, torch):
    """Learned flexible PCG against the mixed and the FP64 multigrid solvers
    on held-out samples: iterations and wall time to rtol 1e-6 (one solve
    each, synchronised host clock), after training the net on the GPU on a
    bounded sample of the data set."""
    nx, ny, nz = (int(v) for v in a.learned_grid.split("x"))
    levels = 4
    t0 = time.perf_counter()
    train = learned_samples(G, nx, ny, nz, a.learned_train, 21, levels)
    t_data = time.perf_counter() - t0
    net = G.Net(seed=5)
    losses = []
    t1 = time.perf_counter()
    for ep in range(a.learned_epochs):
        losses.append(float(np.mean([net.train_step(c, r, f, u, 2e-3) for c, r, f, u in train])))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    steps = a.learned_epochs * len(train)
    out = {"grid": [nx, ny, nz], "mg_levels": levels, "train_samples": len(train),
           "epochs": a.learned_epochs, "data_generation_s": t_data, "train_s": t_train,
           "train_ms_per_step": 1000.0 * t_train / max(steps, 1), "epoch_losses": losses,
           "loss": "1 - cos^2 (scale-free) + 0.01 (|y|^2 - 1)^2", "held_out": []}
    for c, r, f, u in learned_samples(G, nx, ny, nz, 3, 22, levels):
        c.set_net(net)
        row = {}
        for name, meth in (("learned_fpcg", G.LEARNED_FPCG), ("mixed", G.MIXED_IR),
                           ("fp64_mg_pcg", G.MG_PCG)):
            c.solve(G.solve_opts(meth, 1e-6, 10000, levels, 2), want_val=False)  # warm-up
            torch.cuda.synchronize()
            ts = time.perf_counter()
            _, info = c.solve(G.solve_opts(meth, 1e-6, 10000, levels, 2), want_val=False)
            torch.cuda.synchronize()
            row[name] = {"iterations": info.iterations, "ms": 1000.0 * (time.perf_counter() - ts),
                         "status": info.status}
            if meth == G.LEARNED_FPCG:
                row[name]["net_preconditioned_iterations"] = info.learned_iterations
        out["held_out"].append(row)
    # the same net at the mixed-precision grid: inference time and the solve
    gx, gy, gz = (int(v) for v in a.mixed_grid.split("x")) if a.mixed_grid else (0, 0, 0)
    if gx:
        c = G.Context(gx, gy, gz)
        rho = np.random.default_rng(0).uniform(0.1, 0.5, gx * gy * gz)
        c.set_design(rho)
        f = c.fext()
        # one inference on device vectors, CUDA events on the context's stream
        fd = torch.tensor(f, dtype=torch.float64, device="cuda")
        ud = torch.empty_like(fd)
        s = torch.cuda.ExternalStream(c.stream_ptr())
        net.infer_dev(c, fd.data_ptr(), ud.data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        net.infer_dev(c, fd.data_ptr(), ud.data_ptr())
        e1.record(s)
        e1.synchronize()
        big = {"grid": [gx, gy, gz], "net_inference_ms": e0.elapsed_time(e1),
               "note": "net trained at the smaller grid; inference on device vectors, "
                       "CUDA events (includes one host read of |f|)"}
        c.set_net(net)
        for name, meth in (("learned_fpcg", G.LEARNED_FPCG), ("mixed", G.MIXED_IR),
                           ("fp64_mg_pcg", G.MG_PCG)):
            c.solve(G.solve_opts(meth, 1e-6, 10000, a.mixed_levels, 2), want_val=False)
            torch.cuda.synchronize()
            ts = time.perf_counter()
            _, info = c.solve(G.solve_opts(meth, 1e-6, 10000, a.mixed_levels, 2),
                              want_val=False)
            torch.cuda.synchronize()
            big[name] = {"iterations": info.iterations,
                         "ms": 1000.0 * (time.perf_counter() - ts), "status": info.status}
        out["at_mixed_grid"] = big
        c.close()
    net.close()
    return out


def gpu_arm(a):
    import torch
    import torch.distributed as dist
    import icarat2_b200 as G
    from icarat2_b200.replicas import job_rate

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    cpu_line = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        # separate process: the oracle's OpenMP pool never shares this one
        r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--cpu-sample",
                            "--grid", a.grid, "--radius", str(a.radius), "--rtol",
                            str(a.rtol)], capture_output=True, text=True)
        if r.returncode == 0:
            cpu_line = json.loads(r.stdout.strip().splitlines()[-1])

    nx, ny, nz = grid_of(a)
    opts = G.solve_opts(G.MG_PCG, a.rtol, 10000, a.levels, a.smooth, coarse_lag=a.coarse_lag,
                        warm_start=a.warm_start)

    def make_ctx():
        return G.Context(nx, ny, nz, device=local)

    # ---------------- value: device-resident loop
    ctx = make_ctx()
    ctx.loop_init(0.3, method="mma", filter_radius=a.radius, move=0.2, solve=opts)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB
    for _ in range(a.warmup):
        ctx.loop_step()
    barrier()
    torch.cuda.synchronize()
    bus = getattr(torch.cuda.get_device_properties(dev), "pci_bus_id", None)
    clocks = ClockSampler(bus)
    clocks.start()
    l0 = G.kernel_launches()
    evs, infos = [], []
    for _ in range(a.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        infos.append(ctx.loop_step())
        e1.record(stream)
        evs.append((e0, e1))
        with torch.cuda.stream(stream):
            flush.zero_()
    torch.cuda.synchronize()
    launches = G.kernel_launches() - l0
    barrier()
    clk = clocks.stop()
    ms_steps = [e0.elapsed_time(e1) for e0, e1 in evs]
    value, total_ms = job_rate(sum(ms_steps), a.steps, world, dist, dev)

    def alt_loop(levels, lag, warm=None, coarse_op=0):
        warm = a.warm_start if warm is None else warm
        ca = make_ctx()
        ca.loop_init(0.3, method="mma", filter_radius=a.radius, move=0.2,
                     solve=G.solve_opts(G.MG_PCG, a.rtol, 10000, levels, a.smooth,
                                        coarse_lag=lag, warm_start=warm, coarse_op=coarse_op))
        sa = torch.cuda.ExternalStream(ca.stream_ptr(), device=dev)
        for _ in range(a.warmup):
            ca.loop_step()
        torch.cuda.synchronize()
        alt_ms, its = 0.0, []
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(sa)
            its.append(ca.loop_step().cg_iterations)
            e1.record(sa)
            e1.synchronize()
            alt_ms += e0.elapsed_time(e1)
            with torch.cuda.stream(sa):
                flush.zero_()
        torch.cuda.synchronize()
        v, alt_ms = job_rate(alt_ms, a.steps, world, dist, dev)
        ca.close()
        return {"mg_levels": levels, "coarse_lag": lag, "warm_start": warm,
                "coarse_operators": "Galerkin" if coarse_op else "rediscretised", "value": v,
                "unit": "design-iter/s", "ms_per_step": alt_ms / a.steps,
                "cg_iterations_per_step": its}

    # ---------------- the same loop with the coarsest factor of each design
    # computed before its solve, and with one more multigrid level (coarsest
    # level 8x4x4 instead of 16x8x8: a 600-DOF dense solve instead of 3,888)
    other_coarse = alt_loop(a.levels, 1 - a.coarse_lag) if a.alt_levels else None
    other_warm = alt_loop(a.levels, a.coarse_lag, 1 - a.warm_start) if a.alt_levels else None
    alt = alt_loop(a.alt_levels, a.coarse_lag) if a.alt_levels else None
    alt_gal = alt_loop(a.levels, a.coarse_lag, coarse_op=G.COARSE_GALERKIN) \
        if a.alt_levels else None

    # ---------------- dominant kernel: FP64 stencil K u on the final design
    ms_op = ctx.time_operator(30)
    nelx, nd = nx * ny * nz, 3 * (nx + 1) * (ny + 1) * (nz + 1)
    flops = 1152.0 * nelx
    bytes_alg = 16.0 * nd + 8.0 * nelx
    peak64 = fp64_peak_tflops(torch, dev)
    achieved = flops / (ms_op * 1e-3) / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)

    # ---------------- e2e: host-pointer reference-facing calls
    e2e = None
    if not a.no_e2e:
        c2 = make_ctx()
        c2.filter_setup(a.radius)
        mma = G.MMASolver(nelx, 1, device=local)
        mma.SetMoveLimit(0.2)

        def pinned(n, fill=0.0):
            a = torch.empty(max(n, 1), dtype=torch.float64, pin_memory=True).numpy()[:n]
            a[:] = fill
            return a

        # every host buffer of the step in pinned memory (the inputs' and
        # outputs' copies run at DMA speed), allocated once
        x, xmin, xmax = pinned(nelx, 0.3), pinned(nelx, 1e-4), pinned(nelx, 1.0)
        xfil, val = pinned(nelx), pinned(c2.numeq)
        dfds, dgds, dfds_f, dgds_f = pinned(nelx), pinned(nelx), pinned(nelx), pinned(nelx)
        vol = c2.element_stiffness()[1]
        s2 = torch.cuda.ExternalStream(c2.stream_ptr(), device=dev)
        state = {"V0": None, "h2d": 0, "d2h": 0}

        def host_step(k):
            h2d = d2h = 0
            c2.density_filter(x, False, out=xfil)
            h2d += x.nbytes
            d2h += xfil.nbytes
            c2.set_design(xfil)
            h2d += xfil.nbytes
            c2.solve(opts, out=val)
            d2h += val.nbytes
            comp = c2.compliance()
            d2h += 8
            v = float((xfil * vol).sum())
            if state["V0"] is None:
                state["V0"] = v
                g = 0.0
            else:
                g = v / state["V0"] - 1.0
            c2.sensitivity(1.0 / state["V0"], out=(dfds, dgds))
            d2h += dfds.nbytes + dgds.nbytes
            c2.density_filter(dfds, True, out=dfds_f)
            c2.density_filter(dgds, True, out=dgds_f)
            h2d += 2 * dfds.nbytes
            d2h += 2 * dfds.nbytes
            mma.Update(x, dfds_f, np.array([g]), dgds_f, xmin, xmax)
            h2d += 5 * x.nbytes + 8
            d2h += x.nbytes
            state["h2d"], state["d2h"] = h2d, d2h
            return comp

        for k in range(a.warmup):
            host_step(k)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_ms = 0.0
        for k in range(a.steps):
            e0.record(s2)
            host_step(a.warmup + k)
            e1.record(s2)
            e1.synchronize()
            e_ms += e0.elapsed_time(e1)
            with torch.cuda.stream(s2):
                flush.zero_()
            torch.cuda.synchronize()
        e2e = {"value": job_rate(e_ms, a.steps, world, dist, dev)[0], "unit": "design-iter/s",
               "h2d_bytes_per_step": state["h2d"], "d2h_bytes_per_step": state["d2h"],
               "host_memory": "pinned"}
        del mma
        c2.close()

    mixed = None
    if a.mixed_grid:
        mixed = mixed_section(a, G, torch, dev, flush, world, dist)
    batched = None
    if a.batch_steps > 0:
        batched = batch_section(a, G, torch, dev)
    learned = None
    if a.learned_grid:
        learned = learned_section(a, G, torch)
    helm = None
    if a.helm_grid:
        helm = helmholtz_section(a, G, torch, dev, flush, world, dist)
    multi = multi_gal = None
    if a.multi_load:
        multi = multi_load_section(a, G, torch, dev, flush, world, dist)
        multi_gal = multi_load_section(a, G, torch, dev, flush, world, dist,
                                       coarse_op=G.COARSE_GALERKIN)
    vox = voxel_section(a, G, dev) if a.multi_load else None
    conf1 = config1_section(a, G, torch, dev) if (a.config1 and world == 1) else None

    if rank == 0:
        cg = [i.cg_iterations for i in infos]
        line = {
            "metric": METRIC, "value": value, "unit": "design-iter/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": config(a, {"l2": "256 MiB flush between steps, outside the per-step "
                                       "CUDA events", "parallelism": "replicas" if world > 1
                                 else "single GPU"}),
            "e2e": e2e, "gpu_launches": int(launches),
            "roofline": {"bound": "fp64", "kernel": "FP64 K u stencil (k_apply_K_f64 / "
                         "k_cg_spmv)", "achieved": achieved, "peak": peak64,
                         "unit": "TFLOP/s", "frac": achieved / peak64,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                         "traffic": traffic_from_profiles(a.grid),
                         "flops_per_launch": flops, "ms_per_launch": ms_op,
                         "caches": "cold: each timed launch follows a 256 MiB write "
                                   "that evicts L2"},
            "roofline_hbm": {"achieved": bytes_alg / (ms_op * 1e-3) / 1e9, "peak": hbm_peak,
                             "unit": "GB/s", "frac": bytes_alg / (ms_op * 1e-3) / 1e9 / hbm_peak,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                             "bytes_per_launch": bytes_alg},
            "ku_gdof_s": nd / (ms_op * 1e-3) / 1e9,
            "cg_iterations_per_step": cg,
            "alt_levels": alt,
            "alt_coarse_lag": other_coarse,
            "alt_warm_start": other_warm,
            "alt_galerkin": alt_gal,
            "mixed_256x128x128": mixed,
            "batched_80_designs": batched,
            "learned": learned,
            "helmholtz_filter": helm,
            "multi_load": multi,
            "multi_load_galerkin": multi_gal,
            "voxelize": vox,
            "config1_oc_32x16x16": conf1,
            "compliance_last": infos[-1].compliance,
            "clocks": clk,
        }
        if cpu_line:
            line["cpu_baseline"] = {
                "value": 1.0 / cpu_line["t"], "unit": "design-iter/s",
                "cores": cpu_line["threads"], "kind": "port",
                "sample": "first design iteration of the same workload on the CPU "
                          "restatement (oracle/): filter, CSR assembly, Jacobi-PCG to rtol "
                          "%g (%d iterations, reference Eigen_CG semantics), sensitivity, "
                          "filter^T, MMA" % (a.rtol, cpu_line["cg_iters"])}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    a = parse()
    if a.cpu_sample:
        return cpu_sample(a)
    if a.cpu_helm:
        return cpu_helm(a)
    if a.cpu_config1:
        return cpu_config1(a)
    if a.impl == "reference":
        return reference_arm(a)
    return gpu_arm(a)


if __name__ == "__main__":
    sys.exit(main())
