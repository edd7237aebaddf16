#!/usr/bin/env python
"""SIMP design iterations per second on one B200 (per GPU replica).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one full SIMP design iteration on the 2 mm arm grid (110 x 14 x 12
voxels, 64 935 DOF): density filter, four load cases solved as one block
(FP64 PCG preconditioned by an FP32 multigrid V-cycle, relative residual
1e-8), six lowest modes (FP64 LOBPCG with the FP32 multigrid preconditioner,
eigenvalues converged to ~1e-10), MAC tracking, eigenvalue and compliance
sensitivities, the augmented-Lagrangian frequency penalty and the OC update.
The static and the modal solve of an iteration are issued concurrently on two
streams (tof_b200.topopt.SIMPOptimizer, concurrent=True); --sequential-solves
issues them from one thread (same work; for profilers).
Inputs are synthetic (seeded) with the shapes of the reference's arm; see
tof_b200/workloads.py.  With N GPUs every rank runs an independent replica
(the path does not shard); value = N * K / max-rank time.

Also reported: the same iteration in the plain FP64 form (Jacobi PCG per load
case, Jacobi LOBPCG: the reference's algorithms), seconds per PCG / LOBPCG
solve in both forms on the hollow-box arm with their errors against the
reference's FP64 results (tests/golden/arm.npz), the dominant kernel's
roofline, and the reference algorithm timed on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "to-f450-arm_b200"))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "SIMP iter/s"
WORKLOAD = ("arm 110x14x12 @2mm, one SIMP design iteration: 4 load cases (block PCG, rel. residual 1e-8) "
            "+ 6 modes (LOBPCG, eigenvalues to ~1e-10) + adjoint sensitivities + filter r=1.5 + OC, vf 0.08")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="own", choices=["own", "reference"])
    ap.add_argument("--ref-budget-s", type=float, default=600.0,
                    help="wall-clock budget of the --impl reference run (steps after it are not started)")
    ap.add_argument("--no-extras", action="store_true", help="skip FP64/solver/CPU comparisons")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer and kernel-roofline runs "
                    "(profiling runs)")
    ap.add_argument("--sequential-solves", action="store_true",
                    help="issue the static and the modal solve of an iteration one after the other from one "
                         "thread instead of concurrently (profiling runs; same work)")
    return ap.parse_args()


# --------------------------------------------------------------------------- #
def reference_arm(a, rank, world):
    """The reference's algorithm on the host cores (the oracle's restatement
    of src/topopt.py:267-411 with the reference's own SciPy solver calls,
    oracle/cpu_bench.py), on the same workload as the device arm: every step
    is one complete design iteration, the W warm-up steps are design
    iterations 1..W, so the timed steps are the same design iterations the
    device arm times.  A wall-clock budget (--ref-budget-s) bounds the run:
    steps that would start after it are not run, and the line reports the
    steps actually timed."""
    if rank != 0:
        return
    from oracle.cpu_bench import ReferenceSIMPRun, arm_workload
    from tof_b200 import configs as C
    geom, x0, F = arm_workload()
    run = ReferenceSIMPRun(geom, C.PA12.E, C.PA12.nu, C.PA12.rho, F, x0)
    t_start = time.perf_counter()
    warm = [run.step() for _ in range(a.warmup)]
    steps = []
    for _ in range(a.steps):
        last = (steps or warm or [None])[-1]
        est = last["t_s"] if last else 0.0
        if steps and time.perf_counter() - t_start + est > a.ref_budget_s:
            break
        steps.append(run.step())
    run.close()
    total = sum(r["t_s"] for r in steps)
    n = len(steps)
    v = n / total
    stopped = n < a.steps
    sample = (f"complete design iterations {a.warmup + 1}..{a.warmup + n} of the arm workload (same start design, "
              f"4 load cases as Jacobi-CG to 1e-8 with the reference's maxiter 5000 / direct fall-back, 6 modes by "
              f"Jacobi-LOBPCG tol 1e-4 maxiter 500, sensitivities, filter, OC), after {a.warmup} warm-up iterations; "
              f"the 4 static solves and the modal solve run in {run.workers} single-threaded worker processes; "
              f"no extrapolation" + (f"; stopped after {n} of {a.steps} requested steps at the {a.ref_budget_s:.0f} s "
                                     f"budget" if stopped else ""))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s", "n_gpus": a.gpus, "steps": n,
            "warmup": a.warmup, "ms_per_step": total / n * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [110, 14, 12], "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": "iter/s", "cores": run.workers, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "steps_requested": a.steps, "budget_stopped": stopped,
            "step_s": [r["t_s"] for r in steps],
            "history": {"compliance": [r["compliance"] for r in steps], "omega_1_Hz": [r["omega1_Hz"] for r in steps],
                        "cg_iters": [r["cg_iters"] for r in steps], "cg_direct": [r["cg_direct"] for r in steps]}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- #
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons, busy = [], 0.0, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in out.strip().splitlines():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
            if len(parts) > 7:
                try:
                    busy.append(float(parts[7]))
                except ValueError:
                    pass
        if not sm:
            return None
        out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}
        if busy:   # nvidia-smi utilization.gpu: share of time a kernel was running
            out["gpu_busy_mean_pct"] = statistics.mean(busy)
        return out


def l2_flush(buf):
    buf.add_(1.0)


def time_steps(fn, n, flush_buf, torch):
    """Sum of per-step device times (CUDA events on the current stream); the
    L2 flush between steps is outside the timed events."""
    total = 0.0
    per = []
    for _ in range(n):
        l2_flush(flush_buf)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.nvtx.range_push("simp_step")     # lets a profiler select the timed steps
        e0.record()
        fn()
        e1.record()
        torch.cuda.nvtx.range_pop()
        e1.synchronize()
        dt = e0.elapsed_time(e1) / 1e3
        per.append(dt)
        total += dt
    return total, per


def _peak_hbm():
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        return float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_rooflines(ctx, torch, L, reps=100):
    """Live per-launch device time (tof_time_kernel: a CUDA graph of `reps`
    back-to-back launches between CUDA events on the current stream) and the
    HBM roofline fraction of the kernels that dominate a design iteration,
    largest share first: the coarse-level multigrid operator (levels 1 and
    2; 4 vectors as in the static block solve, 8 as in the LOBPCG
    preconditioner), the Rayleigh-Ritz eigensolver, the fine-level FP32
    matrix-free operator (8 and 4 vectors).
    `traffic`: DRAM bytes per launch from the committed ncu capture
    (profiles/roofline_traffic.json), where captured."""
    import ctypes
    lib = ctx.lib
    peak, src = _peak_hbm()
    tpath = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    traffic = json.load(open(tpath)) if os.path.exists(tpath) else {}
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    n_levels = ctx.lib.tof_mg_query(ctx.h, -1, None, None, s)
    cases = [("k_mgs_op level 1, 4 vectors", "k_mgs_op_l1_r4", L.KERNEL_MG_LEVEL_OP, 1, 4, "latency (L2-resident level)"),
             ("k_mgs_op level 1, 8 vectors", "k_mgs_op_l1_r8", L.KERNEL_MG_LEVEL_OP, 1, 8, "latency (L2-resident level)"),
             ("k_mgs_op level 2, 4 vectors", "k_mgs_op_l2_r4", L.KERNEL_MG_LEVEL_OP, 2, 4, "latency (L2-resident level)"),
             ("k_small_eig (Rayleigh-Ritz, one CTA)", "k_small_eig", L.KERNEL_RAYLEIGH_RITZ, 0, 1,
              "latency (one CTA, barrier-separated Jacobi rounds)"),
             ("k_matvec<float,8> fine level", "k_matvec_f32_r8", L.KERNEL_MATVEC_F32, 0, 8, "FP32 issue / L2"),
             ("k_matvec<float,4> fine level", "k_matvec_f32_r4", L.KERNEL_MATVEC_F32, 0, 4, "FP32 issue / L2")]
    out = []
    for name, key, kind, level, R, why in cases:
        if kind == L.KERNEL_MG_LEVEL_OP and level > n_levels - 2:
            continue
        t = L.KernelTiming()
        rc = lib.tof_time_kernel(ctx.h, kind, level, R, reps, ctypes.byref(t), s)
        if rc != 0:
            continue
        us = t.us
        ach = t.bytes / (us * 1e-6) / 1e9 if us > 0 else 0.0
        out.append({"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "traffic": traffic.get(key), "peak_source": src, "launch_us": us,
                    "algorithmic_bytes_per_launch": t.bytes, "flops_per_launch": t.flops,
                    "achieved_tflops": t.flops / (us * 1e-6) / 1e12 if us > 0 else 0.0, "units": int(t.units),
                    "what_bounds_it": why})
    t = L.KernelTiming()
    if lib.tof_time_kernel(ctx.h, L.KERNEL_VCYCLE, 0, 8, 20, ctypes.byref(t), s) == 0 and out:
        out[0]["vcycle_r8_us"] = t.us
    return out


def solver_comparison(torch, L, C):
    """PCG / LOBPCG on the hollow-box arm in both forms, errors vs the
    reference's FP64 results."""
    from tof_b200.workloads import arm_hollow_analysis
    from tof_b200.modal import effective_mass_voxel
    golden = dict(np.load(os.path.join(ROOT, "tests", "golden", "arm.npz")))
    out = {}
    for form in ("mixed", "fp64"):
        geom, fem, rho, F = arm_hollow_analysis(mode=form)
        fem.SOLVE_RTOL = 1e-8
        R = 4 if form == "mixed" else 1
        fem.solve_block(rho, [F] * R, rtol=1e-8)              # warm (graph capture, multigrid setup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        us, st = fem.solve_block(rho, [F] * R, rtol=1e-8)
        torch.cuda.synchronize()
        t_pcg = time.perf_counter() - t0
        c = float(F @ us[0])
        t0 = time.perf_counter()
        freqs, modes, lam = fem.modal_analysis(rho, n_modes=6, tip_mass_kg=C.TIP_MASS_KG, tol=1e-5)
        torch.cuda.synchronize()
        t_lob = time.perf_counter() - t0
        lst = fem.last_stats
        eff = effective_mass_voxel(fem, geom, rho, modes, C.TIP_MASS_KG, direction=2)
        out[form] = {
            "pcg_s": t_pcg, "pcg_rhs": R, "pcg_iters": st[0]["iters"], "pcg_relres": st[0]["relres"],
            "compliance_rel_err": abs(c / float(golden["compliance"]) - 1.0),
            "lobpcg_s": t_lob, "lobpcg_iters": lst["iters"], "lobpcg_max_rel_resid": lst["relres"],
            "freq_rel_err_max": float(np.max(np.abs(freqs / golden["freqs"] - 1.0))),
            "eff_mass_abs_err_max": float(np.max(np.abs(eff - golden["eff"]))),
        }
        fem.device().close()
    return out


def production_domain_extra(torch):
    """The reference's production domain (ArmGeometry3D, 198k free DOF, solid,
    60 g tip mass): seconds per static solve (thrust + motor torque, true
    relative residual 1e-8) in both forms and per 6-mode modal solve
    (relative residual 1e-8) in the mixed form, after a warm-up solve."""
    from tof_b200 import configs as C
    from tof_b200.fem import FEM3D
    from tof_b200.geometry3d import ArmGeometry3D
    g = ArmGeometry3D()
    F = g.load_vector(F=(0.0, 0.0, -15.0), Mz=0.3)
    out = {"grid": [g.nx, g.ny, g.nz]}
    for mode in ("mixed", "fp64"):
        fem = FEM3D(g, C.PA12, mode=mode)
        rho = np.ones(fem.n_active)
        fem.SOLVE_RTOL = 1e-8
        fem.solve(rho, F)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        u = fem.solve(rho, F)
        torch.cuda.synchronize()
        out[f"static_s_{mode}"] = time.perf_counter() - t0
        out[f"compliance_{mode}"] = float(F @ u)
        if mode == "mixed":
            out["free_dofs"] = int(len(fem.free_dofs))
            fem.modal_analysis(rho, n_modes=6, tip_mass_kg=C.TIP_MASS_KG, tol=1e-8)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            freqs, _, _ = fem.modal_analysis(rho, n_modes=6, tip_mass_kg=C.TIP_MASS_KG, tol=1e-8)
            torch.cuda.synchronize()
            out["modal_s_mixed"] = time.perf_counter() - t0
            out["freqs_Hz"] = [float(f) for f in freqs]
        fem.device().close()
    out["timing"] = "wall clock between device synchronisations, one solve each after a warm-up solve"
    return out


def design_sweep_extra(torch, steps=2):
    """The uneven design sweep (five 2 mm arm designs at vf 0.08-0.50 and one
    1 mm design, 4 load cases and 8 modes each): design iterations per second
    with the designs advanced concurrently (one stream and host thread each)
    and one after another, from the same start, after one warm-up iteration."""
    from tof_b200.batch import DesignSweep
    from tof_b200.workloads import sweep_designs
    res = {}
    for mode in ("concurrent", "sequential"):
        designs = sweep_designs()
        sw = DesignSweep(designs)
        sw.step(concurrent=(mode == "concurrent"))
        t = sum(sw.step(concurrent=(mode == "concurrent")) for _ in range(steps))
        res[mode] = len(designs) * steps / t
        if mode == "concurrent":
            res["designs"] = [dict(name=n, grid=[g.nx, g.ny, g.nz], dofs=int(g.n_dofs), tile=list(f.device().tile))
                              for n, g, f, _ in designs]
        for _, _, f, _ in designs:
            f.device().close()
    res.update(unit="design iter/s", steps=steps,
               speedup_concurrent=res["concurrent"] / res["sequential"],
               timing="wall clock between device synchronisations around each sweep iteration")
    return res


def reduce_max(x: float, torch, device) -> float:
    """Max of a per-rank scalar over all ranks (a replica job is as fast as
    its slowest rank); the value itself on a single process."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return x
    if torch.distributed.get_world_size() == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, steps: int, max_total_s: float) -> float:
    """Whole-job throughput of N independent replicas: N * steps / max time."""
    return world * steps / max_total_s


def own_arm(a, rank, world, local_rank):
    import torch
    from tof_b200 import _lib as L
    from tof_b200 import configs as C
    from tof_b200.workloads import arm_simp

    torch.cuda.set_device(local_rank)
    lib = L.load()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    geom, fem, opt = arm_simp(mode="mixed")
    opt.concurrent = not a.sequential_solves
    for _ in range(a.warmup):
        opt.step()
    torch.cuda.synchronize()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2
    flush.zero_()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    n0 = lib.tof_launch_count()
    total, per = time_steps(opt.step, a.steps, flush, torch)
    launches = lib.tof_launch_count() - n0
    torch.cuda.synchronize()
    total = reduce_max(total, torch, "cuda")
    if world > 1:
        torch.distributed.barrier()
    clocks = sampler.stop() if sampler else None
    value = replica_value(world, a.steps, total)
    hist = opt.history

    if a.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
                              "steps": a.steps, "warmup": a.warmup, "ms_per_step": total / a.steps * 1e3,
                              "gpu_launches": int(launches), "profiling_run": True}), flush=True)
        return
    # ---- end to end through the public API with host buffers, over the same
    # design iterations as the device-timed run (reset, same warm-up)
    opt.reset()
    for _ in range(a.warmup):
        opt.step()
    torch.cuda.synchronize()
    n_design = int(opt.design_ids.numel())
    x_host = torch.empty(n_design, dtype=torch.float64, pin_memory=True)
    x_host.copy_(opt.x[opt.design_ids].cpu())
    F_host = torch.from_numpy(np.stack(opt.F_list)).pin_memory()
    out_host = torch.empty(n_design, dtype=torch.float64, pin_memory=True)

    def e2e_step():
        xd = x_host.to("cuda", non_blocking=True)
        opt.x[opt.design_ids] = xd
        opt.b4 = opt.ctx.pack(F_host.to("cuda", non_blocking=True))
        opt.step()
        out_host.copy_(opt.x[opt.design_ids], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        x_host.copy_(out_host)

    n_e2e = a.steps
    e2e_total, _ = time_steps(e2e_step, n_e2e, flush, torch)
    e2e_total = reduce_max(e2e_total, torch, "cuda")
    e2e = {"value": replica_value(world, n_e2e, e2e_total), "unit": "iter/s",
           "h2d_bytes_per_step": int(n_design * 8 + F_host.numel() * 8),
           "d2h_bytes_per_step": int(n_design * 8 + 8 * 4)}

    # ---- roofline of the kernels with the largest shares of a design
    # iteration's device time (profiles/simp_iteration_arm_launches.md):
    # each timed live, with CUDA events around a graph of back-to-back
    # launches on this stream, on the state the timed steps left behind
    roofline_top = kernel_rooflines(opt.ctx, torch, L)
    roofline = dict(roofline_top[0]) if roofline_top else None

    line = {"metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": total / a.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [geom.nx, geom.ny, geom.nz], "dofs": geom.n_dofs,
                       "load_cases": len(opt.F_list), "modes": opt.n_modes_track, "pcg_rtol": 1e-8,
                       "l2": "flushed between timed steps (256 MiB write outside the timed events)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "e2e": e2e, "roofline": roofline, "roofline_top": roofline_top, "gpu_launches": int(launches),
            "step_ms": [p * 1e3 for p in per],
            "history": {"compliance": hist["compliance"][-a.steps:], "omega_1_Hz": hist["omega_1_Hz"][-a.steps:]},
            "convergence": {"design_iterations": [a.warmup + 1, a.warmup + a.steps],
                            "modal_converged": [bool(v) for v in hist["modal_converged"][-a.steps:]],
                            "modal_iters": [int(v) for v in hist["modal_iters"][-a.steps:]],
                            "modal_relres_max": float(max(hist["modal_relres"][-a.steps:])),
                            "modal_tol": opt.modal_tol,
                            "pcg_iters": [int(v) for v in hist["pcg_iters"][-a.steps:]],
                            "pcg_relres_max": float(max(hist["pcg_relres"][-a.steps:]))}}
    if clocks:
        line["clocks"] = clocks

    if rank == 0 and world == 1 and not a.no_extras:
        # each comparison is recorded as {"error": ...} if it fails, so the
        # measured line above is printed whatever happens to them
        def extra(key, fn):
            try:
                fn()
            except Exception as e:                   # noqa: BLE001 (recorded in the line)
                line[key] = {"error": f"{type(e).__name__}: {e}"}

        extra("fp64_plain", lambda: fp64_extra(a, line, flush, per, total, torch))
        extra("solvers_hollow_arm", lambda: line.__setitem__("solvers_hollow_arm", solver_comparison(torch, L, C)))
        extra("design_sweep", lambda: line.__setitem__("design_sweep", design_sweep_extra(torch)))
        extra("production_domain", lambda: line.__setitem__("production_domain", production_domain_extra(torch)))
        extra("cpu_baseline", lambda: cpu_baseline_extra(line))
    if rank == 0:
        print(json.dumps(line), flush=True)


def fp64_extra(a, line, flush, per, total, torch):
    """The plain FP64 form (Jacobi PCG per load case, Jacobi LOBPCG) over the
    SAME design iterations as the mixed value: same start, the same warm-up
    count, then the same number of timed steps."""
    from tof_b200.workloads import arm_simp
    _, fem64, opt64 = arm_simp(mode="fp64", batch_loads=False)
    try:
        for _ in range(a.warmup):
            opt64.step()
        torch.cuda.synchronize()
        t64, per64 = time_steps(opt64.step, a.steps, flush, torch)
        h64 = opt64.history
        it0 = a.warmup + 1
        line["fp64_plain"] = {
            "iter_s": a.steps / t64, "ms_per_step": t64 / a.steps * 1e3, "steps": a.steps, "warmup": a.warmup,
            "design_iterations": [it0, it0 + a.steps - 1], "step_ms": [p * 1e3 for p in per64],
            "modal_converged": [bool(v) for v in h64["modal_converged"][-a.steps:]],
            "modal_iters": [int(v) for v in h64["modal_iters"][-a.steps:]],
            "pcg_iters": [int(v) for v in h64["pcg_iters"][-a.steps:]],
            "pcg_relres_max": float(max(h64["pcg_relres"][-a.steps:])),
            "compliance": h64["compliance"][-a.steps:], "omega_1_Hz": h64["omega_1_Hz"][-a.steps:]}
        line["speedup_mixed_vs_fp64"] = {
            "total": t64 / total, "design_iterations": [it0, it0 + a.steps - 1],
            "per_step": [p64 / pm for p64, pm in zip(per64, per)],
            "min_per_step": min(p64 / pm for p64, pm in zip(per64, per))}
    finally:
        fem64.device().close()


def cpu_baseline_extra(line):
    """The reference algorithm on the host cores: design iteration 1 of the
    same workload, one complete iteration (oracle/cpu_bench.py)."""
    from oracle.cpu_bench import ReferenceSIMPRun, arm_workload
    from tof_b200 import configs as C
    g_c, x0_c, F_c = arm_workload()
    run = ReferenceSIMPRun(g_c, C.PA12.E, C.PA12.nu, C.PA12.rho, F_c, x0_c)
    r = run.step()
    run.close()
    line["cpu_baseline"] = {
        "value": 1.0 / r["t_s"], "unit": "iter/s", "cores": run.workers, "kind": "port",
        "sample": (f"design iteration 1 of the same arm workload, one complete iteration of the reference "
                   f"algorithm in {r['t_s']:.1f} s (4 Jacobi-CG solves to 1e-8, {max(r['cg_iters'])} "
                   f"iterations max, and the 500-iteration Jacobi-LOBPCG, in {run.workers} single-threaded "
                   f"worker processes; no extrapolation)")}


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        backend = "nccl" if a.impl == "own" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    try:
        if a.impl == "reference":
            reference_arm(a, rank, world)
        else:
            own_arm(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
