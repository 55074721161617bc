#!/usr/bin/env python
"""Benchmark of the B200 edge-based finite-volume hot path.

Workload (one "step" = one evaluation): the FP64 second-order residual of
AERO-F's SpaceOperator::computeResidual on a 101^3-node jittered Kuhn tet
mesh (N=1,030,301, E=7,090,300, F_b=120,000), LSQ gradients + van Albada
MUSCL + Roe flux, slip walls on y/z, Steger-Warming far field on x, Mach 0.8,
seeded 1% perturbation of the free stream.  Synthetic, seeded inputs stand in
for the reference's sower meshes (no public dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value   = residual evaluations x E / device time (Medges/s), inputs resident
          in HBM, K back-to-back asynchronous calls timed with CUDA events.
e2e     = the same through the public API with pinned host buffers: each
          step copies U host->device, evaluates, copies R device->host.
roofline: the finite-volume-term pass (edge fluxes + assembly), algorithmic
          bytes 32E + 232N + 40F_b per launch, against the measured HBM copy
          bandwidth; roofline_residual: the whole evaluation against
          B_res2 = 40E + 464N + 40F_b.
--impl reference: the CPU oracle (a C++ restatement of the reference's
          loops; the reference itself needs Fortran/MPI and cannot be built)
          timed with all host threads on the same workload.
Multi-GPU (torchrun): independent replicas, one per GPU, weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "residual Medges/s, %HBM peak; mixed vs FP64 Newton time-to-1e-8; adjoint cost"
FALLBACK_HBM_GBS = 6650.0


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        # nvidia-smi can take a second to print its first sample on a fresh
        # box: the timed region starts once sampling runs
        t0 = time.time()
        while not self.lines and self.proc.poll() is None and time.time() - t0 < 5.0:
            time.sleep(0.01)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        # a timed region shorter than the sampling period still gets the
        # sample that follows it
        n0, t0 = len(self.lines), time.time()
        while len(self.lines) == n0 and self.proc.poll() is None and time.time() - t0 < 1.0:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(local: int):
    import torch
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        return None


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def build_workload(n: int):
    from aerof_dev_b200 import workloads as W
    mesh = W.make_lattice_mesh(n, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    U = W.perturbed_state(mesh["X"].shape[0], 0.8)
    return W, mesh, Ub, U


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(mesh, Ub, U, E: int, budget_s: float = 20.0, max_evals: int = 20, o=None,
                 out=None) -> dict:
    """CPU oracle (restatement of the reference's loops), all host threads,
    on a bounded number of full evaluations of the same workload.  The last
    evaluation is left in `out` (the parity check reads it)."""
    from oracle.oracle import Oracle
    o = o or Oracle(mesh)
    cores = os.cpu_count() or 1
    out = np.empty_like(U) if out is None else out
    o.residual_threaded(U, Ub, 2, nthreads=cores, out=out)  # warm-up
    t0 = time.perf_counter()
    k = 0
    while k < max_evals:
        o.residual_threaded(U, Ub, 2, nthreads=cores, out=out)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return {"value": E * k / dt / 1e6, "unit": "Medges/s", "cores": cores, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"{k} full second-order residual evaluations of the 101^3 mesh after 1 warm-up "
                      f"({dt:.1f} s), OpenMP over {cores} threads, g++ -O3 -march=x86-64-v3"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    W, mesh, Ub, U = build_workload(args.n)
    s = W.lattice_sizes(args.n)
    from oracle.oracle import Oracle
    o = Oracle(mesh)
    cores = os.cpu_count() or 1
    out = np.empty_like(U)
    # the requested warm-up evaluations, within a bounded share of the budget
    t0 = time.perf_counter()
    nw = 0
    for _ in range(max(args.warmup, 1)):
        o.residual_threaded(U, Ub, 2, nthreads=cores, out=out)
        nw += 1
        if time.perf_counter() - t0 > 0.25 * args.ref_budget:
            break
    # each step is one full evaluation; the number of timed steps is capped
    # so the run stays within a few minutes
    t0 = time.perf_counter()
    k = 0
    while k < args.steps:
        o.residual_threaded(U, Ub, 2, nthreads=cores, out=out)
        k += 1
        if time.perf_counter() - t0 > args.ref_budget:
            break
    dt = time.perf_counter() - t0
    value = s["E"] * k / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Medges/s", "n_gpus": args.gpus,
        "steps": k, "requested_steps": args.steps, "warmup": nw, "ms_per_step": dt / k * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, s),
        "cpu_baseline": {"value": value, "unit": "Medges/s", "cores": cores, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": f"{k} full evaluations (capped at {args.ref_budget:.0f} s of the "
                                   f"{args.steps} requested), OpenMP over {cores} threads"},
        "e2e": {"value": value, "unit": "Medges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, s) -> dict:
    return {"workload": f"FP64 second-order residual (LSQ + van Albada + Roe), {args.n}^3 jittered Kuhn tet mesh "
                        f"N={s['N']} E={s['E']} F_b={s['F']}, slip walls y/z, far field x, Mach 0.8",
            "mesh_n": args.n, "N": s["N"], "E": s["E"], "F_b": s["F"], "evals_per_step": 1,
            "l2": "working set > 126 MB L2 (node data 0.2 GB + edge data 0.5 GB); no flush",
            "parallelism": f"replicas x{args.gpus}", "kernel": getattr(args, "kernel", "blocked")}


def timed_on(stream, fn, reps: int, warm: int = 3) -> float:
    """Mean device milliseconds of fn() over reps calls, CUDA events on the
    stream the library runs on, after warm calls."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def parity_part(A, ctx, o, U, Rgpu, Rref) -> dict:
    """Relative L2 of the GPU residual (the timed evaluations' output) and of
    the LSQ gradients (aerof_gpu_gradients) against the CPU oracle on the
    benchmark's own state and mesh."""
    def rel(a, b):
        a = np.asarray(a, dtype=np.float64)
        b = np.asarray(b, dtype=np.float64)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))
    V = o.prim(U)
    got = A.SpaceOperator(ctx).computeGradients(V)
    ref = o.gradients(V)
    return {"residual_rel_l2": rel(Rgpu, Rref),
            "gradients_rel_l2": [rel(a, b) for a, b in zip(got, ref)],
            "tolerance": 1e-12,
            "oracle": "C++ restatement of the reference's CPU loops (FP64), same U and mesh"}


def newton_part(A, ctx, U, args, uuid) -> dict:
    """Mixed-precision vs all-FP64 pseudo-transient Newton-GMRES to
    ||R||/||R0|| <= 1e-8 (CFL 10 -> 1e4, RESIDUAL law ser 0.7, GMRES(30)
    eps 1e-2, block-Jacobi) on the benchmark's mesh and state; device time of
    aerof_gpu_newton, clocks sampled during both solves."""
    import torch
    res, states = {}, {}
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.2)
    for name, prec in (("mixed", A.PREC_FP32), ("fp64", A.PREC_FP64)):
        sol = A.ImplicitSteadySolver(ctx, precision=prec, cfl0=10.0, cfl_max=1e4, ser=0.7, ksp_eps=1e-2,
                                     krylov=30, maxits=30, tol=1e-8, max_steps=args.max_steps)
        ctx.timers()
        ctx.profile(True)
        Uo, info = sol.solve(torch.from_numpy(U).cuda())
        tm = ctx.timers()
        ctx.profile(False)
        states[name] = Uo
        res[name] = {"seconds": info["seconds"], "steps": info["steps"], "gmres_its": info["linear_its"],
                     "rel_residual": info["rel_residual"],
                     "timers_s": {k: v[0] / 1e3 for k, v in tm.items() if v[1]}}
    clk = clocks.stop()
    d = (torch.linalg.norm(states["mixed"] - states["fp64"]) / torch.linalg.norm(states["fp64"])).item()
    return {"speedup_mixed_vs_fp64": res["fp64"]["seconds"] / res["mixed"]["seconds"],
            "unit": "x (FP64 time / mixed time to ||R||/||R0|| <= 1e-8)",
            "mixed": res["mixed"], "fp64": res["fp64"], "state_rel_l2_mixed_vs_fp64": d,
            "config": "second-order FP64 residual, first-order H1 Jacobian (FP32 or FP64 blocks), block-Jacobi, "
                      "GMRES(30) eps 1e-2, CFL 10 -> 1e4; timers are disjoint device-time categories",
            "clocks": clk}


def fp64_peak_tflops() -> float:
    """FP64 peak of this GPU as measured here: cuBLAS DGEMM 8192^3 (FP64
    tensor path, the same rate as the FP64 pipes on this part), best of
    three after one warm-up, CUDA events."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def fp64_roofline(flops_per_edge, E: int, ms_edges: float) -> dict | None:
    """The edge-flux kernel against the FP64 roofline: FP64 operations per
    edge (DADD + DMUL + 2 DFMA thread instructions per edge from one ncu
    capture of the kernel) x E / its CUDA-event time per evaluation."""
    if not flops_per_edge or not ms_edges:
        return None
    peak = fp64_peak_tflops()
    ach = flops_per_edge * E / (ms_edges * 1e-3) / 1e12
    return {"bound": "fp64", "kernel": "edge fluxes (k_fv_blocked)", "achieved": ach, "peak": peak,
            "unit": "TFLOP/s", "frac": ach / peak, "flops_per_edge": flops_per_edge, "ms_per_launch": ms_edges,
            "peak_source": "measured: cuBLAS DGEMM 8192^3 in this run"}


def adjoint_cost_part(A, ctx, Ud, stream, uuid) -> dict:
    """Device time of the adjoint products over one primal residual on the
    benchmark's mesh and state: both products of the adjoint gradient from
    one reverse sweep (J^T lambda and dR/dX^T lambda), and J^T w / J p from
    the stored exact linearisation (the operator the adjoint GMRES applies)."""
    import torch
    sp, S = A.SpaceOperator(ctx), A.Sensitivity(ctx)
    lam = torch.from_numpy(np.random.default_rng(3).standard_normal((ctx.N, 5))).cuda()
    R = torch.empty_like(Ud)
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.2)
    t_res = timed_on(stream, lambda: sp.computeResidual(Ud, R), 20)
    t_both = timed_on(stream, lambda: S.adjoint_products(Ud, lam), 10)
    S.h2_evaluate(Ud)
    t_h2t = timed_on(stream, lambda: S.h2_apply(lam, transpose=True), 20)
    t_h2 = timed_on(stream, lambda: S.h2_apply(lam), 20)
    S.h2_release()
    clk = clocks.stop()
    return {"adjoint_products_over_residual": t_both / t_res,
            "stored_JT_over_residual": t_h2t / t_res, "stored_J_over_residual": t_h2 / t_res,
            "ms": {"residual_sync_call": t_res, "adjoint_products": t_both, "stored_JT": t_h2t, "stored_J": t_h2},
            "unit": "x one primal residual (synchronous calls, device time)", "clocks": clk}


def run_ours(args):
    import torch
    import aerof_dev_b200 as A
    from aerof_dev_b200.replicas import aggregate_rate, max_over_ranks
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    W, mesh, Ub, U = build_workload(args.n)
    s = W.lattice_sizes(args.n)
    kern = {"blocked": A.KERNEL_BLOCKED, "edge": A.KERNEL_EDGE}[args.kernel]
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=A.REC_VANALBADA, device=local, residual_kernel=kern)
    assert ctx.E == s["E"]
    # one dedicated stream: the library's kernels and the timing events are
    # ordered on it
    stream = torch.cuda.Stream(device=local)
    ctx.set_stream(stream)
    sp = A.SpaceOperator(ctx)
    Ud = torch.from_numpy(U).cuda()
    Rd = torch.empty_like(Ud)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        sp.computeResidualAsync(Ud, Rd)
    bad = ctx.status()
    ctx.timers()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.3)
    ctx.profile(True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    A.launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        sp.computeResidualAsync(Ud, Rd)
    e1.record(stream)
    launches = A.launch_count()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if pg:
        pg.barrier()
    bad += ctx.status()
    tm = ctx.timers()
    ctx.profile(False)
    clk = clocks.stop()
    ms = max_over_ranks(ms, "cuda")
    value = aggregate_rate(s["E"] * args.steps, world, ms) / 1e6

    # end to end through the public API with pinned host buffers
    Uh = torch.from_numpy(U).pin_memory()
    Rh = torch.empty_like(Uh).pin_memory()
    k2 = max(1, min(args.steps, args.e2e_steps))
    sp.computeResidual(Uh, Rh)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(k2):
        sp.computeResidual(Uh, Rh)
    a1.record(stream)
    torch.cuda.synchronize()
    ms2 = a0.elapsed_time(a1)
    ms2 = max_over_ranks(ms2, "cuda")
    e2e = aggregate_rate(s["E"] * k2, world, ms2) / 1e6

    peaks = measured_peaks()
    # the finite-volume term (edge fluxes, boundary fluxes, node assembly)
    # is timed by several event pairs per evaluation: divide by evaluations
    # the edge fluxes (fv_edges) and the boundary fluxes + node assembly
    # (fv_term) are disjoint timer categories
    edges_ms = tm.get("fv_edges", (0.0, 0))[0]
    fv_ms = tm["fv_term"][0] + edges_ms
    t_fv = fv_ms / args.steps * 1e-3
    B_fv = 32 * s["E"] + 232 * s["N"] + 40 * s["F"]
    ach = B_fv / t_fv / 1e9
    B_res = 40 * s["E"] + 464 * s["N"] + 40 * s["F"]
    t_eval = ms * 1e-3 / args.steps
    traffic, flops_per_edge = None, None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            prof = json.load(f)
        traffic = prof.get("fv_term_bytes_per_launch")
        flops_per_edge = prof.get("flux_kernel_fp64_flops_per_edge")
    line = {
        "metric": METRIC, "value": value, "unit": "Medges/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(args, s),
        "roofline": {"bound": "hbm", "kernel": "finite-volume term (edge fluxes + assembly)",
                     "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                     "traffic": traffic, "algorithmic_bytes": B_fv, "ms_per_launch": t_fv * 1e3,
                     "peak_source": peaks["source"]},
        "roofline_residual": {"bound": "hbm", "achieved": B_res / t_eval / 1e9, "peak": peaks["hbm_gbs"],
                              "unit": "GB/s", "frac": B_res / t_eval / 1e9 / peaks["hbm_gbs"],
                              "algorithmic_bytes": B_res},
        "timers_ms_per_eval": {k: v[0] / args.steps for k, v in tm.items() if v[1]},
        "roofline_fp64": fp64_roofline(flops_per_edge, s["E"], edges_ms / args.steps),
        "e2e": {"value": e2e, "unit": "Medges/s", "h2d_bytes_per_step": U.nbytes, "d2h_bytes_per_step": U.nbytes,
                "steps": k2},
        "gpu_launches": launches,
        "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                   "samples": clk["samples"]},
        "unphysical_states": bad,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import Oracle
        o = Oracle(mesh)
        Rref = np.empty_like(U)
        line["cpu_baseline"] = cpu_baseline(mesh, Ub, U, s["E"], o=o, out=Rref)
        line["parity"] = parity_part(A, ctx, o, U, Rd.cpu().numpy(), Rref)
        del o
    if world == 1 and not args.no_adjoint_cost:
        line["adjoint_cost"] = adjoint_cost_part(A, ctx, Ud, stream, uuid)
    if world == 1 and not args.no_newton:
        # the configuration the Newton metric names (161^3, block-Jacobi)
        # on its own mesh, and the benchmark's 101^3 mesh
        sizes = [int(v) for v in args.newton_meshes.split(",") if v]
        for nm in sizes:
            if nm == args.n:
                part = newton_part(A, ctx, U, args, uuid)
            else:
                t0 = time.perf_counter()
                Wn, mesh_n, Ub_n, U_n = build_workload(nm)
                ctx_n = A.Context.from_mesh(mesh_n, Ub_n, reconstruction=A.REC_VANALBADA, device=local)
                ctx_n.set_stream(stream)
                setup_s = time.perf_counter() - t0
                part = newton_part(A, ctx_n, U_n, args, uuid)
                part["mesh_setup_s"] = setup_s
                ctx_n.close()
            sn = Wn.lattice_sizes(nm) if nm != args.n else s
            part["mesh"] = f"{nm}^3 jittered Kuhn tet mesh N={sn['N']} E={sn['E']}"
            line["newton" if nm == sizes[-1] else f"newton_{nm}"] = part
    ctx.close()
    if pg:
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_newton(args):
    """Mixed-precision vs all-FP64 pseudo-transient Newton-GMRES, relative
    residual 1e-8 (CFL 10 -> 1e4, RESIDUAL law ser 0.7, GMRES(30) eps 1e-2,
    block-Jacobi).  Times are device time of aerof_gpu_newton (CUDA events)."""
    import torch
    import aerof_dev_b200 as A
    torch.cuda.set_device(0)
    clocks = ClockSampler(gpu_uuid(0))
    clocks.start()
    W, mesh, Ub, U = build_workload(args.n)
    s = W.lattice_sizes(args.n)
    t0 = time.perf_counter()
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=A.REC_VANALBADA)
    setup_s = time.perf_counter() - t0
    if args.pc == "ilu":
        ctx.set_preconditioner(A.PC_ILU0)
    res = {}
    states = {}
    for name, prec in (("mixed", A.PREC_FP32), ("fp64", A.PREC_FP64)):
        sol = A.ImplicitSteadySolver(ctx, precision=prec, cfl0=10.0, cfl_max=1e4, ser=0.7, ksp_eps=1e-2,
                                     krylov=30, maxits=30, tol=1e-8, max_steps=args.max_steps)
        ctx.profile(True)
        Uo, info = sol.solve(torch.from_numpy(U).cuda())
        tm = ctx.timers()
        ctx.profile(False)
        states[name] = Uo
        res[name] = {"seconds": info["seconds"], "steps": info["steps"], "gmres_its": info["linear_its"],
                     "rel_residual": info["rel_residual"],
                     "timers_s": {k: v[0] / 1e3 for k, v in tm.items() if v[1]}}
    d = (torch.linalg.norm(states["mixed"] - states["fp64"]) / torch.linalg.norm(states["fp64"])).item()
    line = {"metric": METRIC, "workload": "newton", "value": res["fp64"]["seconds"] / res["mixed"]["seconds"],
            "unit": "x (FP64 time / mixed time to ||R||/||R0|| <= 1e-8)", "higher_is_better": True,
            "config": {"workload": f"steady Newton-GMRES, {args.n}^3 jittered Kuhn tet mesh N={s['N']} E={s['E']}, "
                                   "second-order FP64 residual, first-order H1 Jacobian, "
                                   + ("block ILU(0), multicolour" if args.pc == "ilu" else "block-Jacobi") + ", GMRES(30)",
                       "preconditioner": args.pc, "mesh_setup_s": setup_s},
            "mixed": res["mixed"], "fp64": res["fp64"], "state_rel_l2_mixed_vs_fp64": d}
    line["clocks"] = clocks.stop()
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_adjoint(args):
    """Adjoint shape sensitivities of the z-force on z=0 (32 Gaussian-bump
    modes) on a converged Mach 0.8 flow, checked against finite differences;
    cost of (J^T v + dR/dX^T lambda) against one primal residual."""
    import torch
    import aerof_dev_b200 as A
    from aerof_dev_b200 import sensitivity as S
    torch.cuda.set_device(0)
    clocks = ClockSampler(gpu_uuid(0))
    clocks.start()
    W = __import__("aerof_dev_b200.workloads", fromlist=["x"])
    mesh = W.make_lattice_mesh(args.n, jitter=0.2, codes="channel")
    X = mesh["X"] + W.shape_modes(mesh["X"], 1, sigma=0.25, amplitude=0.04, seed=7)[0]
    mesh = dict(mesh, X=X)
    Ub = W.freestream(0.8)
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=args.rec)
    N = X.shape[0]
    U0 = torch.from_numpy(np.tile(Ub, (N, 1))).cuda()
    t0 = time.perf_counter()
    U, info = S.converge(ctx, U0, tol=1e-10, max_steps=args.max_steps)
    conv_s = time.perf_counter() - t0
    zf = np.nonzero(mesh["sides"] == 4)[0]
    F = S.ZForce(mesh["faces"], zf)
    modes = W.shape_modes(X, args.modes, seed=11, amplitude=1.0)
    Uh = U.cpu().numpy()
    # cost ratio, device-resident, CUDA events
    sp, sens = A.SpaceOperator(ctx), A.Sensitivity(ctx)
    lam = torch.from_numpy(np.random.default_rng(3).standard_normal((N, 5))).cuda()
    R = torch.empty_like(U)

    def timed(fn, k=10):
        fn(); torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True); e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            fn()
        e1.record(); torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    t_res = timed(lambda: sp.computeResidual(U, R))
    t_vjp = timed(lambda: sens.vjp(U, lam))
    t_dxt = timed(lambda: sens.dRdX_T(U, lam))
    t_jvp = timed(lambda: sens.jvp(U, lam))
    t_both = timed(lambda: sens.adjoint_products(U, lam))
    sens.h2_evaluate(U)
    t_h2t = timed(lambda: sens.h2_apply(lam, transpose=True))
    t_h2 = timed(lambda: sens.h2_apply(lam))
    sens.h2_release()
    t1 = time.perf_counter()
    ga, ainfo = S.adjoint_gradient(ctx, U, X, F, modes)
    adj_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    gs, sinfo = S.adjoint_gradient(ctx, U, X, F, modes, stored_operator=True)
    adj_stored_s = time.perf_counter() - t1
    nfd = min(args.fd_modes, args.modes)
    gr = S.fd_gradient(ctx, Uh, X, F, modes[:nfd], h=(2e-4, 1e-4), tol=1e-10, max_steps=args.max_steps)
    g6 = S.fd_gradient(ctx, Uh, X, F, modes[:nfd], h=1e-6, tol=1e-10, max_steps=args.max_steps)
    line = {"metric": METRIC, "workload": "adjoint", "value": t_both / t_res,
            "unit": "x one primal residual (J^T lambda and dR/dX^T lambda, one reverse sweep)",
            "higher_is_better": False,
            "separate_calls_ratio": (t_vjp + t_dxt) / t_res,
            "config": {"workload": f"adjoint z-force sensitivities, {args.n}^3 jittered mesh with a base bump, "
                                   f"{args.modes} Gaussian-bump modes, Mach 0.8",
                       "reconstruction": {1: "constant", 2: "van Albada", 3: "linear"}[args.rec], "N": N},
            "ms": {"residual": t_res, "vjp": t_vjp, "dRdX_T": t_dxt, "jvp": t_jvp, "adjoint_products": t_both,
                   "h2_vjp": t_h2t, "h2_jvp": t_h2},
            "h2_vjp_over_residual": t_h2t / t_res,
            "converge_s": conv_s, "adjoint_gradient_s": adj_s,
            "adjoint": {k: v for k, v in ainfo.items() if k != "lambda"},
            "adjoint_gradient_stored_operator_s": adj_stored_s,
            "adjoint_stored_operator": {k: v for k, v in sinfo.items() if k != "lambda"},
            "stored_vs_matrix_free_grad_max_rel": float(np.abs(gs - ga).max() / np.abs(ga).max()),
            "J": F.value(Uh, X), "grad": ga.tolist(),
            "fd_richardson": gr.tolist(), "fd_step_1e-6": g6.tolist(),
            "max_rel_err_vs_richardson": float(np.abs(ga[:nfd] - gr).max() / np.abs(gr).max()),
            "max_rel_err_vs_fd_1e-6": float(np.abs(ga[:nfd] - g6).max() / np.abs(g6).max()),
            "newton": {k: v for k, v in info.items() if k != "history"}}
    line["clocks"] = clocks.stop()
    # all modes against the oracle: its dual-number dR/dX . Xdot_k with the
    # adjoint state of the solve above (after the timed and clocked parts)
    t1 = time.perf_counter()
    g_or = oracle_directional(args.n, args.rec, Uh, ainfo["lambda"], args.modes, min(8, os.cpu_count() or 1))
    line["oracle_directional"] = {
        "what": "dJ/dX . Xdot_k - lambda . (dR/dX . Xdot_k), the oracle's forward-mode dual numbers with the "
                "GPU adjoint state, every mode",
        "modes": args.modes, "max_rel_err": float(np.abs(ga - g_or).max() / np.abs(g_or).max()),
        "grad": g_or.tolist(), "seconds": time.perf_counter() - t1}
    print(json.dumps(line), flush=True)
    return 0


def _oracle_modes_worker(job):
    """One worker of the oracle check: rebuild the mesh (seeded, as the
    workload did), then per mode dJ/dX . Xdot_k - lambda . (dR/dX . Xdot_k)
    by the oracle's forward-mode dual numbers."""
    n, rec, U, lam, idx = job
    from aerof_dev_b200 import workloads as W
    from oracle.oracle import Oracle
    mesh = W.make_lattice_mesh(n, jitter=0.2, codes="channel")
    X = mesh["X"] + W.shape_modes(mesh["X"], 1, sigma=0.25, amplitude=0.04, seed=7)[0]
    mesh = dict(mesh, X=X)
    modes = W.shape_modes(X, max(idx) + 1, seed=11, amplitude=1.0)
    o = Oracle(mesh)
    zf = np.nonzero(mesh["sides"] == 4)[0].astype(np.int32)
    Ub = W.freestream(0.8)
    out = []
    for k in idx:
        dR, _ = o.dRdX(U, Ub, modes[k], order=rec)
        out.append((k, o.zforce_dX(U, zf, modes[k]) - float(np.sum(lam * dR))))
    return out


def oracle_directional(n: int, rec: int, U, lam, nmodes: int, nproc: int) -> np.ndarray:
    """Every mode's gradient from the adjoint state lambda with the oracle's
    exact directional derivatives (CPU, spawned worker processes)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    nproc = max(1, min(nproc, nmodes))
    jobs = [(n, rec, U, lam, list(range(w, nmodes, nproc))) for w in range(nproc)]
    g = np.empty(nmodes)
    with ProcessPoolExecutor(max_workers=nproc, mp_context=mp.get_context("spawn")) as ex:
        for part in ex.map(_oracle_modes_worker, jobs):
            for k, v in part:
                g[k] = v
    return g


def run_sensitivities(args):
    """Batched direct shape sensitivities (16 Gaussian-bump modes of the
    z-force on z=0) on a converged Mach 0.8 flow: every right-hand side
    -dR/dX . Xdot_k solved in one call with the exact linearisation stored
    once (FP64 flexible GMRES with the stored products, FP32 first-order
    inner GMRES); checked against the adjoint gradient (all modes) and
    central finite differences of the re-converged flow (first --fd-modes)."""
    import torch
    import aerof_dev_b200 as A
    from aerof_dev_b200 import sensitivity as S
    torch.cuda.set_device(0)
    clocks = ClockSampler(gpu_uuid(0))
    clocks.start()
    W = __import__("aerof_dev_b200.workloads", fromlist=["x"])
    mesh = W.make_lattice_mesh(args.n, jitter=0.2, codes="channel")
    X = mesh["X"] + W.shape_modes(mesh["X"], 1, sigma=0.25, amplitude=0.04, seed=7)[0]
    mesh = dict(mesh, X=X)
    Ub = W.freestream(0.8)
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=args.rec)
    if args.pc == "ilu":
        ctx.set_preconditioner(A.PC_ILU0)
    N = X.shape[0]
    U0 = torch.from_numpy(np.tile(Ub, (N, 1))).cuda()
    t0 = time.perf_counter()
    U, info = S.converge(ctx, U0, tol=1e-10, max_steps=args.max_steps)
    conv_s = time.perf_counter() - t0
    zf = np.nonzero(mesh["sides"] == 4)[0]
    F = S.ZForce(mesh["faces"], zf)
    modes = W.shape_modes(X, args.modes, seed=11, amplitude=1.0)
    Uh = U.cpu().numpy()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    gb, binfo = S.direct_gradient_batch(ctx, Uh, X, F, modes, inner_its=args.inner_its)
    batch_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    g1, info1 = S.direct_gradient(ctx, Uh, X, F, modes[:1], inner_its=args.inner_its)
    single_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    ga, ainfo = S.adjoint_gradient(ctx, Uh, X, F, modes, inner_its=args.inner_its)
    adj_s = time.perf_counter() - t1
    nfd = min(args.fd_modes, args.modes)
    g6 = S.fd_gradient(ctx, Uh, X, F, modes[:nfd], h=1e-6, tol=1e-10, max_steps=args.max_steps) if nfd else None
    s = W.lattice_sizes(args.n)
    line = {"metric": METRIC, "workload": "sensitivities", "value": batch_s / args.modes,
            "unit": "s per right-hand side (batched direct sensitivities, host wall clock)",
            "higher_is_better": False,
            "config": {"workload": f"batched direct shape sensitivities, {args.n}^3 jittered mesh with a base bump "
                                   f"N={s['N']} E={s['E']}, {args.modes} Gaussian-bump modes, Mach 0.8",
                       "reconstruction": {1: "constant", 2: "van Albada", 3: "linear"}[args.rec],
                       "preconditioner": args.pc, "inner_its": args.inner_its},
            "batch_s": batch_s, "batch": binfo, "single_rhs_matrix_free_s": single_s,
            "single_rhs_its": info1["direct_its"], "converge_s": conv_s, "adjoint_gradient_s": adj_s,
            "adjoint": {k: v for k, v in ainfo.items() if k != "lambda"}, "grad_batched_direct": gb.tolist(),
            "grad_adjoint": ga.tolist(),
            "max_rel_batched_vs_adjoint": float(np.abs(gb - ga).max() / np.abs(ga).max()),
            "max_rel_batched_vs_single": float(abs(gb[0] - g1[0]) / abs(g1[0])),
            "newton": {k: v for k, v in info.items() if k != "history"}}
    if g6 is not None:
        line["fd_step_1e-6"] = g6.tolist()
        line["max_rel_batched_vs_fd_1e-6"] = float(np.abs(gb[:nfd] - g6).max() / np.abs(g6).max())
    line["clocks"] = clocks.stop()
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_adjoint_products(args):
    """Per-call device times of the residual and of the exact linearised
    products on a smooth state (no flow solve): J v, J^T w, (dR/dX)^T lam and
    both adjoint products from one reverse sweep; 3 warm-up + 10 timed calls
    each, CUDA events on the context's stream."""
    import torch
    import aerof_dev_b200 as A
    from aerof_dev_b200 import workloads as W
    torch.cuda.set_device(0)
    clocks = ClockSampler(gpu_uuid(0))
    clocks.start()
    mesh = W.make_lattice_mesh(args.n, jitter=0.2, codes="channel")
    Ub = W.freestream(0.8)
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=args.rec)
    ctx.set_stream(torch.cuda.current_stream())
    U = torch.from_numpy(W.smooth_state(mesh["X"], 0.8)).cuda()
    lam = torch.from_numpy(np.random.default_rng(3).standard_normal((ctx.N, 5))).cuda()
    sp, S = A.SpaceOperator(ctx), A.Sensitivity(ctx)
    R = torch.empty_like(U)
    out = {}
    calls = (("residual", lambda: sp.computeResidual(U, R)), ("jvp", lambda: S.jvp(U, lam)),
             ("vjp", lambda: S.vjp(U, lam)), ("dRdX_T", lambda: S.dRdX_T(U, lam)),
             ("adjoint_products", lambda: S.adjoint_products(U, lam)),
             # the stored operator (MatVecProdH2): one evaluation, then products
             ("h2_evaluate", lambda: S.h2_evaluate(U)), ("h2_vjp", lambda: S.h2_apply(lam, transpose=True)),
             ("h2_jvp", lambda: S.h2_apply(lam)))
    for name, fn in calls:
        reps = 3 if name == "h2_evaluate" else 10
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    S.h2_release()
    s = W.lattice_sizes(args.n)
    line = {"metric": METRIC, "workload": "adjoint_products", "value": out["adjoint_products"] / out["residual"],
            "unit": "x one primal residual (J^T lambda and dR/dX^T lambda, one reverse sweep)",
            "higher_is_better": False, "ms": out,
            "h2_vjp_over_residual": out["h2_vjp"] / out["residual"],
            "h2_jvp_over_residual": out["h2_jvp"] / out["residual"],
            "config": {"workload": f"{args.n}^3 jittered Kuhn tet mesh N={s['N']} E={s['E']}, smooth Mach 0.8 state",
                       "reconstruction": {1: "constant", 2: "van Albada", 3: "linear"}[args.rec]}}
    line["clocks"] = clocks.stop()
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_sa_residual(args):
    """Spalart-Allmaras residual (six variables, van Albada, Sutherland
    viscosity, Re 1e6 per unit length, nu~ 3 nu_inf with a bump, wall
    distance to z = 0) on the lattice mesh: device time per evaluation with
    device arrays (CUDA events), against the five-variable laminar residual
    of the same mesh and flow."""
    import torch
    import aerof_dev_b200 as A
    torch.cuda.set_device(0)
    clocks = ClockSampler(gpu_uuid(0))
    clocks.start()
    W, mesh, Ub, U = build_workload(args.n)
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=A.REC_VANALBADA)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream)
    ctx.set_viscosity(model=2, reynolds_mu=1e6, prandtl=0.72, sutherland_alpha=1.4 * 0.4 * 0.64,
                      sutherland_Ts=0.37)
    X = mesh["X"]
    nu = 3e-6 * (1.0 + 4.0 * np.exp(-((X - 0.5) ** 2).sum(1) / 0.05))
    U6 = np.column_stack([U, U[:, 0] * nu])
    Ub6 = np.concatenate([Ub, [3e-6 * Ub[0]]])
    ctx.set_turbulence(np.abs(X[:, 2]) + 1e-3, Ub6)
    sp = A.SpaceOperator(ctx)
    U6d = torch.from_numpy(U6).cuda()
    R6d = torch.empty_like(U6d)
    Ud = torch.from_numpy(U).cuda()
    Rd = torch.empty_like(Ud)
    t_sa = timed_on(stream, lambda: sp.computeResidualSA(U6d, R6d), args.steps, args.warmup)
    t_lam = timed_on(stream, lambda: sp.computeResidual(Ud, Rd), args.steps, args.warmup)
    ctx.set_viscosity(model=0)
    t_inv = timed_on(stream, lambda: sp.computeResidual(Ud, Rd), args.steps, args.warmup)
    s = W.lattice_sizes(args.n)
    line = {"metric": METRIC, "workload": "sa_residual", "value": s["E"] / (t_sa * 1e-3) / 1e6,
            "unit": "Medges/s", "higher_is_better": True, "ms_per_eval": t_sa,
            "laminar_ms_per_eval": t_lam, "sa_over_laminar": t_sa / t_lam, "inviscid_ms_per_eval": t_inv,
            "laminar_galerkin_ms": t_lam - t_inv,
            "config": {"workload": f"Spalart-Allmaras residual (6 variables, van Albada + LSQ + Roe, Sutherland "
                                   f"viscosity), {args.n}^3 jittered Kuhn tet mesh N={s['N']} E={s['E']}",
                       "organisation": "edge (thread per edge, per-node gather)"}}
    line["clocks"] = clocks.stop()
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_e2e_timeline(args):
    """Device timeline of the residual of page-locked host arrays (the e2e
    call): three calls traced with CUPTI (torch.profiler), per call its span
    and, per kind of work, the summed device time of the copies in, the
    copies out and the kernels (they overlap); for the second call every
    event as [kind, start us, duration us]."""
    import torch
    import aerof_dev_b200 as A
    from torch.profiler import ProfilerActivity, profile
    torch.cuda.set_device(0)
    W, mesh, Ub, U = build_workload(args.n)
    ctx = A.Context.from_mesh(mesh, Ub, reconstruction=A.REC_VANALBADA)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream)
    sp = A.SpaceOperator(ctx)
    Uh = torch.from_numpy(U).pin_memory()
    Rh = torch.empty_like(Uh).pin_memory()
    for _ in range(max(args.warmup, 3)):
        sp.computeResidual(Uh, Rh)
    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(3):
            sp.computeResidual(Uh, Rh)
        torch.cuda.synchronize()
    ev = sorted((e for e in prof.events() if e.device_type.name == "CUDA"), key=lambda e: e.time_range.start)
    # every call starts with the memset of its counters
    calls = []
    for e in ev:
        if "Memset" in e.name or not calls:
            calls.append([e])
        else:
            calls[-1].append(e)
    out = []
    for c in calls:
        t0 = min(e.time_range.start for e in c)
        t1 = max(e.time_range.end for e in c)
        kinds = {"h2d_us": 0.0, "d2h_us": 0.0, "kernel_us": 0.0}
        for e in c:
            d = e.time_range.end - e.time_range.start
            if "HtoD" in e.name:
                kinds["h2d_us"] += d
            elif "DtoH" in e.name:
                kinds["d2h_us"] += d
            elif "Memset" not in e.name:
                kinds["kernel_us"] += d
        out.append({"span_us": t1 - t0, **{k: round(v, 1) for k, v in kinds.items()},
                    "kernels": sum(1 for e in c if "Memcpy" not in e.name and "Memset" not in e.name)})
    def kind(name):
        return "copy_in" if "HtoD" in name else "copy_out" if "DtoH" in name else name.split("(")[0][:48]
    mid = calls[len(calls) // 2]
    m0 = min(e.time_range.start for e in mid)
    events = [[kind(e.name), round(e.time_range.start - m0, 1), round(e.time_range.end - e.time_range.start, 1)]
              for e in mid]
    s = W.lattice_sizes(args.n)
    print(json.dumps({"metric": METRIC, "workload": "e2e_timeline", "n": args.n, "E": s["E"],
                      "bytes_each_way": int(U.nbytes), "calls": out, "events": events}), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=101, help="lattice nodes per side")
    ap.add_argument("--e2e-steps", type=int, default=200)
    ap.add_argument("--ref-budget", type=float, default=120.0, help="seconds of timed CPU work (reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-newton", action="store_true", help="leave the Newton part out of the residual line")
    ap.add_argument("--newton-meshes", default="101,161",
                    help="lattice sizes of the Newton part (the last one is reported as 'newton')")
    ap.add_argument("--no-adjoint-cost", action="store_true",
                    help="leave the adjoint-cost part out of the residual line")
    ap.add_argument("--workload", choices=["residual", "newton", "adjoint", "adjoint_products", "sensitivities",
                                           "e2e_timeline", "sa_residual"],
                    default="residual")
    ap.add_argument("--max-steps", type=int, default=400)
    ap.add_argument("--modes", type=int, default=32)
    ap.add_argument("--fd-modes", type=int, default=4)
    ap.add_argument("--rec", type=int, choices=[1, 2, 3], default=2,
                    help="adjoint workload reconstruction: 1 constant, 2 van Albada, 3 linear")
    ap.add_argument("--inner-its", type=int, default=20,
                    help="inner FP32 GMRES iterations of the sensitivity solves")
    ap.add_argument("--pc", choices=["jacobi", "ilu"], default="jacobi",
                    help="preconditioner of the Newton and sensitivity workloads")
    ap.add_argument("--kernel", choices=["blocked", "edge"], default="blocked",
                    help="residual kernel organisation (see include/aerof_gpu.h)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "newton":
        return run_newton(args)
    if args.workload == "adjoint":
        return run_adjoint(args)
    if args.workload == "adjoint_products":
        return run_adjoint_products(args)
    if args.workload == "e2e_timeline":
        return run_e2e_timeline(args)
    if args.workload == "sa_residual":
        return run_sa_residual(args)
    if args.workload == "sensitivities":
        return run_sensitivities(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
