#!/usr/bin/env python
"""Benchmark of the multigrid solve path on the 256^3 variable-coefficient Q1
diffusion problem (-div(k grad u) = 1, log k a seeded 64-mode Fourier field,
16.97M nodes): time to reduce the residual by 1e-10 with CG + V(1,1) Jacobi
multigrid, and the throughput of one V-cycle.

One step = one solve from the device-resident assembled hierarchy (x = 0 to
||r||/||r0|| < 1e-10 in the FP64 residual) with the mixed-precision path (FP32
V-cycle with BF16 coarse residuals inside FP64 iterative refinement) and the
per-node damping of the damping network (gnu_femlisp_b200/weights).
value = top-level DoF / time-to-solution (MDoF/s, whole job: summed over
replicas); the plain FP64 path and the mixed path without the network are
timed beside it.  e2e = the same solve through the C-ABI from pinned host
buffers: coefficient upload, assembly of all levels, damping network and
judge, solve and the solution copied back, every step (wall clock).

--impl reference times the CPU restatement of the reference algorithm
(oracle/, C++ with OpenMP) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to 1e-10 rel. residual + MDoF/s per V-cycle: mixed/learned vs FP64 GMG"
WEIGHTS = os.path.join(ROOT, "gnu_femlisp_b200", "weights", "damping3d.fmgnet")
HBM_FALLBACK_GBS = 6650.0
JUDGE_STEPS = 1  # CG steps after each (re)start on which the plain cycle judges the learned one
# DRAM bytes per top-level node of one launch (read + write), from the ncu
# capture of the 257^3 case (profiles/k_mfc_q1_3d_mixed_257cube.md): mode 2
# 668.7 MB, FP64 mode 0 322.2 MB, mode 1 273.0 MB over 16,974,593 nodes
TOP_TRAFFIC_B_PER_NODE = {"k_mfc<float,double,float,2,1,7>": 668.7e6 / 16974593,
                          "k_mfc<double,float,float,0,1,0>": 322.2e6 / 16974593,
                          "k_mfc<float,double,float,1,0,0>": 273.0e6 / 16974593}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--level", type=int, default=8, help="top level (256^3 cells = 8)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget", type=float, default=300.0,
                    help="--impl reference: seconds of timed steps after which no further step starts")
    ap.add_argument("--matvec-reps", type=int, default=20)
    ap.add_argument("--no-learned", action="store_true", help="mixed precision without the damping network")
    ap.add_argument("--config", choices=["c2", "c3", "c4", "c5"], default="c3",
                    help=("c2: plain FP64 Q2 SOR multigrid on 64^3 cells vs the oracle; c4: the learned "
                          "smoother on 128^2 block fields, 256 held-out seeds; c5: vector-Q2 elasticity on "
                          "48^3 cells, FP64 CG + block-Jacobi V(2,2); each its own JSON line"))
    ap.add_argument("--c5-level", type=int, default=4, help="c5: 3 x 2^level cells per direction")
    ap.add_argument("--c4-fields", type=int, default=256)
    ap.add_argument("--c4-batch", type=int, default=1024, help="c4: fields solved together in one batch")
    ap.add_argument("--profile", choices=["solve", "net", "c5", "c5mv", "ssc", "mfs", "c2"], default=None,
                    help="no timing: a workload for an ncu capture (solve: setup, two mixed+learned solves, "
                         "the launch count, one more solve; net: the damping network on every level, 8 times; "
                         "c5: the elasticity setup, two mixed+learned solves, the launch count, one more; "
                         "c5mv: the elasticity FP64 block matvec, 5 times; mfs: one mixed solve, then inside "
                         "the NVTX range 'mfs' one launch of each top-level kernel of the mixed solve)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def allreduce_max(v: float, world: int) -> float:
    """The maximum of v over the ranks (the job's time is the slowest rank's)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, t_local: float, world: int) -> tuple:
    """Whole-job throughput of `world` independent replicas (weak scaling):
    all ranks' units over the slowest rank's time; returns (value, t_max)."""
    t_max = allreduce_max(t_local, world)
    return world * units_per_rank / t_max, t_max


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def plain_cfg(G, maxsteps=200):
    C = G._capi
    return G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, maxsteps,
                      C.FMG_MULTIPLICATIVE)


def _rel(a, b) -> float:
    """max |a - b| / max |b| (0 when both are zero)."""
    den = float(np.max(np.abs(b))) if np.size(b) else 0.0
    num = float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if np.size(b) else 0.0
    return num / den if den > 0 else num


def parity_block(o, ref, g, gpu_hist, gpu_x, levels) -> dict:
    """The GPU's plain FP64 path against the oracle on the same workload:
    every assembled level matrix and the top-level rhs (bitwise count and the
    largest relative difference), the complete :defnorm history and the
    solution of the solve to 1e-10 (bitwise and relative).  The bar is 1e-12
    relative; the GPU path follows the oracle's operation order, so bitwise
    equality is expected."""
    nbit, worst = 0, 0.0
    for lev in levels:
        a, b = g.matrix(lev), o.matrix(lev)
        nbit += int(np.array_equal(a, b))
        worst = max(worst, _rel(a, b))
        del a, b
    rg, ro = g.rhs(), o.rhs()
    hist_same = len(gpu_hist) == len(ref.history) and np.array_equal(gpu_hist, ref.history)
    hist_rel = (float(np.max(np.abs(gpu_hist - ref.history) / np.abs(ref.history)))
                if len(gpu_hist) == len(ref.history) else float("inf"))
    x_rel = _rel(gpu_x, ref.x)
    return {"levels": len(levels), "levels_bitwise": nbit, "matrix_rel": worst,
            "rhs_bitwise": bool(np.array_equal(rg, ro)), "rhs_rel": _rel(rg, ro),
            "steps_gpu": int(len(gpu_hist) - 1), "steps_oracle": int(ref.steps),
            "history_bitwise": bool(hist_same), "history_rel": hist_rel,
            "x_bitwise": bool(np.array_equal(gpu_x, ref.x)), "x_rel": x_rel, "_x_oracle": ref.x,
            "ok": bool(hist_rel <= 1e-12 and x_rel <= 1e-12 and worst <= 1e-12),
            "bar": "1e-12 relative (history, solution, level matrices)"}


def oracle_c3(wl):
    """The oracle on the benchmark workload: a hierarchy with its
    coefficients (not yet assembled)."""
    from oracle import oracle as O
    o = O.Oracle(3, 1, wl.level, base_level=wl.base_level)
    o.set_coefficient(O.K_CELL, wl.kcell)
    return o


def oracle_cg_cfg(rtol=1e-10):
    from oracle import oracle as O
    return O.solve_cfg(method=O.METHOD_CG_MG, damp=0.6, compat=False, rtol=rtol, maxsteps=200)


def cpu_baseline(wl, g, gpu_hist, gpu_x) -> tuple:
    """The oracle (C++ restatement, OpenMP, all host threads) on the same
    workload, measured, not extrapolated: assembly of every level, then one
    complete CG + V(1,1) Jacobi(0.6) solve to 1e-10 with the oracle's own step
    count.  The same oracle run pins the GPU's plain FP64 path at full size
    (``parity_block``).  Beside it, one complete solve on one thread one level
    down (129^3 nodes), timed whole."""
    from oracle import oracle as O
    o = oracle_c3(wl)
    t0 = time.perf_counter()
    o.assemble()
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref = o.solve(oracle_cg_cfg())
    t_solve = time.perf_counter() - t0
    par = parity_block(o, ref, g, gpu_hist, gpu_x, range(wl.base_level, wl.level + 1))
    del o
    n = wl.nodes
    cpu = {"value": n / t_solve / 1e6, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
           "cores": O.num_threads(), "kind": "port",
           "sample": (f"oracle C++ restatement, {O.num_threads()} OpenMP threads: one complete solve to 1e-10 "
                      f"({ref.steps} CG steps, {t_solve:.1f} s) from the assembled hierarchy (assembly of levels "
                      f"{wl.base_level}..{wl.level}: {t_asm:.1f} s, not in value)"),
           "assembly_s": t_asm, "time_to_solution_s": t_solve, "cg_steps": int(ref.steps),
           "e2e_s": t_asm + t_solve, "host": host_info(), "one_thread": one_thread_solve(wl)}
    return cpu, par


def host_info() -> dict:
    """nproc and the CPU model of the host the baseline ran on."""
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model, "omp_threads": os.environ.get("OMP_NUM_THREADS")}


def one_thread_solve(wl) -> dict:
    """One complete solve of the same algorithm on one thread, one level below
    the workload (8x fewer unknowns), timed whole (assembly and solve)."""
    from gnu_femlisp_b200 import problems
    from oracle import oracle as O
    nthreads = O.num_threads()
    small = problems.c3(seed=0, level=wl.level - 1)
    O.set_num_threads(1)
    try:
        o = oracle_c3(small)
        t0 = time.perf_counter()
        o.assemble()
        t_asm = time.perf_counter() - t0
        t0 = time.perf_counter()
        r = o.solve(oracle_cg_cfg())
        t_solve = time.perf_counter() - t0
    finally:
        O.set_num_threads(nthreads)
    return {"nodes": small.nodes, "assembly_s": t_asm, "time_to_solution_s": t_solve, "cg_steps": int(r.steps),
            "mdof_per_s": small.nodes / t_solve / 1e6,
            "sample": f"1 thread, one complete solve to 1e-10 at {small.nodes} unknowns ({r.steps} CG steps)"}


def run_reference(args, world, rank):
    """The reference algorithm on the host cores: the CPU restatement (C++,
    OpenMP, all host threads).  The hierarchy is assembled once (timed and
    reported beside the line); one step = one complete CG + V(1,1)
    Jacobi(0.6) solve from it to 1e-10 with the oracle's own step count,
    timed whole -- the definition of the GPU arm's value.  Steps run until
    --steps are done or the timed region has used --ref-budget seconds (at
    least one); "steps" is the number actually timed."""
    if rank != 0:
        return
    from gnu_femlisp_b200 import problems
    from oracle import oracle as O
    O.build()
    wl = problems.c3(seed=0, level=args.level)
    n = wl.nodes
    o = oracle_c3(wl)
    t0 = time.perf_counter()
    o.assemble()
    t_asm = time.perf_counter() - t0
    cfg = oracle_cg_cfg()

    def step():
        t0 = time.perf_counter()
        r = o.solve(cfg)
        dt = time.perf_counter() - t0
        if r.status != 0:
            raise RuntimeError(f"oracle solve did not converge in {r.steps} steps")
        return dt, r.steps

    nwarm = min(args.warmup, 1)  # one warm-up solve touches every page; more add nothing on the host
    for _ in range(nwarm):
        step()
    sol, steps = [], 0
    t_start = time.perf_counter()
    while len(sol) < args.steps:
        dt, steps = step()
        sol.append(dt)
        if time.perf_counter() - t_start + dt > args.ref_budget:
            break
    t_solve = float(np.mean(sol))
    val = n / t_solve / 1e6
    line = {
        "metric": METRIC, "value": val, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
        "impl": "reference", "n_gpus": world, "steps": len(sol), "warmup": nwarm,
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": t_solve * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": wl.name, "nodes": n, "solver": "CG + V(1,1) Jacobi(0.6), base level 2",
                   "inputs": "larger than L2"},
        "time_to_solution_s": t_solve, "cg_steps": int(steps),
        "assembly_s": t_asm, "assembly_note": "assembly of all levels, once before the timed steps (not in value)",
        "cpu_baseline": {"value": val, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
                         "cores": O.num_threads(), "kind": "port", "host": host_info(),
                         "sample": (f"{len(sol)} timed steps, each one complete solve to 1e-10 from the assembled "
                                    f"hierarchy ({steps} CG steps, {t_solve:.2f} s); the oracle C++ restatement of "
                                    f"the reference algorithm")},
        "e2e": {"value": val, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_mine(args, world, rank, local):
    import torch

    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.learn import DampingNet
    C = G._capi
    torch.cuda.set_device(local)
    wl = problems.c3(seed=0, level=args.level)
    n = wl.nodes
    ctx = G.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    g = G.Grid(ctx, 3, 1, wl.level, base_level=wl.base_level)
    k_host = torch.from_numpy(wl.kcell).pin_memory()          # pinned host input
    x_host = torch.empty(n, dtype=torch.float64).pin_memory()  # pinned host output
    k_np, x_np = k_host.numpy(), x_host.numpy()
    cfg = plain_cfg(G)
    net = None if args.no_learned else DampingNet.load(ctx, WEIGHTS)
    x, xm = g.vector(), g.vector()

    def clear_damping():
        for lev in range(g.base + 1, g.top + 1):
            g.set_node_damping(lev, None)

    def install_learned():
        # the damping network on every level; the plain cycle judges it inside
        # the solve (JUDGE_STEPS shadowed CG steps after each (re)start)
        net.apply(g)

    def setup():
        g.set_coefficient(C.FMG_K_CELL, k_np)
        g.assemble()
        if net is not None:
            install_learned()

    def plain_step():
        x.fill(0.0)
        return g.solve(cfg, x)

    judge_steps = JUDGE_STEPS if net is not None else 0

    def mixed_step():
        xm.fill(0.0)
        return g.solve_mixed(cfg, xm, matrix_free=True, judge=judge_steps)

    def e2e_step():
        setup()
        out = mixed_step()
        xm.get(out=x_np)
        return out

    def timed(fn, reps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier(world)
        ctx.synchronize()
        torch.cuda.synchronize()
        ev0.record(stream)
        out = None
        for _ in range(reps):
            out = fn()
        ev1.record(stream)
        ev1.synchronize()
        ctx.synchronize()
        return ev0.elapsed_time(ev1) / 1e3 / reps, out

    def wall(fn, reps):
        barrier(world)
        ctx.synchronize()
        t0 = time.perf_counter()
        out = None
        for _ in range(reps):
            out = fn()
        ctx.synchronize()
        return (time.perf_counter() - t0) / reps, out

    # ---- plain FP64 path (scalar damping 0.6): the baseline of the speed-up
    g.set_coefficient(C.FMG_K_CELL, k_np)
    g.assemble()
    clear_damping()
    for _ in range(max(args.warmup, 1)):
        plain_step()
    clocks = ClockSampler(local)
    clocks.start()
    t_plain, (hist, steps, status) = timed(plain_step, args.steps)
    if status != 0:
        raise RuntimeError(f"plain solve did not converge: {steps} steps")
    x_plain = x.get()
    # ---- mixed precision without the learned damping
    for _ in range(max(args.warmup, 1)):
        mixed_step()
    t_mixed_plain, (mh, no_p, ni_p, st_p) = timed(mixed_step, args.steps)
    # ---- mixed precision + learned damping: the headline
    t_setup = t_setup_solve = None
    if net is not None:
        install_learned()  # first use: the network's buffers and kernels
        t_setup, _ = timed(install_learned, 3)

        def setup_and_solve():
            install_learned()
            return mixed_step()
        setup_and_solve()
        t_setup_solve, _ = timed(setup_and_solve, args.steps)
    for _ in range(max(args.warmup, 1)):
        mixed_step()
    launches0 = ctypes_count(C)
    t_head, (mhist, nouter, ninner, mstatus) = timed(mixed_step, args.steps)
    launches = (ctypes_count(C) - launches0) // max(args.steps, 1)
    clk = clocks.stop()
    if mstatus != 0:
        raise RuntimeError(f"mixed solve did not converge: {nouter} outer steps")
    status_learned = g.learned_status()
    value, t_head_max = replica_value(n / 1e6, t_head, world)  # MDoF/s over all replicas
    t_plain_max = allreduce_max(t_plain, world)
    t_mp_max = allreduce_max(t_mixed_plain, world)

    # error of the headline solution against FP64 solutions: the plain path at
    # the same tolerance and a tight (1e-13) FP64 solve
    x_head = xm.get()
    tight = plain_cfg(G)
    tight.rtol = 1e-13
    x.fill(0.0)
    g.solve(tight, x)
    x_tight = x.get()
    err_plain = float(np.linalg.norm(x_head - x_plain) / np.linalg.norm(x_plain))
    err_tight = float(np.linalg.norm(x_head - x_tight) / np.linalg.norm(x_tight))
    err_plain_tight = float(np.linalg.norm(x_plain - x_tight) / np.linalg.norm(x_tight))

    # ---- end to end through the C-ABI from pinned host buffers: coefficient
    # upload, assembly of all levels, learned damping + judge, mixed solve,
    # solution download
    e2e_step()
    t_e2e, _ = wall(e2e_step, max(1, min(args.steps, 3)))
    t_e2e_max = allreduce_max(t_e2e, world)

    # ---- one plain FP64 V-cycle (the preconditioner application) on the top level
    clear_damping()
    mg = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 0.0, 0.0, 1, C.FMG_MULTIPLICATIVE)
    B = g.vector(values=g.rhs())
    R = g.vector()
    X = g.vector()

    def vcyc():
        g.vcycle(mg, X, B, R)
    for _ in range(3):
        vcyc()
    t_cycle, _ = timed(vcyc, 10)

    # ---- the headline step's top-level kernels, each timed alone (CUDA events
    # on the library's stream, inputs larger than L2) against the measured
    # copy peak: per launch, algorithmic bytes / mean launch time
    peak, peak_kind = measured_peaks()
    xm.fill(0.0)
    g.solve_mixed(cfg, xm, matrix_free=True)  # leaves the buffers the kernels run on
    cells = wl.n_cells ** 3
    top_kernels = []
    for kind, name, alg, per_solve in (
            (C.FMG_MXK_SMOOTH, "k_mfc<float,double,float,2,1,7> (top-level post-smoothing + the flexible CG's (z,r), (z,a))",
             n * (5 * 4 + 2 * 8) + 4 * cells, ninner),
            (C.FMG_MXK_MATVEC64, "k_mfc<double,float,float,0,1,0> (FP64 a = A p of the FP32 direction + (a,p))",
             n * (4 + 8) + 8 * cells, ninner + 1),
            (C.FMG_MXK_RESIDUAL, "k_mfc<float,double,float,1,0,0> (top-level FP32 residual)", n * 3 * 4 + 4 * cells, ninner + 1)):
        g.mixed_top_kernel(kind, 3)
        t_k, _ = timed(lambda kind=kind: g.mixed_top_kernel(kind, args.matvec_reps), 1)
        t_k /= args.matvec_reps
        top_kernels.append({"kernel": name, "algorithmic_bytes": int(alg), "launch_ms": t_k * 1e3,
                            "achieved_gbs": alg / t_k / 1e9, "frac": alg / t_k / 1e9 / peak,
                            "launches_per_solve": int(per_solve), "ms_per_solve": t_k * 1e3 * per_solve})
    dom = max(top_kernels, key=lambda r: r["ms_per_solve"])
    # ---- the north star's matvec criterion: the plain path's FP64 stencil
    # matvec of the top level (assembled matrix)
    P = g.vector(values=np.random.default_rng(1).standard_normal(n))
    Y = g.vector()

    def mv():
        g.matvec(P, Y)
    for _ in range(3):
        mv()
    t_mv, _ = timed(mv, args.matvec_reps)
    nnz = (3 * wl.n_cells + 1) ** 3
    alg_bytes = 8 * nnz + 16 * n
    achieved = alg_bytes / t_mv / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_head_max * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 outer residual/update + f32 V-cycle + bf16 coarse residuals", "data": "synthetic",
        "config": {"workload": wl.name, "nodes": n,
                   "path": ("mixed+learned: FP64 flexible CG (true FP64 residual restarts) preconditioned by "
                            "an FP32 V(1,1) Jacobi cycle (matrix-free top level) with per-node damping from "
                            "the damping network, BF16 coarse rhs/residuals, FP64 dense LU on 5^3"
                            if net is not None else
                            "mixed: FP64 flexible CG preconditioned by an FP32 V(1,1) Jacobi(0.6) cycle"),
                   "outer_steps": int(nouter), "inner_iterations": int(ninner),
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (3.9 GB FP64 matrix, 134 MB FP64 coefficients)"},
        "time_to_solution_s": t_head_max,
        "plain_fp64": {"time_to_solution_s": t_plain_max, "mdof_per_s": world * n / t_plain_max / 1e6,
                       "cg_steps": int(steps), "solver": "CG + V(1,1) Jacobi(0.6) on assembled FP64 levels"},
        "mixed_without_learned": {"time_to_solution_s": t_mp_max, "inner_iterations": int(ni_p),
                                  "speedup_vs_plain_fp64": t_plain_max / t_mp_max},
        "speedup_vs_plain_fp64": t_plain_max / t_head_max,
        "time_to_solution_incl_learned_setup_s": allreduce_max(t_setup_solve or t_head, world),
        "speedup_incl_learned_setup_vs_plain_fp64": t_plain_max / allreduce_max(t_setup_solve or t_head, world),
        "error_vs_fp64": {"vs_plain_same_tol": err_plain, "vs_fp64_1e-13": err_tight,
                          "plain_vs_fp64_1e-13": err_plain_tight},
        "mdof_per_s_per_vcycle": n / t_cycle / 1e6,
        "vcycle_ms": t_cycle * 1e3,
        "ms_per_inner_iteration": t_head_max * 1e3 / max(int(ninner), 1),
        "roofline": {"bound": "hbm", "achieved": dom["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": dom["frac"], "traffic": TOP_TRAFFIC_B_PER_NODE.get(dom["kernel"].split(" ")[0], 0) * n or None,
                     "kernel": dom["kernel"], "peak_kind": peak_kind,
                     "algorithmic_bytes": dom["algorithmic_bytes"], "launch_ms": dom["launch_ms"],
                     "top_level_kernels": top_kernels},
        "matvec_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": 233.7 * n,
                            "kernel": "k_spmv<3,1> (top-level FP64 matvec of the assembled matrix, plain path)",
                            "peak_kind": peak_kind, "algorithmic_bytes": alg_bytes, "launch_ms": t_mv * 1e3},
        "e2e": {"value": world * n / t_e2e_max / 1e6, "unit": "MDoF/s to 1e-10 (N_top / time-to-solution)",
                "h2d_bytes_per_step": int(k_np.nbytes), "d2h_bytes_per_step": int(x_np.nbytes),
                "time_s": t_e2e_max,
                "includes": ("coefficient upload + assembly of all levels + damping network on all levels + "
                             "judge + mixed solve + solution download (wall clock)")},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if net is not None:
        line["learned"] = {"weights": os.path.relpath(WEIGHTS, ROOT), "setup_s": t_setup,
                           "judge": {"kind": "in-solve: the plain cycle shadows the learned one on the first "
                                             f"{JUDGE_STEPS} CG steps after each (re)start, a step along each "
                                             "direction scored by its energy decrease (z,r)^2/(z,Az)",
                                     "accepted": status_learned["reverts"] == 0,
                                     "energy_decrease_learned": status_learned["rho_learned"],
                                     "energy_decrease_plain": status_learned["rho_plain"]},
                           "status": status_learned,
                           "setup": "damping network on levels 3..8 (tcgen05 convolutions); the judge runs in the solve",
                           "setup_timing": ("setup_s: the network alone; time_to_solution_incl_learned_setup_s: the "
                                            "network followed by the judged solve, CUDA events on the library's "
                                            "stream")}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, par = cpu_baseline(wl, g, hist, x_plain)
        line["cpu_baseline"] = cpu
        line["parity"] = par
        head = line["error_vs_fp64"]
        xo = par.pop("_x_oracle")
        head["mixed_vs_oracle"] = float(np.linalg.norm(x_head - xo) / np.linalg.norm(xo))
        head["mixed_vs_oracle_max_rel"] = _rel(x_head, xo)
    if rank == 0:
        print(json.dumps(line), flush=True)
    del P, Y, B, R, X, x, xm
    if net is not None:
        net.close()
    g.close()
    ctx.close()


WEIGHTS_ELASTIC = os.path.join(ROOT, "gnu_femlisp_b200", "weights", "damping3d_elastic.fmgnet")
WEIGHTS2D = os.path.join(ROOT, "gnu_femlisp_b200", "weights", "damping2d.fmgnet")


def run_c4(args):
    """The learned smoother on the block-field set: 2D Q1, 128^2 cells, k
    piecewise constant on 8 x 8 blocks with log10 k ~ U[-3, 3]; for each of
    the held-out seeds 1,000,000 .. the plain V(1,1) Jacobi(0.6) cycle and the
    learned damping (network on every level, then the judge), as the
    iteration (GMG) and as the CG preconditioner, from x = 0 to 1e-10."""
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import learn
    C = G._capi
    ctx = G.Context(0)
    net = learn.DampingNet.load(ctx, WEIGHTS2D)
    seeds = range(1000000, 1000000 + args.c4_fields)
    out = {}
    for method, name, maxsteps in ((C.FMG_METHOD_MG, "gmg", 400), (C.FMG_METHOD_CG_MG, "cg_gmg", 200)):
        cfg = G.SolveCfg(method, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, maxsteps, C.FMG_MULTIPLICATIVE)
        rows = learn.evaluate_on_fields(net, ctx, learn.block_field, seeds, cfg, 2, 7, 2, top_only=False)
        ps = np.array([r["plain_steps"] for r in rows], float)
        ls = np.array([r["learned_steps"] for r in rows], float)
        pt = np.array([r["plain_s"] for r in rows])
        lt = np.array([r["learned_s"] for r in rows])
        out[name] = {
            "plain": {"cycles_mean": ps.mean(), "cycles_median": float(np.median(ps)),
                      "failed": int(sum(r["plain_status"] for r in rows)), "ms_mean": 1e3 * pt.mean()},
            "learned": {"cycles_mean": ls.mean(), "cycles_median": float(np.median(ls)),
                        "failed": int(sum(r["learned_status"] for r in rows)), "ms_mean": 1e3 * lt.mean(),
                        "setup_ms_mean": 1e3 * float(np.mean([r["setup_s"] for r in rows]))},
            "judge_accepted": float(np.mean([r["accepted"] for r in rows])),
            "fields_learned_fewer_cycles": int(np.sum(ls < ps)), "fields_learned_more_cycles": int(np.sum(ls > ps)),
        }
    out["batch"] = run_c4_batch(args, G, net, ctx)
    line = {"metric": "C4 learned smoother: cycles and time to 1e-10, learned damping vs plain w=0.6 GMG",
            "value": out["cg_gmg"]["plain"]["cycles_mean"] / out["cg_gmg"]["learned"]["cycles_mean"],
            "unit": "plain / learned mean CG+GMG cycles", "higher_is_better": True, "n_gpus": 1,
            "data": "synthetic", "dtype": "f64",
            "config": {"workload": "2D Q1 128^2 cells, 8x8 blocks, log10 k ~ U[-3,3]",
                       "fields": f"held-out seeds 1000000..{1000000 + args.c4_fields - 1}",
                       "weights": os.path.relpath(WEIGHTS2D, ROOT),
                       "solve": "one field at a time (fmg_solve), base level 2; batch: "
                                f"{args.c4_batch} fields in one fmg_batch_solve"},
            "results": out}
    print(json.dumps(line), flush=True)
    net.close()
    ctx.close()


def run_c4_batch(args, G, net, ctx):
    """The C4 fields solved as one batch (fmg_batch_solve: every kernel launch
    covers all fields): seeds 1,000,000 .. + c4_batch - 1, CG + V(1,1) Jacobi
    to 1e-10, with the plain damping 0.6 and with the network's damping on
    every level (no judge); the time of the batched solve (CUDA events on the
    library's stream) against the same fields solved one at a time."""
    import torch

    from gnu_femlisp_b200 import learn
    C = G._capi
    B = args.c4_batch
    seeds = list(range(1000000, 1000000 + B))
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, 0.6, 1, 1, 1, 0, 1.0, 1e-10, 0.0, 200, C.FMG_MULTIPLICATIVE)
    stream = torch.cuda.ExternalStream(ctx.stream)
    g = G.Grid(ctx, 2, 1, 7, 2)
    res = {"fields": B, "unknowns_per_field": g.nnodes(), "unknowns_total": B * g.nnodes()}
    for name, learned in (("plain", False), ("learned", True)):
        batch = G.Grid.batch(g, B)
        t0 = time.perf_counter()
        for k, sd in enumerate(seeds):
            g.set_coefficient(C.FMG_K_CELL, learn.block_field(sd))
            g.assemble()
            if learned:
                net.apply(g)
            else:
                for lev in range(g.base + 1, g.top + 1):
                    g.set_node_damping(lev, None)
            batch.batch_load(k, g)
        ctx.synchronize()
        t_setup = time.perf_counter() - t0
        x = batch.vector()
        ts = []
        for rep in range(3):
            x.fill(0.0)
            ctx.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            _, steps, status = batch.batch_solve(cfg, x)
            ev1.record(stream)
            ev1.synchronize()
            ts.append(ev0.elapsed_time(ev1) / 1e3)
        t = min(ts)
        # the first 32 fields one at a time (fmg_solve on their own grid), for the per-field time
        xs = g.vector()
        t_one = []
        for k, sd in enumerate(seeds[:32]):
            g.set_coefficient(C.FMG_K_CELL, learn.block_field(sd))
            g.assemble()
            if learned:
                net.apply(g)
            else:
                for lev in range(g.base + 1, g.top + 1):
                    g.set_node_damping(lev, None)
            xs.fill(0.0)
            ctx.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            _, st1, _ = g.solve(cfg, xs)
            ev1.record(stream)
            ev1.synchronize()
            t_one.append(ev0.elapsed_time(ev1) / 1e3)
            assert st1 == steps[k], (k, st1, steps[k])
        xs.close()
        per_one = float(np.mean(t_one))
        res[name] = {"batch_solve_s": t, "per_field_ms": 1e3 * t / B, "cg_steps_mean": float(np.mean(steps)),
                     "cg_steps_max": int(np.max(steps)), "failed": int(np.sum(status != 0)),
                     "mdof_per_s": B * g.nnodes() / t / 1e6, "setup_s": t_setup,
                     "one_at_a_time_ms_per_field": 1e3 * per_one,
                     "batch_speedup_per_field": per_one / (t / B)}
        x.close()
        batch.close()
    g.close()
    return res


def run_profile_c5(args):
    """The elasticity workloads for ncu captures at `--c5-level`."""
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.learn import DampingNet
    C = G._capi
    wl = problems.c5(level=args.c5_level)
    ctx = G.Context(0)
    g = G.Grid(ctx, 3, wl.order, wl.level, base_level=wl.base_level, n0=wl.n0, ncomp=3,
               dirichlet_mask=wl.dirichlet_mask)
    g.set_coefficient(C.FMG_LAMBDA_MU_CELL, wl.ecell)
    g.set_coefficient(C.FMG_F_VEC, list(wl.force))
    g.assemble()
    if args.profile == "c5mv":
        P = g.vector(values=np.random.default_rng(1).standard_normal(wl.dofs))
        Y = g.vector()
        for _ in range(5):
            g.matvec(P, Y)
        ctx.synchronize()
        print("launches", ctypes_count(C), flush=True)
        return
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, wl.damp, wl.pre, wl.post, 1, 0, 1.0, wl.rtol, 0.0, 300,
                     C.FMG_MULTIPLICATIVE)
    net = DampingNet.load(ctx, WEIGHTS_ELASTIC)
    net.apply(g)
    g.learned_judge_mixed(cfg)
    x = g.vector()
    for _ in range(2):
        x.fill(0.0)
        g.solve_mixed(cfg, x)
    ctx.synchronize()
    print("launches_before_last", ctypes_count(C), flush=True)
    x.fill(0.0)
    _, _, ninner, _ = g.solve_mixed(cfg, x)
    ctx.synchronize()
    print("launches_after", ctypes_count(C), "inner_iterations", ninner, flush=True)


def run_profile_ssc(args):
    """Geometric SSC sweeps on the C2 problem (3D Q2 Poisson) at `--level`:
    the block factorisation once, then 4 sweeps (4 x 8 colour launches)."""
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.iteration import sample_at_gauss_points
    C = G._capi
    wl = problems.c2()
    level = min(args.level, wl.level)
    ctx = G.Context(0)
    g = G.Grid(ctx, 3, 2, level, base_level=wl.base_level)
    g.set_coefficient(C.FMG_F_IP, sample_at_gauss_points(wl.source, 3, 2, 1 << level))
    g.assemble()
    n = g.nnodes()
    x, b, r = g.vector(), g.vector(values=g.rhs()), g.vector()
    for _ in range(4):
        g.ssc(x, b, r, 1.0)
    ctx.synchronize()
    print("launches", ctypes_count(C), "nodes", n, flush=True)
    g.close()
    ctx.close()


def run_profile_c2(args):
    """The C2 V-cycles for ncu captures: the 3D Q2 hierarchy of the C2
    problem at `--level` (6: the configuration), two V(2,2) SOR(1.2) cycles
    and a matvec to warm up, then (after the printed launch count) one
    V(2,2) SOR cycle, one V(1,1) SSC cycle and one top-level matvec inside
    the NVTX range 'c2' (ncu --nvtx --nvtx-include c2/)."""
    import torch

    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.iteration import sample_at_gauss_points
    C = G._capi
    wl = problems.c2()
    level = min(args.level, wl.level)
    ctx = G.Context(0)
    g = G.Grid(ctx, 3, 2, level, base_level=wl.base_level)
    g.set_coefficient(C.FMG_F_IP, sample_at_gauss_points(wl.source, 3, 2, 1 << level))
    g.assemble()
    sor = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SOR, wl.damp, wl.pre, wl.post, 1, 0, 1.0, 0.0, 0.0, 1,
                     C.FMG_MULTIPLICATIVE)
    ssc = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SSC, 1.0, 1, 1, 1, 0, 1.0, 0.0, 0.0, 1, C.FMG_MULTIPLICATIVE)
    n = g.nnodes()
    B = g.vector(values=g.rhs())
    R, X, Y = g.vector(), g.vector(), g.vector()
    for _ in range(2):
        g.vcycle(sor, X, B, R)
    g.vcycle(ssc, X, B, R)
    g.matvec(X, Y)
    ctx.synchronize()
    print("launches_before", ctypes_count(C), "nodes", n, flush=True)
    torch.cuda.nvtx.range_push("c2")
    g.vcycle(sor, X, B, R)
    ctx.synchronize()
    print("launches_after_sor_cycle", ctypes_count(C), flush=True)
    g.vcycle(ssc, X, B, R)
    g.matvec(X, Y)
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    print("launches_after", ctypes_count(C), flush=True)
    g.close()
    ctx.close()


def run_profile_mfs(args):
    """The matrix-free top-level kernels of the mixed solve at `--level`: one
    plain mixed solve (no damping network) leaves their buffers, then one
    launch of each (FMG_MXK_SMOOTH, FMG_MXK_MATVEC64, FMG_MXK_RESIDUAL, and the
    top-level transfers FMG_MXK_RESTRICT, FMG_MXK_PROLONG) inside the NVTX
    range 'mfs' (ncu --nvtx --nvtx-include mfs/)."""
    import torch

    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    C = G._capi
    wl = problems.c3(seed=0, level=args.level)
    ctx = G.Context(0)
    g = G.Grid(ctx, 3, 1, wl.level, base_level=wl.base_level)
    g.set_coefficient(C.FMG_K_CELL, wl.kcell)
    g.assemble()
    x = g.vector()
    g.solve_mixed(plain_cfg(G), x, matrix_free=True)
    ctx.synchronize()
    torch.cuda.nvtx.range_push("mfs")
    for kind in (C.FMG_MXK_SMOOTH, C.FMG_MXK_MATVEC64, C.FMG_MXK_RESIDUAL, C.FMG_MXK_RESTRICT,
                 C.FMG_MXK_PROLONG):
        g.mixed_top_kernel(kind, 1)
    ctx.synchronize()
    torch.cuda.nvtx.range_pop()
    print("mfs kernels launched", flush=True)
    g.close()
    ctx.close()


def run_profile(args):
    """Workloads for ncu captures (profiles/ names the commands)."""
    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.learn import DampingNet
    C = G._capi
    if args.profile in ("c5", "c5mv"):
        return run_profile_c5(args)
    if args.profile == "ssc":
        return run_profile_ssc(args)
    if args.profile == "mfs":
        return run_profile_mfs(args)
    if args.profile == "c2":
        return run_profile_c2(args)
    wl = problems.c3(seed=0, level=args.level)
    ctx = G.Context(0)
    g = G.Grid(ctx, 3, 1, wl.level, base_level=wl.base_level)
    g.set_coefficient(C.FMG_K_CELL, wl.kcell)
    g.assemble()
    cfg = plain_cfg(G)
    net = DampingNet.load(ctx, WEIGHTS)
    if args.profile == "net":
        for _ in range(8):
            net.apply(g)
        ctx.synchronize()
        print("launches", ctypes_count(C), flush=True)
    else:
        net.apply(g)
        g.learned_judge_mixed(cfg)
        x = g.vector()
        for _ in range(2):
            x.fill(0.0)
            g.solve_mixed(cfg, x)
        ctx.synchronize()
        print("launches_before_last", ctypes_count(C), flush=True)
        x.fill(0.0)
        _, _, ninner, _ = g.solve_mixed(cfg, x)
        ctx.synchronize()
        print("launches_after", ctypes_count(C), "inner_iterations", ninner, flush=True)
    net.close()
    g.close()
    ctx.close()


def ctypes_count(C) -> int:
    import ctypes
    v = ctypes.c_longlong(0)
    C.load().fmg_launch_count(ctypes.byref(v))
    return v.value


def run_c2(args):
    """3D Poisson, f = sin(pi x) sin(pi y) sin(pi z), Q2 on 64^3 cells
    (2,146,689 nodes), the multigrid iteration with V(2,2) multicolour
    SOR(1.2), base level 2 (4^3 cells, dense LU), from x = 0 to 1e-10: the
    plain FP64 GPU path, with the oracle (C++ restatement, all host threads)
    timed on a bounded sample of the same solve beside it."""
    import torch

    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from gnu_femlisp_b200.iteration import sample_at_gauss_points
    from oracle import oracle as O
    C = G._capi
    wl = problems.c2()
    n = wl.nodes
    fip = sample_at_gauss_points(wl.source, 3, 2, wl.n_cells)
    ctx = G.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)
    g = G.Grid(ctx, 3, 2, wl.level, base_level=wl.base_level)
    g.set_coefficient(C.FMG_F_IP, fip)
    cfg = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SOR, wl.damp, wl.pre, wl.post, 1, 0, 1.0, wl.rtol, 0.0, 200,
                     C.FMG_MULTIPLICATIVE)

    def timed(fn, reps):
        ctx.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        out = None
        for _ in range(reps):
            out = fn()
        ev1.record(stream)
        ev1.synchronize()
        ctx.synchronize()
        return ev0.elapsed_time(ev1) / 1e3 / reps, out

    for _ in range(2):
        g.assemble()
    t_asm, _ = timed(lambda: g.assemble(), 3)
    x = g.vector()

    def solve():
        x.fill(0.0)
        return g.solve(cfg, x)
    for _ in range(max(args.warmup, 1)):
        solve()
    clocks = ClockSampler(0)
    clocks.start()
    t_solve, (hist, cycles, status) = timed(solve, args.steps)
    B = g.vector(values=g.rhs())
    R, X = g.vector(), g.vector()
    one = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SOR, wl.damp, wl.pre, wl.post, 1, 0, 1.0, 0.0, 0.0, 1,
                     C.FMG_MULTIPLICATIVE)
    for _ in range(3):
        g.vcycle(one, X, B, R)
    t_cycle, _ = timed(lambda: g.vcycle(one, X, B, R), 10)
    P = g.vector(values=np.random.default_rng(1).standard_normal(n))
    Y = g.vector()
    for _ in range(3):
        g.matvec(P, Y)
    t_mv, _ = timed(lambda: g.matvec(P, Y), args.matvec_reps)
    # the reference's own default smoother for Q2 (select-smoother,
    # geomg.lisp:48-60): the vertex-centred geometric SSC, V(1,1), omega 1
    cfg_ssc = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SSC, 1.0, 1, 1, 1, 0, 1.0, wl.rtol, 0.0, 200,
                         C.FMG_MULTIPLICATIVE)

    def solve_ssc():
        x.fill(0.0)
        return g.solve(cfg_ssc, x)
    solve_ssc()
    t_ssc, (hist_ssc, cycles_ssc, status_ssc) = timed(solve_ssc, args.steps)
    one_ssc = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_SSC, 1.0, 1, 1, 1, 0, 1.0, 0.0, 0.0, 1, C.FMG_MULTIPLICATIVE)
    g.vcycle(one_ssc, X, B, R)
    t_cycle_ssc, _ = timed(lambda: g.vcycle(one_ssc, X, B, R), 5)
    clk = clocks.stop()
    if status != 0:
        raise RuntimeError(f"C2 solve did not converge in {cycles} cycles")
    ssc = {"solver": "MG iteration, V(1,1) geometric SSC (vertex-centred 3^3 blocks, omega 1)",
           "time_to_solution_s": t_ssc, "cycles": int(cycles_ssc), "status": int(status_ssc),
           "vcycle_ms": t_cycle_ssc * 1e3, "history_tail": [float(v) for v in hist_ssc[-2:]]}
    nnz = (8 * wl.n_cells + 1) ** 3
    alg_bytes = 8 * nnz + 16 * n
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / t_mv / 1e9
    # CPU: the same algorithm restated in C++ (bitwise the GPU path's
    # arithmetic): assembly, then one complete solve to 1e-10 timed whole; the
    # same run pins the GPU's plain FP64 path at this size (every level matrix,
    # the rhs, the cycle history and the solution)
    cpu, par = None, None
    if not args.no_cpu_baseline:
        O.build()
        x.fill(0.0)
        hist_gpu, _, _ = g.solve(cfg, x)
        x_gpu = x.get()
        o = O.Oracle(3, 2, wl.level, base_level=wl.base_level)
        o.set_coefficient(O.F_IP, fip)
        t0 = time.perf_counter()
        o.assemble()
        t_asm_cpu = time.perf_counter() - t0
        ocfg = O.solve_cfg(method=O.METHOD_MG, smoother=O.SOR, damp=wl.damp, pre=wl.pre, post=wl.post,
                           compat=False, rtol=wl.rtol, maxsteps=200)
        t0 = time.perf_counter()
        ref = o.solve(ocfg)
        t_cpu = time.perf_counter() - t0
        par = parity_block(o, ref, g, hist_gpu, x_gpu, range(wl.base_level, wl.level + 1))
        par.pop("_x_oracle")
        del o
        cpu = {"value": n / t_cpu / 1e6, "unit": "MDoF/s to 1e-10 (N / time-to-solution)",
               "cores": O.num_threads(), "kind": "port",
               "sample": (f"oracle C++ restatement, {O.num_threads()} OpenMP threads: one complete solve to 1e-10 "
                          f"({ref.steps} cycles, {t_cpu:.1f} s) from the assembled hierarchy (assembly "
                          f"{t_asm_cpu:.1f} s, not in value)"),
               "assembly_s": t_asm_cpu, "time_to_solution_s": t_cpu, "cycles": int(ref.steps),
               "host": host_info()}
    line = {"metric": "C2 time to 1e-10 (plain FP64 GPU multigrid, Q2 SOR V(2,2))",
            "value": n / t_solve / 1e6, "unit": "MDoF/s to 1e-10 (N / time-to-solution)", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_solve * 1e3, "higher_is_better": True,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": wl.name, "nodes": n, "nnz": nnz,
                       "solver": "MG iteration, V(2,2) multicolour SOR(1.2), base level 2 dense LU",
                       "l2": "inputs larger than L2 (2.2 GB level-6 matrix)"},
            "time_to_solution_s": t_solve, "cycles": int(cycles), "assembly_s": t_asm,
            "vcycle_ms": t_cycle * 1e3, "mdof_per_s_per_vcycle": n / t_cycle / 1e6,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_spmv<3,2> (top-level FP64 Q2 matvec)", "peak_kind": peak_kind,
                         "algorithmic_bytes": alg_bytes, "launch_ms": t_mv * 1e3},
            "cpu_baseline": cpu, "parity": par, "clocks": clk,
            "history_tail": [float(v) for v in hist[-3:]], "ssc": ssc}
    print(json.dumps(line), flush=True)


def run_c5(args):
    """3D linear elasticity, vector Q2 with 3 x 3 nodal blocks on 48^3 cells
    (2,738,019 DoF), lambda = mu = E log-normal (sigma 0.5), the x = 0 face
    clamped, body force -z: CG preconditioned by the block-Jacobi V(2,2)
    cycle, FP64 on the GPU, from x = 0 to 1e-10; the oracle (C++
    restatement, all host threads) timed beside it on the same problem one
    level down (24^3 cells), its per-step time scaled by the DoF ratio."""
    import torch

    import gnu_femlisp_b200 as G
    from gnu_femlisp_b200 import problems
    from oracle import oracle as O
    C = G._capi
    wl = problems.c5(level=args.c5_level)
    nd = wl.dofs
    ctx = G.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream)

    def timed(fn, reps):
        ctx.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        out = None
        for _ in range(reps):
            out = fn()
        ev1.record(stream)
        ev1.synchronize()
        ctx.synchronize()
        return ev0.elapsed_time(ev1) / 1e3 / reps, out

    g = G.Grid(ctx, 3, wl.order, wl.level, base_level=wl.base_level, n0=wl.n0, ncomp=3,
               dirichlet_mask=wl.dirichlet_mask)
    g.set_coefficient(C.FMG_LAMBDA_MU_CELL, wl.ecell)
    g.set_coefficient(C.FMG_F_VEC, list(wl.force))
    g.assemble()
    t_asm, _ = timed(lambda: g.assemble(), 2)
    cfg = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, wl.damp, wl.pre, wl.post, 1, 0, 1.0, wl.rtol, 0.0, 300,
                     C.FMG_MULTIPLICATIVE)
    x = g.vector()

    def solve():
        x.fill(0.0)
        return g.solve(cfg, x)
    xm = g.vector()

    def solve_mixed():
        xm.fill(0.0)
        return g.solve_mixed(cfg, xm)
    for _ in range(max(args.warmup, 1)):
        solve()
        solve_mixed()
    clocks = ClockSampler(0)
    clocks.start()
    t_solve, (hist, steps, status) = timed(solve, args.steps)
    t_mixed_plain, (_, _, ninner_plain, _) = timed(solve_mixed, args.steps)
    # the learned per-node damping of the block Jacobi (every level), judged by
    # the plain cycle with the mixed solve's CG probe
    from gnu_femlisp_b200.learn import DampingNet
    net = DampingNet.load(ctx, WEIGHTS_ELASTIC)
    ctx.synchronize()
    t0 = time.perf_counter()
    net.apply(g)
    ctx.synchronize()
    t_apply = time.perf_counter() - t0
    ok, rp, rl = g.learned_judge_mixed(cfg)
    ctx.synchronize()
    t_setup = time.perf_counter() - t0
    for _ in range(max(args.warmup, 1)):
        solve_mixed()
    t_mixed, (mhist, nouter, ninner, mstatus) = timed(solve_mixed, args.steps)
    learned_info = {"weights": os.path.relpath(WEIGHTS_ELASTIC, ROOT), "accepted": ok, "rho_plain": rp,
                    "rho_learned": rl, "setup_s": t_setup, "net_apply_s": t_apply, "judge_s": t_setup - t_apply,
                    "status": g.learned_status(),
                    "mixed_without_learned": {"time_to_solution_s": t_mixed_plain,
                                              "inner_iterations": int(ninner_plain)}}
    x64, xmx = x.get(), xm.get()
    tight = G.SolveCfg(C.FMG_METHOD_CG_MG, C.FMG_JACOBI, wl.damp, wl.pre, wl.post, 1, 0, 1.0, 1e-13, 0.0, 400,
                       C.FMG_MULTIPLICATIVE)
    xt = g.vector()
    g.solve(tight, xt)
    xtt = xt.get()
    err_mixed = float(np.linalg.norm(xmx - xtt) / np.linalg.norm(xtt))
    err_plain = float(np.linalg.norm(x64 - xtt) / np.linalg.norm(xtt))
    B = g.vector(values=g.rhs())
    R, X = g.vector(), g.vector()
    one = G.SolveCfg(C.FMG_METHOD_MG, C.FMG_JACOBI, wl.damp, wl.pre, wl.post, 1, 0, 1.0, 0.0, 0.0, 1,
                     C.FMG_MULTIPLICATIVE)
    for _ in range(3):
        g.vcycle(one, X, B, R)
    t_cycle, _ = timed(lambda: g.vcycle(one, X, B, R), 5)
    P = g.vector(values=np.random.default_rng(1).standard_normal(nd))
    Y = g.vector()
    for _ in range(3):
        g.matvec(P, Y)
    t_mv, _ = timed(lambda: g.matvec(P, Y), args.matvec_reps)
    clk = clocks.stop()
    if status != 0 or mstatus != 0:
        raise RuntimeError(f"C5 solve did not converge ({steps} FP64 steps, {ninner} mixed iterations)")
    nnz = 9 * ((8 if wl.order == 2 else 3) * wl.n_cells + 1) ** 3  # scalar nonzeros of the 3 x 3 blocks
    alg_bytes = 8 * nnz + 16 * nd
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / t_mv / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        O.build()
        sl = max(wl.level - 1, 1)
        ws = problems.c5(level=sl)
        o = O.Oracle(3, ws.order, sl, base_level=ws.base_level, ncomp=3, n0=ws.n0, dirichlet_mask=ws.dirichlet_mask)
        o.set_coefficient(O.LAMBDA_MU_CELL, ws.ecell)
        o.set_coefficient(O.F_VEC, list(ws.force))
        t0 = time.perf_counter()
        o.assemble()
        t_asm_cpu = time.perf_counter() - t0
        ocfg = O.solve_cfg(method=O.METHOD_CG_MG, smoother=O.JACOBI, damp=ws.damp, pre=ws.pre, post=ws.post,
                           compat=False, rtol=ws.rtol, maxsteps=2)
        t0 = time.perf_counter()
        r = o.solve(ocfg)
        per_step = (time.perf_counter() - t0) / max(r.steps, 1) * (nd / ws.dofs)
        t_cpu = per_step * steps
        cpu = {"value": nd / t_cpu / 1e6, "unit": "MDoF/s to 1e-10 (DoF / time-to-solution)",
               "cores": O.num_threads(), "kind": "port",
               "sample": (f"oracle C++ restatement, {O.num_threads()} OpenMP threads, on the same problem at "
                          f"{ws.n_cells}^3 cells ({ws.dofs} DoF): assembly {t_asm_cpu:.1f} s, {r.steps} CG steps; "
                          f"per-step time x {nd / ws.dofs:.2f} (DoF ratio) x {steps} steps"),
               "time_to_solution_est_s": t_cpu}
    line = {"metric": ("C5 time to 1e-10 (vector-Q2 elasticity: FP32 block-Jacobi V(2,2) with learned per-node "
                       "damping inside FP64 flexible CG)"),
            "value": nd / t_mixed / 1e6, "unit": "MDoF/s to 1e-10 (DoF / time-to-solution)", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mixed * 1e3, "higher_is_better": True,
            "dtype": "f64 outer residual/update + f32 V-cycle", "data": "synthetic",
            "config": {"workload": wl.name, "dofs": nd, "nnz_scalar": nnz,
                       "solver": (f"FP64 flexible CG + FP32 V({wl.pre},{wl.post}) 3x3 block Jacobi with per-node "
                                  f"damping from the damping network (plain {wl.damp}), base level 0 FP64 dense LU"),
                       "l2": "inputs larger than L2 (8.2 GB level matrix)"},
            "time_to_solution_s": t_mixed, "inner_iterations": int(ninner), "outer_steps": int(nouter),
            "error_vs_fp64": {"mixed_vs_fp64_1e-13": err_mixed, "plain_vs_fp64_1e-13": err_plain},
            "plain_fp64": {"time_to_solution_s": t_solve, "cg_steps": int(steps),
                           "speedup_mixed_vs_plain": t_solve / t_mixed},
            "learned": learned_info,
            "cg_steps": int(steps), "assembly_s": t_asm,
            "vcycle_ms": t_cycle * 1e3, "mdof_per_s_per_vcycle": nd / t_cycle / 1e6,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "kernel": "k_spmv3<2> (top-level FP64 block matvec)", "peak_kind": peak_kind,
                         "algorithmic_bytes": alg_bytes, "launch_ms": t_mv * 1e3},
            "cpu_baseline": cpu, "clocks": clk,
            "history_tail": [float(v) for v in hist[-3:]]}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    try:
        if args.profile:
            if rank == 0:
                run_profile(args)
        elif args.config == "c4":
            if rank == 0:
                run_c4(args)
        elif args.config == "c2":
            if rank == 0:
                run_c2(args)
        elif args.config == "c5":
            if rank == 0:
                run_c5(args)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_mine(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
