"""Throughput of the lbm-fem hot path on B200.

Workload (default): the Taylor-Green throughput scan -- periodic unit square,
Q3 elements on 1024 x 1024 cells (3072^2 = 9,437,184 distinct nodes), D2Q9,
Lee-Lin predictor-corrector, consistent mass: FP64 by Jacobi-PCG to 1e-8 (the
reference default), mixed precision by FP64-residual refinement around the
FP32 tensor-product window solve to 1e-6. Re 100, U0 = 0.05, CFL 0.5,
u = U0 sin(2 pi x) cos(2 pi y) with the matching pressure, f = feq. Synthetic
(analytic) input, state resident in HBM (about 7 GB, far larger than L2, so no
flush is needed between steps). Steps are graph-launched (device-side solver
loops).

A step is one Scheme::step of the whole mesh. Metric: Q.DoF updates/s =
9 x distinct nodes x steps / seconds.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

  python bench.py --streaming tg3|tg3-split [--cfl C]   (Bardow FP64 TG3 step at
  CFL C against TG2 at CFL 0.25 over the same simulated time)

--impl reference times the CPU implementation of the same path on the host
cores (the deal.II reference cannot be built here; the FP64 oracle port of its
algorithm, OpenMP on all cores, stands in for it).
Under torchrun (N > 1) the mesh is cut into N y-strips, one per rank
(lbfem_gpu.strips): ghost rows and CG sums over NCCL, value = the mesh's
units / max-over-ranks device time (strong scaling).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "lbm-fem_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Q·DoF updates/s, mixed vs FP64 on 1 B200 at ≤1e-5 rel. L2; % HBM roofline"
UNIT = "Q·DoF updates/s"


def workload(args):
    from lbfem_gpu import cases, d2q9

    tc = cases.TaylorGreenVortex(0.05 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
    tc.set_reynolds(100)
    mesh = cases.build_mesh(tc, args.cells, args.degree)
    dt, lam = mesh.time_step(0.5), tc.relaxation_time()
    x, y = mesh.nodes()
    f0 = tc.initial_populations(x, y, lam)
    cfg = {
        "workload": f"taylor-green periodic, Q{args.degree} {args.cells}x{args.cells} cells, "
                    f"{args.scheme}, consistent mass (Jacobi-PCG {args.cg_tol:g})",
        "degree": args.degree, "cells": args.cells, "nodes_distinct": mesh.n_unique(), "nodes_stored": mesh.n_dofs,
        "scheme": args.scheme, "mass": "cg", "cg_tolerance": args.cg_tol, "Re": 100, "U0": 0.05, "cfl": 0.5,
        "l2": "state > L2 (no flush needed)",
    }
    return tc, mesh, dt, lam, f0, cfg


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.proc, self.path = device, None, None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "samples": len(rows), "reasons": reasons}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def allreduce_max(pg, v):
    if pg is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_run(tc, mesh, dt, lam, f0, args, budget_s, max_steps, keep=False):
    """The FP64 oracle port on the host cores: warm-up 1 step, then steps until
    budget_s or max_steps. keep: also return the oracle's populations after its
    1 + n steps (the parity check of the FP64 GPU path on the same mesh)."""
    import oracle
    from lbfem_gpu import make_params

    threads = oracle.set_threads(os.cpu_count() or 1)
    h = oracle.Oracle(mesh, make_params(args.scheme, "cg", cg_tolerance=args.cg_tol))
    h.set_time_step(dt, lam)
    h.set_initial_populations(f0)
    h.step(1)
    n, t0 = 0, time.perf_counter()
    while n < max_steps:
        h.step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    sec = time.perf_counter() - t0
    f_end = h.get_populations() if keep else None
    h.close()
    out = (9 * mesh.n_unique() * n / sec, n, sec, threads)
    return out + (f_end,) if keep else out


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    world, rank, local, pg = dist_setup()
    if rank != 0:
        return 0
    tc, mesh, dt, lam, f0, cfg = workload(args)
    budget = float(os.environ.get("LBFEM_CPU_BUDGET_S", "150"))
    value, n, sec, threads = cpu_run(tc, mesh, dt, lam, f0, args, budget, args.steps)
    sample = (f"{n} Lee-Lin steps of the full {args.cells}x{args.cells} Q{args.degree} mesh after 1 warm-up step "
              f"(bounded to {budget:.0f} s), CPU FP64 oracle port, {threads} OpenMP threads, {cpu_model()}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": n,
            "warmup": 1, "ms_per_step": 1e3 * sec / max(n, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# DRAM traffic per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the default
# workload's kernels, from one-pass ncu captures of a launch on the 1024^2 Q3 mesh itself
# (profiles/traffic_tgv_q3_1024.md gives the commands and the read / write split).
STREAMING_TRAFFIC = {"fp64": 1269.1e6, "mixed": 608.9e6}
WINDOW_TRAFFIC = 1476.0e6


def mixed_tol(cg_tol):
    """The relative tolerance of the mixed-precision mass solve (LBFEM_MIXED_TOLERANCE = 1e-6)."""
    return max(cg_tol, 1e-6)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def gpu_states(args, mesh, dt, lam, f0, local, steps, precision="fp64", cg_tol=None):
    """A fresh GPU context of the workload stepped `steps` times from f0 (untimed);
    its populations (FP64, stored numbering)."""
    import lbfem_gpu
    from lbfem_gpu import make_params

    prm = make_params(args.scheme, "cg", cg_tolerance=cg_tol or args.cg_tol, precision=precision, device=local)
    h = lbfem_gpu.Solver(mesh, prm)
    h.set_time_step(dt, lam)
    h.set_initial_populations(f0)
    h.step(steps)
    f = h.get_populations()
    h.close()
    return f


def accuracy_leg(args, mesh, dt, lam, f0, local, steps):
    """Mixed against FP64 on the GPU after `steps` steps of both from f0: relative L2
    of the velocity and of the density deviation over the independent nodes, and
    each run's drift of the mean density."""
    from lbfem_gpu import d2q9

    ind = mesh.independent()
    mom = {}
    for precision in ("fp64", "mixed"):
        f = gpu_states(args, mesh, dt, lam, f0, local, steps, precision)[:, ind]
        mom[precision] = d2q9.moments(f)
    (r64, ux64, uy64), (rm, uxm, uym) = mom["fp64"], mom["mixed"]
    u64 = np.stack([ux64, uy64])
    return {"steps": steps,
            "rel_l2_u_mixed_vs_fp64": float(np.linalg.norm(np.stack([uxm, uym]) - u64) / np.linalg.norm(u64)),
            "rel_l2_drho_mixed_vs_fp64": float(np.linalg.norm(rm - r64) / np.linalg.norm(r64 - 1.0)),
            "mean_density_drift": {"fp64": float(np.mean(r64) - 1.0), "mixed": float(np.mean(rm) - 1.0)},
            "target": 1e-5}


def run_precision(args, precision, tc, mesh, dt, lam, f0, local, pg, world, cg_tol=None, rooflines=True):
    """One timed run of the workload in one precision; returns its figures and final velocity."""
    import ctypes as C

    import lbfem_gpu
    from lbfem_gpu import make_params

    lib = lbfem_gpu.library()
    cg_tol = cg_tol or args.cg_tol
    prm = make_params(args.scheme, "cg", cg_tolerance=cg_tol, precision=precision, device=local)
    h = lbfem_gpu.Solver(mesh, prm)
    h.set_time_step(dt, lam)
    h.set_initial_populations(f0)
    ctx = h.h

    def elapsed(a, b):
        ms = C.c_float()
        h._call("event_elapsed", ctx, a, b, C.byref(ms))
        return ms.value * 1e-3

    h.step(args.warmup)
    lib.lbfem_gpu_synchronize(ctx)
    barrier(pg)
    with Clocks(local) as clocks:
        lib.lbfem_gpu_synchronize(ctx)
        h._call("event_record", ctx, 0)
        h.step(args.steps)
        h._call("event_record", ctx, 1)
        lib.lbfem_gpu_synchronize(ctx)
    sec = allreduce_max(pg, elapsed(0, 1))
    barrier(pg)
    its, launches = C.c_double(), C.c_int64()
    h._call("last_step_stats", ctx, C.byref(its), C.byref(launches))
    cons = h.conservation()
    rho, ux, uy = (np.empty(mesh.n_dofs) for _ in range(3))
    P = C.POINTER(C.c_double)
    h._call("moments", ctx, rho.ctypes.data_as(P), ux.ctypes.data_as(P), uy.ctypes.data_as(P))

    if not rooflines:
        h.close()
        return {"sec": sec, "its": its.value, "launches": int(launches.value), "clocks": clocks.summary()}

    # rooflines, each kernel timed alone on the context's stream (CUDA events, 10 launches)
    reps = 10
    peak, peak_kind = measured_peaks()

    def timed(entry):
        h._call(entry, ctx)
        lib.lbfem_gpu_synchronize(ctx)
        h._call("event_record", ctx, 2)
        for _ in range(reps):
            h._call(entry, ctx)
        h._call("event_record", ctx, 3)
        return elapsed(2, 3) / reps

    def roofline(kernel, alg_bytes, t, traffic):
        achieved = alg_bytes / t / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": kernel, "algorithmic_bytes_per_launch": alg_bytes,
                "launch_ms": 1e3 * t, "peak_kind": f"{peak_kind} HBM copy bandwidth (burst)"}

    tuning = None
    if precision == "mixed":
        shape, tms = C.c_int32(), (C.c_float * 3)()
        h._call("tuning", ctx, C.byref(shape), tms)
        names = ["default", "alternative", "small (3 CTAs per SM)"]
        tuning = {"chosen": names[shape.value] if shape.value >= 0 else None,
                  "ms_per_launch": dict(zip(names, list(tms))),
                  "how": "the three compiled tile shapes timed on the context before its first step (CUDA events)"}
    # the streaming kernel (K1): reads f (9 arrays), writes r (8; Bardow also the 9 collided populations)
    real = 4 if precision == "mixed" else 8
    n_writes = 8 if args.scheme == "leelin" else 17
    default_workload = args.cells == 1024 and args.degree == 3 and args.scheme == "leelin"
    k1 = roofline(f"k_stream_pair<{args.degree}, {args.scheme}> (FP32, population pairs)" if precision == "mixed"
                  else f"k_advection<{args.degree}, {args.scheme} fused, double>",
                  real * mesh.n_dofs * (9 + n_writes), timed("advection_resident"),
                  (STREAMING_TRAFFIC[precision] if default_workload else None))
    if precision == "mixed":
        # the dominant kernel of the mixed step: one round of the mixed solve, 8 systems, reading r, x, b and
        # writing x, r (FP32)
        roof = roofline(f"k_window_correct<{args.degree}> (window solve + FP64 residual, 8 systems)",
                        5 * 4 * 8 * mesh.n_dofs, timed("solve_round_resident"),
                        WINDOW_TRAFFIC if default_workload else None)
    else:
        roof = k1
    if tuning is not None:
        k1["tile_tuning"] = tuning
    out = {"sec": sec, "its": its.value, "launches": int(launches.value), "roofline": roof, "streaming": k1,
           "clocks": clocks.summary(), "mass": cons[1] / cons[0], "u": np.stack([ux, uy]), "handle": h}
    return out


def run_strips(args, world, rank, local, pg):
    """The workload on N GPUs as one mesh cut into N y-strips (lbfem_gpu.strips):
    each rank steps its strip's context; ghost rows and CG sums move over NCCL
    (DistComm). Both precisions, device time on each rank's context stream (CUDA
    events around the K steps, which include the collectives' waits), max over
    ranks. Strong scaling: the mesh is the same for every N."""
    import ctypes as C
    import datetime

    import torch
    import torch.distributed as dist

    import lbfem_gpu
    from lbfem_gpu import make_params, strips

    torch.cuda.set_device(local)
    nccl = dist.new_group(backend="nccl", timeout=datetime.timedelta(seconds=120))
    tc, mesh, dt, lam, f0, cfg = workload(args)
    lib = lbfem_gpu.library()
    st = strips.partition(mesh, world)[rank]
    device = f"cuda:{local}"
    units = 9 * mesh.n_unique() * args.steps
    out = {}
    for precision in ("fp64", "mixed"):
        prm = make_params(args.scheme, "cg", cg_tolerance=args.cg_tol, precision=precision, device=local)
        s = strips.StripSolver(mesh, st, prm, lambda mm, pp: lbfem_gpu.Solver(mm, pp), device,
                               lambda solver: strips.DistComm(st, solver.bufs, nccl))
        s.set_time_step(dt, lam)
        s.set_initial_populations(f0)
        h = s.h
        s.step(args.warmup)
        lib.lbfem_gpu_synchronize(h.h)
        barrier(pg)
        with Clocks(local) as clocks:
            h._call("event_record", h.h, 0)
            s.step(args.steps)
            h._call("event_record", h.h, 1)
            lib.lbfem_gpu_synchronize(h.h)
        ms = C.c_float()
        h._call("event_elapsed", h.h, 0, 1, C.byref(ms))
        sec = allreduce_max(pg, ms.value * 1e-3)
        its, launches = C.c_double(), C.c_int64()
        h._call("last_step_stats", h.h, C.byref(its), C.byref(launches))
        r = {"sec": sec, "its": its.value, "launches": int(launches.value), "clocks": clocks.summary()}
        if precision == "mixed":
            # end to end through the strip's host-buffer calls: this rank's local
            # populations in, one step, its owned populations out
            n_e2e = max(1, min(args.steps, 5))
            loc = s._local(f0)
            barrier(pg)
            t0 = time.perf_counter()
            for _ in range(n_e2e):
                h.set_populations(loc)
                s.step(1)
                s.owned_populations()
            r["e2e_sec"] = allreduce_max(pg, time.perf_counter() - t0)
            r["e2e_steps"] = n_e2e
            lb = 9 * 8 * st.mesh.n_dofs
            ob = 9 * 8 * len(st.owned_index(mesh)[0])
            t = torch.tensor([lb, ob], dtype=torch.float64)
            if pg is not None:
                pg.all_reduce(t)
            r["h2d"], r["d2h"] = int(t[0]), int(t[1])
        s.close()
        out[precision] = r
    if rank != 0:
        return 0
    mix, f64 = out["mixed"], out["fp64"]
    line = {
        "metric": METRIC, "value": units / mix["sec"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * mix["sec"] / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 mixed (FP32 deviations, FP32 streaming/collision and FP32 tensor-product window "
                 "correction; FP64 refinement residuals, dot products and conservation sums)",
        "data": "synthetic (analytic Taylor-Green initial state)",
        "config": dict(cfg, precision="mixed (headline) and fp64",
                       parallelism=f"y-strips x{world} (one mesh; ghost rows and CG sums over NCCL)",
                       mixed_tolerance=mixed_tol(args.cg_tol),
                       solver_iterations_per_solve={"mixed (window corrections)": mix["its"],
                                                    "fp64 (Jacobi-PCG)": f64["its"]}),
        "fp64": {"value": units / f64["sec"], "ms_per_step": 1e3 * f64["sec"] / args.steps,
                 "cg_tolerance": args.cg_tol, "gpu_launches": f64["launches"]},
        "mixed_vs_fp64_speedup": f64["sec"] / mix["sec"],
        "roofline": None, "cpu_baseline": None,
        "e2e": {"value": 9 * mesh.n_unique() * mix["e2e_steps"] / mix["e2e_sec"], "unit": UNIT,
                "h2d_bytes_per_step": mix["h2d"], "d2h_bytes_per_step": mix["d2h"], "steps": mix["e2e_steps"],
                "call": "each rank: set_populations of its local mesh, one strip step, its owned populations out"},
        "clocks": mix["clocks"], "gpu_launches": mix["launches"],
        "timing": "device time per rank (CUDA events on the strip context's stream), max over ranks",
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import ctypes as C

    import lbfem_gpu

    world, rank, local, pg = dist_setup()
    if world > 1:
        return run_strips(args, world, rank, local, pg)
    tc, mesh, dt, lam, f0, cfg = workload(args)
    lib = lbfem_gpu.library()
    ind = mesh.independent()
    runs = {}
    for precision in ("fp64", "mixed"):
        r = run_precision(args, precision, tc, mesh, dt, lam, f0, local, pg, world)
        if precision == "fp64":
            r.pop("handle").close()
        runs[precision] = r
    mix, f64 = runs["mixed"], runs["fp64"]
    h = mix.pop("handle")
    du = mix["u"][:, ind] - f64["u"][:, ind]
    rel_u = float(np.linalg.norm(du) / np.linalg.norm(f64["u"][:, ind]))
    units = 9 * mesh.n_unique() * args.steps * world

    # end to end through the host-buffer C ABI call: upload f, one step, download f
    ctx = h.h
    n_e2e = max(1, min(args.steps, 5))
    fbuf_ptr = lib.lbfem_gpu_host_alloc(9 * mesh.n_dofs * 8)
    fbuf = np.ctypeslib.as_array((C.c_double * (9 * mesh.n_dofs)).from_address(fbuf_ptr))
    fbuf[:] = h.get_populations().ravel()
    P = C.POINTER(C.c_double)
    lib.lbfem_gpu_synchronize(ctx)
    barrier(pg)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        h._call("step_host", ctx, C.cast(fbuf_ptr, P), 1)
    e2e_sec = allreduce_max(pg, time.perf_counter() - t0)
    e2e_value = 9 * mesh.n_unique() * n_e2e * world / e2e_sec
    lib.lbfem_gpu_host_free(fbuf_ptr)
    h.close()

    # the FP64 path at config 0's CG tolerance (1e-12), beside the reference default 1e-8 above
    f64_tight = None
    if not args.no_accuracy:
        f64_tight = run_precision(args, "fp64", tc, mesh, dt, lam, f0, local, pg, world, cg_tol=1e-12,
                                  rooflines=False)

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        budget = float(os.environ.get("LBFEM_CPU_BUDGET_S", "20"))
        cval, cn, csec, threads, f_oracle = cpu_run(tc, mesh, dt, lam, f0, args, budget, 1000, keep=True)
        cpu = {"value": cval, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{cn} step(s) of the full mesh after 1 warm-up step ({csec:.1f} s), CPU FP64 oracle port, "
                         f"{threads} OpenMP threads, {cpu_model()}"}
        # the FP64 GPU path against the oracle on the same mesh, from the same f0, after the same steps
        f_gpu = gpu_states(args, mesh, dt, lam, f0, local, 1 + cn)
        parity = {"rel_l2_fp64_vs_oracle": float(np.linalg.norm(f_gpu - f_oracle) / np.linalg.norm(f_oracle)),
                  "max_abs_fp64_vs_oracle": float(np.max(np.abs(f_gpu - f_oracle))), "steps": 1 + cn,
                  "target": 1e-12, "note": "all 9 population arrays, images included, CG tolerance "
                                           f"{args.cg_tol:g} in both"}
    accuracy_long = None
    if rank == 0 and not args.no_accuracy:
        accuracy_long = accuracy_leg(args, mesh, dt, lam, f0, local, args.accuracy_steps)
    batched = None
    if rank == 0 and world == 1 and not args.no_batch:
        batched = batch_measure(64, 100, 5)
        batched.pop("instances")
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": units / mix["sec"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * mix["sec"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 mixed (FP32 deviations, FP32 streaming/collision and FP32 tensor-product window "
                 "correction; FP64 refinement residuals, dot products and conservation sums)",
        "data": "synthetic (analytic Taylor-Green initial state)",
        "config": dict(cfg, precision="mixed (headline) and fp64", parallelism="single GPU",
                       mixed_tolerance=mixed_tol(args.cg_tol),
                       solver_iterations_per_solve={"mixed (window corrections)": mix["its"],
                                                    "fp64 (Jacobi-PCG)": f64["its"]}),
        "fp64": {"value": units / f64["sec"], "ms_per_step": 1e3 * f64["sec"] / args.steps,
                 "cg_tolerance": args.cg_tol, "roofline": f64["roofline"], "gpu_launches": f64["launches"]},
        "fp64_cg_1e-12": None if f64_tight is None else {
            "value": units / f64_tight["sec"], "ms_per_step": 1e3 * f64_tight["sec"] / args.steps,
            "cg_iterations_per_solve": f64_tight["its"], "gpu_launches": f64_tight["launches"],
            "mixed_vs_this_speedup": f64_tight["sec"] / mix["sec"],
            "note": "config 0's CG tolerance, the other reading of the throughput scan's unstated one"},
        "streaming_kernel": mix["streaming"],
        "accuracy": {"rel_l2_u_mixed_vs_fp64": rel_u, "target": 1e-5, "mean_density_fp64": f64["mass"],
                     "mean_density_mixed": mix["mass"],
                     "note": f"after {args.warmup + args.steps} steps of both runs from the same initial state"},
        "accuracy_long": accuracy_long,
        "parity": parity,
        "mixed_vs_fp64_speedup": f64["sec"] / mix["sec"],
        "roofline": mix["roofline"],
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 9 * 8 * mesh.n_dofs,
                "d2h_bytes_per_step": 9 * 8 * mesh.n_dofs, "steps": n_e2e,
                "call": "lbfem_gpu_step_host on the mixed context (FP64 host populations in, one step, out)"},
        "clocks": mix["clocks"],
        "gpu_launches": mix["launches"],
        "batched": batched,
    }
    print(json.dumps(line))
    return 0


class MT19937_64:
    """The 64-bit Mersenne Twister of Matsumoto and Nishimura (2000), with the
    parameters and seeding of C++'s std::mt19937_64: w = 64, n = 312, m = 156,
    r = 31, a = 0xB5026F5AA96619E9, tempering (u, d) = (29, 0x5555555555555555),
    (s, b) = (17, 0x71D67FFFEDA60000), (t, c) = (37, 0xFFF7EEE000000000), l = 43,
    initialisation multiplier f = 6364136223846793005. __call__ returns the
    engine's next 64-bit output (tests/test_host.py checks the stream against
    std::mt19937_64 compiled here)."""

    N, M = 312, 156
    MASK = (1 << 64) - 1
    UPPER, LOWER = 0xFFFFFFFF80000000, 0x7FFFFFFF

    def __init__(self, seed):
        self.mt = [seed & self.MASK]
        for i in range(1, self.N):
            prev = self.mt[-1]
            self.mt.append((6364136223846793005 * (prev ^ (prev >> 62)) + i) & self.MASK)
        self.i = self.N

    def _twist(self):
        mt = self.mt
        for k in range(self.N):
            y = (mt[k] & self.UPPER) | (mt[(k + 1) % self.N] & self.LOWER)
            v = mt[(k + self.M) % self.N] ^ (y >> 1)
            mt[k] = v ^ 0xB5026F5AA96619E9 if y & 1 else v
        self.i = 0

    def __call__(self):
        if self.i >= self.N:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & self.MASK

    def uniform(self):
        """A double in [0, 1) from the top 53 bits of one output."""
        return (self() >> 11) * (1.0 / (1 << 53))

    def choice(self, values):
        """One of values, uniform: the output modulo len(values) (bias below 1e-18)."""
        return values[self() % len(values)]


def batch_instances(n, seed=20261203):
    """The batched workload: n independent instances drawn from
    std::mt19937_64(seed) (MT19937_64): half lid-driven cavities, half
    Taylor-Green vortices (alternating); then per instance, in this order, the
    mesh edge from {32, 48, 64, 96, 128, 192, 256} cells, the degree 1 or 2,
    Re log-uniform in [100, 1000] and U0 uniform in [0.05, 0.1] (MT19937_64.choice
    and .uniform); mixed precision, consistent mass; Bardow for cavities,
    Lee-Lin for vortices; CFL 0.4."""
    from lbfem_gpu import cases, d2q9, make_params

    rng = MT19937_64(seed)
    out = []
    for k in range(n):
        case = "cavity" if k % 2 == 0 else "tgv"
        edge = int(rng.choice([32, 48, 64, 96, 128, 192, 256]))
        p = int(rng.choice([1, 2]))
        re = float(100.0 * 10 ** rng.uniform())
        u0 = float(0.05 + 0.05 * rng.uniform())
        if case == "cavity":
            tc = cases.LidDrivenCavity(u0, 1.2)
        else:
            tc = cases.TaylorGreenVortex(u0 / math.sqrt(d2q9.CS2), 1, 1, shift=(0.25, 0.25), chapman_enskog=False)
        tc.set_reynolds(re)
        mesh = cases.build_mesh(tc, edge, p)
        scheme = "bardow" if case == "cavity" else "leelin"
        out.append({"case": case, "edge": edge, "p": p, "Re": re, "U0": u0, "scheme": scheme, "tc": tc,
                    "mesh": mesh, "params": make_params(scheme, "cg", precision="mixed")})
    return out


def batch_measure(n, steps, warmup, accuracy_steps=1000):
    """The batched workload of n instances: batched steps (one graph launch per step
    of all of them) in mixed precision and on the plain FP64 path, the same instances
    stepped one at a time in both precisions, and each batched mixed instance's
    relative L2 velocity error against its FP64 run. Device time: CUDA events on the
    batch stream around the batched launches, and on each instance's stream around
    its steps one at a time (summed)."""
    import ctypes as C

    import lbfem_gpu
    from lbfem_gpu import d2q9, make_params

    inst = batch_instances(n)
    lib = lbfem_gpu.library()

    def make(fp64=False):
        hs = []
        for it in inst:
            m, tc = it["mesh"], it["tc"]
            h = lbfem_gpu.Solver(m, make_params(it["scheme"], "cg") if fp64 else it["params"])
            dt, lam = m.time_step(0.4), tc.relaxation_time()
            x, y = m.nodes()
            h.set_time_step(dt, lam)
            h.set_initial_populations(tc.initial_populations(x, y, lam))
            hs.append(h)
        return hs

    def one_at_a_time(hs):
        total = 0.0
        for h in hs:
            h.step(warmup)
            h._call("event_record", h.h, 0)
            h.step(steps)
            h._call("event_record", h.h, 1)
            ms = C.c_float()
            h._call("event_elapsed", h.h, 0, 1, C.byref(ms))
            total += ms.value * 1e-3
        return total

    def batched(hs, more=0, grouped=True):
        # LBFEM_BATCH_GROUP is read when the batch is created
        old = os.environ.get("LBFEM_BATCH_GROUP")
        os.environ["LBFEM_BATCH_GROUP"] = "1" if grouped else "0"
        try:
            b = lbfem_gpu.Batch(hs)
        finally:
            if old is None:
                del os.environ["LBFEM_BATCH_GROUP"]
            else:
                os.environ["LBFEM_BATCH_GROUP"] = old
        b.step(warmup)
        b.step(steps)  # returns after the device finished (one synchronisation)
        sec = b.last_ms() * 1e-3
        launches = b.last_launches()
        if more:
            b.step(more)  # untimed: the longer run of the accuracy check
        b.close()
        return sec, launches

    units = 9 * sum(it["mesh"].n_unique() for it in inst) * steps
    more = max(0, accuracy_steps - warmup - steps)
    hs = make()
    t_batch, n_launch = batched(hs, more)
    f_mixed = [h.get_populations() for h in hs]  # the batched mixed run's end states
    for h in hs:
        h.close()
    hs = make()
    t_branches, n_launch_branches = batched(hs, grouped=False)
    for h in hs:
        h.close()
    hs = make(fp64=True)
    t_batch_fp64, _ = batched(hs, more)
    f_fp64 = [h.get_populations() for h in hs]  # the batched FP64 run (bitwise the one-at-a-time run)
    for h in hs:
        h.close()
    hs = make()
    t_single = one_at_a_time(hs)
    for h in hs:
        h.close()
    hs = make(fp64=True)
    t_fp64 = one_at_a_time(hs)
    for h in hs:
        h.close()
    errs, errs0, decays = [], [], []
    for it, fr, fm in zip(inst, f_fp64, f_mixed):
        ind = it["mesh"].independent()
        _, uxm, uym = d2q9.moments(fm[:, ind])
        _, uxr, uyr = d2q9.moments(fr[:, ind])
        x, y = it["mesh"].nodes()
        _, ux0, uy0 = d2q9.moments(it["tc"].initial_populations(x, y, it["tc"].relaxation_time())[:, ind])
        du = float(np.linalg.norm(np.stack([uxm - uxr, uym - uyr])))
        u_now, u_0 = float(np.linalg.norm(np.stack([uxr, uyr]))), float(np.linalg.norm(np.stack([ux0, uy0])))
        errs.append(du / u_now)
        # against the larger of the initial and the current velocity (cavities start at rest)
        errs0.append(du / max(u_0, u_now))
        decays.append(u_now / u_0 if u_0 > 0 else None)
    worst = int(np.argmax(errs))
    return {"value": units / t_batch, "ms_per_step": 1e3 * t_batch / steps, "steps": steps, "warmup": warmup,
            "gpu_launches": n_launch,
            "branches": {"value": units / t_branches, "ms_per_step": 1e3 * t_branches / steps,
                         "gpu_launches": n_launch_branches,
                         "note": "every instance a graph branch of its own step graph (LBFEM_BATCH_GROUP=0)"},
            "gain_of_grouping": t_branches / t_batch,
            "one_at_a_time": {"value": units / t_single, "ms_per_step": 1e3 * t_single / steps},
            "speedup_vs_one_at_a_time": t_single / t_batch,
            "fp64_one_at_a_time": {"value": units / t_fp64, "ms_per_step": 1e3 * t_fp64 / steps},
            "speedup_vs_fp64_one_at_a_time": t_fp64 / t_batch,
            "fp64_batched": {"value": units / t_batch_fp64, "ms_per_step": 1e3 * t_batch_fp64 / steps},
            "gain_of_precision_batched": t_batch_fp64 / t_batch,
            "gain_of_batching_mixed": t_single / t_batch,
            "gain_of_batching_fp64": t_fp64 / t_batch_fp64,
            "accuracy": {"max_rel_l2_u_mixed_vs_fp64": max(errs), "median": float(np.median(errs)), "target": 1e-5,
                         "instances_above_target": int(sum(e > 1e-5 for e in errs)),
                         "worst": {"instance": worst, "rel_l2_u": errs[worst], "velocity_now_over_initial": decays[worst],
                                   "error_over_larger_of_initial_and_current_velocity": errs0[worst]},
                         "max_error_over_larger_of_initial_and_current_velocity": max(errs0),
                         "rel_l2_u_per_instance": [float(f"{e:.3g}") for e in errs],
                         "velocity_now_over_initial_per_instance": [None if v is None else float(f"{v:.3g}")
                                                                    for v in decays],
                         "note": f"per instance, after {warmup + steps + more} steps of both batched runs; "
                                 "rel_l2_u divides by the FP64 velocity at that time, which decays"},
            "workload": f"{n} instances (cavities and Taylor-Green vortices)",
            "nodes_distinct_total": int(sum(it["mesh"].n_unique() for it in inst)),
            "instances": [{k: it[k] for k in ("case", "edge", "p", "Re", "U0", "scheme")} for it in inst],
            "grouping": "the mixed instances' steps run as grouped kernels, each over the tiles of all "
                        "instances of its degree (one solver loop for all); the FP64 batch is graph branches",
            "timing": "device time: CUDA events on the batch stream around the batched graph launches; "
                      "one at a time, events on each instance's stream around its steps, summed"}


def run_batch(args):
    """Aggregate throughput of the batched instances, against stepping them one at a
    time, in mixed precision and on the plain FP64 path."""
    world, rank, local, pg = dist_setup()
    r = batch_measure(args.batch, args.steps, args.warmup, args.batch_accuracy_steps)
    if rank == 0:
        line = {"metric": "aggregate Q·DoF updates/s of batched independent instances (one graph launch per step)",
                "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": r["ms_per_step"], "higher_is_better": True,
                "one_at_a_time": r["one_at_a_time"], "speedup_vs_one_at_a_time": r["speedup_vs_one_at_a_time"],
                "fp64_one_at_a_time": r["fp64_one_at_a_time"],
                "speedup_vs_fp64_one_at_a_time": r["speedup_vs_fp64_one_at_a_time"], "accuracy": r["accuracy"],
                "gpu_launches": r["gpu_launches"], "branches": r["branches"],
                "gain_of_grouping": r["gain_of_grouping"], "grouping": r["grouping"],
                "fp64_batched": r["fp64_batched"], "gain_of_precision_batched": r["gain_of_precision_batched"],
                "gain_of_batching_mixed": r["gain_of_batching_mixed"],
                "gain_of_batching_fp64": r["gain_of_batching_fp64"],
                "dtype": "f32 mixed", "data": "synthetic",
                "config": {"workload": r["workload"], "nodes_distinct_total": r["nodes_distinct_total"],
                           "instances": r["instances"]},
                "timing": r["timing"]}
        print(json.dumps(line))
    return 0


def run_ladder(args):
    """The Reynolds-continuation ladder of the throughput scan: args.ladder lid-driven
    cavities on args.ladder_cells^2 Q2 cells (Ma 0.1, stretch 1.2, CFL 0.4, Bardow,
    lumped mass as in the reference's cavity continuations, mixed precision), Re
    geometric from 100 to 3200, each rung warm-started from the previous one
    (driver.batched_ladder), args.steps steps per stage. The batched ladder is timed
    against the same ladder stepped one rung at a time. The default mesh is 128^2:
    on 256^2 the Re = 100 rung of this scheme grows without bound within 100 steps
    (both schemes, both masses, CFL 0.4 and 0.2, in the FP64 oracle as well), while
    128^2 holds every rung."""
    import lbfem_gpu
    from lbfem_gpu import cases, driver, make_params

    world, rank, local, pg = dist_setup()
    lib = lbfem_gpu.library()
    reynolds = driver.reynolds_ladder(100.0, 3200.0, args.ladder)
    tc = cases.LidDrivenCavity(0.1, 1.2)
    mesh = cases.build_mesh(tc, args.ladder_cells, 2)
    dt = mesh.time_step(0.4)
    x, y = mesh.nodes()

    def make():
        hs = []
        for k, re in enumerate(reynolds):
            tc.set_reynolds(re)
            h = lbfem_gpu.Solver(mesh, make_params("bardow", "lumped", precision="mixed", device=local))
            h.set_time_step(dt, tc.relaxation_time())
            if k == 0:
                h.set_initial_populations(tc.initial_populations(x, y, tc.relaxation_time()))
            hs.append(h)
        return hs

    def timed(batch):
        hs = make()
        lib.lbfem_gpu_synchronize(hs[0].h)
        barrier(pg)
        t0 = time.perf_counter()
        taken = driver.batched_ladder(hs, args.steps, batch=batch)
        for h in hs:
            lib.lbfem_gpu_synchronize(h.h)
        sec = allreduce_max(pg, time.perf_counter() - t0)
        rho = [float(h.conservation()[1] / h.conservation()[0]) for h in hs]
        for h in hs:
            h.close()
        return sec, taken, rho

    t_batch, taken, rho = timed(True)
    t_single, _, _ = timed(False)
    units = 9 * mesh.n_unique() * sum(taken) * world
    if rank == 0:
        line = {"metric": "aggregate Q·DoF updates/s of a batched Reynolds-continuation ladder (warm-started rungs)",
                "value": units / t_batch, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": 0, "ms_per_stage": 1e3 * t_batch / len(reynolds), "higher_is_better": True,
                "scaling": "weak",
                "one_at_a_time": {"value": units / t_single, "sec": t_single},
                "speedup_vs_one_at_a_time": t_single / t_batch,
                "dtype": "f32 mixed", "data": "synthetic",
                "config": {"workload": f"ladder of {len(reynolds)} lid-driven cavities, Q2 "
                                       f"{args.ladder_cells}x{args.ladder_cells} cells, Re 100 -> 3200",
                           "reynolds": [round(r, 2) for r in reynolds], "steps_per_rung": taken,
                           "nodes_distinct_per_rung": int(mesh.n_unique()), "scheme": "bardow", "mass": "lumped",
                           "cfl": 0.4, "mean_density_per_rung": rho},
                "timing": "host wall clock around the whole ladder, warm starts and graph captures included; "
                          "the first stage steps from the cavity at rest"}
        print(json.dumps(line))
    return 0


def run_streaming(args):
    """TG3 streaming (--streaming tg3 | tg3-split): the Bardow scheme in FP64 on the
    Taylor-Green workload at CFL args.cfl, against TG2 at CFL 0.25 over the same
    simulated time (the reference's comparison, docs/results.md:97-160)."""
    import ctypes as C

    import lbfem_gpu
    from lbfem_gpu import cases, make_params

    world, rank, local, pg = dist_setup()
    tc, mesh, _, lam, f0, cfg = workload(args)
    lib = lbfem_gpu.library()

    def timed_run(streaming, cfl, steps, warmup):
        dt = mesh.time_step(cfl)
        prm = make_params("bardow", "cg", cg_tolerance=args.cg_tol, streaming=streaming, device=local)
        h = lbfem_gpu.Solver(mesh, prm)
        h.set_time_step(dt, lam)
        h.set_initial_populations(f0)
        h.step(warmup)
        lib.lbfem_gpu_synchronize(h.h)
        barrier(pg)
        with Clocks(local) as clocks:
            h._call("event_record", h.h, 0)
            h.step(steps)
            h._call("event_record", h.h, 1)
            lib.lbfem_gpu_synchronize(h.h)
        ms = C.c_float()
        h._call("event_elapsed", h.h, 0, 1, C.byref(ms))
        sec = allreduce_max(pg, ms.value * 1e-3)
        its, launches = C.c_double(), C.c_int64()
        h._call("last_step_stats", h.h, C.byref(its), C.byref(launches))
        t = (warmup + steps) * dt
        err = cases.diagnostics(tc, mesh, h.node_weight(), h.get_populations(), t)["rel_l2_u"]
        h.close()
        return {"sec": sec, "dt": dt, "its": its.value, "launches": int(launches.value), "clocks": clocks.summary(),
                "rel_l2_u_vs_exact": err, "t": t}

    tg3 = timed_run(args.streaming, args.cfl, args.steps, args.warmup)
    ratio = int(round(args.cfl / 0.25))  # TG2 steps per TG3 step over the same simulated time
    tg2 = timed_run("tg2", 0.25, args.steps * ratio, args.warmup * ratio)
    if rank != 0:
        return 0
    units = 9 * mesh.n_unique() * args.steps * world
    sim_rate = lambda r, n: n * r["dt"] / r["sec"]  # noqa: E731 (simulated time per second)
    line = {
        "metric": f"Q·DoF updates/s, Bardow {args.streaming} FP64 at CFL {args.cfl:g} (and time to solution "
                  f"against TG2 at CFL 0.25)",
        "value": units / tg3["sec"], "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tg3["sec"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic Taylor-Green initial state)",
        "config": dict(cfg, workload=cfg["workload"].replace(args.scheme, "bardow"), scheme="bardow",
                       streaming=args.streaming, cfl=args.cfl,
                       solver_iterations_per_solve=tg3["its"], parallelism=f"replicas x{world}" if world > 1
                       else "single GPU"),
        "tg2_cfl_0.25": {"value": 9 * mesh.n_unique() * args.steps * ratio * world / tg2["sec"],
                         "ms_per_step": 1e3 * tg2["sec"] / (args.steps * ratio), "steps": args.steps * ratio,
                         "solver_iterations_per_solve": tg2["its"], "rel_l2_u_vs_exact": tg2["rel_l2_u_vs_exact"]},
        "rel_l2_u_vs_exact": tg3["rel_l2_u_vs_exact"],
        "simulated_time_per_second": {args.streaming: sim_rate(tg3, args.steps),
                                      "tg2": sim_rate(tg2, args.steps * ratio)},
        "time_to_solution_speedup_vs_tg2": tg2["sec"] / tg3["sec"],
        "clocks": tg3["clocks"], "gpu_launches": tg3["launches"],
    }
    print(json.dumps(line))
    return 0


def run_contraction_study(args):
    """The x-pass contraction of the streaming right-hand side alone, on CUDA
    cores and on tensor cores (lbfem_gpu_contraction_study), degree 2 and 3,
    FP32 (TF32 three-term split) and FP64 (DMMA), on the node rows of the
    --cells^2 mesh of each degree. Device time per launch (CUDA events) and the
    relative difference of the two forms' output checksums."""
    import ctypes as C

    import lbfem_gpu

    world, rank, local, pg = dist_setup()
    lib = lbfem_gpu.library()
    fn = lib.lbfem_gpu_contraction_study
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32] * 7 + [C.POINTER(C.c_float), C.POINTER(C.c_double)]
    out = []
    for p in (2, 3):
        rows = p * args.cells + 1
        for fp64 in (0, 1):
            res = {}
            for tensor in (0, 1):
                ms, cs = C.c_float(), C.c_double()
                st = fn(local, p, fp64, tensor, rows, args.cells, args.study_reps, C.byref(ms), C.byref(cs))
                if st != 0:
                    raise RuntimeError(f"contraction study p={p} fp64={fp64} tensor={tensor}: status {st}")
                res[tensor] = (ms.value, cs.value)
            real = 8 if fp64 else 4
            nbytes = 4 * rows * (p * args.cells + 1) * real  # u, h in; y1, y2 out
            out.append({"degree": p, "precision": "fp64 (DMMA)" if fp64 else "fp32 (TF32 x3)",
                        "cuda_core_ms": res[0][0], "tensor_core_ms": res[1][0],
                        "tensor_over_cuda_time": res[1][0] / res[0][0],
                        "cuda_core_gbs": nbytes / res[0][0] / 1e6, "tensor_core_gbs": nbytes / res[1][0] / 1e6,
                        "checksum_rel_diff": abs(res[1][1] - res[0][1]) / abs(res[0][1])})
    if rank == 0:
        print(json.dumps({"study": "x-pass sum-factorisation contraction, CUDA cores vs tensor cores",
                          "grid": f"(p {args.cells} + 1)^2 nodes, two fields in, two assembled rows out",
                          "reps": args.study_reps, "results": out}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=1024)
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--scheme", default="leelin", choices=["leelin", "bardow"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-workload leg (64 instances, mixed batched vs one at a time and FP64)")
    ap.add_argument("--batch-accuracy-steps", type=int, default=10000,
                    help="steps per instance of the --batch leg's mixed-vs-FP64 accuracy check (both batched)")
    ap.add_argument("--batch", type=int, default=0,
                    help="time N batched independent instances (the batched workload) instead of the default")
    ap.add_argument("--ladder", type=int, default=0,
                    help="time a Reynolds-continuation ladder of N cavities (Re 100 -> 3200) instead of the default")
    ap.add_argument("--ladder-cells", type=int, default=128, help="cells per side of each ladder cavity (Q2)")
    ap.add_argument("--streaming", default="tg2", choices=["tg2", "tg3", "tg3-split"],
                    help="tg3 / tg3-split: time the Bardow FP64 TG3 step against TG2 at CFL 0.25 instead")
    ap.add_argument("--cfl", type=float, default=1.0, help="CFL number of the --streaming tg3* run")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the untimed accuracy legs (mixed vs FP64 over --accuracy-steps, FP64 at CG 1e-12)")
    ap.add_argument("--accuracy-steps", type=int, default=500,
                    help="steps of the mixed-vs-FP64 accuracy leg (the throughput scan's 500)")
    ap.add_argument("--cg-tol", type=float, default=1e-8,
                    help="relative CG tolerance of both precisions (MassSettings default 1e-8, mass.h:33)")
    ap.add_argument("--contraction-study", action="store_true",
                    help="time the x-pass contraction on CUDA cores and tensor cores instead of the default")
    ap.add_argument("--study-reps", type=int, default=20)
    args = ap.parse_args()
    if args.contraction_study:
        return run_contraction_study(args)
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.batch and args.impl == "ours":
        return run_batch(args)
    if args.ladder and args.impl == "ours":
        return run_ladder(args)
    if args.streaming != "tg2" and args.impl == "ours":
        return run_streaming(args)
    return run_reference(args) if args.impl == "reference" else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
