#!/usr/bin/env python
"""Benchmark of the alpha-AMG + flexible-CG solve path.

Metric: solves/s to rtol 1e-8.  One step = one complete solve of the
workload: bootstrap setup (matching, aggregation, Galerkin hierarchy) plus
FCG from x0 = 0 plus teardown, i.e. what the reference's solve(A, p, rhs)
does (src/SOLVER/solver.cu:20-129).

  value  inputs (A, b) already resident in HBM (bcmg_setup_device +
         bcmg_solve on device pointers); CUDA events on the library stream.
  e2e    the reference-shaped C-ABI call bcmg_solve_legacy with pinned HOST
         buffers: host->device copies of A, b and x0 and the device->host copy
         of x are inside the timed region.
  roofline  the dominant kernel (level-0 l1-Jacobi sweep) timed live with CUDA
         events; algorithmic bytes from the sweep formula in DESIGN.md.
  cpu_baseline  the CPU oracle (multithreaded FP64 restatement of the same
         method) on a bounded sample of the same workload.

--impl reference times the CPU implementation of the path (the oracle; the
reference itself has no CPU path and its CUDA build needs cuSPARSE routines
removed from CUDA 11+) on the host cores.

Multi-GPU: one solve never shards (global dots every iteration), so N GPUs
run N independent replicas ("scaling": "weak"); value = all solves / the
slowest rank's time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "solves/s to rtol 1e-8, mixed vs FP64 AMG-FCG"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def c1_settings(bc):
    p = bc.Params.default()
    p.solver_type, p.max_hrc, p.conv_ratio = 0, 1, 0.8
    p.aggrsweeps, p.aggrtype, p.max_levels, p.cycle_type = 2, 0, 20, 0
    p.relax_type, p.coarse_solver = 4, 4
    p.prerelax_sweeps, p.postrelax_sweeps, p.relaxnumber_coarse = 4, 4, 16
    p.itnlim, p.rtol = 1000, 1e-8
    return p


def make_workload(bc, name):
    """Synthetic inputs with the shapes and distributions of the configs."""
    p = c1_settings(bc)
    if name == "poisson27_128":
        A = bc.poisson(27, 128, 128, 128)
        b = bc.vector(1, 1, A.n)
        desc = "3-D 27-point Poisson 128^3 (center 26, neighbours -1), b ~ N(0,1) seed 1"
    elif name == "poisson7_32":
        A = bc.poisson(7, 32, 32, 32)
        b = bc.vector(0, 0, A.n)
        desc = "3-D 7-point Poisson 32^3, Dirichlet, b = 1"
    elif name == "fv2d_2048":
        A = bc.fv2d(2048, 2048, seed=2, aniso=1e-3)
        b = bc.vector(2, 2, A.n)
        p.max_hrc, p.conv_ratio, p.solver_type = 3, 0.5, 0
        desc = ("2-D anisotropic FV -div(K grad u) 2048^2, K=exp(2g), g boxed N(0,1), "
                "y-faces x1e-3, bootstrap max_hrc 3 rho 0.5, b ~ U[-1,1] seed 2")
    elif name == "poisson7_96":
        A = bc.poisson(7, 96, 96, 96)
        b = bc.vector(1, 3, A.n)
        desc = "3-D 7-point Poisson 96^3, b ~ N(0,1) seed 3"
    else:
        raise SystemExit(f"unknown workload {name}")
    return A, b, p, desc


def params_dict(p):
    return {k: getattr(p, k) for k in ("solver_type", "max_hrc", "conv_ratio", "aggrsweeps",
                                       "aggrtype", "max_levels", "cycle_type",
                                       "coarse_solver", "relax_type", "relaxnumber_coarse",
                                       "prerelax_sweeps", "postrelax_sweeps", "itnlim",
                                       "rtol")}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel, workload):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(f"{kernel}@{workload}")


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, out_path):
        self.out_path = out_path
        self.proc = None

    def start(self):
        try:
            self.f = open(self.out_path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self, gpu_index=0):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.out_path) as f:
            for line in f:
                parts = [s.strip() for s in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    if int(parts[0]) != gpu_index:
                        continue
                    rows.append(parts)
                except ValueError:
                    continue
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4)
                          if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
def run_cpu_baseline(bc, orc, A, b, p, iters_hint, threads):
    """Oracle on a bounded sample: full setup + 3 FCG iterations, scaled to a
    complete solve with the same iteration count as the GPU FP64 run."""
    orc.set_threads(threads)
    t0 = time.perf_counter()
    h = orc.OracleHandle(A, p)
    setup_s = time.perf_counter() - t0
    k = 3
    # itnlim=k runs the first FCG step plus k loop passes: k+1 preconditioned
    # iterations, the unit the reference's num_iter counts (FCG.cu:569).
    it_s = h.fcg_sample(b, k) / (k + 1)
    h.close()
    per_solve = setup_s + iters_hint * it_s
    return {"value": 1.0 / per_solve, "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": (f"oracle setup ({setup_s:.2f} s) + {k} FCG iterations "
                       f"({it_s:.3f} s each), scaled to {iters_hint} iterations")}


def run_reference(args):
    """CPU implementation of the path (the oracle) on the box's host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import bootcmatchg_b200 as bc
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    A, b, p, desc = make_workload(bc, args.workload)
    t0 = time.perf_counter()
    h = orc.OracleHandle(A, p)
    setup_s = time.perf_counter() - t0
    # One full solve (untimed) gives the iteration count of this workload.
    x, info, _ = h.solve(b)
    iters = info["iters"]
    for _ in range(args.warmup):
        h.fcg_sample(b, 1)
    # itnlim=1 = first FCG step + one loop pass = 2 preconditioned iterations.
    samples = [h.fcg_sample(b, 1) / 2 for _ in range(args.steps)]
    it_s = statistics.median(samples)
    per_solve = setup_s + iters * it_s
    value = 1.0 / per_solve
    sample = (f"setup {setup_s:.2f} s once + {iters} iterations x median of {args.steps} "
              f"two-iteration samples ({it_s:.3f} s per iteration)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": it_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": desc,
                       "params": params_dict(p), "n": A.n, "nnz": A.nnz},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "detail": {"iters": iters, "setup_s": setup_s, "iter_s": it_s}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    import bootcmatchg_b200 as bc
    from bootcmatchg_b200._lib import check, lib, Csr

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    A, b_h, p, desc = make_workload(bc, args.workload)
    prec = bc.PREC_MIXED if args.precision == "mixed" else bc.PREC_FP64
    stream = torch.cuda.Stream(device=dev)
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0, device=local,
                        stream=stream.cuda_stream)

    with torch.cuda.stream(stream):
        row = torch.from_numpy(A.row).to(dev)
        col = torch.from_numpy(A.col).to(dev)
        val = torch.from_numpy(A.val).to(dev)
        b = torch.from_numpy(b_h).to(dev)
        x = torch.zeros(A.n, dtype=torch.float64, device=dev)
    stream.synchronize()

    def step():
        h = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(),
                                  p, ext)
        with torch.cuda.stream(stream):
            x.zero_()
        info = h.solve_device(b.data_ptr(), x.data_ptr())
        h.close()
        return info

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        info = step()
    if not info.converged:
        raise SystemExit(f"warm-up solve did not converge: {info}")

    sampler = ClockSampler(os.path.join(ROOT, "gpurun_out" if os.path.isdir(
        os.path.join(ROOT, "gpurun_out")) else ".", f"clocks_rank{rank}.csv"))
    barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    l0 = lib.bcmg_kernel_launches()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    infos = [step() for _ in range(args.steps)]
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    launches = lib.bcmg_kernel_launches() - l0
    clocks = sampler.stop(local)
    ms = t_start.elapsed_time(t_end)
    ms_max = ms
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * args.steps / (ms_max / 1e3)
    info = infos[-1]
    xs = x.cpu().numpy()
    res = b_h - A.to_scipy() @ xs
    true_rel = float(np.linalg.norm(res) / np.linalg.norm(b_h))

    # ---- e2e: reference-shaped C-ABI call with pinned host buffers -----------
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    h_row, h_col, h_val, h_b = pin(A.row), pin(A.col), pin(A.val), pin(b_h)
    h_x = torch.zeros(A.n, dtype=torch.float64).pin_memory()
    c = Csr()
    c.n, c.m, c.nnz = A.n, A.n, A.nnz
    c.row = C.cast(h_row.data_ptr(), C.POINTER(C.c_int32))
    c.col = C.cast(h_col.data_ptr(), C.POINTER(C.c_int32))
    c.val = C.cast(h_val.data_ptr(), C.POINTER(C.c_double))
    pc, ec = p.to_c(), ext.to_c()
    from bootcmatchg_b200._lib import SolveInfo

    def e2e_step():
        si = SolveInfo()
        check(lib.bcmg_solve_legacy(C.byref(c), C.byref(pc), C.byref(ec),
                                    C.c_void_p(h_b.data_ptr()), C.c_void_p(h_x.data_ptr()),
                                    C.byref(si)), "bcmg_solve_legacy")
        return si

    e2e_steps = max(1, min(args.steps, 3))
    e2e_step()
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    e2e_value = world * e2e_steps / (e_ms / 1e3)
    h2d = (A.n + 1) * 4 + A.nnz * 12 + A.n * 8 * 2
    d2h = A.n * 8

    # ---- roofline: level-0 smoother sweep, timed live ---------------------
    # The dominant kernel of the solve: the level-0 l1-Jacobi sweep, run
    # through bcmg_level_relax exactly as the cycle runs it (solve format and
    # precision), timed with CUDA events on the library stream.
    h = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(), p, ext)
    slots, cslots = C.c_int64(), C.c_int64()
    nsl, vbytes = C.c_int32(), C.c_int32()
    check(lib.bcmg_level_format(h.ptr, 0, 0, C.byref(slots), C.byref(cslots), C.byref(nsl),
                                C.byref(vbytes)), "level_format")
    xdt = torch.float32 if prec == bc.PREC_MIXED else torch.float64
    xbytes = 4 if prec == bc.PREC_MIXED else 8
    with torch.cuda.stream(stream):
        f = torch.from_numpy(b_h).to(dev).to(xdt)
        u = torch.from_numpy(bc.vector(1, 5, A.n)).to(dev).to(xdt)
    stream.synchronize()
    sweeps = 20
    check(lib.bcmg_level_relax(h.ptr, 0, 0, C.c_void_p(f.data_ptr()), C.c_void_p(u.data_ptr()),
                               2), "level_relax warmup")
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    check(lib.bcmg_level_relax(h.ptr, 0, 0, C.c_void_p(f.data_ptr()), C.c_void_p(u.data_ptr()),
                               sweeps), "level_relax")
    r1.record(stream)
    torch.cuda.synchronize(dev)
    h.close()
    sweep_s = r0.elapsed_time(r1) / 1e3 / sweeps
    if vbytes.value:
        # sliced copy: values incl. padding, explicit columns, per-slice
        # metadata, and u (gathered once), f, d read + u' written
        sweep_bytes = (vbytes.value * 32 * slots.value + 4 * 32 * cslots.value +
                       16 * nsl.value + 4 * xbytes * A.n)
        kname = "k_sl_relax (level-0 l1-Jacobi sweep, sliced)"
    else:
        sweep_bytes = 12 * A.nnz + 4 * (A.n + 1) + 36 * A.n
        kname = "k_relax_t (level-0 l1-Jacobi sweep, CSR)"
    csr_equiv = 12 * A.nnz + 4 * (A.n + 1) + 36 * A.n
    achieved = sweep_bytes / sweep_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic = committed_traffic("k_sl_relax", f"{args.workload}:{args.precision}")

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        try:
            cpu = run_cpu_baseline(bc, orc, A, b_h, p, info.iters, os.cpu_count() or 1)
        except Exception as exc:  # the baseline never blocks the GPU line
            cpu = {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {exc}"}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    dtype = "f32+f64" if prec == bc.PREC_MIXED else "f64"
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "precision": args.precision,
                   "params": params_dict(p), "n": A.n, "nnz": A.nnz,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs (%.0f MB matrix) larger than the 126 MB L2; no flush" %
                         ((A.nnz * 12) / 1e6),
                   "step": "setup (bootstrap hierarchy) + FCG solve + teardown"},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": {"kernel": kname, "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes": sweep_bytes,
                     "csr_fp64_equivalent_bytes": csr_equiv,
                     "launch_ms": sweep_s * 1e3},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "detail": {"iters": info.iters, "setup_ms": info.setup_ms, "solve_ms": info.solve_ms,
                   "rel_residual": info.rel_residual, "true_rel_residual": true_rel,
                   "e2e_steps": e2e_steps},
    }
    print(json.dumps(line), flush=True)
    log(f"[bench] {args.workload} {args.precision}: {value:.3f} solves/s "
        f"({ms_max / args.steps:.1f} ms/solve, iters {info.iters}, setup {info.setup_ms:.1f} ms,"
        f" solve {info.solve_ms:.1f} ms), e2e {e2e_value:.3f} solves/s, "
        f"sweep {achieved:.0f} GB/s ({achieved / peak:.2f} of {peak_kind} peak)")
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="poisson27_128",
                    choices=["poisson27_128", "poisson7_32", "fv2d_2048", "poisson7_96"])
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        log("[bench] warm-up raised to the minimum of 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
