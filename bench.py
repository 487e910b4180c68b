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
         events; algorithmic bytes = stored values (slots x 32 x value bytes)
         + explicit columns + 16 B of metadata per 32-row slice + u, f, d read
         and u' written (4 n x vector bytes).
  cpu_baseline  the CPU oracle (multithreaded FP64 restatement of the same
         method): one complete, timed solve of the workload on all host
         threads, plus a 1-thread figure (setup timed in full, FCG iterations
         from a timed sample); its solution also gives detail.err_vs_oracle.

--impl reference times the CPU implementation of the path on the host cores:
the oracle (the reference has no CPU path, and its own GPU solve stopped with
an illegal memory access on these inputs, so it is not run); every step is
one complete solve.  It loads no product library.

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

import workloads as wl  # noqa: E402  (seeded synthetic inputs; not the product)

METRIC = "solves/s to rtol 1e-8, mixed vs FP64 AMG-FCG"
BATCH_RHS = 32


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def c1_settings():
    """The 7-point Poisson 32^3 settings (single hierarchy, aggrsweeps 2,
    unsmoothed, 20 levels, V-cycle, l1 smoother and l1 coarse solver, 4/4
    sweeps, 16 coarse sweeps, itnlim 1000, rtol 1e-8); the other workloads
    take them for every field they do not name.  A plain namespace, so the
    CPU arm never loads the product library; the GPU arms convert it with
    product_params()."""
    import types
    return types.SimpleNamespace(
        solver_type=0, max_hrc=1, conv_ratio=0.8, matchtype=3, aggrsweeps=2, aggrtype=0,
        max_levels=20, cycle_type=0, coarse_solver=4, relax_type=4, prerelax_sweeps=4,
        postrelax_sweeps=4, itnlim=1000, rtol=1e-8, relaxnumber_coarse=16)


def product_params(bc, p):
    return bc.Params(**vars(p))


def make_workload(name):
    """Synthetic inputs with the shapes and distributions of the configs."""
    p = c1_settings()
    if name == "poisson27_128":
        A = wl.poisson(27, 128, 128, 128)
        b = wl.vector(1, 1, A.n)
        desc = "3-D 27-point Poisson 128^3 (center 26, neighbours -1), b ~ N(0,1) seed 1"
    elif name == "poisson7_32":
        A = wl.poisson(7, 32, 32, 32)
        b = wl.vector(0, 0, A.n)
        desc = "3-D 7-point Poisson 32^3, Dirichlet, b = 1"
    elif name == "fv2d_2048":
        A = wl.fv2d(2048, 2048, seed=2, aniso=1e-3)
        b = wl.vector(2, 2, A.n)
        p.max_hrc, p.conv_ratio, p.solver_type = 3, 0.5, 0
        desc = ("2-D anisotropic FV -div(K grad u) 2048^2, K=exp(2g), g boxed N(0,1), "
                "y-faces x1e-3, bootstrap max_hrc 3 rho 0.5, b ~ U[-1,1] seed 2")
    elif name == "poisson7_96":
        A = wl.poisson(7, 96, 96, 96)
        b = wl.vector(1, 3, A.n)
        desc = "3-D 7-point Poisson 96^3, b ~ N(0,1) seed 3"
    elif name == "rgg_2m":
        A = wl.rgg(2_000_000, seed=4)
        b = wl.vector(1, 4, A.n)
        desc = ("random geometric graph Laplacian, 2,000,000 points in the unit cube, mean "
                "degree 12, weights U[0.5, 2], shift 1e-3 (the largest graphs of the served "
                "stream), b ~ N(0,1) seed 4")
    elif name == "poisson7_96_x32":
        A = wl.poisson(7, 96, 96, 96)
        # 32 right-hand sides: one N(0,1) stream from seed 3, column-major.
        b = np.asfortranarray(wl.vector(1, 3, A.n * BATCH_RHS).reshape(A.n, BATCH_RHS,
                                                                       order="F"))
        desc = ("3-D 7-point Poisson 96^3 with 32 simultaneous right-hand sides "
                "~ N(0,1) seed 3 (column-major), one shared hierarchy")
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
        """Starts sampling every 100 ms and returns once the first sample is
        written (up to 5 s), so that a timed region of a few hundred
        milliseconds is covered from its start."""
        try:
            self.f = open(self.out_path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            try:
                with open(self.out_path) as f:
                    if any(line.count(",") >= 8 for line in f):
                        break
            except OSError:
                pass
            time.sleep(0.02)

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


def aggregate_over_ranks(ms_local, steps, units_per_step, world, dist=None, device=None):
    """Whole-job throughput of N replicas: the slowest rank's device time
    (MAX over ranks) and all ranks' units divided by it."""
    ms = ms_local
    if world > 1:
        import torch
        t = torch.tensor([ms_local], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * steps * units_per_step / (ms / 1e3)


# ---------------------------------------------------------------------------
def clock_dir():
    """Where the nvidia-smi clock samples of the timed region go
    (BCMG_CLOCK_DIR, else the system temporary directory)."""
    import tempfile
    return os.environ.get("BCMG_CLOCK_DIR") or tempfile.gettempdir()


def oracle_full_solve(orc, A, b, p, threads):
    """One complete oracle solve (bootstrap setup + FCG from x0 = 0 to rtol)
    on `threads` host threads, timed on the host clock."""
    orc.set_threads(threads)
    t0 = time.perf_counter()
    h = orc.OracleHandle(A, p)
    t1 = time.perf_counter()
    x, info, st = h.solve(b)
    t2 = time.perf_counter()
    if st != 0 or not info["converged"]:
        raise RuntimeError(f"oracle solve did not converge (status {st}, {info})")
    return {"x": x, "iters": info["iters"], "setup_s": t1 - t0, "solve_s": t2 - t1,
            "total_s": t2 - t0, "handle": h}


def one_core_figure(orc, A, b, p, iters):
    """The 1-thread figure beside the all-core one: 1-thread setup, timed in
    full, plus a timed 2-iteration FCG sample scaled to `iters` iterations
    (a complete 1-thread solve of the large workloads takes minutes)."""
    orc.set_threads(1)
    try:
        t0 = time.perf_counter()
        h = orc.OracleHandle(A, p)
        setup_s = time.perf_counter() - t0
        # itnlim=1 = first FCG step + one loop pass: 2 preconditioned
        # iterations, the unit the reference's num_iter counts (FCG.cu:569).
        it_s = h.fcg_sample(b, 1) / 2
        h.close()
    finally:
        orc.set_threads(os.cpu_count() or 1)
    per = setup_s + iters * it_s
    return {"value": 1.0 / per, "unit": "solves/s", "cores": 1,
            "sample": (f"1-thread setup ({setup_s:.2f} s, timed) + a timed 2-iteration FCG "
                       f"sample ({it_s:.3f} s per iteration) scaled to {iters} iterations")}


def run_cpu_baseline(orc, A, b, p, threads, nrhs=1):
    """The oracle on the host cores: one complete, timed solve of the
    workload (setup + FCG to convergence) on all threads; for nrhs > 1 the
    setup is shared and every column's solve is counted at that one column's
    solve time.  Also returns the oracle's solution for the error figure."""
    full = oracle_full_solve(orc, A, b, p, threads)
    full["handle"].close()
    per = (full["setup_s"] + nrhs * full["solve_s"]) / nrhs
    sample = (f"one complete oracle solve timed on {threads} threads: setup "
              f"{full['setup_s']:.2f} s + {full['iters']} FCG iterations {full['solve_s']:.2f} s")
    if nrhs > 1:
        sample += f"; one setup shared by {nrhs} right-hand sides, each at that solve time"
    out = {"value": 1.0 / per, "unit": "solves/s", "cores": threads, "kind": "port",
           "sample": sample, "setup_s": full["setup_s"], "solve_s": full["solve_s"],
           "iters": full["iters"]}
    out["one_core"] = one_core_figure(orc, A, b, p, full["iters"])
    return out, full["x"]


def run_reference(args):
    """The reference's method on the host cores: the multithreaded FP64 CPU
    oracle (the reference has no CPU path of its own, and its GPU solve is not
    run: it stopped with an illegal memory access on these inputs).  One step
    = one complete solve (setup + FCG to rtol) of the workload, timed on the
    host clock; the multi-right-hand-side workload shares one setup among its
    32 columns and solves every column."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    if args.workload == "serve_stream":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the served stream has no CPU counterpart: the oracle solves "
                          "one request at a time and the reference has no server"}))
        return 0
    A, b, p, desc = make_workload(args.workload)
    cols = [b] if b.ndim == 1 else [np.ascontiguousarray(b[:, j]) for j in range(b.shape[1])]
    nrhs = len(cols)

    def step():
        t0 = time.perf_counter()
        h = orc.OracleHandle(A, p)
        iters = []
        for c in cols:
            x, info, st = h.solve(c)
            if st != 0 or not info["converged"]:
                raise RuntimeError(f"oracle solve did not converge: {info}")
            iters.append(info["iters"])
        h.close()
        return time.perf_counter() - t0, iters

    for _ in range(args.warmup):
        step()
    times, iters = [], []
    for _ in range(args.steps):
        t, it = step()
        times.append(t)
        iters = it
    total = sum(times)
    value = args.steps * nrhs / total
    sample = (f"{args.steps} complete oracle solves (setup + FCG to rtol) timed on {threads} "
              f"threads, median {statistics.median(times):.2f} s")
    if nrhs > 1:
        sample = (f"{args.steps} steps of one oracle setup + {nrhs} complete column solves, "
                  f"timed on {threads} threads, median {statistics.median(times):.2f} s")
    one = one_core_figure(orc, A, cols[0], p, iters[0])
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": desc,
                       "params": params_dict(p), "n": A.n, "nnz": A.nnz, "nrhs": nrhs},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads,
                             "kind": "port", "sample": sample, "one_core": one},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "detail": {"iters": iters, "step_s": times}}
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

    A, b_h, p_plain, desc = make_workload(args.workload)
    p = product_params(bc, p_plain)
    prec = bc.PREC_MIXED if args.precision == "mixed" else bc.PREC_FP64
    stream = torch.cuda.Stream(device=dev)
    # The anisotropic FV workload stores its coarse levels in BF16 (FP32
    # accumulation); the others keep FP32 coarse values.
    storage = bc.STORE_BF16 if args.workload == "fv2d_2048" else bc.STORE_FP32
    ext = bc.Extensions(precision=prec, coarse_storage=storage, replace_every=10 if prec else 0,
                        device=local, stream=stream.cuda_stream)

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

    sampler = ClockSampler(os.path.join(clock_dir(), f"clocks_rank{rank}.csv"))
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
    ms_max, value = aggregate_over_ranks(t_start.elapsed_time(t_end), args.steps, 1, world,
                                         dist, dev)
    info = infos[-1]
    xs = x.cpu().numpy()
    res = b_h - A.to_scipy() @ xs
    true_rel = float(np.linalg.norm(res) / np.linalg.norm(b_h))

    # ---- comparison legs (same process, same inputs, untimed by the driver) ----
    def timed_ms(fn, reps):
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = [fn() for _ in range(reps)]
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps, out

    def cached_ms(ext_):
        # solves on one hierarchy, setup excluded (the reference's solve_time)
        hh = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(),
                                   p, ext_)

        def one():
            with torch.cuda.stream(stream):
                x.zero_()
            return hh.solve_device(b.data_ptr(), x.data_ptr())
        one()
        ms, out = timed_ms(one, max(3, args.steps))
        hh.close()
        return ms, out[-1].iters

    # The comparison denominator is the plain FP64 path: FP64 values, no
    # exact narrowing of the stored values.
    ext64 = bc.Extensions(precision=bc.PREC_FP64, device=local, stream=stream.cuda_stream,
                          narrow_values=0)
    compare = {}
    x64 = None
    if prec == bc.PREC_MIXED:
        ext_saved = ext
        ext = ext64
        step()
        fp64_ms, fp64_infos = timed_ms(step, args.steps)
        ext = ext_saved
        x64 = x.cpu().numpy()
        compare["fp64_full_solve"] = {"solves_per_s": 1e3 / fp64_ms, "ms_per_solve": fp64_ms,
                                      "iters": fp64_infos[-1].iters,
                                      "setup_ms": fp64_infos[-1].setup_ms}
        compare["mixed_over_fp64_full_solve"] = fp64_ms / (ms_max / args.steps)
    mixed_c, mixed_it = cached_ms(ext)
    compare["cached_hierarchy"] = {"ms_per_solve": mixed_c, "solves_per_s": 1e3 / mixed_c,
                                   "iters": mixed_it}
    if prec == bc.PREC_MIXED:
        fp64_c, fp64_it = cached_ms(ext64)
        compare["cached_hierarchy"].update({"fp64_ms_per_solve": fp64_c,
                                            "fp64_solves_per_s": 1e3 / fp64_c,
                                            "fp64_iters": fp64_it,
                                            "mixed_over_fp64": fp64_c / mixed_c})
        ext64n = bc.Extensions(precision=bc.PREC_FP64, device=local, stream=stream.cuda_stream)
        fp64n_c, _ = cached_ms(ext64n)
        compare["cached_hierarchy"]["fp64_narrowed_ms_per_solve"] = fp64n_c

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
    e_ms, e2e_value = aggregate_over_ranks(e0.elapsed_time(e1), e2e_steps, 1, world, dist,
                                           dev)
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
        u = torch.from_numpy(wl.vector(1, 5, A.n)).to(dev).to(xdt)
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
        kname = "k_sl_pipe<EpiRelax> (level-0 l1-Jacobi sweep, sliced, pipelined)"
    else:
        sweep_bytes = 12 * A.nnz + 4 * (A.n + 1) + 36 * A.n
        kname = "k_relax_t (level-0 l1-Jacobi sweep, CSR)"
    csr_equiv = 12 * A.nnz + 4 * (A.n + 1) + 36 * A.n
    achieved = sweep_bytes / sweep_s / 1e9
    peak, peak_kind = measured_peaks()
    # keyed by the copy's value width: a capture of another storage format
    # (FP32 values, BF16 values) does not describe this launch
    traffic = committed_traffic("k_sl_pipe",
                                f"{args.workload}:{args.precision}:{vbytes.value}B")

    cpu, err = None, {}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        try:
            cpu, x_orc = run_cpu_baseline(orc, A, b_h, p_plain, os.cpu_count() or 1)
            # error of the GPU solutions against the FP64 oracle's solution of
            # the same PCG + AMG (same settings, same right-hand side)
            nrm = np.linalg.norm(x_orc)
            err["err_vs_oracle"] = float(np.linalg.norm(xs - x_orc) / nrm)
            if x64 is not None:
                err["fp64_err_vs_oracle"] = float(np.linalg.norm(x64 - x_orc) / nrm)
            err["oracle_iters"] = cpu["iters"]
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
                   **err, "e2e_steps": e2e_steps, "compare": compare,
                   "level0_cycle_value_bytes": vbytes.value},
    }
    print(json.dumps(line), flush=True)
    log(f"[bench] {args.workload} {args.precision}: {value:.3f} solves/s "
        f"({ms_max / args.steps:.1f} ms/solve, iters {info.iters}, setup {info.setup_ms:.1f} ms,"
        f" solve {info.solve_ms:.1f} ms), e2e {e2e_value:.3f} solves/s, "
        f"sweep {achieved:.0f} GB/s ({achieved / peak:.2f} of {peak_kind} peak)")
    return 0


def run_batch(args):
    """Multi-right-hand-side workload: one step = setup of the shared
    hierarchy + bcmg_solve_batch of all 32 columns + teardown; value counts
    every column as one solve."""
    import torch
    import torch.distributed as dist

    import bootcmatchg_b200 as bc
    from bootcmatchg_b200._lib import check, lib, Csr, SolveInfo

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
    A, B_h, p_plain, desc = make_workload(args.workload)
    p = product_params(bc, p_plain)
    nrhs = B_h.shape[1]
    prec = bc.PREC_MIXED if args.precision == "mixed" else bc.PREC_FP64
    stream = torch.cuda.Stream(device=dev)
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0, device=local,
                        stream=stream.cuda_stream)
    with torch.cuda.stream(stream):
        row = torch.from_numpy(A.row).to(dev)
        col = torch.from_numpy(A.col).to(dev)
        val = torch.from_numpy(A.val).to(dev)
        # Column-major n x nrhs on the device: row j of a (nrhs, n) tensor is
        # column j.
        Bd = torch.from_numpy(np.ascontiguousarray(B_h.T)).to(dev)
        Xd = torch.zeros_like(Bd)
    stream.synchronize()

    def step():
        h = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(),
                                  p, ext)
        with torch.cuda.stream(stream):
            Xd.zero_()
        infos = h.solve_batch_device(nrhs, Bd.data_ptr(), A.n, Xd.data_ptr(), A.n)
        h.close()
        return infos

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        infos = step()
    if not all(i.converged for i in infos):
        raise SystemExit("warm-up batch did not converge")
    sampler = ClockSampler(os.path.join(clock_dir(), f"clocks_rank{rank}.csv"))
    barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    l0 = lib.bcmg_kernel_launches()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    all_infos = [step() for _ in range(args.steps)]
    t1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    launches = lib.bcmg_kernel_launches() - l0
    clocks = sampler.stop(local)
    ms_max, value = aggregate_over_ranks(t0.elapsed_time(t1), args.steps, nrhs, world, dist,
                                         dev)
    infos = all_infos[-1]
    X = Xd.cpu().numpy().T
    As = A.to_scipy()
    true_rel = max(float(np.linalg.norm(B_h[:, j] - As @ X[:, j]) / np.linalg.norm(B_h[:, j]))
                   for j in range(nrhs))

    # Solve-only rate (hierarchy kept) and the one-column-at-a-time rate on
    # the same handle, for the batching gain.
    h = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(), p, ext)
    h.solve_batch_device(nrhs, Bd.data_ptr(), A.n, Xd.data_ptr(), A.n)
    torch.cuda.synchronize(dev)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    with torch.cuda.stream(stream):
        Xd.zero_()
    h.solve_batch_device(nrhs, Bd.data_ptr(), A.n, Xd.data_ptr(), A.n)
    s1.record(stream)
    torch.cuda.synchronize(dev)
    batch_solve_ms = s0.elapsed_time(s1)
    with torch.cuda.stream(stream):
        xs = torch.zeros(A.n, dtype=torch.float64, device=dev)
    stream.synchronize()
    single = []
    for j in range(min(nrhs, 8)):
        with torch.cuda.stream(stream):
            xs.zero_()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        si = h.solve_device(Bd[j].data_ptr(), xs.data_ptr())
        g1.record(stream)
        torch.cuda.synchronize(dev)
        single.append((g0.elapsed_time(g1), si.iters))
    cfg = [h.batch_config(nrhs, 0, l) for l in range(h.hierarchy_info(0)["num_levels"])]
    # The plain FP64 path (FP64 hierarchy and cycle, no value narrowing), one
    # column at a time on its own handle: the denominator of the batching and
    # mixed-precision gain.
    ext64 = bc.Extensions(precision=bc.PREC_FP64, narrow_values=0, device=local,
                          stream=stream.cuda_stream)
    h64 = bc.Handle.from_device(A.n, A.nnz, row.data_ptr(), col.data_ptr(), val.data_ptr(), p,
                                ext64)
    fp64_single = []
    for j in range(4):
        with torch.cuda.stream(stream):
            xs.zero_()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        si = h64.solve_device(Bd[j].data_ptr(), xs.data_ptr())
        g1.record(stream)
        torch.cuda.synchronize(dev)
        fp64_single.append((g0.elapsed_time(g1), si.iters))
    # The same plain FP64 path batched: all columns in one solve on the FP64
    # handle (warmed once), so batching and precision gains are separable.
    with torch.cuda.stream(stream):
        Xd.zero_()
    h64.solve_batch_device(nrhs, Bd.data_ptr(), A.n, Xd.data_ptr(), A.n)
    with torch.cuda.stream(stream):
        Xd.zero_()
    torch.cuda.synchronize(dev)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    infos64 = h64.solve_batch_device(nrhs, Bd.data_ptr(), A.n, Xd.data_ptr(), A.n)
    g1.record(stream)
    torch.cuda.synchronize(dev)
    fp64_batch_ms = g0.elapsed_time(g1)
    h64.close()
    fp64_ms = float(np.median([t for t, _ in fp64_single[1:]]))
    # Roofline: the level-0 batched smoother sweep on 32 interleaved columns.
    W = cfg[0]["width"]
    xdt, xbytes = (torch.float32, 4) if prec == bc.PREC_MIXED else (torch.float64, 8)
    vbytes = 4 if prec == bc.PREC_MIXED else 8
    with torch.cuda.stream(stream):
        f = torch.from_numpy(B_h[:, :W].copy()).to(dev).to(xdt).contiguous()
        u = torch.zeros_like(f)
    stream.synchronize()
    sweeps = 20
    check(lib.bcmg_level_relax_batch(h.ptr, 0, 0, W, C.c_void_p(f.data_ptr()),
                                     C.c_void_p(u.data_ptr()), 2), "relax_batch warmup")
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    check(lib.bcmg_level_relax_batch(h.ptr, 0, 0, W, C.c_void_p(f.data_ptr()),
                                     C.c_void_p(u.data_ptr()), sweeps), "relax_batch")
    r1.record(stream)
    torch.cuda.synchronize(dev)
    h.close()
    sweep_s = r0.elapsed_time(r1) / 1e3 / sweeps
    # values + columns + row pointers + d, then f and u read and u' written
    # for W columns (u gathered once).
    sweep_bytes = A.nnz * (vbytes + 4) + (A.n + 1) * 4 + A.n * xbytes + 3 * A.n * W * xbytes
    achieved = sweep_bytes / sweep_s / 1e9
    peak, peak_kind = measured_peaks()

    # e2e: host CSR + host right-hand sides through the C ABI.
    pin = lambda a: torch.from_numpy(a).pin_memory()  # noqa: E731
    h_row, h_col, h_val = pin(A.row), pin(A.col), pin(A.val)
    h_B = pin(np.ascontiguousarray(B_h.T))
    h_X = torch.zeros((nrhs, A.n), dtype=torch.float64).pin_memory()
    c = Csr()
    c.n, c.m, c.nnz = A.n, A.n, A.nnz
    c.row = C.cast(h_row.data_ptr(), C.POINTER(C.c_int32))
    c.col = C.cast(h_col.data_ptr(), C.POINTER(C.c_int32))
    c.val = C.cast(h_val.data_ptr(), C.POINTER(C.c_double))
    pc, ec = p.to_c(), ext.to_c()

    def e2e_step():
        hh = C.c_void_p()
        check(lib.bcmg_setup(C.byref(c), C.byref(pc), C.byref(ec), C.byref(hh)), "setup")
        h_X.zero_()
        infos_c = (SolveInfo * nrhs)()
        check(lib.bcmg_solve_batch(hh, nrhs, C.c_void_p(h_B.data_ptr()), A.n,
                                   C.c_void_p(h_X.data_ptr()), A.n, 0, infos_c), "solve_batch")
        lib.bcmg_destroy(hh)

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
    e_ms, e2e_value = aggregate_over_ranks(e0.elapsed_time(e1), e2e_steps, nrhs, world, dist,
                                           dev)
    h2d = (A.n + 1) * 4 + A.nnz * 12 + 2 * A.n * nrhs * 8
    d2h = A.n * nrhs * 8

    cpu, err = None, {}
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        try:
            cpu, x_orc = run_cpu_baseline(orc, A, B_h[:, 0].copy(), p_plain,
                                          os.cpu_count() or 1, nrhs=nrhs)
            err["err_vs_oracle_column0"] = float(np.linalg.norm(X[:, 0] - x_orc)
                                                 / np.linalg.norm(x_orc))
        except Exception as exc:
            cpu = {"value": None, "unit": "solves/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"failed: {exc}"}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    single_ms = statistics.median(t for t, _ in single)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec == bc.PREC_MIXED else "f64", "data": "synthetic",
        "config": {"workload": args.workload, "description": desc, "precision": args.precision,
                   "params": params_dict(p), "n": A.n, "nnz": A.nnz, "nrhs": nrhs,
                   "parallelism": f"replicas{world}",
                   "l2": "interleaved 32-column blocks (%.0f MB each in FP32) exceed "
                         "the 126 MB L2; no flush" % (A.n * nrhs * 4 / 1e6),
                   "step": "setup (shared hierarchy) + batched FCG of all columns + "
                           "teardown",
                   "autotune": "row-kernel shapes timed once per level shape and width in "
                               "the process (warm-up steps), reused by later setups"},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "k_bt_rowop (level-0 batched l1-Jacobi sweep, %d columns)" % W,
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": committed_traffic("k_bt_rowop",
                                                  f"{args.workload}:{args.precision}"),
                     "algorithmic_bytes": sweep_bytes, "launch_ms": sweep_s * 1e3},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "detail": {"iters": [i.iters for i in infos], "setup_ms": infos[0].setup_ms,
                   "batch_solve_ms": batch_solve_ms,
                   "solve_only_solves_per_s": nrhs / (batch_solve_ms / 1e3),
                   "single_rhs_solve_ms_median": single_ms,
                   "single_rhs_solves_per_s": 1e3 / single_ms,
                   "single_rhs_iters": [it for _, it in single],
                   "fp64_single_rhs_solve_ms_median": fp64_ms,
                   "fp64_single_rhs_solves_per_s": 1e3 / fp64_ms,
                   "fp64_single_rhs_iters": [it for _, it in fp64_single],
                   "fp64_batch_solve_ms": fp64_batch_ms,
                   "fp64_batch_solves_per_s": nrhs / (fp64_batch_ms / 1e3),
                   "fp64_batch_iters": [i.iters for i in infos64],
                   "batched_mixed_over_fp64_batched": fp64_batch_ms / batch_solve_ms,
                   "batched_mixed_over_fp64_single": (nrhs / (batch_solve_ms / 1e3))
                   / (1e3 / fp64_ms),
                   "max_true_rel_residual": true_rel, **err, "shapes": cfg,
                   "e2e_steps": e2e_steps},
    }
    print(json.dumps(line), flush=True)
    log(f"[bench] {args.workload} {args.precision}: {value:.1f} solves/s "
        f"({ms_max / args.steps:.1f} ms per {nrhs}-column step), solve-only "
        f"{nrhs / (batch_solve_ms / 1e3):.1f} solves/s vs one-at-a-time "
        f"{1e3 / single_ms:.1f} (plain FP64 {1e3 / fp64_ms:.1f}); sweep {achieved:.0f} GB/s "
        f"({achieved / peak:.2f})")
    return 0


def serve_requests(count, seed):
    """The serving stream: per request a matrix spec and a right-hand-side
    seed.  New matrices are 7-point or 27-point 3-D Poisson grids with side
    log-uniform in [16, 160] or random geometric graph Laplacians (unit
    cube, mean degree 12, weights U[0.5, 2], shift 1e-3) with n log-uniform
    in [1e4, 2e6]; 30% of requests reuse a previously seen matrix (one of the
    64 most recent) with a new N(0,1) right-hand side."""
    rng = np.random.default_rng(seed)
    reqs, seen = [], []
    for k in range(count):
        if seen and rng.random() < 0.3:
            key = seen[int(rng.integers(0, len(seen)))]
        else:
            kind = int(rng.integers(0, 3))
            if kind < 2:
                side = int(np.exp(rng.uniform(np.log(16), np.log(160))))
                spec = ("poisson", 7 if kind == 0 else 27, side)
            else:
                n = int(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
                spec = ("rgg", n, int(rng.integers(1, 1 << 30)))
            key = (len(reqs) + 1, spec)
            seen.append(key)
            seen = seen[-64:]
        reqs.append((key, 7919 * (k + 1)))
    return reqs


def make_matrix(spec):
    if spec[0] == "poisson":
        return wl.poisson(spec[1], spec[2], spec[2], spec[2])
    return wl.rgg(spec[1], seed=spec[2])


def serve_once(bc, lib, p, ext, reqs, rate, slots):
    """One pass of the request stream through a fresh bcmg_server at `rate`
    Poisson arrivals per second; returns its throughput and latencies."""
    import threading
    from concurrent.futures import ThreadPoolExecutor

    rng = np.random.default_rng(12)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
    # Host matrices are generated ahead of their arrival by a thread pool and
    # kept while a later request may reuse them.
    pool = ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 4))
    futures = {}
    last_use = {}
    for i, (key, _) in enumerate(reqs):
        last_use[key] = i
    ahead = 0  # requests whose matrices are being generated

    def prefetch(upto):
        nonlocal ahead
        while ahead < min(upto, len(reqs)):
            key = reqs[ahead][0]
            if key not in futures:
                futures[key] = pool.submit(make_matrix, key[1])
            ahead += 1
    srv = bc.Server(p, ext, slots=slots, mem_cap_gb=150.0, cache_cap_gb=60.0, max_batch=32)
    l0 = lib.bcmg_kernel_launches()
    results = [None] * len(reqs)
    lag = []
    lock = threading.Lock()

    def waiter(i, t, A):
        x, r = srv.wait(t)
        with lock:
            results[i] = r
        del A

    threads = []
    t0 = time.perf_counter()
    prefetch(48)
    for i, (key, rseed) in enumerate(reqs):
        prefetch(i + 48)
        A = futures[key].result()
        b = wl.vector(1, rseed, A.n)
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        lag.append(max(0.0, (time.perf_counter() - t0) - arrivals[i]))
        t = srv.submit(A, b, key=hash(key) & 0x7FFFFFFFFFFFFFFF)
        th = threading.Thread(target=waiter, args=(i, t, A))
        th.start()
        threads.append(th)
        if last_use[key] == i:
            # The host copy is no longer needed once no later request uses it
            # (the server reads A only while setting it up, which the waiter
            # thread's reference keeps alive until the request is done).
            futures[key] = None
    for th in threads:
        th.join()
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    pool.shutdown()
    lat = np.array([r.latency_ms for r in results])
    qms = np.array([r.queue_ms for r in results])
    return {"rate_per_s": rate, "solves_per_s": len(reqs) / wall, "wall_s": wall,
            "latency_ms": {"p50": float(np.percentile(lat, 50)),
                           "p99": float(np.percentile(lat, 99)), "mean": float(lat.mean()),
                           "max": float(lat.max())},
            "queue_ms": {"p50": float(np.percentile(qms, 50)),
                         "p99": float(np.percentile(qms, 99))},
            "converged": int(sum(r.solve.converged for r in results)),
            "arrival_lag_ms_p99": 1e3 * float(np.percentile(lag, 99)),
            "groups": int(sum(1 for r in results if r.group > 1)),
            "cache_hits": int(sum(r.cache_hit for r in results)),
            "launches": int(lib.bcmg_kernel_launches() - l0), "server": st}


def run_serve(args):
    """Serving stream: the requests go to a bcmg_server (continuous batching,
    hierarchy cache, admission under a 150 GB footprint cap) with Poisson
    arrivals, once per rate of --rate (a comma-separated list).  value = the
    throughput at the highest rate (completed solves / (last completion -
    first submission)); latency = submission -> solution on the host, p50 and
    p99 at every rate."""
    import bootcmatchg_b200 as bc
    from bootcmatchg_b200._lib import lib

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0  # replicas of the stream add nothing: one GPU per server
    p = product_params(bc, c1_settings())
    prec = bc.PREC_MIXED if args.precision == "mixed" else bc.PREC_FP64
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0)
    reqs = serve_requests(args.requests, 11)
    rates = sorted(float(r) for r in str(args.rate).split(","))
    runs = []
    for rate in rates:
        r = serve_once(bc, lib, p, ext, reqs, rate, args.slots)
        runs.append(r)
        log(f"[bench] serve_stream {len(reqs)} requests at {rate}/s: "
            f"{r['solves_per_s']:.1f} solves/s, latency p50 {r['latency_ms']['p50']:.1f} ms "
            f"p99 {r['latency_ms']['p99']:.1f} ms, queue p50 {r['queue_ms']['p50']:.1f} ms, "
            f"{r['converged']}/{len(reqs)} converged, setups {r['server']['setups']}, "
            f"hits {r['server']['cache_hits']}, batches {r['server']['batches']}")
    top = runs[-1]
    line = {
        "metric": "solves/s to rtol 1e-8 and p50/p99 latency, served stream",
        "value": top["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "steps": len(reqs), "warmup": 0, "ms_per_step": 1e3 * top["wall_s"] / len(reqs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if prec else "f64", "data": "synthetic",
        "config": {"workload": "serve_stream", "requests": len(reqs), "rates_per_s": rates,
                   "slots": args.slots, "mem_cap_gb": 150, "cache_cap_gb": 60,
                   "max_batch": 32, "precision": args.precision,
                   "description": serve_requests.__doc__.split("\n\n")[0].replace("\n", " ")},
        "latency_ms": top["latency_ms"], "queue_ms": top["queue_ms"],
        "by_rate": [{k: v for k, v in r.items() if k != "server"} | {"server": r["server"]}
                    for r in runs],
        "e2e": {"value": top["solves_per_s"], "unit": "solves/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "gpu_launches": int(sum(r["launches"] for r in runs)),
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- profiling cases (--case): small fixed workloads for ncu --------------
def run_case(args):
    """Small, fixed workloads for profiling single kernels under ncu.

    sweep_fp32   level-0 smoother sweeps (--sweeps, default 3) of 27-point
                 Poisson 128^3, mixed precision (FP32 sliced values)
    sweep_fp64   the same in FP64
    sweep_fv2d   level-0 smoother sweeps of the 2-D FV 2048^2 matrix
                 (5-point), mixed precision
    batch_fp32   batched smoother sweeps of 7-point Poisson 96^3 on 32
                 interleaved columns (FP32), autotuning off
    solve_mixed  one complete mixed-precision solve of 27-point Poisson
                 GRID^3 (--grid, default 128), FCG loop driven from the host
                 (every kernel is a plain launch a profiler can see)
    solve_rgg    one complete solve of the 2,000,000-node random geometric
                 graph Laplacian (the rgg_2m workload) in --precision, FCG
                 loop driven from the host
    batch_solve  one 32-column batched solve of 7-point Poisson 96^3 (mixed),
                 FCG loop driven from the host
    setup        one FP64 setup of 27-point Poisson GRID^3 (--grid, default
                 96): matching, aggregation and Galerkin kernels

    Each case sets up its hierarchy first and then runs the kernels of
    interest; filter on kernel names such as k_sl_pipe or k_bt_rowop."""
    import torch

    import bootcmatchg_b200 as bc
    from bootcmatchg_b200._lib import check, lib

    p = product_params(bc, c1_settings())
    case, k = args.case, args.sweeps
    if case in ("sweep_fp32", "sweep_fp64", "sweep_fv2d"):
        prec = bc.PREC_FP64 if case == "sweep_fp64" else bc.PREC_MIXED
        A = wl.fv2d(2048, 2048, seed=2) if case == "sweep_fv2d" else wl.poisson(27, 128, 128, 128)
        dt = torch.float32 if prec == bc.PREC_MIXED else torch.float64
        with bc.Handle(A, p, bc.Extensions(precision=prec, replace_every=10)) as h:
            f = torch.randn(A.n, dtype=dt, device="cuda:0")
            u = torch.zeros(A.n, dtype=dt, device="cuda:0")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            check(lib.bcmg_level_relax(h.ptr, 0, 0, C.c_void_p(f.data_ptr()),
                                       C.c_void_p(u.data_ptr()), k), "bcmg_level_relax")
            print(f"{k} sweeps: {1e3 * (time.perf_counter() - t0):.3f} ms")
    elif case == "batch_fp32":
        A = wl.poisson(7, 96, 96, 96)
        ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, autotune=0)
        with bc.Handle(A, p, ext) as h:
            f = torch.randn(A.n * 32, dtype=torch.float32, device="cuda:0")
            u = torch.zeros(A.n * 32, dtype=torch.float32, device="cuda:0")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            check(lib.bcmg_level_relax_batch(h.ptr, 0, 0, 32, C.c_void_p(f.data_ptr()),
                                             C.c_void_p(u.data_ptr()), k), "relax_batch")
            print(f"{k} batched sweeps: {1e3 * (time.perf_counter() - t0):.3f} ms")
    elif case == "solve_mixed":
        g = args.grid or 128
        A = wl.poisson(27, g, g, g)
        b = wl.vector(1, 1, A.n)
        ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, use_graphs=0)
        with bc.Handle(A, p, ext) as h:
            x, info = h.solve(b)
        print(f"iters {info.iters} converged {info.converged} setup {info.setup_ms:.1f} ms "
              f"solve {info.solve_ms:.1f} ms")
    elif case == "solve_rgg":
        A = wl.rgg(2_000_000, seed=4)
        b = wl.vector(1, 1, A.n)
        prec = bc.PREC_MIXED if args.precision == "mixed" else bc.PREC_FP64
        ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0, use_graphs=0)
        with bc.Handle(A, p, ext) as h:
            x, info = h.solve(b)
        print(f"{args.precision}: iters {info.iters} converged {info.converged} "
              f"setup {info.setup_ms:.1f} ms solve {info.solve_ms:.1f} ms")
    elif case == "batch_solve":
        A = wl.poisson(7, 96, 96, 96)
        B = np.asfortranarray(wl.vector(1, 3, A.n * 32).reshape(A.n, 32, order="F"))
        ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, use_graphs=0)
        with bc.Handle(A, p, ext) as h:
            X, infos = h.solve_batch(B)
        print(f"iters {max(i.iters for i in infos)} converged "
              f"{all(i.converged for i in infos)} solve {infos[0].solve_ms:.1f} ms")
    elif case == "setup":
        g = args.grid or 96
        A = wl.poisson(27, g, g, g)
        with bc.Handle(A, p, bc.Extensions(precision=bc.PREC_FP64)) as h:
            info = h.hierarchy_info(0)
        print(f"levels {info['num_levels']} op_cmplx {info['op_cmplx']:.3f}")
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="poisson27_128",
                    choices=["poisson27_128", "poisson7_32", "fv2d_2048", "poisson7_96", "rgg_2m",
                             "poisson7_96_x32", "serve_stream"])
    ap.add_argument("--requests", type=int, default=300, help="serve_stream: requests")
    ap.add_argument("--rate", default="20", help="serve_stream: arrivals per s (a comma list "
                    "runs the stream once per rate)")
    ap.add_argument("--slots", type=int, default=4, help="serve_stream: solves in flight")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--case", choices=["sweep_fp32", "sweep_fp64", "sweep_fv2d", "batch_fp32",
                                       "solve_mixed", "solve_rgg", "batch_solve", "setup"],
                    help="run one small profiling case instead of the benchmark")
    ap.add_argument("--sweeps", type=int, default=3, help="--case: sweeps per launch")
    ap.add_argument("--grid", type=int, default=None, help="--case setup/solve_mixed: side")
    args = ap.parse_args()
    if args.case:
        return run_case(args)
    if args.warmup < 3:
        log("[bench] warm-up raised to the minimum of 3 steps")
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serve_stream":
        return run_serve(args)
    if args.workload.endswith("_x32"):
        return run_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
