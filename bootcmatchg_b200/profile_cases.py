"""Small, fixed workloads for profiling single kernels under ncu.

    python -m bootcmatchg_b200.profile_cases CASE [--sweeps K]

CASE:
  sweep_fp32    level-0 smoother sweeps of 27-point Poisson 128^3, mixed
                precision (FP32 sliced values)
  sweep_fp64    the same in FP64
  sweep_fv2d    level-0 smoother sweeps of the 2-D FV 2048^2 matrix (5-point),
                mixed precision
  batch_fp32    batched smoother sweeps of 7-point Poisson 96^3 on 32
                interleaved columns (FP32), autotuning off
  solve_mixed   one complete mixed-precision solve of 27-point Poisson
                GRID^3 (--grid, default 128) with the FCG loop driven from the
                host (every kernel is a plain launch a profiler can see)
  batch_solve   one 32-column batched solve of 7-point Poisson 96^3 (mixed),
                FCG loop driven from the host
  setup         one FP64 setup of 27-point Poisson GRID^3 (--grid, default
                96): matching, aggregation and Galerkin kernels

Each case sets up its hierarchy first and then runs the kernels of interest;
the kernel names to filter on are k_sl_relax, k_bt_rowop and so on.
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
import time

import numpy as np

from . import api as bc
from ._lib import check, lib


def c1_params() -> bc.Params:
    p = bc.Params.default()
    p.solver_type, p.max_hrc, p.conv_ratio = 0, 1, 0.8
    p.aggrsweeps, p.aggrtype, p.max_levels, p.cycle_type = 2, 0, 20, 0
    p.relax_type, p.coarse_solver = 4, 4
    p.prerelax_sweeps, p.postrelax_sweeps, p.relaxnumber_coarse = 4, 4, 16
    p.itnlim, p.rtol = 1000, 1e-8
    return p


def sweeps(prec: int, k: int, fv2d: bool = False) -> None:
    import torch
    A = bc.fv2d(2048, 2048, seed=2) if fv2d else bc.poisson(27, 128, 128, 128)
    dt = torch.float32 if prec == bc.PREC_MIXED else torch.float64
    with bc.Handle(A, c1_params(), bc.Extensions(precision=prec, replace_every=10)) as h:
        f = torch.randn(A.n, dtype=dt, device="cuda:0")
        u = torch.zeros(A.n, dtype=dt, device="cuda:0")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.bcmg_level_relax(h.ptr, 0, 0, C.c_void_p(f.data_ptr()),
                                   C.c_void_p(u.data_ptr()), k), "bcmg_level_relax")
        print(f"{k} sweeps: {1e3 * (time.perf_counter() - t0):.3f} ms")


def batch_sweeps(k: int) -> None:
    import torch
    A = bc.poisson(7, 96, 96, 96)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, autotune=0)
    with bc.Handle(A, c1_params(), ext) as h:
        f = torch.randn(A.n * 32, dtype=torch.float32, device="cuda:0")
        u = torch.zeros(A.n * 32, dtype=torch.float32, device="cuda:0")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        check(lib.bcmg_level_relax_batch(h.ptr, 0, 0, 32, C.c_void_p(f.data_ptr()),
                                         C.c_void_p(u.data_ptr()), k), "relax_batch")
        print(f"{k} batched sweeps: {1e3 * (time.perf_counter() - t0):.3f} ms")


def solve_mixed(grid: int = 128) -> None:
    A = bc.poisson(27, grid, grid, grid)
    b = bc.vector(1, 1, A.n)
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, use_graphs=0)
    with bc.Handle(A, c1_params(), ext) as h:
        x, info = h.solve(b)
    print(f"iters {info.iters} converged {info.converged} setup {info.setup_ms:.1f} ms "
          f"solve {info.solve_ms:.1f} ms")


def batch_solve() -> None:
    A = bc.poisson(7, 96, 96, 96)
    B = np.asfortranarray(bc.vector(1, 3, A.n * 32).reshape(A.n, 32, order="F"))
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10, use_graphs=0)
    with bc.Handle(A, c1_params(), ext) as h:
        X, infos = h.solve_batch(B)
    print(f"iters {max(i.iters for i in infos)} converged "
          f"{all(i.converged for i in infos)} solve {infos[0].solve_ms:.1f} ms")


def setup(grid: int) -> None:
    A = bc.poisson(27, grid, grid, grid)
    with bc.Handle(A, c1_params(), bc.Extensions(precision=bc.PREC_FP64)) as h:
        info = h.hierarchy_info(0)
    print(f"levels {info['num_levels']} op_cmplx {info['op_cmplx']:.3f}")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="profiling workloads")
    ap.add_argument("case", choices=["sweep_fp32", "sweep_fp64", "sweep_fv2d", "batch_fp32",
                                     "solve_mixed",
                                     "batch_solve", "setup"])
    ap.add_argument("--sweeps", type=int, default=3)
    ap.add_argument("--grid", type=int, default=None,
                    help="grid side for setup (default 96) and solve_mixed (default 128)")
    a = ap.parse_args(argv)
    if a.case == "sweep_fp32":
        sweeps(bc.PREC_MIXED, a.sweeps)
    elif a.case == "sweep_fp64":
        sweeps(bc.PREC_FP64, a.sweeps)
    elif a.case == "sweep_fv2d":
        sweeps(bc.PREC_MIXED, a.sweeps, fv2d=True)
    elif a.case == "batch_fp32":
        batch_sweeps(a.sweeps)
    elif a.case == "solve_mixed":
        solve_mixed(a.grid or 128)
    elif a.case == "setup":
        setup(a.grid or 96)
    else:
        batch_solve()
    return 0


if __name__ == "__main__":
    sys.exit(main())
