"""Times BootCMatchG's own GPU solve (the stock solve(A, p, rhs) of
oracle/_ref/libref.so) on the benchmark workloads: the reference GPU baseline.

Each measured call is the whole solve() -- upload of A, bootstrap setup, FCG,
teardown -- plus the copy of x back to the host, i.e. the same work as the
e2e number of bench.py.  Every workload runs in a child process so the
reference's stdout (#META lines) can be parsed.  Prints one JSON line per
workload.  Usage (GPU box): python oracle/ref/time_ref_solve.py [workload ...]
On a B200 the stock solve() stopped with an illegal memory access
(src/matrix/CSR.cu:140) on both default workloads, so it is not run again;
the script is kept as the record of that attempt.
TEST INFRASTRUCTURE ONLY.
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

CHILD = r"""
import ctypes as C, json, sys, time
import numpy as np
sys.path.insert(0, ROOT)
import bench
import bootcmatchg_b200 as bc
lib = C.CDLL(REF)
A, b, p, desc = bench.make_workload(bc, WORKLOAD)
prm = np.array([p.solver_type, p.max_hrc, p.aggrsweeps, p.aggrtype, p.max_levels,
                p.cycle_type, p.coarse_solver, p.relax_type, p.relaxnumber_coarse,
                p.prerelax_sweeps, p.postrelax_sweeps, p.itnlim], np.int32)
dprm = np.array([p.conv_ratio, p.rtol])
P = lambda a: C.c_void_p(a.ctypes.data)
x = np.zeros(A.n)
times = []
for k in range(REPS + 1):
    t0 = time.perf_counter()
    st = lib.ref_solve(A.n, A.nnz, P(A.row), P(A.col), P(A.val), P(prm), P(dprm), P(b), P(x))
    times.append(time.perf_counter() - t0)
    assert st == 0, st
res = b - A.to_scipy() @ x
sys.stdout.flush()
print("RESULT " + json.dumps({"times": times[1:], "n": A.n, "nnz": A.nnz, "desc": desc,
      "true_rel_residual": float(np.linalg.norm(res) / np.linalg.norm(b))}), flush=True)
"""


def run(workload, reps):
    code = (f"ROOT = {ROOT!r}\nREF = {os.path.join(ROOT, 'oracle', '_ref', 'libref.so')!r}\n"
            f"WORKLOAD = {workload!r}\nREPS = {reps}\n" + CHILD)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=1800)
    if out.returncode != 0:
        return {"workload": workload, "error": out.stderr[-1500:]}
    res = json.loads(re.search(r"RESULT (.*)", out.stdout).group(1))
    iters = re.findall(r"#META sol;num_iteration int (\d+)", out.stdout)
    boot = re.findall(r"#META time;bootstrap_time float (\S+)", out.stdout)
    solve = re.findall(r"#META time;solve_time float (\S+)", out.stdout)
    t = sorted(res["times"])
    med = t[len(t) // 2]
    return {"workload": workload, "impl": "reference-gpu (stock solve(), sm_100a build)",
            "n": res["n"], "nnz": res["nnz"], "iters": int(iters[-1]) if iters else None,
            "bootstrap_ms": float(boot[-1]) if boot else None,
            "solve_ms": float(solve[-1]) if solve else None,
            "wall_s_median": med, "solves_per_s": 1.0 / med, "reps": len(t),
            "true_rel_residual": res["true_rel_residual"]}


def main():
    workloads = sys.argv[1:] or ["poisson7_32", "poisson27_128"]
    for w in workloads:
        print(json.dumps(run(w, 3)), flush=True)


if __name__ == "__main__":
    main()
