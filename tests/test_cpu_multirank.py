"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

The solve path does not shard ("replicas only"): N GPUs run N independent
replicas and the only cross-rank steps are a barrier and the MAX of the
ranks' elapsed device times.  These tests run that reduction with the gloo
backend, and check that the reference arm does no work on ranks other than 0.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms_local = 10.0 * (rank + 1)  # rank 1 is the slowest
        ms, value = bench.aggregate_over_ranks(ms_local, steps=5, units_per_step=32,
                                               world=world, dist=dist, device="cpu")
        dist.barrier()
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_throughput():
    world = 2
    port = free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=rank_main, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in out:
        assert ms == 20.0  # the slowest rank's time on every rank
        assert value == pytest.approx(world * 5 * 32 / 0.020)


def test_reference_arm_idles_on_other_ranks(monkeypatch):
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(workload="poisson27_128", steps=1, warmup=3, gpus=2)
    assert bench.run_reference(args) == 0


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    ms, value = bench.aggregate_over_ranks(12.5, steps=4, units_per_step=1, world=1)
    assert ms == 12.5 and value == pytest.approx(4 / 0.0125)


def test_reference_arm_json_line():
    """bench.py --impl reference on the CPU: one JSON line with the metric of
    the GPU arm, the CPU baseline it times and an e2e block without
    transfers."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference",
                          "--workload", "poisson7_32", "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, check=True, env=env, timeout=600)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "solves/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] in ("port", "reference")
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "solves/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "poisson7_32"
    assert "one complete oracle solve" in line["cpu_baseline"]["sample"] or \
        "complete oracle solves" in line["cpu_baseline"]["sample"]
    assert line["cpu_baseline"]["one_core"]["cores"] == 1


def test_reference_arm_loads_no_product_library():
    """The reference arm runs the oracle only: neither the product package
    nor libbcmg.so is loaded in its process."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'poisson7_32',"
        " '--steps', '1', '--warmup', '3']\n"
        "try:\n"
        f"    runpy.run_path({os.path.join(root, 'bench.py')!r}, run_name='__main__')\n"
        "except SystemExit as e:\n"
        "    assert not e.code, e.code\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT_LOADED' if ('libbcmg.so' in maps or 'bootcmatchg_b200' in sys.modules)"
        " else 'NO_PRODUCT')\n")
    env = dict(os.environ, RANK="0", WORLD_SIZE="1")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         check=True, env=env, timeout=600, cwd=root)
    assert out.stdout.strip().splitlines()[-1] == "NO_PRODUCT"
