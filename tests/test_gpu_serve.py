"""GPU tests of the solve server (bcmg_server_*): continuous batching with a
hierarchy cache and memory-capped admission.

A request run alone (its own handle, nothing else on the GPU) and the same
request run in a mix of concurrent requests must give the same solution:
bit for bit when it runs by itself on a slot (max_batch 1: solves are
deterministic and never share state), and within the batched solve's
tolerance (1e-5 relative, converged to rtol) when it was grouped with other
requests on the same matrix.
"""
import time

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from helpers import c1_params

pytestmark = pytest.mark.gpu


def mix():
    mats = [wl.poisson(7, 10, 10, 10), wl.poisson(27, 8, 8, 8), wl.rgg(2000, seed=7),
            wl.fv2d(24, 24, seed=2), wl.poisson(7, 20, 20, 20)]
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(24):
        m = int(rng.integers(0, len(mats)))
        reqs.append((m, wl.vector(1, 1000 + k, mats[m].n)))
    return mats, reqs


def alone(mats, reqs, p):
    out = []
    for m, b in reqs:
        with bc.Handle(mats[m], p) as h:
            x, info = h.solve(b)
        out.append(x)
    return out


def test_same_alone_and_in_the_mix():
    p = c1_params()
    mats, reqs = mix()
    with bc.Server(p, slots=4, max_batch=1) as srv:
        tickets = [srv.submit(mats[m], b, key=m + 1) for m, b in reqs]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
    ref = alone(mats, reqs, p)
    for (x, r), xr in zip(res, ref):
        assert r.solve.converged and r.group == 1
        assert np.array_equal(x, xr)
        assert 0.0 <= r.queue_ms <= r.latency_ms
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["setups"] == len({m for m, _ in reqs})
    assert st["cache_hits"] == len(reqs) - st["setups"]


def test_grouped_requests_match_their_single_solves():
    p = c1_params()
    A = wl.poisson(7, 16, 16, 16)
    bs = [wl.vector(1, 2000 + k, A.n) for k in range(12)]
    with bc.Server(p, slots=1, max_batch=32) as srv:
        first = srv.submit(A, bs[0], key=7)
        tickets = [srv.submit(A, b, key=7) for b in bs[1:]]  # queue behind the setup
        res = [srv.wait(first)] + [srv.wait(t) for t in tickets]
        st = srv.stats()
    assert st["setups"] == 1 and st["batches"] >= 1
    assert max(r.group for _, r in res) > 1
    with bc.Handle(A, p) as h:
        for (x, r), b in zip(res, bs):
            xs, si = h.solve(b)
            assert r.solve.converged
            assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-5
            res_b = b - A.to_scipy() @ x
            assert np.linalg.norm(res_b) / np.linalg.norm(b) <= 1.05 * p.rtol


def test_cache_budget_evicts_and_keeps_results():
    p = c1_params()
    mats, reqs = mix()
    with bc.Server(p, slots=2, max_batch=1, cache_cap_gb=1e-6) as srv:
        tickets = [srv.submit(mats[m], b, key=m + 1) for m, b in reqs[:10]]
        res = [srv.wait(t) for t in tickets]
        st = srv.stats()
    ref = alone(mats, reqs[:10], p)
    for (x, r), xr in zip(res, ref):
        assert np.array_equal(x, xr)
    assert st["evictions"] > 0 and st["cached_hierarchies"] == 0


def test_admission_rejects_what_cannot_fit():
    p = c1_params()
    small = wl.poisson(7, 8, 8, 8)
    big = wl.poisson(7, 64, 64, 64)  # ~0.14 GB estimated
    with bc.Server(p, slots=2, mem_cap_gb=0.05) as srv:
        tb = srv.submit(big, np.ones(big.n), key=1)
        ts = srv.submit(small, np.ones(small.n), key=2)
        with pytest.raises(bc.BcmgError) as e:
            srv.wait(tb)
        assert e.value.status == bc.ERR_ALLOC
        x, r = srv.wait(ts)
        assert r.solve.converged
        with pytest.raises(bc.BcmgError):
            srv.wait(tb)  # ticket released


def test_wait_timeout_and_stats():
    p = c1_params()
    A = wl.poisson(7, 40, 40, 40)
    with bc.Server(p, slots=1) as srv:
        t = srv.submit(A, np.ones(A.n), key=3)
        polls = 0
        while True:
            try:
                x, r = srv.wait(t, timeout=0.0)
                break
            except TimeoutError:
                polls += 1
                time.sleep(0.001)
        assert r.solve.converged and r.latency_ms > 0
        st = srv.stats()
        assert st["submitted"] == 1 and st["completed"] == 1
        assert st["resident_bytes"] > 0 and st["cached_hierarchies"] == 1
