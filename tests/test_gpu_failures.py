"""Failure detection, exercised without faulting or hanging the GPU.

The reference stops the process on every error (exit()/assert,
src/utility/utils.h:36-71); this library returns a status and stays usable.

Bounded device waits.  Every wait of a pipelined row pass is bounded by the
handle's max_device_seconds.  On a healthy pipeline a wait never runs out
(mbarrier.try_wait holds the thread until the staged copy lands), so the
bound is exercised by bcmg_wait_selftest: the pipeline's own wait functions
on a barrier that nothing completes, beside a real staged copy that must
drain; it returns BCMG_ERR_DEVICE_TIMEOUT after the bound and the device
keeps working.  Changing the bound on a live handle keeps its results.  A
matching step limit of one makes every suitor-matching thread run out: setup
returns BCMG_ERR_DEVICE_TIMEOUT and the next setup on the device succeeds.

Allocation failures.  bcmg_debug_fail_alloc fails one chosen device
allocation on the host side (nothing reaches the GPU).  Failing each
allocation of a setup + solve in turn, every call returns BCMG_ERR_ALLOC,
the library holds no device allocation afterwards, and the next setup +
solve gives the bits of the first.  The same for the first batched solve of
a handle, whose state is allocated on demand: the handle stays usable.
"""
import ctypes as C

import numpy as np
import pytest

import bootcmatchg_b200 as bc
import workloads as wl
from bootcmatchg_b200._lib import lib
from helpers import c1_params

pytestmark = pytest.mark.gpu

ERR_ALLOC, ERR_DEVICE_TIMEOUT = 3, 7


def alloc_stats():
    live, made = C.c_int64(), C.c_int64()
    lib.bcmg_debug_alloc_stats(C.byref(live), C.byref(made))
    return live.value, made.value


def test_bounded_wait_runs_out_and_device_stays_usable():
    """bcmg_wait_selftest: a pipeline wait that nothing completes gives up
    after its bound (here 20 ms) and the call reports it as a solve would."""
    import time
    t0 = time.perf_counter()
    st = lib.bcmg_wait_selftest(0, 0.02)
    elapsed = time.perf_counter() - t0
    assert st == ERR_DEVICE_TIMEOUT, (st, lib.bcmg_last_error())
    assert elapsed >= 0.02
    A = wl.poisson(7, 16, 16, 16)
    with bc.Handle(A, c1_params()) as h:
        x, info = h.solve(np.ones(A.n))
    assert info.converged


@pytest.mark.parametrize("prec", [bc.PREC_FP64, bc.PREC_MIXED])
def test_wait_bound_change_keeps_results(prec):
    """bcmg_set_max_device_seconds on a live handle (the captured FCG loop is
    rebuilt with the new bound): same bits as a fresh handle."""
    A = wl.poisson(27, 32, 32, 32)
    b = wl.vector(1, 1, A.n)
    p = c1_params()
    ext = bc.Extensions(precision=prec, replace_every=10 if prec else 0)
    with bc.Handle(A, p, ext) as h0:
        x0, i0 = h0.solve(b)
    with bc.Handle(A, p, ext) as h:
        x1, i1 = h.solve(b)
        h.set_max_device_seconds(0.5)
        x2, i2 = h.solve(b)
        with pytest.raises(bc.BcmgError) as e:
            h.set_max_device_seconds(0.0)
        assert e.value.status == 1
    assert i0.converged and i0.iters == i1.iters == i2.iters
    assert np.array_equal(x1, x0) and np.array_equal(x2, x0)


def test_matching_step_limit_runs_out():
    A = wl.poisson(7, 24, 24, 24)
    p = c1_params()
    with pytest.raises(bc.BcmgError) as e:
        bc.Handle(A, p, bc.Extensions(match_step_limit=1))
    assert e.value.status == ERR_DEVICE_TIMEOUT, str(e.value)
    assert "matching" in str(e.value)
    with bc.Handle(A, p) as h:
        x, info = h.solve(np.ones(A.n))
    assert info.converged


def test_every_allocation_failure_is_reported_without_leaks():
    A = wl.poisson(7, 12, 12, 12)
    b = wl.vector(1, 1, A.n)
    p = c1_params()
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)
    live0, made0 = alloc_stats()
    with bc.Handle(A, p, ext) as h:
        x_ref, i_ref = h.solve(b)
    live1, made1 = alloc_stats()
    assert live1 == live0
    total = made1 - made0
    assert total > 10
    try:
        for k in range(total):
            lib.bcmg_debug_fail_alloc(k)
            with pytest.raises(bc.BcmgError) as e:
                with bc.Handle(A, p, ext) as h:
                    h.solve(b)
            assert e.value.status == ERR_ALLOC and "injected" in str(e.value), (k, str(e.value))
            assert alloc_stats()[0] == live0, f"allocation {k}: device memory leaked"
    finally:
        lib.bcmg_debug_fail_alloc(-1)
    with bc.Handle(A, p, ext) as h:
        x, info = h.solve(b)
    assert info.iters == i_ref.iters and np.array_equal(x, x_ref)
    assert alloc_stats()[0] == live0


@pytest.mark.parametrize("max_hrc", [1, 2])
def test_copies_built_beside_the_setup_fail_cleanly_and_repeat_bits(max_hrc):
    """7-point Poisson 52^3 (140,608 rows) is large enough for a setup to
    build its solve-phase copies on a helper thread and stream while it
    coarsens (inputs of 131,072 rows and more).  Repeated setups + solves
    give the same bits; failing each allocation of a setup + solve in turn,
    whichever thread makes it, returns BCMG_ERR_ALLOC and leaks nothing.
    With max_hrc 2 (conv_ratio 0.01, so the second hierarchy is built) the
    copies are installed before the bootstrap's inner iterations."""
    A = wl.poisson(7, 52, 52, 52)
    b = wl.vector(1, 4, A.n)
    p = c1_params()
    p.max_hrc, p.conv_ratio = max_hrc, 0.01
    ext = bc.Extensions(precision=bc.PREC_MIXED, replace_every=10)
    live0, made0 = alloc_stats()
    with bc.Handle(A, p, ext) as h:
        x_ref, i_ref = h.solve(b)
        assert h.num_hierarchies()[0] == max_hrc
    live1, made1 = alloc_stats()
    assert live1 == live0 and i_ref.converged
    for _ in range(3):
        with bc.Handle(A, p, ext) as h:
            x, info = h.solve(b)
        assert info.iters == i_ref.iters and np.array_equal(x, x_ref)
    total = made1 - made0
    assert total > 10
    try:
        for k in range(total):
            lib.bcmg_debug_fail_alloc(k)
            with pytest.raises(bc.BcmgError) as e:
                with bc.Handle(A, p, ext) as h:
                    h.solve(b)
            assert e.value.status == ERR_ALLOC and "injected" in str(e.value), (k, str(e.value))
            assert alloc_stats()[0] == live0, f"allocation {k}: device memory leaked"
    finally:
        lib.bcmg_debug_fail_alloc(-1)
    with bc.Handle(A, p, ext) as h:
        x, info = h.solve(b)
    assert info.iters == i_ref.iters and np.array_equal(x, x_ref)
    assert alloc_stats()[0] == live0


def test_batched_state_allocation_failure_leaves_handle_usable():
    A = wl.poisson(7, 16, 16, 16)
    B = np.asfortranarray(wl.vector(1, 3, A.n * 4).reshape(A.n, 4, order="F"))
    p = c1_params()
    ext = bc.Extensions(autotune=0)  # a fixed row-kernel shape rule: no timing runs
    live0, _ = alloc_stats()
    with bc.Handle(A, p, ext) as h:
        X_ref, inf_ref = h.solve_batch(B)
    with bc.Handle(A, p, ext) as h:
        live_h, made_h = alloc_stats()
        h.solve_batch(B)  # counts the state's allocations on a scratch handle
        n_state = alloc_stats()[1] - made_h
    assert n_state > 0
    with bc.Handle(A, p, ext) as h:
        live_h, _ = alloc_stats()
        try:
            for k in range(n_state):
                lib.bcmg_debug_fail_alloc(k)
                with pytest.raises(bc.BcmgError) as e:
                    h.solve_batch(B)
                assert e.value.status == ERR_ALLOC, str(e.value)
                assert alloc_stats()[0] == live_h, f"allocation {k}: batch state leaked"
        finally:
            lib.bcmg_debug_fail_alloc(-1)
        X, infos = h.solve_batch(B)
    assert [i.iters for i in infos] == [i.iters for i in inf_ref]
    assert np.array_equal(X, X_ref)
    assert alloc_stats()[0] == live0
