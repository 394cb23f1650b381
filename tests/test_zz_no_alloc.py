"""sfb200_run_noalloc against sfb200_run, through the C ABI.

sfb200_run_noalloc serves callers that must not allocate device memory while they run (a loop that
reserved its whole device budget up front, or a process sharing the device where an allocation could
fail or make the device wait): its scratch is a fixed array inside the library. This file is
collected last on purpose, and the test must hold both in a fresh process and after every other GPU
test. Two calls in a row must each agree with sfb200_run on the same device inputs: counts identical,
sums within the precision's tolerance times the CPU oracle's per-bin sum |v| (both run the same pair
kernel in the caller's point order; only the order of the floating-point atomics differs), and each
must match the oracle within that tolerance too. A call larger than the fixed scratch must be refused
with a clear error.
"""
import functools

import numpy as np
import pytest

import oracle_py
from helpers import TOL_FP64, TOL_MIXED, compare
from sfb200 import _abi, _lib, synthetic
from sfb200.api import plan_description
from sfb200.errors import ArgumentError

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def device_inputs(w):
    # column-major (W, N) == row-major (N, W)
    xd = torch.from_numpy(np.ascontiguousarray(w.x.T)).cuda()
    ud = torch.from_numpy(np.ascontiguousarray(w.u.T)).cuda()
    return xd, ud


def run_plain(plan, ctx, xd, ud, n):
    sums = torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda")
    counts = torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")
    flags = _abi.RUN_DEVICE_INPUT | _abi.RUN_DEVICE_OUTPUT
    plan.run(xd.data_ptr(), ud.data_ptr(), n, flags, sums.data_ptr(), counts.data_ptr(), ctx.stream)
    torch.cuda.synchronize()
    return sums.cpu().numpy(), counts.cpu().numpy()


def run_noalloc(plan, ctx, xd, ud, n):
    sums = torch.full((plan.n_sums,), 7.0, dtype=torch.float64, device="cuda")  # overwritten by the call
    counts = torch.full((plan.n_counts,), 7, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.load().sfb200_run_noalloc(plan.ptr, xd.data_ptr(), ud.data_ptr(), int(n), 0, sums.data_ptr(),
                                              counts.data_ptr(), ctx.stream), ctx.ptr, "run_noalloc")
    torch.cuda.synchronize()
    return sums.cpu().numpy(), counts.cpu().numpy()


@functools.lru_cache(maxsize=None)
def oracle_of(name, n):
    w = synthetic.config(name, n=n)
    desc, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, None, w.metric, "fp64", w.x.dtype,
                                  w.u.dtype)
    return oracle_py.run(desc, w.x, w.u, with_abs=True)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("name,n", [("c0", 4096), ("c1", 10000)])
def test_noalloc_matches_run_on_two_calls(precision, name, n):
    w = synthetic.config(name, n=n)
    ctx = _lib.Context(0)
    desc, keep = plan_description(w.ops, w.u.shape[0], w.distance_bins, None, w.metric, precision, w.x.dtype,
                                  w.u.dtype)
    plan = _lib.Plan(ctx, desc, keep)
    plan.set_option(_abi.OPT_POINT_ORDER, 0)  # the caller's point order, as the no-allocation path
    tol = TOL_MIXED if precision == "mixed" else TOL_FP64
    os_, oc, oa = oracle_of(name, n)
    nb = len(w.distance_bins) - 1
    xd, ud = device_inputs(w)
    try:
        ref_s, ref_c = run_plain(plan, ctx, xd, ud, w.n)
        for _ in range(2):
            s, c = run_noalloc(plan, ctx, xd, ud, w.n)
            assert np.array_equal(c, ref_c)
            assert int(c.sum()) > 0
            for k in range(len(w.ops)):
                sl = slice(k * nb, (k + 1) * nb)
                compare(s[sl], c, os_[sl], oc, oa[sl], tol)
                compare(s[sl], c, ref_s[sl], ref_c, oa[sl], 2 * tol)
    finally:
        plan.close()
        ctx.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_noalloc_at_the_scratch_limit_allocates_nothing(precision):
    """The largest call the scratch takes: 3D, 65536 points (the packed coordinates and velocities then
    end exactly where the accumulators begin), the c1 workload's four operators. Against sfb200_run
    and the oracle, and with the device's free memory unchanged by a call (after a first call has
    loaded the kernels)."""
    from full_oracle import oracle_for

    w = synthetic.config("c1")
    assert w.n == 65536 and w.u.shape[0] == 3
    os_, oc, oa, _src = oracle_for("c1", w)
    ctx = _lib.Context(0)
    desc, keep = plan_description(w.ops, 3, w.distance_bins, None, w.metric, precision, w.x.dtype, w.u.dtype)
    plan = _lib.Plan(ctx, desc, keep)
    plan.set_option(_abi.OPT_POINT_ORDER, 0)
    tol = TOL_MIXED if precision == "mixed" else TOL_FP64
    nb = len(w.distance_bins) - 1
    xd, ud = device_inputs(w)
    lib = _lib.load()
    try:
        ref_s, ref_c = run_plain(plan, ctx, xd, ud, w.n)
        run_noalloc(plan, ctx, xd, ud, w.n)  # loads the kernels of this plan
        sums = torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda")
        counts = torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")
        free0, free1, total = _abi.C.c_int64(), _abi.C.c_int64(), _abi.C.c_int64()
        torch.cuda.synchronize()
        _lib.check(lib.sfb200_device_memory(ctx.ptr, _abi.C.byref(free0), _abi.C.byref(total)), ctx.ptr)
        _lib.check(lib.sfb200_run_noalloc(plan.ptr, xd.data_ptr(), ud.data_ptr(), w.n, 0, sums.data_ptr(),
                                          counts.data_ptr(), ctx.stream), ctx.ptr, "run_noalloc")
        torch.cuda.synchronize()
        _lib.check(lib.sfb200_device_memory(ctx.ptr, _abi.C.byref(free1), _abi.C.byref(total)), ctx.ptr)
        assert free1.value == free0.value
        s, c = sums.cpu().numpy(), counts.cpu().numpy()
        assert np.array_equal(c, ref_c)
        assert int(c.sum()) == w.pairs
        for k in range(len(w.ops)):
            sl = slice(k * nb, (k + 1) * nb)
            compare(s[sl], c, os_[sl], oc, oa[sl], tol)
            compare(s[sl], c, ref_s[sl], ref_c, oa[sl], 2 * tol)
    finally:
        plan.close()
        ctx.close()


def test_noalloc_refuses_what_does_not_fit():
    ctx = _lib.Context(0)
    w = synthetic.config("c0", n=70000)  # above the fixed scratch of 65536 points
    desc, keep = plan_description(w.ops, 2, w.distance_bins, None, w.metric, "mixed", w.x.dtype, w.u.dtype)
    plan = _lib.Plan(ctx, desc, keep)
    xd, ud = device_inputs(w)
    out = torch.zeros(plan.n_sums, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(plan.n_counts, dtype=torch.int64, device="cuda")
    try:
        with pytest.raises(ArgumentError, match="exceed its fixed scratch"):
            _lib.check(_lib.load().sfb200_run_noalloc(plan.ptr, xd.data_ptr(), ud.data_ptr(), w.n, 0,
                                                      out.data_ptr(), cnt.data_ptr(), ctx.stream), ctx.ptr)
    finally:
        plan.close()
        ctx.close()
