"""The two-dimensional single pass on the GPU (calculate_structure_functions_single_pass_2d[!]): every
row (S2, L2, T2, S3, L3, L1T2) as a joint distance x value histogram of that invariant, against the
oracle's restatement of the reference's single-pass scatter (src/Calculations/serial_single_pass.jl:
876-909 flat, 820-849 other metrics). Counts bit-exact per cell and row; sums within the precision's
tolerance times the cell's sum of |value|."""
import math

import numpy as np
import pytest

import oracle_py
from helpers import TOL_FP32, TOL_FP64, TOL_MIXED, compare, sphere_tol
import sfb200 as SF
from sfb200 import synthetic
from sfb200.api import plan_description
from sfb200.single_pass import _single_pass_2d_raw

pytestmark = pytest.mark.gpu

PRECISIONS = [("fp64", TOL_FP64), ("mixed", TOL_MIXED), ("fp32", TOL_FP32)]
NAMES = ("S2", "L2", "T2", "S3", "L3", "L1T2")


def oracle_rows(x, u, dist, rows, metric=None):
    out = []
    for t in range(6):
        desc, keep = plan_description((SF.SinglePass2DRow(t),), u.shape[0], dist, rows[t], metric, "fp64",
                                      x.dtype, u.dtype)
        out.append(oracle_py.run(desc, x, u, with_abs=True))
    return out


def check(x, u, dist, value_bins, metric=None, precision="mixed", tol=TOL_MIXED):
    be = SF.B200Backend(precision=precision)
    sp = SF.calculate_structure_functions_single_pass_2d(x, u, dist, value_bins, backend=be, distance_metric=metric,
                                                         count_eltype=np.uint64)
    assert list(sp) == list(NAMES)
    rows = value_bins if isinstance(value_bins, tuple) else (value_bins,) * 6
    # the library's FP64 rows against the oracle at the precision's tolerance; the public containers
    # hold them in the reference's accumulator type, promote_type(float(FT1), float(FT2)) (Float32 for
    # Float32 inputs, which adds that rounding, 2^-24 of the sum)
    raw_s, raw_c, _ = _single_pass_2d_raw(be, x, u, dist, value_bins, SF.Euclidean() if metric is None else metric)
    f32 = x.dtype == np.float32 and u.dtype == np.float32
    for t, (name, (rs, rc, ra)) in enumerate(zip(NAMES, oracle_rows(x, u, dist, rows, metric))):
        compare(np.ravel(raw_s[t], order="F"), np.ravel(raw_c[t], order="F"), rs, rc, ra, tol)
        r = sp[name]
        assert isinstance(r, SF.StructureFunction2DSumsAndCounts)
        assert r.sums.dtype == (np.float32 if f32 else np.float64) and r.counts.dtype == np.uint64
        compare(np.ravel(r.sums, order="F"), np.ravel(r.counts, order="F"), rs, rc, ra,
                max(tol, 2.0 ** -23) if f32 else tol)
    assert int(sp["S2"].counts.sum()) > 0
    return sp


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_2d_shared_value_axis(precision, tol):
    w = synthetic.config("c3", n=2500)  # 2D, Float32 inputs
    sigma = float(np.std(w.u.astype(np.float64))) * math.sqrt(2.0)
    vb = SF.LinearBinEdges(-5.0 * sigma ** 2, 5.0 * sigma ** 2, 65)
    check(w.x, w.u, w.distance_bins.edges, vb, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_3d_per_row_value_axes(precision, tol):
    """A 6-tuple of value axes: log edges for the non-negative rows, a plain vector and a
    LinearBinEdges for the signed ones (test/test_single_pass_2d.jl:202-229)."""
    w = synthetic.config("c1", n=1800)
    lg = np.exp(np.linspace(np.log(1e-6), np.log(10.0), 33))
    raw = np.linspace(-3.0, 3.0, 33)
    lin = SF.LinearBinEdges(-3.0, 3.0, 33)
    check(w.x, w.u, w.distance_bins.edges, (lg, lg, lg, lin, raw, lin), precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_sphere(precision, tol):
    w = synthetic.config("c2", n=900)
    vb = np.linspace(-4.0, 8.0, 49)
    check(w.x, w.u, w.distance_bins.edges, vb, metric=w.metric, precision=precision, tol=sphere_tol(precision, tol))


def test_inplace_accumulates_and_matches():
    rng = np.random.default_rng(8)
    x = rng.random((2, 1500))
    u = rng.standard_normal((2, 1500))
    dist = synthetic.log_edges(1e-3, math.sqrt(2.0), 16)
    vb = np.linspace(-4.0, 6.0, 21)
    be = SF.B200Backend(precision="mixed")
    sp = SF.calculate_structure_functions_single_pass_2d(x, u, dist, vb, backend=be, count_eltype=np.uint64)
    sums = np.zeros((6, 16, 20))
    counts = np.zeros((6, 16, 20), dtype=np.uint64)
    for _ in range(2):
        SF.calculate_structure_functions_single_pass_2d_inplace(sums, counts, x, u, dist, vb, backend=be)
    for t, name in enumerate(NAMES):
        assert np.array_equal(counts[t], 2 * sp[name].counts)
        assert np.allclose(sums[t], 2 * sp[name].sums, rtol=1e-12, atol=0)


def test_auxiliary_axis_slices():
    """(D, N, B) velocities over shared positions: each slice's rows equal the point-field call."""
    rng = np.random.default_rng(9)
    x = rng.random((2, 900))
    u = rng.standard_normal((2, 900, 2))
    dist = synthetic.log_edges(1e-3, math.sqrt(2.0), 12)
    vb = np.linspace(-4.0, 6.0, 17)
    be = SF.B200Backend(precision="fp64")
    sp = SF.calculate_structure_functions_single_pass_2d(x, u, dist, vb, backend=be, count_eltype=np.uint64)
    for b in range(2):
        one = SF.calculate_structure_functions_single_pass_2d(x, np.ascontiguousarray(u[:, :, b]), dist, vb,
                                                              backend=be, count_eltype=np.uint64)
        for name in NAMES:
            assert np.array_equal(sp[name].counts[:, :, b], one[name].counts)
            assert np.allclose(sp[name].sums[:, :, b], one[name].sums, rtol=1e-13, atol=0)


def test_flat_mixed_rows_run_the_fp64_kernel():
    """Flat rows requested at precision MIXED run the FP64 joint kernel: the oracle's FP64 tolerance holds,
    nothing is rechecked, and such a plan refuses to become a batched slice."""
    import ctypes

    from sfb200 import _lib
    rng = np.random.default_rng(12)
    x = rng.random((2, 2000))
    u = rng.standard_normal((2, 2000))
    dist = synthetic.log_edges(1e-3, math.sqrt(2.0), 20)
    vb = SF.LinearBinEdges(-40.0, 40.0, 41)
    be = SF.B200Backend(precision="mixed")
    raw_s, raw_c, _ = _single_pass_2d_raw(be, x, u, dist, vb, SF.Euclidean())
    for t, (rs, rc, ra) in enumerate(oracle_rows(x, u, dist, (vb,) * 6)):
        compare(np.ravel(raw_s[t], order="F"), np.ravel(raw_c[t], order="F"), rs, rc, ra, TOL_FP64)
    ctx = _lib.Context(0)
    try:
        desc, keep = plan_description((SF.SinglePass2DRow(4),), 2, dist, vb, None, "mixed", x.dtype, u.dtype)
        plan = _lib.Plan(ctx, desc, keep)
        xs = np.asfortranarray(x)  # (D, N) column-major, the C ABI's layout
        us = np.asfortranarray(u)
        sums = np.zeros(plan.n_sums)
        counts = np.zeros(plan.n_counts, dtype=np.uint64)
        plan.run(xs.ctypes.data, us.ctypes.data, x.shape[1], 0, sums.ctypes.data, counts.ctypes.data)
        assert plan.stats()["rechecked"] == 0
        with pytest.raises(SF.ArgumentError, match="FP64 joint kernel"):
            _lib.Slice(plan, xs.ctypes.data_as(ctypes.c_void_p), us.ctypes.data_as(ctypes.c_void_p), x.shape[1])
    finally:
        ctx.close()


@pytest.mark.parametrize("D", [2, 3])
def test_row_group_plan_equals_single_row_plans(D):
    """A joint plan of consecutive flat rows (here rows 1-3, one launch) gives each row's single-row plan
    result: counts bit-exact, sums to FP64 rounding (the cell updates come in another order); rows that
    are not consecutive are refused."""
    from sfb200 import _lib
    rng = np.random.default_rng(13 + D)
    n = 1800
    x = np.asfortranarray(rng.random((D, n)))
    u = np.asfortranarray(rng.standard_normal((D, n)))
    dist = synthetic.log_edges(1e-3, math.sqrt(float(D)), 24)
    vb = SF.LinearBinEdges(-6.0, 10.0, 33)
    ctx = _lib.Context(0)
    try:
        def run(rows):
            desc, keep = plan_description(tuple(SF.SinglePass2DRow(t) for t in rows), D, dist, vb, None, "mixed",
                                          x.dtype, u.dtype)
            plan = _lib.Plan(ctx, desc, keep)
            sums = np.zeros(plan.n_sums)
            counts = np.zeros(plan.n_counts, dtype=np.uint64)
            plan.run(x.ctypes.data, u.ctypes.data, n, 0, sums.ctypes.data, counts.ctypes.data)
            return sums, counts

        gs, gc = run((1, 2, 3))
        m = 24 * 32
        assert gs.size == 3 * m and gc.size == 3 * m
        for g, t in enumerate((1, 2, 3)):
            s1, c1 = run((t,))
            assert np.array_equal(gc[g * m:(g + 1) * m], c1)
            # the value axis has an edge at 0, so a cell's values share one sign (no cancellation)
            assert np.allclose(gs[g * m:(g + 1) * m], s1, rtol=1e-11, atol=1e-300)
        assert int(gc.sum()) > 0
        with pytest.raises(SF.ArgumentError, match="consecutive"):
            run((1, 3))
    finally:
        ctx.close()
