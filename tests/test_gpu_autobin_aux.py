"""Automatic binning and auxiliary-axis inputs through the library (the reference's rows beside the
pair loop: dispatch.jl:153-298 and the (D, N, aux...) shapes of shapes.jl:17-20 / batch.jl:201-217).

- The device scan of the pair-distance range equals a brute-force scan of all pairs (Euclidean in FP64
  exactly; the sphere to 1e-12 relative), and an integer `distance_bins` gives the histogram of the
  explicit edges built from that range (log and linear spacing).
- Shared-position and varying-position auxiliary axes give, slice by slice, the oracle's histogram
  of that slice (1D and joint), in the (n_bins, aux...) layout.
"""
import math

import numpy as np
import pytest

import oracle_py
from helpers import TOL_FP64, TOL_MIXED, compare, sphere_tol
import sfb200 as SF
from sfb200 import synthetic
from sfb200.api import plan_description

pytestmark = pytest.mark.gpu


def brute_range(x, metric=None):
    x = np.asarray(x, dtype=np.float64)
    n = x.shape[1]
    lo, hi = math.inf, 0.0
    if metric is None:
        for i in range(n - 1):
            d = x[:, i + 1:] - x[:, i:i + 1]
            r2 = d[0] * d[0]
            for k in range(1, x.shape[0]):
                r2 = r2 + d[k] * d[k]
            lo, hi = min(lo, float(r2.min())), max(hi, float(r2.max()))
        return math.sqrt(lo), math.sqrt(hi)
    lon, lat = np.radians(x[0]), np.radians(x[1])
    p = np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])
    for i in range(n - 1):
        d = p[:, i + 1:] - p[:, i:i + 1]
        c2 = (d * d).sum(axis=0)
        lo, hi = min(lo, float(c2.min())), max(hi, float(c2.max()))
    arc = lambda c: metric.radius * 2.0 * math.atan2(math.sqrt(c), math.sqrt(max(4.0 - c, 0.0)))  # noqa: E731
    return arc(lo), arc(hi)


@pytest.mark.parametrize("D", [2, 3])
def test_distance_range_flat_is_exact(D):
    rng = np.random.default_rng(60 + D)
    x = rng.random((D, 3000))
    u = rng.standard_normal((D, 3000))
    lo, hi = SF.distance_range(x, u)
    blo, bhi = brute_range(x)
    assert lo == blo and hi == bhi


def test_distance_range_sphere():
    w = synthetic.config("c2", n=2500)
    lo, hi = SF.distance_range(w.x, w.u, w.metric)
    blo, bhi = brute_range(w.x, w.metric)
    assert math.isclose(lo, blo, rel_tol=1e-6) and math.isclose(hi, bhi, rel_tol=1e-6)


@pytest.mark.parametrize("spacing", [None, SF.LinearBinEdges])
def test_integer_bins_equal_explicit_edges(spacing):
    rng = np.random.default_rng(70)
    x = rng.random((2, 2000))
    u = rng.standard_normal((2, 2000))
    r = SF.calculate_structure_function(SF.L2SF, x, u, 20, bin_spacing=spacing,
                                        output_type=SF.StructureFunctionSumsAndCounts)
    lo, hi = SF.distance_range(x, u)
    edges = SF.auto_distance_bins(lo, hi, 20, spacing)
    assert len(r.distance) == 21 and np.array_equal(np.asarray(r.distance), np.asarray(edges))
    desc, keep = plan_description((SF.L2SF,), 2, edges, None, None, "fp64", x.dtype, u.dtype)
    rs, rc, ra = oracle_py.run(desc, x, u, with_abs=True)
    compare(r.sums, r.counts, rs, rc, ra, TOL_MIXED)
    # the edges span the pairs: prevfloat(min) lies below the closest pair and max is the last edge. A
    # LogBinEdges rebuilds its edges as exp of a log-uniform grid (src/BinEdges.jl:180-183), so the
    # last edge can round an ulp below the largest distance and drop the farthest pair, as in the
    # reference; linear edges keep max exactly
    if spacing is SF.LinearBinEdges:
        assert int(rc.sum()) == 2000 * 1999 // 2
    else:
        assert int(rc.sum()) >= 2000 * 1999 // 2 - 2


def _slice_oracle(ops, xb, ub, bins, value_bins=None, metric=None):
    desc, keep = plan_description(ops, ub.shape[0], bins, value_bins, metric, "fp64", xb.dtype, ub.dtype)
    return oracle_py.run(desc, np.asarray(xb), np.asarray(ub), with_abs=True)


@pytest.mark.parametrize("precision,tol", [("mixed", TOL_MIXED), ("fp64", TOL_FP64)])
def test_shared_positions_auxiliary_axes(precision, tol):
    rng = np.random.default_rng(80)
    n = 1200
    x = rng.random((2, n))
    u = rng.standard_normal((2, n, 3, 2))
    bins = synthetic.log_edges(1e-3, math.sqrt(2.0), 12)
    be = SF.B200Backend(precision=precision)
    r = SF.calculate_structure_function(SF.L2SF, x, u, bins, backend=be, count_eltype=np.uint64,
                                        output_type=SF.StructureFunctionSumsAndCounts)
    assert r.sums.shape == (12, 3, 2) and r.counts.shape == (12, 3, 2)
    for a in range(3):
        for b in range(2):
            rs, rc, ra = _slice_oracle((SF.L2SF,), x, u[:, :, a, b], bins)
            compare(r.sums[:, a, b], r.counts[:, a, b], rs, rc, ra, tol)
    # the geometry is shared: every slice has the same counts
    assert (r.counts == r.counts[:, :1, :1]).all()


@pytest.mark.parametrize("precision,tol", [("mixed", TOL_MIXED), ("fp64", TOL_FP64)])
def test_varying_positions_joint_and_sphere(precision, tol):
    rng = np.random.default_rng(81)
    n, B = 900, 3
    x = rng.random((2, n, B))
    u = rng.standard_normal((2, n, B))
    bins = synthetic.log_edges(1e-3, math.sqrt(2.0), 10)
    vb = SF.LinearBinEdges(-3.0, 3.0, 25)
    be = SF.B200Backend(precision=precision)
    op = SF.ProjectedStructureFunctionType(1, 0)
    r = SF.calculate_structure_function(op, x, u, bins, vb, backend=be)
    assert r.sums.shape == (10, 24, B)
    for b in range(B):
        rs, rc, ra = _slice_oracle((op,), x[:, :, b], u[:, :, b], bins, vb)
        compare(r.sums[:, :, b].ravel(order="F"), r.counts[:, :, b].ravel(order="F"), rs, rc, ra, tol)
    w = synthetic.config("c2", n=800)
    xs = np.stack([w.x, w.x[:, ::-1]], axis=-1).astype(np.float64)
    us = np.stack([w.u, w.u[:, ::-1]], axis=-1).astype(np.float64)
    r = SF.calculate_structure_function(SF.L2SF, xs, us, w.distance_bins.edges, backend=be, distance_metric=w.metric,
                                        output_type=SF.StructureFunctionSumsAndCounts, count_eltype=np.uint64)
    for b in range(2):
        rs, rc, ra = _slice_oracle((SF.L2SF,), xs[:, :, b], us[:, :, b], w.distance_bins.edges, metric=w.metric)
        compare(r.sums[:, b], r.counts[:, b], rs, rc, ra, sphere_tol(precision, tol))


def test_inplace_auxiliary_axes_accumulate():
    rng = np.random.default_rng(82)
    x = rng.random((3, 700))
    u = rng.standard_normal((3, 700, 4))
    bins = synthetic.log_edges(1e-3, math.sqrt(3.0), 8)
    sums = np.zeros((8, 4))
    counts = np.zeros((8, 4), dtype=np.uint64)
    for _ in range(2):
        SF.calculate_structure_function_inplace(sums, counts, SF.L3SF, x, u, bins)
    for b in range(4):
        rs, rc, ra = _slice_oracle((SF.L3SF,), x, u[:, :, b], bins)
        compare(sums[:, b], counts[:, b], 2 * rs, 2 * rc, 2 * ra, TOL_MIXED)
