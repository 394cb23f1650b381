"""GPU parity: libsfb200.so through the C ABI against the CPU oracle on the same seeded inputs.

Counts must be identical (bit-exact, joint cells included); sums must agree per bin within
TOL_FP64 (FP64 kernels) or TOL_MIXED (FP32 kernels) times the oracle's per-bin sum of |value|.
"""
import math

import numpy as np
import pytest

import oracle_py
from helpers import TOL_FP32, TOL_FP64, TOL_FP64_SPHERE, TOL_MIXED, compare, sphere_tol
import sfb200 as SF
from sfb200 import _abi, _lib, synthetic
from sfb200.api import plan_description

pytestmark = pytest.mark.gpu

PRECISIONS = [("fp64", TOL_FP64), ("mixed", TOL_MIXED), ("fp32", TOL_FP32)]


def run_gpu(ops, x, u, bins, metric=None, value_bins=None, precision="mixed", tile=0, priv=None, options=None):
    be = SF.B200Backend(precision=precision, tile=tile)
    desc, keep = plan_description(ops, u.shape[0], bins, value_bins, metric, precision, x.dtype, u.dtype)
    plan = _lib.Plan(be.context, desc, keep)
    if tile or priv is not None:
        plan.set_launch(tile, -1 if priv is None else priv, 0)
    for opt, val in (options or {}).items():
        plan.set_option(opt, val)
    sums = np.zeros(plan.n_sums)
    counts = np.zeros(plan.n_counts, dtype=np.uint64)
    xa = np.asfortranarray(x)
    ua = np.asfortranarray(u)
    plan.run(xa.ctypes.data, ua.ctypes.data, x.shape[1], 0, sums.ctypes.data, counts.ctypes.data)
    st = plan.stats()
    plan.close()
    return sums, counts, st


def run_oracle(ops, x, u, bins, metric=None, value_bins=None):
    desc, keep = plan_description(ops, u.shape[0], bins, value_bins, metric, "fp64", x.dtype, u.dtype)
    return oracle_py.run(desc, x, u, with_abs=True)


def check(ops, x, u, bins, metric=None, value_bins=None, precision="mixed", tol=TOL_MIXED, tile=0):
    gs, gc, st = run_gpu(ops, x, u, bins, metric, value_bins, precision, tile)
    rs, rc, ra = run_oracle(ops, x, u, bins, metric, value_bins)
    nb = len(bins) - 1
    if value_bins is None:
        scale = ra
        for k in range(len(ops)):
            compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], tol)
    else:
        compare(gs, gc, rs, rc, ra, tol)
    return st


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("D", [2, 3])
def test_flat_l2_random(precision, tol, D):
    rng = np.random.default_rng(10 + D)
    x = rng.random((D, 1500))
    u = rng.standard_normal((D, 1500))
    bins = synthetic.log_edges(1e-3, math.sqrt(D), 24)
    check((SF.L2SF,), x, u, bins, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_quad_3d(precision, tol):
    w = synthetic.config("c1", n=2048)
    check(w.ops, w.x, w.u, w.distance_bins.edges, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_c0_full(precision, tol):
    w = synthetic.config("c0")
    check(w.ops, w.x, w.u, w.distance_bins.edges, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("opset", [
    (SF.S2SF,), (SF.T2SF,), (SF.L3SF,), (SF.T3SF,), (SF.S3SF,), (SF.L1T2SF,), (SF.L2T1SF,), (SF.T2ComponentSF,),
    (SF.L1T2ComponentSF,), (SF.FullVectorStructureFunctionType(3),), (SF.ProjectedStructureFunctionType(1, 1),),
    (SF.L2SF, SF.T2SF), (SF.S2SF, SF.L2SF, SF.T2SF, SF.S3SF, SF.L3SF, SF.L1T2SF),
])
@pytest.mark.parametrize("D", [2, 3])
def test_flat_operator_matrix(precision, tol, opset, D):
    rng = np.random.default_rng(100 + D)
    x = rng.random((D, 700))
    u = rng.standard_normal((D, 700))
    bins = np.linspace(0.0, math.sqrt(D), 17)
    check(opset, x, u, bins, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_linear_bins(precision, tol):
    rng = np.random.default_rng(7)
    x = rng.random((2, 1200))
    u = rng.standard_normal((2, 1200))
    bins = SF.LinearBinEdges(0.0, 1.4, 11)
    check((SF.L2SF,), x, u, bins, precision=precision, tol=tol)


_LINEAR_CASE = {}


def _linear_case():
    """18500 points with LinearBinEdges(0, 0.3, 33) (the shape of the reference's own GPU benchmark) and
    a row of points whose distances from one point fall on the edges and one ulp either side."""
    if not _LINEAR_CASE:
        rng = np.random.default_rng(21)
        x = rng.random((2, 18500))
        bins = SF.LinearBinEdges(0.0, 0.3, 33)
        row = [0.5]
        for e in bins.edges:
            for v in (e, np.nextafter(e, 1.0), np.nextafter(e, 0.0)):
                row.append(0.5 + v)
        x[0, :len(row)] = row
        x[1, :len(row)] = 0.5
        u = rng.standard_normal((2, 18500))
        _LINEAR_CASE["case"] = (x, u, bins, run_oracle((SF.L2SF,), x, u, bins))
    return _LINEAR_CASE["case"]


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_linear_bins_large(precision, tol):
    """A LinearBinEdges distance axis at a size with many tile pairs per block: the oracle's FMA search
    on the rounded distance, bit for bit, edges and edge +- 1 ulp included."""
    x, u, bins, (rs, rc, ra) = _linear_case()
    gs, gc, st = run_gpu((SF.L2SF,), x, u, bins, precision=precision)
    compare(gs, gc, rs, rc, ra, tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_flat_float32_inputs(precision, tol):
    rng = np.random.default_rng(8)
    x = rng.random((2, 1500)).astype(np.float32)
    u = rng.standard_normal((2, 1500)).astype(np.float32)
    bins = np.linspace(0.0, 1.4, 11).astype(np.float32)
    check((SF.L2SF,), x, u, bins, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("D", [2, 3])
def test_sphere_l2(precision, tol, D):
    w = synthetic.config("c2", n=1500)
    u = w.u
    if D == 3:
        u = np.vstack([w.u, np.random.default_rng(5).standard_normal((1, w.n)).astype(np.float32)])
    check((SF.L2SF, SF.T2SF, SF.S2SF) if D == 3 else w.ops, w.x, u, w.distance_bins.edges, metric=w.metric,
          precision=precision, tol=sphere_tol(precision, tol))


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_sphere_radians_and_odd_ops(precision, tol):
    rng = np.random.default_rng(9)
    lon = rng.uniform(-math.pi, math.pi, 900)
    lat = np.arcsin(rng.uniform(-1, 1, 900))
    x = np.stack([lon, lat])
    u = rng.standard_normal((2, 900))
    bins = np.linspace(0.0, math.pi, 13)
    check((SF.L3SF, SF.T3SF, SF.L2T1SF), x, u, bins, metric=SF.SphericalAngle(), precision=precision,
          tol=sphere_tol(precision, tol))


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_joint_c3_subset(precision, tol):
    w = synthetic.config("c3", n=3000)
    check(w.ops, w.x, w.u, w.distance_bins.edges, value_bins=w.value_bins, precision=precision, tol=tol)


@pytest.mark.parametrize("tile", [512, 768])
def test_joint_mixed_tiles(tile):
    """The mixed joint kernel's 512- and 768-thread forms (flat 2D and 3D, sphere) give the oracle's
    histogram; the 768-point tile is the flat default from 32768 points."""
    w = synthetic.config("c3", n=2600)
    check(w.ops, w.x, w.u, w.distance_bins.edges, value_bins=w.value_bins, tol=TOL_MIXED, tile=tile)
    w3 = synthetic.config("c1", n=1700)
    check((SF.ProjectedStructureFunctionType(1, 0),), w3.x, w3.u, w3.distance_bins.edges,
          value_bins=SF.LinearBinEdges(-4.0, 4.0, 97), tol=TOL_MIXED, tile=tile)
    ws = synthetic.config("c2", n=1500)
    check((SF.ProjectedStructureFunctionType(1, 0),), ws.x, ws.u, ws.distance_bins.edges, metric=ws.metric,
          value_bins=SF.LinearBinEdges(-3.0, 3.0, 61), tol=TOL_MIXED, tile=tile)


def test_joint_fp64_vector_value_bins():
    rng = np.random.default_rng(11)
    x = rng.random((2, 800))
    u = rng.standard_normal((2, 800))
    check((SF.L2SF,), x, u, np.linspace(0, 1.4, 9), value_bins=np.linspace(0.0, 4.0, 11), precision="fp64",
          tol=TOL_FP64)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_joint_sphere(precision, tol):
    w = synthetic.config("c2", n=1200)
    vb = SF.LinearBinEdges(-3.0, 3.0, 61)
    check((SF.ProjectedStructureFunctionType(1, 0),), w.x, w.u, w.distance_bins.edges, metric=w.metric,
          value_bins=vb, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("priv", [0, 1, 2, 3, 4, 6, 8, 32])
@pytest.mark.parametrize("tile", [32, 64, 256])
def test_privatization_modes(precision, tol, priv, tile):
    """Every histogram privatization depth and tile size gives the oracle's histogram."""
    w = synthetic.config("c1", n=1500)
    gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, precision=precision, tile=tile, priv=priv)
    # two open runs (6) exist in the flat FP64 and MIXED kernels; FP32-bulk plans take the run table
    assert st["privatization"] == (3 if priv == 6 and precision == "fp32" else priv) and st["tile"] <= tile
    rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges)
    nb = len(w.distance_bins) - 1
    for k in range(len(w.ops)):
        compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], tol)
    ws = synthetic.config("c2", n=700)
    gs, gc, st = run_gpu(ws.ops, ws.x, ws.u, ws.distance_bins.edges, metric=ws.metric, precision=precision,
                         tile=tile, priv=priv)
    rs, rc, ra = run_oracle(ws.ops, ws.x, ws.u, ws.distance_bins.edges, metric=ws.metric)
    compare(gs, gc, rs, rc, ra, sphere_tol(precision, tol))


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("cols", [1, 8, 32])
def test_point_order_and_table_columns(precision, tol, order, cols):
    """Morton-ordered storage and every run-length table width give the oracle's histogram."""
    opts = {_abi.OPT_POINT_ORDER: order, _abi.OPT_HIST_COLUMNS: cols}
    w = synthetic.config("c1", n=2000)
    gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, precision=precision, priv=3, options=opts)
    rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges)
    nb = len(w.distance_bins) - 1
    for k in range(len(w.ops)):
        compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], tol)
    for name in ("c0", "c2"):
        w = synthetic.config(name, n=2500)
        gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric, precision=precision,
                             priv=3, options=opts)
        rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric)
        compare(gs, gc, rs, rc, ra, sphere_tol(precision, tol) if name == "c2" else tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_joint_point_order(precision, tol):
    """The joint flat histogram is the same in caller and Morton order."""
    w = synthetic.config("c3", n=2500)
    for order in (0, 1, 2):
        gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, value_bins=w.value_bins,
                             precision=precision, options={_abi.OPT_POINT_ORDER: order})
        rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges, value_bins=w.value_bins)
        compare(gs, gc, rs, rc, ra, tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("count", [2, 3, 8])
def test_tile_pair_shards_add_up(precision, tol, count):
    """The shards of SFB200_OPT_SHARD (one per GPU in a multi-GPU run), run one after another and
    added, give the oracle's histogram."""
    for name, n in (("c1", 3000), ("c2", 2000), ("c3", 2500)):
        w = synthetic.config(name, n=n)
        tot_s, tot_c = None, None
        for k in range(count):
            gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric, value_bins=w.value_bins,
                                 precision=precision, options={_abi.OPT_SHARD: (count << 32) | k})
            tot_s = gs if tot_s is None else tot_s + gs
            tot_c = gc if tot_c is None else tot_c + gc
        rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric, value_bins=w.value_bins)
        compare(tot_s, tot_c, rs, rc, ra, sphere_tol(precision, tol) if name == "c2" else tol)


def test_autotuned_backend_gives_the_oracle_histogram():
    """B200Backend(autotune=True): the first call times the launch candidates, applies the fastest
    (cached per shape), and the result still equals the oracle's."""
    from sfb200 import autotune

    autotune.clear()
    be = SF.B200Backend(autotune=True)
    for name, n in (("c1", 3000), ("c0", 4096)):
        w = synthetic.config(name, n=n)
        op = w.ops[0]
        r = SF.calculate_structure_function(op, w.x, w.u, w.distance_bins.edges, backend=be,
                                            output_type=SF.StructureFunctionSumsAndCounts)
        desc, keep = plan_description((op,), w.u.shape[0], w.distance_bins.edges, None, None, "mixed", w.x.dtype,
                                      w.u.dtype)
        assert autotune.lookup(autotune.shape_key(desc, n)) is not None
        rs, rc, ra = run_oracle((op,), w.x, w.u, w.distance_bins.edges)
        compare(np.asarray(r.sums, dtype=np.float64), r.counts, rs, rc, ra, TOL_MIXED)


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_tiny_and_empty(precision):
    be = SF.B200Backend(precision=precision)
    for n in (0, 1, 2, 3):
        x = np.arange(2 * n, dtype=np.float64).reshape(2, n) / 10.0
        u = np.ones((2, n))
        r = SF.calculate_structure_function(SF.L2SF, x, u, [0.0, 3.0], backend=be,
                                            output_type=SF.StructureFunctionSumsAndCounts)
        assert int(r.counts.sum()) == n * (n - 1) // 2


@pytest.mark.parametrize("precision", ["fp64", "mixed", "fp32"])
def test_points_on_edges_exact(precision):
    """Pairs placed exactly on bin edges (right-inclusive) and at edge +- 1 ulp."""
    edges = np.array([0.1, 0.2, 0.3, 0.5])
    xs = [0.0]
    for e in edges:
        xs += [e, np.nextafter(e, 1.0), np.nextafter(e, 0.0)]
    x = np.zeros((2, len(xs)))
    x[0] = xs
    u = np.random.default_rng(3).standard_normal((2, len(xs)))
    check((SF.L2SF,), x, u, edges, precision=precision, tol=TOL_MIXED)


@pytest.mark.parametrize("xscale,uscale", [(1e-15, 1e30), (1e12, 1e-25), (3.0, 7.0)])
def test_mixed_extreme_scales(xscale, uscale):
    """The mixed kernels scale into FP32 range exactly: coordinates and velocities far outside
    FP32's comfortable range (third-order values ~1e90 or ~1e-75) keep the 1e-6 tolerance."""
    w = synthetic.config("c1", n=1200)
    x = w.x * xscale
    u = w.u * uscale
    edges = w.distance_bins.edges * xscale
    check(w.ops, x, u, edges, precision="mixed", tol=TOL_MIXED)
    ws = synthetic.config("c2", n=800)
    check(ws.ops, ws.x, ws.u.astype(np.float64) * uscale, ws.distance_bins.edges, metric=ws.metric,
          precision="mixed", tol=TOL_MIXED)
    wj = synthetic.config("c3", n=1500)
    vb = SF.LinearBinEdges(wj.value_bins.first_edge * uscale, wj.value_bins.last_edge * uscale, len(wj.value_bins))
    check(wj.ops, wj.x.astype(np.float64) * xscale, wj.u.astype(np.float64) * uscale,
          wj.distance_bins.edges * xscale, value_bins=vb, precision="mixed", tol=TOL_MIXED)


@pytest.mark.parametrize("value_bins", [SF.LinearBinEdges(-1.0, 1.0, 9), SF.LinearBinEdges(-0.9, 1.1, 9)])
def test_joint_values_near_zero(value_bins):
    """Values a hundred times smaller than the half bin width, all in the value bins at or next to zero
    (an edge at zero, or a bin straddling it). Every cell, down to the few-pair cells of the smallest
    distances, must stay within 1e-6 of its sum |v|: the coarse fixed-point quantum alone bounds a
    pair's error only by 2^-22 of the half width (3e-8 here, 2e-5 of such a value), so this exercises
    the kernel's fine offsets near zero."""
    rng = np.random.default_rng(17)
    n = 1500
    x = rng.random((2, n))
    u = 1e-3 * rng.standard_normal((2, n))
    edges = synthetic.log_edges(1e-3, math.sqrt(2.0), 12)
    check((SF.ProjectedStructureFunctionType(1, 0),), x, u, edges, value_bins=value_bins)


@pytest.mark.parametrize("form", [1, 2])
def test_fp64_sphere_formulations(form):
    """Precision FP64 on the sphere in both formulations (SFB200_OPT_FORMULATION): 1 the reference's own
    (the pair frame for every pair), 2 the mixed kernel's chord algorithm in FP64 (the chord bin with
    its ambiguity band, increments from the chord and the tangent velocities). Both give the oracle's
    histogram to FP64 rounding."""
    opts = {_abi.OPT_FORMULATION: form}
    TOL = TOL_FP64 if form == 1 else TOL_FP64_SPHERE
    w = synthetic.config("c2", n=1500)
    gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric, precision="fp64", options=opts)
    rs, rc, ra = run_oracle(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric)
    compare(gs, gc, rs, rc, ra, TOL)
    rng = np.random.default_rng(31)
    u = rng.standard_normal((3, 1200))
    lon = rng.uniform(-180, 180, 1200)
    xs = np.stack([lon, np.degrees(np.arcsin(rng.uniform(-1, 1, 1200)))])
    ops = (SF.L2SF, SF.T2SF, SF.L3SF, SF.T3SF)
    bins = np.linspace(0.0, 20000.0, 17)
    gs, gc, st = run_gpu(ops, xs, u, bins, metric=SF.Haversine(6371.0), precision="fp64", options=opts)
    rs, rc, ra = run_oracle(ops, xs, u, bins, metric=SF.Haversine(6371.0))
    nb = len(bins) - 1
    for k in range(len(ops)):
        compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], TOL)
    # radians, odd operators and the single-pass list
    x = np.stack([rng.uniform(-math.pi, math.pi, 900), np.arcsin(rng.uniform(-1, 1, 900))])
    for ops in ((SF.L3SF, SF.T3SF, SF.L2T1SF), (SF.S2SF, SF.L2SF, SF.S3SF, SF.L3SF)):
        uu = rng.standard_normal((2, 900))
        b = np.linspace(0.0, math.pi, 13)
        gs, gc, st = run_gpu(ops, x, uu, b, metric=SF.SphericalAngle(), precision="fp64", options=opts)
        rs, rc, ra = run_oracle(ops, x, uu, b, metric=SF.SphericalAngle())
        nb = len(b) - 1
        for k in range(len(ops)):
            compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], TOL)
