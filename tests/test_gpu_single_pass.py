"""The six-invariant single pass on the GPU (calculate_structure_functions_single_pass): one fused pair
pass accumulating S2, L2, S3, L3, with T2 and L1T2 derived per bin, against the oracle's restatement of
the reference's single-pass loop (src/Calculations/serial_single_pass.jl:238-270, 321-350, 209-219).

Counts bit-exact (all six rows); the accumulated rows within the precision's tolerance times their
per-bin sum of |value|, the derived rows within it times the sum of the two rows' |value| sums (the
scale of a difference, as the reference forms them).
"""
import math

import numpy as np
import pytest

import oracle_py
from helpers import TOL_FP32, TOL_FP64, TOL_MIXED, sphere_tol
import sfb200 as SF
from sfb200 import synthetic
from sfb200.api import plan_description

pytestmark = pytest.mark.gpu

PRECISIONS = [("fp64", TOL_FP64), ("mixed", TOL_MIXED), ("fp32", TOL_FP32)]
NAMES = ("S2", "L2", "T2", "S3", "L3", "L1T2")


def oracle_sp(x, u, bins, metric=None):
    desc, keep = plan_description((SF.L2SF,), u.shape[0], bins, None, metric, "fp64", x.dtype, u.dtype)
    return oracle_py.run_single_pass(desc, x, u)


def check(x, u, bins, metric=None, precision="mixed", tol=TOL_MIXED):
    be = SF.B200Backend(precision=precision)
    sp = SF.calculate_structure_functions_single_pass(x, u, bins, backend=be, distance_metric=metric,
                                                      output_type=SF.StructureFunctionSumsAndCounts,
                                                      count_eltype=np.uint64)
    assert list(sp) == list(NAMES) + ["helmholtz"]
    rs, rc, ra = oracle_sp(x, u, bins, metric)
    for t, name in enumerate(NAMES):
        assert np.array_equal(sp[name].counts, rc[t]), name
        err = np.abs(sp[name].sums.astype(np.float64) - rs[t])
        assert np.all(err <= tol * np.maximum(ra[t], 1e-300)), (name, float(np.max(err / np.maximum(ra[t], 1e-300))))
    assert int(rc[0].sum()) > 0
    return sp


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("D", [2, 3])
def test_single_pass_flat(precision, tol, D):
    rng = np.random.default_rng(40 + D)
    x = rng.random((D, 2500))
    u = rng.standard_normal((D, 2500))
    check(x, u, synthetic.log_edges(1e-3, math.sqrt(D), 24), precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_single_pass_c1_fields_morton_order(precision, tol):
    """20000 points of the 3D benchmark field: Morton point order and sorted tiles are in play."""
    w = synthetic.config("c1", n=20000)
    check(w.x, w.u, w.distance_bins.edges, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_single_pass_linear_distance_axis(precision, tol):
    """The reference's published single-pass shape (20000 points, 32 LinearBinEdges bins over (0, 0.3]):
    the mixed kernel's form compiled for a linear distance axis (bin from the FP32 distance, the FP64
    search near an edge)."""
    w = synthetic.config("rsp1d")
    check(w.x.astype(np.float64), w.u.astype(np.float64), w.distance_bins, precision=precision, tol=tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_single_pass_sphere(precision, tol):
    w = synthetic.config("c2", n=2000)
    # Float64 copies of the Float32 inputs (exact): the results then come back as Float64, so the
    # FP64 tolerance is not hidden by a Float32 output type
    check(w.x.astype(np.float64), w.u.astype(np.float64), w.distance_bins.edges, metric=w.metric,
          precision=precision, tol=sphere_tol(precision, tol))


def test_reference_three_point_case():
    """test/test_single_pass.jl:26-66 through the library: counts [2, 1] and the separate-operator sums."""
    x = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    sp = check(x, x.copy(), np.array([0.1, 1.0, 2.0]))
    assert sp["S2"].counts.tolist() == [2, 1]
    h = sp["helmholtz"]
    d_ll = sp["L2"].sums / sp["L2"].counts
    d_tt = sp["T2"].sums / sp["T2"].counts
    rot = h.rotational_sums / h.rotational_counts
    div = h.divergent_sums / h.divergent_counts
    assert np.allclose(rot + div, d_ll + d_tt, atol=1e-12)


def test_inplace_accumulates_and_rederives():
    rng = np.random.default_rng(5)
    x = rng.random((2, 1500))
    u = rng.standard_normal((2, 1500))
    bins = synthetic.log_edges(1e-3, math.sqrt(2.0), 16)
    sums = np.zeros((6, 16))
    counts = np.zeros((6, 16), dtype=np.uint64)
    for _ in range(2):
        SF.calculate_structure_functions_single_pass_inplace(sums, counts, x, u, bins)
    rs, rc, ra = oracle_sp(x, u, bins)
    assert np.array_equal(counts, 2 * rc)
    assert np.all(np.abs(sums - 2 * rs) <= 2 * TOL_MIXED * np.maximum(ra, 1e-300))
    assert np.allclose(sums[2], sums[0] - sums[1]) and np.allclose(sums[5], sums[3] - sums[4])
