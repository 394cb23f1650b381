"""The two-dimensional single pass on the CPU: the oracle's rows against a plain-Python restatement of
the reference's flat single-pass scatter (src/Calculations/serial_single_pass.jl:876-909, 852-864), the
properties the reference's own tests check (test/test_single_pass_2d.jl: per-invariant equivalence
with the standalone joint operators, marginals equal to the 1D single pass), and the host-side
validation of the value axes."""
import math

import numpy as np
import pytest

import oracle_py
import sfb200 as SF
from sfb200.api import plan_description
from sfb200.single_pass import SINGLE_PASS_OPERATORS, _row_bins, _rows_per_launch, _sp2d_value_bins


def _oracle_rows(x, u, dist_edges, rows, metric=None):
    """(6, nd, nv) sums / counts / sum|v| of the oracle, one joint plan per row."""
    nd = len(dist_edges) - 1
    nv = len(rows[0]) - 1
    s = np.zeros((6, nd, nv))
    c = np.zeros((6, nd, nv), dtype=np.uint64)
    a = np.zeros((6, nd, nv))
    for t in range(6):
        desc, keep = plan_description((SF.SinglePass2DRow(t),), u.shape[0], dist_edges, rows[t], metric, "fp64",
                                      x.dtype, u.dtype)
        rs, rc, ra = oracle_py.run(desc, x, u, with_abs=True)
        s[t] = rs.reshape((nd, nv), order="F")
        c[t] = rc.reshape((nd, nv), order="F")
        a[t] = ra.reshape((nd, nv), order="F")
    return s, c, a


def _python_rows(x, u, dist_edges, rows):
    """Plain-Python restatement of _sp2d_simd_pairs! (flat, vector bins): r2 = dot(dx, dx), bin from
    searchsortedfirst over the squared edges, du_L = dot(du, dx) * inv(sqrt(r2)), dn2 = dot(du, du), the
    six rows, each digitized on its own edges and kept when 1 <= vbin <= n_val."""
    D, N = u.shape
    sq = [float(e) * float(e) for e in dist_edges]
    nd, nv = len(dist_edges) - 1, len(rows[0]) - 1
    s = np.zeros((6, nd, nv))
    c = np.zeros((6, nd, nv), dtype=np.uint64)
    for i in range(N):
        for j in range(i + 1, N):
            dx = [float(x[k, j]) - float(x[k, i]) for k in range(D)]
            du = [float(u[k, j]) - float(u[k, i]) for k in range(D)]
            r2 = dx[0] * dx[0]
            for k in range(1, D):
                r2 = r2 + dx[k] * dx[k]
            # digitize = searchsortedfirst (1-based) - 1 = numpy's 0-based searchsorted
            db = int(np.searchsorted(sq, r2, side="left"))
            if not 1 <= db <= nd:
                continue
            p = du[0] * dx[0]
            dn2 = du[0] * du[0]
            for k in range(1, D):
                p = p + du[k] * dx[k]
                dn2 = dn2 + du[k] * du[k]
            duL = p * (1.0 / math.sqrt(r2))
            duL2 = duL * duL
            duT2 = dn2 - duL2
            vals = (dn2, duL2, duT2, duL * dn2, duL * duL2, duL * duT2)
            for t in range(6):
                vb = int(np.searchsorted(np.asarray(rows[t], dtype=np.float64), vals[t], side="left"))
                if 1 <= vb <= nv:
                    s[t, db - 1, vb - 1] += vals[t]
                    c[t, db - 1, vb - 1] += 1
    return s, c


@pytest.mark.parametrize("D", [2, 3])
def test_oracle_rows_match_python_restatement(D):
    rng = np.random.default_rng(11 + D)
    x = rng.random((D, 90))
    u = rng.standard_normal((D, 90))
    dist = np.exp(np.linspace(np.log(0.02), np.log(2.0), 9))
    shared = np.linspace(-2.0, 3.0, 13)
    rows = [shared] * 6
    s, c, a = _oracle_rows(x, u, dist, rows)
    ps, pc = _python_rows(x, u, dist, rows)
    assert np.array_equal(c, pc)
    assert np.allclose(s, ps, rtol=0, atol=1e-12 * max(1.0, float(np.abs(ps).max())))
    assert int(c.sum()) > 0


def test_per_invariant_value_axes():
    # a 6-tuple of value axes: log edges for the non-negative rows, linear ones for the signed rows
    rng = np.random.default_rng(5)
    x = rng.random((2, 70))
    u = rng.standard_normal((2, 70))
    dist = np.linspace(0.0, 1.5, 7)
    lg = np.exp(np.linspace(np.log(1e-4), np.log(10.0), 9))
    lin = np.linspace(-5.0, 5.0, 9)
    rows = [lg, lg, lg, lin, lin, lin]
    s, c, _ = _oracle_rows(x, u, dist, rows)
    ps, pc = _python_rows(x, u, dist, rows)
    assert np.array_equal(c, pc)
    assert np.allclose(s, ps, rtol=0, atol=1e-11)


def test_rows_match_standalone_joint_operators():
    # test/test_single_pass_2d.jl:44-53: row t equals the standalone joint histogram of the same
    # invariant (to the rounding of the two formulas; counts equal on generic data)
    rng = np.random.default_rng(42)
    x = rng.random((2, 40)) * 50000.0
    u = rng.standard_normal((2, 40)) * 0.5
    dist = np.exp(np.linspace(np.log(1000.0), np.log(50000.0), 6))
    vb = np.linspace(-1.0, 2.0, 11)
    s, c, _ = _oracle_rows(x, u, dist, [vb] * 6)
    for t, op in enumerate(SINGLE_PASS_OPERATORS.values()):
        desc, keep = plan_description((op,), 2, dist, vb, None, "fp64", x.dtype, u.dtype)
        rs, rc = oracle_py.run(desc, x, u)
        assert np.array_equal(c[t], rc.reshape(c[t].shape, order="F"))
        assert np.allclose(s[t], rs.reshape(s[t].shape, order="F"), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("metric", [None, SF.Haversine(6371.0)])
def test_marginals_equal_the_1d_single_pass(metric):
    # test/test_single_pass_2d.jl:55-66: with value axes covering every value, the row marginals are the
    # 1D single pass (counts exactly)
    rng = np.random.default_rng(3)
    if metric is None:
        x = rng.random((2, 60))
        dist = np.exp(np.linspace(np.log(0.01), np.log(1.5), 8))
    else:
        x = np.vstack([rng.uniform(-180, 180, 60), np.degrees(np.arcsin(rng.uniform(-1, 1, 60)))])
        dist = np.exp(np.linspace(np.log(10.0), np.log(20000.0), 8))
    u = rng.standard_normal((2, 60))
    vb = np.array([-1e300, -1.0, 0.0, 1.0, 1e300])
    s, c, _ = _oracle_rows(x, u, dist, [vb] * 6, metric)
    desc, keep = plan_description((SF.L2SF,), 2, dist, None, metric, "fp64", x.dtype, u.dtype)
    s1, c1, _ = oracle_py.run_single_pass(desc, x, u)
    for t in range(6):
        assert np.array_equal(c[t].sum(axis=1), c1[t])
        assert np.allclose(s[t].sum(axis=1), s1[t], rtol=1e-10, atol=1e-10)


def test_value_axis_validation():
    with pytest.raises(SF.DimensionMismatch):
        _sp2d_value_bins((np.linspace(0, 1, 5),) * 5)
    with pytest.raises(SF.DimensionMismatch):
        _sp2d_value_bins((np.linspace(0, 1, 5),) * 5 + (np.linspace(0, 1, 3),))
    n_val, rows = _sp2d_value_bins(np.linspace(0, 1, 5))
    assert n_val == 4 and len(rows) == 6
    n_val, rows = _sp2d_value_bins((np.linspace(0, 1, 5),) + (np.linspace(0, 2, 9),) * 5)
    assert n_val == 4 and len(_row_bins(rows[1], n_val)) == 5
    with pytest.raises(SF.ArgumentError):
        _row_bins(SF.LinearBinEdges(0.0, 2.0, 9), 4)
    x = np.zeros((2, 3))
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_functions_single_pass_2d(x, x, [0.0, 1.0], [0.0, 1.0], output_type=SF.StructureFunction)


def test_rows_per_launch():
    """Rows share one joint run on flat geometry with one shared value axis, as many as 196 KB of cells
    (12 bytes each) hold; per-row axes and the sphere keep one run per row."""
    shared = SF.LinearBinEdges(-1.0, 1.0, 51)
    n, rows = _sp2d_value_bins(shared)
    assert _rows_per_launch(rows, 50, n, SF.Euclidean(), 2) == 6          # 50 x 50: all six rows
    n, rows = _sp2d_value_bins(np.linspace(-1.0, 1.0, 101))
    assert _rows_per_launch(rows, 64, n, SF.Euclidean(), 3) == 2          # 64 x 100: 76.8 KB per row
    assert _rows_per_launch(rows, 512, n, SF.Euclidean(), 2) == 1         # one row's cells exceed the budget
    n, rows = _sp2d_value_bins((shared,) * 6)                             # a tuple of one axis object
    assert _rows_per_launch(rows, 50, n, SF.Euclidean(), 2) == 6
    n, rows = _sp2d_value_bins(tuple(SF.LinearBinEdges(-1.0, 1.0 + k, 51) for k in range(6)))
    assert _rows_per_launch(rows, 50, n, SF.Euclidean(), 2) == 1          # per-row axes
    n, rows = _sp2d_value_bins(shared)
    assert _rows_per_launch(rows, 50, n, SF.Haversine(6371.0), 2) == 1    # sphere


@pytest.mark.parametrize("D", [2, 3])
def test_oracle_row_group_equals_single_rows(D):
    """The oracle's fused pass over consecutive rows (the reference's own loop: du_L and |du|^2 once per
    pair) gives each row's single-row result bit for bit, serial and threaded."""
    rng = np.random.default_rng(60 + D)
    x = rng.random((D, 700))
    u = rng.standard_normal((D, 700))
    dist = np.exp(np.linspace(math.log(1e-3), math.log(math.sqrt(D)), 17))
    vb = SF.LinearBinEdges(-6.0, 10.0, 33)
    m = 16 * 32
    for rows in ((0, 1, 2, 3, 4, 5), (2, 3)):
        desc, keep = plan_description(tuple(SF.SinglePass2DRow(t) for t in rows), D, dist, vb, None, "fp64",
                                      x.dtype, u.dtype)
        gs, gc, ga = oracle_py.run(desc, x, u, with_abs=True)
        ts, tc = oracle_py.run(desc, x, u, threads=4)
        assert gs.size == len(rows) * m and np.array_equal(tc, gc)
        assert np.allclose(ts, gs, rtol=1e-12, atol=0)  # the threaded merge adds partial sums in another order
        for g, t in enumerate(rows):
            d1, k1 = plan_description((SF.SinglePass2DRow(t),), D, dist, vb, None, "fp64", x.dtype, u.dtype)
            s1, c1, a1 = oracle_py.run(d1, x, u, with_abs=True)
            assert np.array_equal(gc[g * m:(g + 1) * m], c1)
            assert np.array_equal(gs[g * m:(g + 1) * m], s1) and np.array_equal(ga[g * m:(g + 1) * m], a1)
        assert int(gc.sum()) > 0
    bad, keep = plan_description((SF.SinglePass2DRow(1), SF.SinglePass2DRow(3)), D, dist, vb, None, "fp64",
                                 x.dtype, u.dtype)
    with pytest.raises(RuntimeError):
        oracle_py.run(bad, x, u)
