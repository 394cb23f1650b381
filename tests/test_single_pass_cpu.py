"""The six-invariant single pass on the CPU: the oracle's restatement of the reference's single-pass
loop against the reference's own single-pass tests (test/test_single_pass.jl:26-121), and the host
arithmetic of the single-pass API (derived rows, the 2D Helmholtz decomposition)."""
import numpy as np

import oracle_py
import sfb200 as SF
from sfb200.api import plan_description
from sfb200.single_pass import SINGLE_PASS_OPERATORS, derive_rows, helmholtz_decompose_2d

OPS6 = tuple(SINGLE_PASS_OPERATORS.values())


def _single_pass(x, u, bins, metric=None):
    desc, keep = plan_description((SF.L2SF,), u.shape[0], bins, None, metric, "fp64", x.dtype, u.dtype)
    return oracle_py.run_single_pass(desc, x, u)


def _separate(x, u, bins, metric=None):
    desc, keep = plan_description(OPS6, u.shape[0], bins, None, metric, "fp64", x.dtype, u.dtype)
    s, c = oracle_py.run(desc, x, u)
    return s.reshape(6, -1), c


def test_three_point_case_matches_separate_operators():
    # test/test_single_pass.jl:26-66: points (0,0), (1,0), (0,1), velocities equal to the positions
    x = np.array([[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    u = x.copy()
    bins = np.array([0.1, 1.0, 2.0])
    s, c, a = _single_pass(x, u, bins)
    rs, rc = _separate(x, u, bins)
    assert np.allclose(s, rs, atol=1e-12)
    assert (c == rc[None, :]).all()
    assert c[0].tolist() == [2, 1]  # two pairs at distance 1, one at sqrt(2)


def test_three_dimensional_float32_case():
    # test/test_single_pass.jl:90-121 (Float32 inputs, widened exactly to Float64 by the oracle)
    x = np.array([[0.0, 1.0, 0.0, 0.3], [0.0, 0.0, 1.0, 0.4], [0.0, 0.0, 0.0, 1.0]], dtype=np.float32)
    u = np.array([[0.0, 0.5, 0.0, 0.0], [0.0, 0.0, 0.5, 0.0], [0.0, 0.0, 0.0, 0.5]], dtype=np.float32)
    bins = np.array([0.1, 1.0, 2.0], dtype=np.float32)
    s, c, a = _single_pass(x, u, bins)
    rs, rc = _separate(x, u, bins)
    assert np.allclose(s, rs, rtol=1e-12, atol=1e-14)
    assert (c == rc[None, :]).all() and int(c[0].sum()) == 6


def test_seeded_flat_and_sphere_match_separate_operators():
    rng = np.random.default_rng(21)
    for D in (2, 3):
        x = rng.random((D, 400))
        u = rng.standard_normal((D, 400))
        bins = np.exp(np.linspace(np.log(1e-2), np.log(np.sqrt(D)), 13))
        s, c, a = _single_pass(x, u, bins)
        rs, rc = _separate(x, u, bins)
        assert (c == rc[None, :]).all()
        assert np.all(np.abs(s - rs) <= 1e-12 * np.maximum(a, 1e-300))
    lon = rng.uniform(-180, 180, 300)
    lat = np.degrees(np.arcsin(rng.uniform(-1, 1, 300)))
    x = np.stack([lon, lat])
    u = rng.standard_normal((2, 300))
    bins = np.exp(np.linspace(0.0, np.log(20000.0), 11))
    s, c, a = _single_pass(x, u, bins, SF.Haversine(6371.0))
    rs, rc = _separate(x, u, bins, SF.Haversine(6371.0))
    assert (c == rc[None, :]).all() and int(c[0].sum()) > 0
    assert np.all(np.abs(s - rs) <= 1e-12 * np.maximum(a, 1e-300))


def test_derive_rows_is_idempotent():
    rng = np.random.default_rng(3)
    s = rng.standard_normal((6, 5))
    c = np.zeros((6, 5), dtype=np.uint64)
    c[0] = [3, 0, 7, 1, 2]
    derive_rows(s, c)
    s1, c1 = s.copy(), c.copy()
    derive_rows(s, c)
    assert np.array_equal(s, s1) and np.array_equal(c, c1)
    assert np.allclose(s[2], s[0] - s[1]) and np.allclose(s[5], s[3] - s[4])
    assert (c == c[0]).all()


def test_helmholtz_rotational_plus_divergent_is_longitudinal_plus_transverse():
    # test/test_single_pass.jl:68-80: D_rot + D_div = D_LL + D_TT wherever a bin has pairs, and the
    # decomposition keeps the raw L2 / T2 means
    edges = np.array([0.05, 0.1, 0.2, 0.4, 0.8, 1.6])
    rng = np.random.default_rng(8)
    counts = np.array([4, 5, 9, 12, 30], dtype=np.uint64)
    l2 = rng.random(5) * counts
    t2 = rng.random(5) * counts
    h = helmholtz_decompose_2d(edges, l2, counts, t2, counts)
    ok = counts > 0
    d_ll = l2[ok] / counts[ok]
    d_tt = t2[ok] / counts[ok]
    rot = h.rotational_sums[ok] / counts[ok]
    div = h.divergent_sums[ok] / counts[ok]
    assert np.allclose(rot + div, d_ll + d_tt, atol=1e-12)
    assert np.allclose(h.longitudinal_values[ok], d_ll)
    assert np.allclose(h.transverse_values[ok], d_tt)
    # an empty bin is NaN, never 0, and the cumulative integral carries it to every larger bin
    # (src/Calculations/serial_single_pass.jl:55-57)
    c0 = counts.copy()
    c0[1] = 0
    h0 = helmholtz_decompose_2d(edges, l2, c0, t2, c0)
    assert np.isnan(h0.longitudinal_values[1]) and np.isnan(h0.rotational_sums[1:]).all()
    assert np.isfinite(h0.rotational_sums[0])
    # with (6, n_bins) single-pass arrays it takes rows L2 and T2
    s6 = np.zeros((6, 5))
    c6 = np.tile(counts, (6, 1))
    s6[1], s6[2] = l2, t2
    h6 = helmholtz_decompose_2d(edges, s6, c6)
    assert np.allclose(np.nan_to_num(h6.rotational_sums), np.nan_to_num(h.rotational_sums))
