"""Pins the CPU oracle against the reference's own known answers (tests/golden/reference_kats.json)
and its property tests (joint marginalization, spherical solid-body rotation, thin shell, flat
limit), and checks the shared transcendentals against 300-bit mpmath."""
import json
import math
import os

import mpmath as mp
import numpy as np
import pytest

import oracle_py
import sfb200 as SF
from sfb200 import _abi
from sfb200.api import plan_description

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT = json.load(open(os.path.join(GOLDEN, "reference_kats.json")))

OPS = {
    "L2": SF.L2SF, "T2": SF.T2SF, "L3": SF.L3SF, "T3": SF.T3SF, "L1T2": SF.L1T2SF, "L2T1": SF.L2T1SF,
    "S2": SF.S2SF, "S3": SF.S3SF, "T2C": SF.T2ComponentSF, "L1T2C": SF.L1T2ComponentSF,
    "FULLVEC3": SF.FullVectorStructureFunctionType(3),
}


def op_from(spec):
    if spec[0] == "PROJECTED":
        return SF.ProjectedStructureFunctionType(spec[1], spec[2])
    return OPS[spec[0]]


def run(ops, x, u, bins, metric=None, value_bins=None):
    x = np.asarray(x, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    desc, keep = plan_description(tuple(ops), u.shape[0], bins, value_bins, metric, "fp64", x.dtype, u.dtype)
    return oracle_py.run(desc, x, u)


@pytest.mark.parametrize("case", KAT["kats"], ids=[k["name"] for k in KAT["kats"]])
def test_reference_known_answers(case):
    s, c = run([op_from(case["op"])], case["x"], case["u"], case["bins"])
    assert c.tolist() == case["counts"]
    if "mean" in case:
        assert np.allclose(s / c, case["mean"], rtol=1e-15, atol=1e-15)
    if "sums" in case:
        assert np.allclose(s, case["sums"], rtol=1e-15)


@pytest.mark.parametrize("case", KAT["functor"], ids=lambda c: c["cite"])
def test_operator_values(case):
    for name, val in case["values"].items():
        got = oracle_py.sf_functor(OPS[name].as_abi(), case["du"], case["rhat"])
        assert math.isclose(got, val, rel_tol=1e-14), (name, got, val)


def test_operator_identities_and_orientation():
    # src/StructureFunctionTypes.jl: S2 = L2 + T2, S3 = L3 + L1T2 (test/test_core_correctness.jl:145-155)
    du, rh = [2.0, 3.0, 4.0], [1.0, 0.0, 0.0]
    f = lambda n: oracle_py.sf_functor(OPS[n].as_abi(), du, rh)  # noqa: E731
    assert math.isclose(f("S2"), f("L2") + f("T2"))
    assert math.isclose(f("S3"), f("L3") + f("L1T2"))
    assert f("S3") != f("FULLVEC3")
    # 2D orientation: rotations keep L2T1/T3, reflections flip them (test/test_core_correctness.jl:157-177)
    du, rh = np.array([2.0, 3.0]), np.array([1.0, 0.0])
    th = 0.7
    R = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]])
    F = np.array([[1.0, 0.0], [0.0, -1.0]])
    for n in ("L2T1", "T3"):
        base = oracle_py.sf_functor(OPS[n].as_abi(), du, rh)
        assert math.isclose(oracle_py.sf_functor(OPS[n].as_abi(), R @ du, R @ rh), base, rel_tol=1e-12)
        assert math.isclose(oracle_py.sf_functor(OPS[n].as_abi(), F @ du, F @ rh), -base, rel_tol=1e-12)
    assert math.isclose(oracle_py.sf_functor(OPS["T2"].as_abi(), F @ du, F @ rh),
                        oracle_py.sf_functor(OPS["T2"].as_abi(), du, rh))


@pytest.mark.parametrize("case", KAT["digitize"], ids=lambda c: c["cite"])
def test_digitize(case):
    for k, q in enumerate(case["queries"]):
        ssf = oracle_py.searchsortedfirst(case["edges"], q)
        if "bins" in case:
            assert ssf - 1 == case["bins"][k]
        else:
            assert ssf == case["ssf"][k]


def test_linear_bin_edges_search_matches_vector_search():
    # test/test_bin_edges.jl:32-47: LinearBinEdges FMA search == generic search on the same edges
    lb = SF.LinearBinEdges(1.0, 10.0, 10)
    abi = lb.value_abi([])
    for q in np.linspace(0.0, 11.0, 100):
        assert oracle_py.digitize(abi, q) == oracle_py.searchsortedfirst(lb.edges, q) - 1
    # the log grid queried at every edge and edge +- 1 ulp (test/test_bin_edges.jl:49-78)
    n = 15
    le = SF.LinearBinEdges(math.log(1.0), math.log(100.0), n)
    abi = le.value_abi([])
    queries = list(np.random.default_rng(1).random(200) * 120.0) + [0.5, 1.0, 100.0, 150.0]
    for e in le.edges:
        v = math.exp(e)
        queries += [v, np.nextafter(v, 0.0), np.nextafter(v, 200.0)]
    for q in queries:
        ref = oracle_py.searchsortedfirst(le.edges, math.log(q)) if q > 0 else 1
        got = oracle_py.digitize(abi, math.log(q)) + 1 if q > 0 else 1
        assert got == ref or abs(math.log(q) - le.edges[min(ref - 1, n - 1)]) < 1e-15


@pytest.mark.parametrize("case", KAT["nhat"], ids=lambda c: c["cite"])
def test_nhat(case):
    # mdu_t(du, r) = du . n_hat(r): probe n_hat with unit du along each axis
    D = len(case["rhat"])
    T1 = SF.ProjectedStructureFunctionType(0, 1).as_abi()
    for k in range(D):
        du = [0.0] * D
        du[k] = 1.0
        assert math.isclose(oracle_py.sf_functor(T1, du, case["rhat"]), case["nhat"][k], abs_tol=1e-15)


def test_count_guard():
    for dt, n in KAT["count_guard"]["ok"]:
        SF.assert_counts_representable(np.dtype(dt), n)
    for dt, n in KAT["count_guard"]["fail"]:
        with pytest.raises(SF.ArgumentError):
            SF.assert_counts_representable(np.dtype(dt), n)


def test_joint_marginal_equals_1d():
    # test/test_2d_binning.jl:32-108 (mass conservation with wide value bins)
    rng = np.random.default_rng(1234)
    x = np.vstack([rng.random(50) * 50000.0, rng.random(50) * 50000.0])
    u = np.vstack([rng.standard_normal(50) * 0.5, rng.standard_normal(50) * 0.5])
    db = [0.0, 10000.0, 20000.0, 30000.0, 50000.0]
    for op, vb in ((SF.L2SF, SF.LinearBinEdges(0.0, 1000.0, 11)), (SF.L3SF, SF.LinearBinEdges(-1000.0, 1000.0, 11))):
        s1, c1 = run([op], x, u, db)
        s2, c2 = run([op], x, u, db, value_bins=vb)
        s2 = s2.reshape((4, 10), order="F")
        c2 = c2.reshape((4, 10), order="F")
        assert np.array_equal(c2.sum(axis=1), c1)
        assert np.allclose(s2.sum(axis=1), s1, rtol=1e-12)


EARTH_R = 6.371e6


def haversine(lo1, la1, lo2, la2, R):
    p1, p2 = math.radians(la1), math.radians(la2)
    dp, dl = p2 - p1, math.radians(lo2 - lo1)
    h = math.sin(dp / 2) ** 2 + math.cos(p1) * math.cos(p2) * math.sin(dl / 2) ** 2
    return 2 * R * math.asin(math.sqrt(h))


def test_spherical_separation_matches_haversine():
    # test/test_spherical_geometry.jl:44-62
    for lo1, la1, lo2, la2 in ((10.0, 45.0, 13.0, 47.0), (-170.0, -33.0, 175.0, 12.0), (0.0, 0.0, 0.0, 90.0),
                               (100.0, 60.0, 100.0, 60.5)):
        A = oracle_py.sphere_point(lo1, la1, 0)
        B = oracle_py.sphere_point(lo2, la2, 0)
        ok, r, tA, tB = oracle_py.sphere_frame(A, B, EARTH_R)
        assert ok
        assert math.isclose(r, haversine(lo1, la1, lo2, la2, EARTH_R), rel_tol=1e-12)
        Ar = oracle_py.sphere_point(math.radians(lo1), math.radians(la1), 1)
        Br = oracle_py.sphere_point(math.radians(lo2), math.radians(la2), 1)
        ok2, r2, tA2, tB2 = oracle_py.sphere_frame(Ar, Br, 1.0)
        assert ok2 and math.isclose(r, EARTH_R * r2, rel_tol=1e-12)
        assert np.allclose(tA, tA2, atol=1e-12) and np.allclose(tB, tB2, atol=1e-12)


def test_solid_body_rotation_has_no_longitudinal_increment():
    # test/test_spherical_geometry.jl:67-90
    rng = np.random.default_rng(20260817)
    N, Om = 250, 7.292e-5
    lon = 360 * rng.random(N) - 180
    lat = 120 * rng.random(N) - 60
    x = np.vstack([lon, lat])
    u = np.vstack([Om * EARTH_R * np.cos(np.radians(lat)), np.zeros(N)])
    bins = np.linspace(0.0, 8.0e6, 21)
    s, c = run([SF.L2SF, SF.S2SF], x, u, bins, metric=SF.Haversine(EARTH_R))
    L2, S2 = s[:20], s[20:]
    occ = c > 0
    assert occ.any()
    assert L2[occ].sum() / S2[occ].sum() < 1e-24


def test_thin_shell_radial_component_never_transported():
    # test/test_spherical_geometry.jl:92-114
    rng = np.random.default_rng(7)
    N, Om = 200, 7.292e-5
    lon = 300 * rng.random(N) - 150
    lat = 100 * rng.random(N) - 50
    x = np.vstack([lon, lat])
    ue = Om * EARTH_R * np.cos(np.radians(lat))
    u2 = np.vstack([ue, np.zeros(N)])
    u3 = np.vstack([ue, np.zeros(N), 3.0 * np.sin(np.radians(2 * lat))])
    bins = np.linspace(0.0, 8.0e6, 21)
    m = SF.Haversine(EARTH_R)
    s2, c2 = run([SF.L2SF], x, u2, bins, metric=m)
    s3, c3 = run([SF.L2SF, SF.S2SF, SF.T2SF], x, u3, bins, metric=m)
    assert np.array_equal(s3[:20], s2) and np.array_equal(c3, c2)
    s2b, _ = run([SF.S2SF], x, u2, bins, metric=m)
    assert s3[20:40].sum() > s2b.sum()
    assert np.allclose(s3[20:40], s3[:20] + s3[40:60], rtol=1e-12, atol=1e-9)


def test_flat_limit_converges_like_r_over_R():
    # test/test_spherical_geometry.jl:150-179. The reference bins into 8 bins; with another random
    # stream the max-over-bins statistic is dominated by the few pairs that cross a bin edge between
    # the two geometries (shot noise, ratio ~2 on average). One bin holding every pair isolates the
    # claim under test: the transported frame departs from the flat tangent-plane frame like r/R.
    N, lat0 = 90, 35.0

    def deviation(hw):
        rng = np.random.default_rng(4242)
        dlon = hw * (2 * rng.random(N) - 1)
        dlat = hw * (2 * rng.random(N) - 1)
        uu = np.vstack([rng.standard_normal(N), rng.standard_normal(N)])
        xs = np.vstack([dlon, lat0 + dlat])
        xf = np.vstack([EARTH_R * np.radians(dlon) * math.cos(math.radians(lat0)), EARTH_R * np.radians(dlat)])
        rmax = 2.2 * EARTH_R * math.radians(hw)
        bins = np.array([0.0, 2.0 * rmax])
        a, ca = run([SF.L2SF], xs, uu, bins, metric=SF.Haversine(EARTH_R))
        b, cb = run([SF.L2SF], xf, uu, bins)
        occ = (ca > 0) & (cb > 0)
        return np.max(np.abs(a[occ] - b[occ])) / np.max(np.abs(b[occ]))

    d_big, d_small = deviation(4.0), deviation(1.0)
    assert d_small < d_big
    assert d_big / d_small > 2.5


# ----------------------------------------------------------------------- transcendentals vs mpmath

mp.mp.prec = 200


def ulp_err(got, exact):
    exact_f = float(exact)
    if exact_f == 0.0:
        return 0.0 if got == 0.0 else float("inf")
    u = math.ulp(exact_f)
    return abs(mp.mpf(got) - exact) / u


def test_sincosd_accuracy():
    rng = np.random.default_rng(0)
    xs = list(rng.uniform(-720, 720, 3000)) + [0.0, 30.0, 45.0, 60.0, 90.0, 180.0, -90.0, 270.0, 359.999999,
                                               1e-300, 12345.678]
    worst = 0.0
    for x in xs:
        s, c = oracle_py.sincosd(x)
        rad = mp.radians(mp.mpf(x))
        worst = max(worst, ulp_err(s, mp.sin(rad)) if abs(s) > 1e-300 else 0.0,
                    ulp_err(c, mp.cos(rad)) if abs(c) > 1e-300 else 0.0)
    assert worst <= 1.5, worst
    assert oracle_py.sincosd(90.0) == (1.0, 0.0) and oracle_py.sincosd(180.0)[1] == -1.0


def test_sincos_radians_accuracy():
    rng = np.random.default_rng(1)
    worst = 0.0
    for x in list(rng.uniform(-10, 10, 3000)) + [0.0, math.pi / 4, math.pi / 2, math.pi]:
        s, c = oracle_py.sincos(x)
        X = mp.mpf(x)
        if abs(s) > 1e-12:
            worst = max(worst, ulp_err(s, mp.sin(X)))
        if abs(c) > 1e-12:
            worst = max(worst, ulp_err(c, mp.cos(X)))
    assert worst <= 1.5, worst


def test_atan2_accuracy():
    rng = np.random.default_rng(2)
    worst = 0.0
    pts = [(abs(a), abs(b)) for a, b in rng.standard_normal((4000, 2))]
    pts += [(1.0, 1.0), (1e-300, 1.0), (1.0, 1e-300), (0.0, 1.0), (2.0, 1e-8), (1e-8, 2.0), (0.0625, 1.0)]
    for y, x in pts:
        got = oracle_py.atan2(y, x)
        worst = max(worst, ulp_err(got, mp.atan2(mp.mpf(y), mp.mpf(x))))
    assert worst <= 1.5, worst
    assert oracle_py.atan2(0.0, 0.0) == 0.0
    for y, x in ((-1.0, 1.0), (1.0, -1.0), (-1.0, -1.0)):
        assert ulp_err(oracle_py.atan2(y, x), mp.atan2(y, x)) <= 1.5


# ----------------------------------------------------------------------- frozen oracle outputs

def test_oracle_matches_frozen_golden():
    g = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    import make_golden

    now = make_golden.oracle_small()
    for k in g.files:
        if k.endswith("_counts"):
            assert np.array_equal(g[k], now[k]), k
        elif k.endswith("_sums"):
            assert np.array_equal(g[k], now[k]), k
