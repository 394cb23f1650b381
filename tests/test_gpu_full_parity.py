"""Parity at the benchmark sizes: the c1 (3D, N = 65536, four fused operators), c2 (sphere,
N = 200000) and c3 (joint 64 x 256, N = 131072) workloads through the C ABI, in every precision,
against the FP64 oracle on the same inputs.

These sizes reach the mechanisms that small cases never do: Morton point order (from 16384 points),
the periodic fold of the FP32 run tables, the joint kernel's fixed-point flush before a cell can hold
2^20 pairs, the chord band of the sphere at 2e10 pairs, and uint64 counts above 2^32 in total. The
oracle result is cached by input hash (tests/golden/full_oracle.npz, written by full_oracle.py in the
same folder); a different hash recomputes it in spawned worker processes.

Tolerances as everywhere: counts bit-exact (joint cells included); sums per bin within TOL x the
oracle's per-bin sum of |value| (mixed 1e-6, fp64 1e-12 (1e-11 on the sphere), fp32 2e-5).
"""
import numpy as np
import pytest

from full_oracle import oracle_for
from helpers import TOL_FP32, TOL_FP64, TOL_MIXED, compare, sphere_tol
from test_gpu_parity import run_gpu
from sfb200 import synthetic

pytestmark = pytest.mark.gpu

_CACHE = {}


def _oracle(name):
    if name not in _CACHE:
        w = synthetic.config(name)
        rs, rc, ra, src = oracle_for(name, w)
        _CACHE[name] = (w, rs, rc, ra, src)
    return _CACHE[name]


@pytest.mark.parametrize("precision,tol", [("mixed", TOL_MIXED), ("fp64", TOL_FP64), ("fp32", TOL_FP32)])
@pytest.mark.parametrize("name", ["c1", "c2", "c3"])
def test_full_size_against_oracle(name, precision, tol):
    w, rs, rc, ra, src = _oracle(name)
    if name == "c2":
        tol = sphere_tol(precision, tol)
    gs, gc, st = run_gpu(w.ops, w.x, w.u, w.distance_bins.edges, metric=w.metric, value_bins=w.value_bins,
                         precision=precision)
    assert int(rc.sum()) > 0
    if w.value_bins is None:
        nb = len(w.distance_bins) - 1
        for k in range(len(w.ops)):
            compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], tol)
    else:
        compare(gs, gc, rs, rc, ra, tol)


def test_full_size_pair_totals():
    """Every pair is binned once: c1's edges cover the unit cube's diameter, so all N(N-1)/2 pairs land in
    range; c2 and c3 lose only pairs beyond their first or last edge."""
    w, rs, rc, ra, src = _oracle("c1")
    assert int(rc.sum()) == w.pairs
    for name in ("c2", "c3"):
        w, rs, rc, ra, src = _oracle(name)
        assert 0.5 * w.pairs < int(rc.sum()) <= w.pairs
        assert rc.dtype == np.uint64
