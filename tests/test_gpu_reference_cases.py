"""The reference's own known answers and its GPU parity cases, run through libsfb200.so.

- Every known-answer case of tests/golden/reference_kats.json (transcribed from the reference's tests:
  test/baseline_correctness.jl:6-22, test/test_core_correctness.jl:23-140) in all three precisions:
  counts equal to the stated ones, means equal to the stated values.
- test/test_gpu_tiled_parity.jl:26-81: linear, log (LogBinEdges on the device against the plain edge
  vector on the CPU) and general monotone bins, N = 50, counts exact against the serial result.
"""
import json
import os

import numpy as np
import pytest

from helpers import TOL_FP32, TOL_FP64, TOL_MIXED, compare
from test_gpu_parity import run_gpu, run_oracle
from test_oracle_kats import op_from
import sfb200 as SF

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KAT = json.load(open(os.path.join(GOLDEN, "reference_kats.json")))
PRECISIONS = [("fp64", TOL_FP64), ("mixed", TOL_MIXED), ("fp32", TOL_FP32)]


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("case", KAT["kats"], ids=[k["name"] for k in KAT["kats"]])
def test_reference_known_answers_on_gpu(case, precision, tol):
    x = np.asarray(case["x"], dtype=np.float64)
    u = np.asarray(case["u"], dtype=np.float64)
    ops = (op_from(case["op"]),)
    gs, gc, _ = run_gpu(ops, x, u, np.asarray(case["bins"]), precision=precision)
    assert gc.tolist() == case["counts"]
    rs, rc, ra = run_oracle(ops, x, u, np.asarray(case["bins"]))
    compare(gs, gc, rs, rc, ra, tol)
    if "mean" in case:
        mean = gs / np.maximum(gc, 1)
        want = np.asarray(case["mean"])
        assert np.all(np.abs(mean - want) <= tol * np.maximum(np.abs(want), ra / np.maximum(gc, 1))), (mean, want)
    if "sums" in case:
        assert np.allclose(gs, case["sums"], rtol=tol, atol=0.0)


def _tiled_case(seed, D, N=50, shift=0.0):
    rng = np.random.default_rng(seed)
    return rng.random((D, N)) + shift, rng.random((D, N))


@pytest.mark.parametrize("precision,tol", PRECISIONS)
def test_reference_tiled_parity_cases(precision, tol):
    # linear 2D and 3D edges as vectors (test/test_gpu_tiled_parity.jl:26-55)
    for D, top in ((2, 1.4), (3, 2.0)):
        x, u = _tiled_case(42 + D, D)
        edges = np.linspace(0.0, top, 11)
        gs, gc, _ = run_gpu((SF.L2SF,), x, u, edges, precision=precision)
        rs, rc, ra = run_oracle((SF.L2SF,), x, u, edges)
        compare(gs, gc, rs, rc, ra, tol)
    # general monotone bins (test/test_gpu_tiled_parity.jl:74-86)
    x, u = _tiled_case(44, 2)
    edges = np.array([0.0, 0.05, 0.12, 0.25, 0.4, 0.55, 0.7, 0.85, 1.0, 1.15, 1.35])
    gs, gc, _ = run_gpu((SF.L2SF,), x, u, edges, precision=precision)
    rs, rc, ra = run_oracle((SF.L2SF,), x, u, edges)
    compare(gs, gc, rs, rc, ra, tol)


@pytest.mark.parametrize("precision,tol", PRECISIONS)
@pytest.mark.parametrize("seed", [45, 46, 47])
def test_reference_log_bin_edges_case(precision, tol, seed):
    """test/test_gpu_tiled_parity.jl:59-72: LogBinEdges on the device, the plain edge vector on the CPU;
    counts must be identical. The library bins on the squared physical edges of the LogBinEdges plan
    (src/BinEdges.jl:447-453), the serial CPU route on the squares of the vector (src/BinEdges.jl:440)."""
    x, u = _tiled_case(seed, 2, shift=0.01)
    log_vec = np.exp(np.linspace(np.log(0.05), np.log(1.4), 11))
    lb = SF.LogBinEdges(log_vec)
    gs, gc, _ = run_gpu((SF.L2SF,), x, u, lb, precision=precision)
    rs, rc, ra = run_oracle((SF.L2SF,), x, u, log_vec)
    compare(gs, gc, rs, rc, ra, tol)
    # and exactly the oracle of the same LogBinEdges plan, at a size with many pairs per bin
    rng = np.random.default_rng(seed)
    x = rng.random((2, 3000)) + 0.01
    u = rng.standard_normal((2, 3000))
    gs, gc, _ = run_gpu((SF.L2SF, SF.T2SF), x, u, lb, precision=precision)
    rs, rc, ra = run_oracle((SF.L2SF, SF.T2SF), x, u, lb)
    nb = len(log_vec) - 1
    for k in range(2):
        compare(gs[k * nb:(k + 1) * nb], gc, rs[k * nb:(k + 1) * nb], rc, ra[k * nb:(k + 1) * nb], tol)
