"""Shared test helpers: oracle/GPU comparison with the stated tolerances."""
import numpy as np

# Tolerances (per bin). Counts: bit-exact. Sums: |gpu - oracle| <= tol * sum|v| (the oracle's per-bin
# sum of absolute values), which is the meaningful scale for signed and near-cancelling bins.
TOL_FP64 = 1e-12
# FP64 on the sphere, chord formulation (the default): the tangent-velocity difference U_B - U_A of
# nearby points cancels, so each FP64 increment carries ~1e-16 |U| / |dU| of relative error, as the
# reference's own frame formula does in its difference uB.tB - uA.tA; the two FP64 formulations then
# differ by ~1e-12 of the sum in bins of a few close pairs.
TOL_FP64_SPHERE = 1e-11
TOL_MIXED = 1e-6
# FP32-bulk kernels: each pair value carries FP32 rounding of its differences, ~1e-7 |du|^k absolute,
# which in bins of a few near-cancelling pairs reaches a few 1e-6 of sum|v|.
TOL_FP32 = 2e-5


def compare(gpu_sums, gpu_counts, ref_sums, ref_counts, scale, tol):
    """Assert counts are identical and sums agree within tol * scale per bin."""
    gpu_counts = np.asarray(gpu_counts).astype(np.uint64)
    ref_counts = np.asarray(ref_counts).astype(np.uint64)
    assert gpu_counts.sum() == ref_counts.sum(), (int(gpu_counts.sum()), int(ref_counts.sum()))
    bad = np.nonzero(gpu_counts != ref_counts)[0]
    assert bad.size == 0, f"counts differ at {bad[:10]}: gpu {gpu_counts[bad[:10]]} ref {ref_counts[bad[:10]]}"
    gs = np.asarray(gpu_sums, dtype=np.float64)
    rs = np.asarray(ref_sums, dtype=np.float64)
    sc = np.maximum(np.asarray(scale, dtype=np.float64), 1e-300)
    err = np.abs(gs - rs) / sc
    both_nan = np.isnan(gs) & np.isnan(rs)
    err[both_nan] = 0.0
    assert np.all(err[~both_nan] <= tol), f"max normalised sum error {np.nanmax(err):.3e} > {tol:.1e}"
    return float(np.nanmax(err)) if err.size else 0.0


def sphere_tol(precision, tol):
    """The tolerance of a spherical plan: FP64 widened to TOL_FP64_SPHERE (see above)."""
    return max(tol, TOL_FP64_SPHERE) if precision == "fp64" else tol
