"""The six-invariant single pass, mirroring src/Calculations/serial_single_pass.jl of the reference.

    calculate_structure_functions_single_pass(x, u, distance_bins; backend, output_type, count_eltype,
                                              distance_metric)
    calculate_structure_functions_single_pass_inplace(sums, counts, x, u, distance_bins; ...)
    helmholtz_decompose_2d(distance_bins, L2_sums, L2_counts, T2_sums, T2_counts)

One pass over the pairs accumulates four rows per distance bin -- S2 = |du|^2, L2 = du_L^2,
S3 = du_L |du|^2 and L3 = du_L^3 -- in one fused kernel (operator list {S2SF, L2SF, S3SF, L3SF});
T2 = S2 - L2 and L1T2 = S3 - L3 are derived per bin afterwards, as the reference does
(`_sp1d_derive_rows!`, src/Calculations/serial_single_pass.jl:209-219): both identities hold pair by
pair, so they hold for the bin sums. The accumulator is the reference's (6, n_bins) layout, rows
S2, L2, T2, S3, L3, L1T2 (SINGLE_PASS_N = 6, src/Calculations/batch_api.jl:98).
"""
import numpy as np

from .api import (B200Backend, _finalize, _output_float_type, _run, _shape_of, assert_counts_representable,
                  default_backend, validate_array_shape)
from .errors import ArgumentError, DimensionMismatch
from .metrics import Euclidean
from .operators import (DiagonalConsistentThirdOrderStructureFunction, LongitudinalSecondOrderStructureFunction,
                        OffDiagonalInconsistentThirdOrderStructureFunction, SecondOrderStructureFunction,
                        ThirdOrderStructureFunction, TransverseSecondOrderStructureFunction)
from .results import AbstractStructureFunction, StructureFunction, StructureFunctionSumsAndCounts, bin_average

SINGLE_PASS_N = 6

# The six invariants in stacked-row order (src/Calculations/serial_single_pass.jl:593-600).
SINGLE_PASS_OPERATORS = {
    "S2": SecondOrderStructureFunction,
    "L2": LongitudinalSecondOrderStructureFunction,
    "T2": TransverseSecondOrderStructureFunction,
    "S3": ThirdOrderStructureFunction,
    "L3": DiagonalConsistentThirdOrderStructureFunction,
    "L1T2": OffDiagonalInconsistentThirdOrderStructureFunction,
}

# the rows the kernel accumulates, in the order of its fused operator list, and where they go
_ACCUMULATED = (SecondOrderStructureFunction, LongitudinalSecondOrderStructureFunction, ThirdOrderStructureFunction,
                DiagonalConsistentThirdOrderStructureFunction)
_ROWS = (0, 1, 3, 4)


class HelmholtzDecomposition2D(AbstractStructureFunction):
    """Rotational / divergent split of binned L2 and T2 (src/StructureFunctionObjects.jl:179-196)."""

    def __init__(self, distance_bins, rotational_sums, rotational_counts, divergent_sums, divergent_counts,
                 longitudinal_values, transverse_values):
        self.distance_bins = distance_bins
        self.rotational_sums = np.asarray(rotational_sums)
        self.rotational_counts = np.asarray(rotational_counts)
        self.divergent_sums = np.asarray(divergent_sums)
        self.divergent_counts = np.asarray(divergent_counts)
        self.longitudinal_values = np.asarray(longitudinal_values)
        self.transverse_values = np.asarray(transverse_values)


def derive_rows(sums, counts):
    """_sp1d_derive_rows! (src/Calculations/serial_single_pass.jl:209-219), in place: T2 = S2 - L2,
    L1T2 = S3 - L3, and the shared count row copied to every row. Idempotent."""
    sums[2] = sums[0] - sums[1]
    sums[5] = sums[3] - sums[4]
    counts[1:] = counts[0]
    return sums, counts


def helmholtz_decompose_2d(distance_bins, L2_sums, L2_counts, T2_sums=None, T2_counts=None):
    """2D isotropic Helmholtz decomposition from binned L2 / T2 (src/Calculations/serial_single_pass.jl:
    31-95): geometric bin midpoints, cumulative trapezoidal integral of (D_TT - D_LL) / r, then
    D_rot = D_TT + r I and D_div = D_LL - r I, as sums over the L2 counts. Called with (6, n_bins)
    single-pass sums and counts it uses rows L2 and T2 (src/Calculations/serial_single_pass.jl:11-23)."""
    if T2_sums is None:
        sums, counts = np.asarray(L2_sums), np.asarray(L2_counts)
        return helmholtz_decompose_2d(distance_bins, sums[1], counts[1], sums[2], counts[2])
    L2_sums, L2_counts = np.asarray(L2_sums), np.asarray(L2_counts)
    T2_sums, T2_counts = np.asarray(T2_sums), np.asarray(T2_counts)
    if len(L2_sums) != len(T2_sums):
        raise DimensionMismatch("L2_sums and T2_sums must have the same length")
    if len(L2_counts) != len(L2_sums):
        raise DimensionMismatch("L2_counts must match L2_sums length")
    if len(T2_counts) != len(T2_sums):
        raise DimensionMismatch("T2_counts must match T2_sums length")
    nb = len(L2_sums)
    edges = np.asarray(distance_bins, dtype=np.float64)
    if len(edges) != nb + 1:
        raise DimensionMismatch("distance_bins must have length n_bins + 1")
    mids = np.array([np.sqrt(edges[k] * edges[k + 1]) if edges[k] > 0 else np.nan for k in range(nb)])
    d_ll = bin_average(L2_sums, L2_counts)
    d_tt = bin_average(T2_sums, T2_counts)
    integral = np.zeros(nb, dtype=d_ll.dtype)
    for k in range(1, nb):
        f_prev = (d_tt[k - 1] - d_ll[k - 1]) / mids[k - 1]
        f_curr = (d_tt[k] - d_ll[k]) / mids[k]
        integral[k] = integral[k - 1] + 0.5 * (f_prev + f_curr) * (mids[k] - mids[k - 1])
    rot_counts = L2_counts.copy()
    div_counts = L2_counts.copy()
    rot = (d_tt + mids * integral) * rot_counts
    div = (d_ll - mids * integral) * div_counts
    return HelmholtzDecomposition2D(distance_bins, rot, rot_counts, div, div_counts, d_ll.copy(), d_tt.copy())


def _single_pass_raw(backend, x, u, distance_bins, distance_metric):
    """(6, n_bins) float64 sums and uint64 counts of one single pass (derived rows filled)."""
    sums, counts, plan, xcode, ucode = _run(backend, list(_ACCUMULATED), x, u, distance_bins, None, distance_metric)
    nb = len(distance_bins) - 1
    s6 = np.zeros((SINGLE_PASS_N, nb))
    c6 = np.zeros((SINGLE_PASS_N, nb), dtype=np.uint64)
    for k, row in enumerate(_ROWS):
        s6[row] = sums[k * nb:(k + 1) * nb]
    c6[0] = counts
    derive_rows(s6, c6)
    return s6, c6, _output_float_type(xcode, ucode)


def calculate_structure_functions_single_pass(x, u, distance_bins, *, backend=None, output_type=StructureFunction,
                                              count_eltype=np.uint32, distance_metric=None):
    """The reference's `calculate_structure_functions_single_pass`
    (src/Calculations/serial_single_pass.jl:663-693): the six invariants in one pair pass, as a dict
    keyed S2, L2, T2, S3, L3, L1T2 of single-operator results of `output_type`, plus "helmholtz" (a
    HelmholtzDecomposition2D) for point-field input."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    if not isinstance(backend, B200Backend):
        raise ArgumentError(f"backend {backend!r} is not a B200Backend")
    if isinstance(distance_bins, (int, np.integer)):
        raise ArgumentError("the single pass takes explicit bin edges")
    validate_array_shape(x, u, distance_metric)
    assert_counts_representable(count_eltype, _shape_of(x)[1])
    s6, c6, ot = _single_pass_raw(backend, x, u, distance_bins, distance_metric)
    ct = np.dtype(count_eltype)
    cc = c6[0].astype(ct)  # the six invariants share one count row
    out = {}
    for row, (name, op) in enumerate(SINGLE_PASS_OPERATORS.items()):
        raw = StructureFunctionSumsAndCounts(op, distance_bins, s6[row].astype(ot), cc.copy())
        out[name] = _finalize(raw, output_type)
    out["helmholtz"] = helmholtz_decompose_2d(distance_bins, s6[1].astype(ot), cc, s6[2].astype(ot), cc)
    return out


def calculate_structure_functions_single_pass_inplace(sums, counts, x, u, distance_bins, *, backend=None,
                                                      distance_metric=None):
    """The reference's mutating `calculate_structure_functions_single_pass!`
    (src/Calculations/serial_single_pass.jl:408-421 with _accumulate_single_pass_1d!, :165-192): adds
    the accumulated rows into the caller's (6, n_bins) `sums` / `counts`, then re-derives rows T2,
    L1T2 and the count rows from them."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    validate_array_shape(x, u, distance_metric)
    nb = len(distance_bins) - 1
    if sums.shape != (SINGLE_PASS_N, nb):
        raise DimensionMismatch(f"sums must have shape ({SINGLE_PASS_N}, n_bins); got {sums.shape}")
    if counts.shape != (SINGLE_PASS_N, nb):
        raise DimensionMismatch(f"counts must have shape ({SINGLE_PASS_N}, n_bins); got {counts.shape}")
    s6, c6, _ = _single_pass_raw(backend, x, u, distance_bins, distance_metric)
    for row in _ROWS:
        sums[row] += s6[row].astype(sums.dtype)
    counts[0] += c6[0].astype(counts.dtype)
    derive_rows(sums, counts)
    return sums, counts
