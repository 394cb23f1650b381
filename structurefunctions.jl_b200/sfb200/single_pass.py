"""The six-invariant single pass, mirroring src/Calculations/serial_single_pass.jl of the reference.

    calculate_structure_functions_single_pass(x, u, distance_bins; backend, output_type, count_eltype,
                                              distance_metric)
    calculate_structure_functions_single_pass_inplace(sums, counts, x, u, distance_bins; ...)
    helmholtz_decompose_2d(distance_bins, L2_sums, L2_counts, T2_sums, T2_counts)
    calculate_structure_functions_single_pass_2d(x, u, distance_bins, value_bins; ...)
    calculate_structure_functions_single_pass_2d_inplace(sums_3d, counts_3d, x, u, distance_bins,
                                                         value_bins; ...)

One pass over the pairs accumulates four rows per distance bin -- S2 = |du|^2, L2 = du_L^2,
S3 = du_L |du|^2 and L3 = du_L^3 -- in one fused kernel (operator list {S2SF, L2SF, S3SF, L3SF});
T2 = S2 - L2 and L1T2 = S3 - L3 are derived per bin afterwards, as the reference does
(`_sp1d_derive_rows!`, src/Calculations/serial_single_pass.jl:209-219): both identities hold pair by
pair, so they hold for the bin sums. The accumulator is the reference's (6, n_bins) layout, rows
S2, L2, T2, S3, L3, L1T2 (SINGLE_PASS_N = 6, src/Calculations/batch_api.jl:98).
"""
import numpy as np

from dataclasses import dataclass

from . import _abi
from .api import (B200Backend, PointField, _aux_slices, _finalize, _output_float_type, _run, _shape_of,
                  assert_counts_representable, default_backend, validate_array_shape)
from .bins import BinEdges, LinearBinEdges, as_bin_edges
from .errors import ArgumentError, DimensionMismatch
from .metrics import Euclidean, pair_geometry_for
from .operators import (AbstractPairwiseStructureFunctionType, DiagonalConsistentThirdOrderStructureFunction,
                        LongitudinalSecondOrderStructureFunction, OffDiagonalInconsistentThirdOrderStructureFunction,
                        SecondOrderStructureFunction, ThirdOrderStructureFunction,
                        TransverseSecondOrderStructureFunction)
from .results import (AbstractStructureFunction, StructureFunction, StructureFunction2DSumsAndCounts,
                      StructureFunctionSumsAndCounts, bin_average)

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


# ------------------------------------------------------------------- two-dimensional single pass
#
# calculate_structure_functions_single_pass_2d (src/Calculations/serial_single_pass.jl:1161-1181) bins
# each of the six invariants of a pair on its own value axis: row t of the (6, n_dist, n_val)
# accumulator is the joint (distance x value) histogram of invariant t, with that invariant's counts
# (_sp2d_scatter!, src/Calculations/serial_single_pass.jl:852-864). Every row runs as one joint histogram on the GPU
# whose value is the invariant in the pass's own formulas (operator kind SFB200_OP_SP2D): flat
# du_L = (du . dx) * inv(sqrt(r2)) (:889-893), other metrics du_L = du . r_hat (:839), |du|^2 = du . du,
# and the rows (|du|^2, du_L^2, |du|^2 - du_L^2, du_L |du|^2, du_L^3, du_L (|du|^2 - du_L^2)) (:843, :905).
# Value bins are digitized as the reference's scatter does (SFH.digitize, :856): a plain vector by
# searchsortedfirst(edges, v) - 1 (src/HelperFunctions.jl:77-84), a LinearBinEdges by its FMA search
# (src/BinEdges.jl:114-131), a LogBinEdges by its exact edge comparisons (a sorted-table search).


@dataclass(frozen=True)
class SinglePass2DRow(AbstractPairwiseStructureFunctionType):
    """Row `t` (0-based: S2, L2, T2, S3, L3, L1T2) of the two-dimensional single pass as the value of a
    joint histogram (C-ABI operator kind SFB200_OP_SP2D)."""

    t: int

    def __post_init__(self):
        if not 0 <= int(self.t) < SINGLE_PASS_N:
            raise ValueError("single-pass row must be in 0..5")

    def as_abi(self):
        return _abi.Operator(_abi.OP_SP2D, int(self.t), 0, 0)

    def order(self):
        return 2 if self.t < 3 else 3


def _sp2d_value_bins(value_bins):
    """Per-row edge vectors and n_val of a SinglePass2DValueBins (a vector shared by the six rows or a
    6-tuple, src/Calculations/batch_api.jl:101-146): n_val = length(first) - 1 and every row needs at
    least n_val + 1 edges (_validate_value_bins!)."""

    if isinstance(value_bins, tuple):
        if len(value_bins) != SINGLE_PASS_N:
            raise DimensionMismatch(
                f"single-pass 2D value_bins tuple must have {SINGLE_PASS_N} entries; got {len(value_bins)}")
        rows = [as_bin_edges(v) for v in value_bins]
    else:
        rows = [as_bin_edges(value_bins)] * SINGLE_PASS_N
    n_val = len(rows[0]) - 1
    _check_rows(rows, n_val)
    return n_val, rows


def _check_rows(rows, n_val):
    if n_val < 1:
        raise DimensionMismatch("value_bins needs at least 2 edges")
    for t, e in enumerate(rows):
        if len(e) < n_val + 1:
            raise DimensionMismatch(f"value_bins[{t + 1}] needs at least {n_val + 1} edges for n_val={n_val} "
                                    f"(got {len(e)})")


def _row_bins(vb, n_val):
    """A row's value axis cut to its first n_val + 1 edges: value bins above n_val are dropped, as the
    reference's scatter does (src/Calculations/serial_single_pass.jl:857)."""
    if len(vb) == n_val + 1:
        return vb
    if isinstance(vb, LinearBinEdges):
        raise ArgumentError("a LinearBinEdges value axis must have exactly n_val + 1 edges on this backend")
    return BinEdges(np.asarray(vb.edges)[:n_val + 1])


# Shared-memory budget of the cells of one launch of several rows (FP64 sum and 32-bit count per cell;
# 227 KB per block on B200, less the J tile).
_ROW_CELL_BYTES = 196 * 1024


def _rows_per_launch(rows, nd, n_val, distance_metric, D):
    """How many consecutive rows one joint run takes: on flat geometry with one value axis shared by the
    six rows, as many as the shared-memory cell budget holds (the pair arithmetic is then done once for
    them); otherwise one."""
    shared = all(r is rows[0] for r in rows) and len(rows[0]) == n_val + 1
    if not shared or pair_geometry_for(distance_metric, D).kind != _abi.GEOM_FLAT:
        return 1
    return int(max(1, min(SINGLE_PASS_N, _ROW_CELL_BYTES // max(1, nd * n_val * 12))))


def _single_pass_2d_slice(backend, x, u, distance_bins, rows, n_val, distance_metric):
    """(6, n_dist, n_val) float64 sums and uint64 counts of one point set, on each row's first n_val + 1
    edges (value bins above n_val are dropped, as the reference's scatter does,
    src/Calculations/serial_single_pass.jl:858): one joint run per group of consecutive rows (several
    rows per run on flat geometry with a shared value axis, see _rows_per_launch; one otherwise)."""
    nd = len(distance_bins) - 1
    s = np.zeros((SINGLE_PASS_N, nd, n_val))
    c = np.zeros((SINGLE_PASS_N, nd, n_val), dtype=np.uint64)
    ot = None
    k = _rows_per_launch(rows, nd, n_val, distance_metric, _shape_of(u)[0])
    for t0 in range(0, SINGLE_PASS_N, k):
        group = range(t0, min(SINGLE_PASS_N, t0 + k))
        vb = _row_bins(rows[t0], n_val)
        sums, counts, _, xcode, ucode = _run(backend, [SinglePass2DRow(t) for t in group], x, u, distance_bins, vb,
                                             distance_metric)
        m = nd * n_val
        for g, t in enumerate(group):
            s[t] = sums[g * m:(g + 1) * m].reshape((nd, n_val), order="F")
            c[t] = counts[g * m:(g + 1) * m].reshape((nd, n_val), order="F")
        ot = _output_float_type(xcode, ucode)
    return s, c, ot


def _single_pass_2d_raw(backend, x, u, distance_bins, value_bins, distance_metric):
    """(6, n_dist, n_val[, aux...]) sums and counts for point-field or auxiliary-axis input."""
    n_val, rows = _sp2d_value_bins(value_bins)
    shape = validate_array_shape(x, u, distance_metric)
    if isinstance(shape, PointField):
        return _single_pass_2d_slice(backend, x, u, distance_bins, rows, n_val, distance_metric)
    nd = len(distance_bins) - 1
    aux = tuple(shape.aux)
    s = np.zeros((SINGLE_PASS_N, nd, n_val) + aux, order="F")
    c = np.zeros((SINGLE_PASS_N, nd, n_val) + aux, dtype=np.uint64, order="F")
    ot = None
    for k, (xb, ub) in zip(np.ndindex(*aux[::-1]), _aux_slices(shape, x, u)):
        idx = (slice(None),) * 3 + tuple(reversed(k))
        sb, cb, ot = _single_pass_2d_slice(backend, xb, ub, distance_bins, rows, n_val, distance_metric)
        s[idx] = sb
        c[idx] = cb
    return s, c, ot


def calculate_structure_functions_single_pass_2d(x, u, distance_bins, value_bins, *, backend=None,
                                                 output_type=StructureFunction2DSumsAndCounts,
                                                 count_eltype=np.uint32, distance_metric=None):
    """The reference's `calculate_structure_functions_single_pass_2d`
    (src/Calculations/serial_single_pass.jl:1161-1181): the six invariants binned on distance x value
    in one call, as a dict keyed S2, L2, T2, S3, L3, L1T2 of StructureFunction2DSumsAndCounts (the
    joint histogram has no averaged form; _single_pass_collection_2d, :1139-1148). `value_bins` is a
    vector shared by the six invariants or a 6-tuple of vectors."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    if not isinstance(backend, B200Backend):
        raise ArgumentError(f"backend {backend!r} is not a B200Backend")
    if output_type is not StructureFunction2DSumsAndCounts:
        raise ArgumentError(f"Cannot produce a {getattr(output_type, '__name__', output_type)} from this "
                            "calculation (got a StructureFunction2DSumsAndCounts). Check the `output_type` keyword.")
    validate_array_shape(x, u, distance_metric)
    assert_counts_representable(count_eltype, _shape_of(x)[1])
    s, c, ot = _single_pass_2d_raw(backend, x, u, distance_bins, value_bins, distance_metric)
    ct = np.dtype(count_eltype)
    out = {}
    for t, (name, op) in enumerate(SINGLE_PASS_OPERATORS.items()):
        vb = value_bins[t] if isinstance(value_bins, tuple) else value_bins
        out[name] = StructureFunction2DSumsAndCounts(op, distance_bins, vb, s[t].astype(ot), c[t].astype(ct))
    return out


def calculate_structure_functions_single_pass_2d_inplace(sums_3d, counts_3d, x, u, distance_bins, value_bins, *,
                                                         backend=None, distance_metric=None):
    """The reference's mutating `calculate_structure_functions_single_pass_2d!`
    (src/Calculations/serial_single_pass.jl:712-728 with _accumulate_single_pass_2d!, :731-754 and
    _sp2d_unpack!, :803-812): adds every row into the caller's (6, n_dist, n_val) `sums_3d` /
    `counts_3d`."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    validate_array_shape(x, u, distance_metric)
    nd = len(distance_bins) - 1
    if sums_3d.ndim != 3 or sums_3d.shape[0] != SINGLE_PASS_N or sums_3d.shape[1] != nd:
        raise DimensionMismatch(f"sums must have shape ({SINGLE_PASS_N}, n_bins, n_val); got {sums_3d.shape}")
    if counts_3d.shape != sums_3d.shape:
        raise DimensionMismatch("counts and sums must have the same shape")
    n_val = sums_3d.shape[2]
    _, rows = _sp2d_value_bins(value_bins)
    _check_rows(rows, n_val)
    s, c, _ = _single_pass_2d_slice(backend, x, u, distance_bins, rows, n_val, distance_metric)
    sums_3d += s.astype(sums_3d.dtype)
    counts_3d += c.astype(counts_3d.dtype)
    return sums_3d, counts_3d
