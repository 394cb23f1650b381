"""Public entry points, mirroring src/Calculations/dispatch.jl of the reference.

    calculate_structure_function(sf, x, u, distance_bins[, value_bins][, count_eltype];
                                 backend=B200Backend(), output_type=..., distance_metric=Euclidean())
    calculate_structure_function_inplace(sums, counts, sf, x, u, distance_bins[, value_bins]; ...)

`x` is (W, N) and `u` is (D, N), with W = D for Euclidean geometry and W = 2 (lon, lat) on the
sphere, as in the reference. NumPy arrays (host) and CUDA torch tensors (device-resident) are
accepted. Validation, error types and result containers follow the reference; the O(N^2) pair loop
runs in libsfb200.so on the GPU (no CPU fallback).

Extension beyond the reference: `sf` may be a tuple/list of operators; the pair loop is then run
once and a tuple of results (one per operator) is returned.
"""
import ctypes as C
import weakref

import numpy as np

from . import _abi, _lib, autotune
from . import operators as ops_module
from .bins import AbstractBinEdges, LinearBinEdges, LogBinEdges, as_bin_edges
from .errors import ArgumentError, DimensionMismatch
from .metrics import Euclidean, pair_geometry_for
from .operators import AbstractDerivedStructureFunctionType, AbstractPairwiseStructureFunctionType
from .results import (StructureFunction, StructureFunction2DSumsAndCounts, StructureFunctionSumsAndCounts,
                      bin_average)

try:  # torch is optional: only used to accept device-resident tensors
    import torch
except Exception:  # pragma: no cover
    torch = None


# ----------------------------------------------------------------------------------- backend

_CONTEXTS = {}


def _context(device):
    ctx = _CONTEXTS.get(device)
    if ctx is None:
        ctx = _lib.Context(device)
        _CONTEXTS[device] = ctx
    return ctx


class B200Backend:
    """Execution backend that runs the pair loop on a B200 through libsfb200.so.

    precision: "mixed" (FP64 differences, squared distance and projection numerators; FP32
    normalisation, powers and accumulation; FP64 merge), "fp64" (every pair in FP64) or "fp32"
    (FP32 bulk with an FP64 recheck of bin membership). Plans are cached per (operator set, bins,
    metric, dtypes). With `autotune=True` the first call of each plan shape and size class times the
    launch candidates on its own inputs (sfb200.autotune) and keeps the fastest.
    """

    def __init__(self, device=0, precision="mixed", tile=0, autotune=False):
        if precision not in _abi.PRECISIONS:
            raise ArgumentError("precision must be 'mixed', 'fp64' or 'fp32'")
        self.device = int(device)
        self.precision = precision
        self.tile = int(tile)
        self.autotune = bool(autotune)
        self._plans = {}

    def __repr__(self):
        return f"B200Backend(device={self.device}, precision={self.precision!r})"

    @property
    def context(self):
        return _context(self.device)

    def plan(self, key, desc, keep):
        p = self._plans.get(key)
        if p is None:
            p = _lib.Plan(self.context, desc, keep)
            if self.tile:
                p.set_launch(self.tile, -1, 0)
            self._plans[key] = p
        return p


_DEFAULT_BACKEND = None


def default_backend():
    global _DEFAULT_BACKEND
    if _DEFAULT_BACKEND is None:
        _DEFAULT_BACKEND = B200Backend()
    return _DEFAULT_BACKEND


# ----------------------------------------------------------------------------------- validation

class PointField:
    """u is (D, N) (src/Calculations/shapes.jl:18)."""

    aux = ()

    def __init__(self, D):
        self.D = D


class SharedPositionField:
    """x is (W, N), u is (D, N, auxiliary...): one geometry, several fields (src/Calculations/shapes.jl:19)."""

    def __init__(self, D, aux):
        self.D = D
        self.aux = tuple(aux)


class VaryingPositionField:
    """x is (W, N, auxiliary...) and u is (D, N, auxiliary...) with the same auxiliary axes
    (src/Calculations/shapes.jl:20)."""

    def __init__(self, D, aux):
        self.D = D
        self.aux = tuple(aux)


def _shape_of(a):
    return tuple(a.shape)


def _validate_spatial_dimension(D):
    if D not in (2, 3):
        raise DimensionMismatch(f"expected spatial/velocity dimension D=2 or D=3 on axis 1; got D={D}")


def validate_array_shape(x, u, distance_metric):
    """_validate_array_shape (src/Calculations/shapes.jl:67-105)."""
    xs, us = _shape_of(x), _shape_of(u)
    if len(xs) < 2:
        raise DimensionMismatch(f"x must have shape (Dx, N) or (Dx, N, auxiliary...); got ndims(x)={len(xs)}")
    if len(us) < 2:
        raise DimensionMismatch(f"u must have shape (D, N) or (D, N, auxiliary...); got ndims(u)={len(us)}")
    D = us[0]
    _validate_spatial_dimension(D)
    W = pair_geometry_for(distance_metric, D).coordinate_width()
    if xs[0] != W:
        raise DimensionMismatch(
            f"this geometry locates a point with {W} coordinate(s) on axis 1 of x, but got size(x,1)={xs[0]} "
            f"(velocity dimension D={D} from size(u,1))")
    if us[1] != xs[1]:
        raise DimensionMismatch(
            f"x and u must share axis-2 point count N; got size(x,2)={xs[1]} and size(u,2)={us[1]}")
    if len(xs) == 2 and len(us) == 2:
        return PointField(D)
    if len(xs) == 2 and len(us) >= 3:
        return SharedPositionField(D, us[2:])
    if len(xs) >= 3 and len(us) >= 3:
        if len(xs) != len(us):
            raise DimensionMismatch(
                f"varying-position inputs must have the same rank; got ndims(x)={len(xs)} and ndims(u)={len(us)}")
        if xs[2:] != us[2:]:
            raise DimensionMismatch(f"varying-position inputs must share auxiliary axes; got {xs[2:]} and {us[2:]}")
        return VaryingPositionField(D, us[2:])
    raise DimensionMismatch(
        f"unsupported shape combination: x has shape {xs}, u has shape {us}; valid forms are (Dx,N)/(D,N), "
        "(Dx,N)/(D,N,auxiliary...), or matched (Dx,N,auxiliary...) arrays")


def assert_counts_representable(count_eltype, n_points):
    """_assert_counts_representable (src/Calculations/serial.jl:111-120)."""
    ct = np.dtype(count_eltype)
    if ct.kind not in "iu":
        raise ArgumentError(f"count_eltype must be an integer type; got {ct}")
    n_pairs = (int(n_points) * (int(n_points) - 1)) // 2
    if n_pairs > int(np.iinfo(ct).max):
        raise ArgumentError(
            f"count_eltype={ct} cannot represent the worst-case pair count {n_pairs} for N={n_points} "
            f"(typemax({ct}) = {np.iinfo(ct).max}); pass count_eltype=np.uint64 or np.int64.")


def _derived_error(sf):
    raise ArgumentError(
        f"{type(sf).__name__} is a derived structure-function quantity, not a pairwise operator. Use "
        "helmholtz_decompose_2d for 2D Helmholtz rotational/divergent quantities.")


# ----------------------------------------------------------------------------------- arrays

def _is_torch(a):
    return torch is not None and isinstance(a, torch.Tensor)


def _dtype_code(dt):
    if dt == np.float64:
        return _abi.F64
    if dt == np.float32:
        return _abi.F32
    raise ArgumentError(f"inputs must be Float32 or Float64; got {dt}")


def _prepare(a):
    """(W, N) array -> (pointer, keepalive, dtype code, on_device) with column-major memory."""
    if _is_torch(a):
        if a.dtype not in (torch.float32, torch.float64):
            raise ArgumentError(f"inputs must be Float32 or Float64; got {a.dtype}")
        t = a.t().contiguous()  # (N, W) row-major == (W, N) column-major
        code = _abi.F64 if a.dtype == torch.float64 else _abi.F32
        if t.is_cuda:
            return t.data_ptr(), t, code, True
        arr = t.numpy()
        return arr.ctypes.data, arr, code, False
    arr = np.asarray(a)
    if arr.dtype not in (np.float32, np.float64):
        if arr.dtype.kind in "iu":
            arr = arr.astype(np.float64)
        else:
            raise ArgumentError(f"inputs must be Float32 or Float64; got {arr.dtype}")
    arr = np.asfortranarray(arr)
    return arr.ctypes.data, arr, _dtype_code(arr.dtype), False


def _output_float_type(x_code, u_code):
    """promote_type(float(FTx), float(FTu)) (src/Calculations/batch.jl:179)."""
    return np.float64 if (x_code == _abi.F64 or u_code == _abi.F64) else np.float32


# ----------------------------------------------------------------------------------- core

def _ops_of(sf):
    if isinstance(sf, (list, tuple)):
        ops = list(sf)
        multi = True
    else:
        ops = [sf]
        multi = False
    for o in ops:
        if isinstance(o, AbstractDerivedStructureFunctionType):
            _derived_error(o)
        if not isinstance(o, AbstractPairwiseStructureFunctionType):
            raise ArgumentError(f"not a structure-function operator: {o!r}")
    if not 1 <= len(ops) <= _abi.MAX_OPS:
        raise ArgumentError(f"between 1 and {_abi.MAX_OPS} operators per call")
    return ops, multi


def plan_description(ops, D, distance_bins, value_bins=None, distance_metric=None, precision="mixed",
                     x_dtype=np.float64, u_dtype=np.float64):
    """The C-ABI plan description (and the arrays it points to) for a call of the public API."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    geom = pair_geometry_for(distance_metric, D)
    keep = []
    dbins = as_bin_edges(distance_bins)
    desc = _abi.PlanDesc()
    desc.geometry = geom.kind
    desc.dim = geom.dim
    desc.angle_unit = geom.angle_unit
    desc.radius = geom.radius
    desc.n_ops = len(ops)
    for k, o in enumerate(ops):
        desc.ops[k] = o.as_abi()
    desc.distance = dbins.distance_abi(geom.kind, keep)
    desc.joint = 1 if value_bins is not None else 0
    if value_bins is not None:
        desc.value = as_bin_edges(value_bins).value_abi(keep)
    desc.precision = _abi.PRECISIONS[precision]
    desc.x_dtype = _dtype_code(np.dtype(x_dtype))
    desc.u_dtype = _dtype_code(np.dtype(u_dtype))
    return desc, keep


def _run(backend, ops, x, u, distance_bins, value_bins, distance_metric):
    """Run the pair loop; returns (sums (float64), counts (uint64), plan, x_code, u_code)."""
    shape = validate_array_shape(x, u, distance_metric)
    geom = pair_geometry_for(distance_metric, shape.D)
    xp, xkeep, xcode, xdev = _prepare(x)
    up, ukeep, ucode, udev = _prepare(u)
    if xdev != udev:
        raise ArgumentError("x and u must both be host arrays or both be device tensors")
    n = _shape_of(x)[1]
    dt = {_abi.F64: np.float64, _abi.F32: np.float32}
    desc, keep = plan_description(ops, shape.D, distance_bins, value_bins, distance_metric, backend.precision,
                                  dt[xcode], dt[ucode])
    key = (tuple(ops), as_bin_edges(distance_bins), value_bins is not None and as_bin_edges(value_bins), geom,
           xcode, ucode)
    plan = backend.plan(key, desc, keep)
    sums = np.zeros(plan.n_sums, dtype=np.float64)
    counts = np.zeros(plan.n_counts, dtype=np.uint64)
    flags = _abi.RUN_DEVICE_INPUT if xdev else 0
    if backend.autotune and n >= 2:
        skey = autotune.shape_key(desc, n)
        if getattr(plan, "_tuned_key", None) != skey:
            choice = autotune.lookup(skey)
            if choice is not None:
                autotune.apply(plan, choice)
            else:
                autotune.tune(plan, desc, lambda: plan.run(xp, up, n, flags, sums.ctypes.data, counts.ctypes.data), n)
            plan._tuned_key = skey
    plan.run(xp, up, n, flags, sums.ctypes.data, counts.ctypes.data)
    return sums, counts, plan, xcode, ucode


def _aux_slices(shape, x, u):
    """The (x_b, u_b) point sets of an auxiliary-axis input, in column-major order of the auxiliary
    axes (b runs fastest along the first auxiliary axis, as Julia's linear indexing)."""
    B = int(np.prod(shape.aux))
    shared = isinstance(shape, SharedPositionField)

    def flat(a):
        if _is_torch(a):
            return a.permute(*range(a.dim() - 1, 1, -1), 0, 1).reshape(B, a.shape[0], a.shape[1]) \
                if a.dim() > 3 else a.permute(2, 0, 1)
        arr = np.asarray(a)
        return np.reshape(arr, (arr.shape[0], arr.shape[1], B), order="F").transpose(2, 0, 1)

    us = flat(u)
    xs = None if shared else flat(x)
    return [(x if shared else xs[b], us[b]) for b in range(B)]


def _run_aux(backend, ops, shape, x, u, distance_bins, value_bins, distance_metric):
    """The pair loop over every auxiliary-axis slice. Precision MIXED runs all slices as resident
    slices in batched rounds (one persistent launch per kernel variant and round; sfb200_batch_run),
    the other precisions one sfb200_run per slice. Returns per-slice (sums, counts) lists plus the
    input codes."""
    pieces = _aux_slices(shape, x, u)
    out = []
    if backend.precision == "mixed" and len(pieces) > 1:
        xp0, _, xcode, xdev = _prepare(pieces[0][0])
        up0, _, ucode, udev = _prepare(pieces[0][1])
        dt = {_abi.F64: np.float64, _abi.F32: np.float32}
        geom = pair_geometry_for(distance_metric, shape.D)
        desc, keep = plan_description(ops, shape.D, distance_bins, value_bins, distance_metric, "mixed", dt[xcode],
                                      dt[ucode])
        key = (tuple(ops), as_bin_edges(distance_bins), value_bins is not None and as_bin_edges(value_bins), geom,
               xcode, ucode)
        plan = backend.plan(key, desc, keep)
        ctx = backend.context
        chunk = 256  # resident slices per round
        for c0 in range(0, len(pieces), chunk):
            slices, keepalive = [], []
            try:
                for xb, ub in pieces[c0:c0 + chunk]:
                    xp, xk, _, _ = _prepare(xb)
                    up, uk, _, _ = _prepare(ub)
                    keepalive.append((xk, uk))
                    slices.append(_lib.Slice(plan, xp, up, _shape_of(xb)[1], _abi.RUN_DEVICE_INPUT if xdev else 0))
                _lib.batch_run(ctx, slices, [0] * len(slices), [sl.tile_pairs for sl in slices])
                _lib.batch_wait(ctx)
                for sl in slices:
                    sb = np.zeros(plan.n_sums)
                    cb = np.zeros(plan.n_counts, dtype=np.uint64)
                    sl.read(sb.ctypes.data, cb.ctypes.data)
                    out.append((sb, cb))
            finally:
                for sl in slices:
                    sl.close()
        return out, xcode, ucode
    xcode = ucode = None
    for xb, ub in pieces:
        sb, cb, plan, xcode, ucode = _run(backend, ops, xb, ub, distance_bins, value_bins, distance_metric)
        out.append((sb, cb))
    return out, xcode, ucode


def _split_args(args):
    """(value_bins?, count_eltype?) from the positional tail, as the reference's methods take them."""
    value_bins, count_eltype = None, np.uint32
    rest = list(args)
    if rest and not _is_dtype_like(rest[0]):
        value_bins = rest.pop(0)
    if rest:
        count_eltype = rest.pop(0)
    if rest:
        raise ArgumentError("too many positional arguments")
    return value_bins, count_eltype


def _is_dtype_like(v):
    if isinstance(v, (AbstractBinEdges, list, tuple, np.ndarray)):
        return False
    try:
        np.dtype(v)
        return True
    except TypeError:
        return False


def distance_range(x, u, distance_metric=None, backend=None):
    """(min, max) distance over all pairs of the points, on the device (sfb200_distance_range): the
    scan of the reference's auto-binning (_minmax_matrix_for_autobins / minmax_i,
    src/Calculations/dispatch.jl:205-298), in the inputs' float type."""
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    shape = validate_array_shape(x, u, distance_metric)
    geom = pair_geometry_for(distance_metric, shape.D)
    xp, xkeep, xcode, xdev = _prepare(x)
    up, ukeep, ucode, udev = _prepare(u)
    if xdev != udev:
        raise ArgumentError("x and u must both be host arrays or both be device tensors")
    n = _shape_of(x)[1]
    if n < 2:
        raise ArgumentError("automatic binning needs at least 2 points")
    dt = {_abi.F64: np.float64, _abi.F32: np.float32}
    # a plan over placeholder edges: the scan needs only the geometry and the input layout
    desc, keep = plan_description((ops_module.L2SF,), shape.D, [0.0, 1.0], None, distance_metric, backend.precision,
                                  dt[xcode], dt[ucode])
    plan = backend.plan(("distance_range", geom, xcode, ucode), desc, keep)
    lo, hi = plan.distance_range(xp, up, n, _abi.RUN_DEVICE_INPUT if xdev else 0)
    ft = np.float32 if xcode == _abi.F32 else np.float64  # float(eltype(x))
    return ft(lo), ft(hi)


def auto_distance_bins(min_distance, max_distance, n_bins, bin_spacing=None):
    """_auto_distance_bins (src/Calculations/dispatch.jl:190-203): `n_bins` log-spaced (default) or
    linear bins from prevfloat(min) to max, in the distances' float type."""
    bin_spacing = LogBinEdges if bin_spacing is None else bin_spacing
    ft = type(min_distance) if isinstance(min_distance, np.floating) else np.float64
    lo = np.nextafter(ft(min_distance), ft(-np.inf))
    hi = ft(max_distance)
    if bin_spacing is LinearBinEdges:
        return LinearBinEdges(float(lo), float(hi), int(n_bins) + 1)
    if bin_spacing is LogBinEdges:
        e = 10.0 ** np.linspace(np.log10(float(lo)), np.log10(float(hi)), int(n_bins) + 1)
        e[0], e[-1] = lo, hi
        return LogBinEdges(e)
    raise ArgumentError(f"bin_spacing must be LinearBinEdges or LogBinEdges; got {bin_spacing}")


def calculate_structure_function(structure_function_type, x, u, distance_bins, *args, backend=None,
                                 output_type=None, distance_metric=None, count_eltype=None, verbose=False,
                                 show_progress=False, bin_spacing=None):
    """The reference's `calculate_structure_function` (src/Calculations/dispatch.jl:64-91, 108-136); with
    an integer `distance_bins`, the auto-binning method (dispatch.jl:153-184): the pair-distance range
    is scanned on the device and `distance_bins` log-spaced (or, with bin_spacing=LinearBinEdges,
    linear) bins span it."""
    if isinstance(x, tuple) or isinstance(u, tuple):
        raise ArgumentError("tuple-of-component-vector inputs are not part of the stabilized public API; "
                            "pass arrays with shape (D, N) or (D, N, auxiliary...) instead")
    if isinstance(distance_bins, (int, np.integer)) and not isinstance(distance_bins, bool):
        lo, hi = distance_range(x, u, distance_metric, backend)
        edges = auto_distance_bins(lo, hi, int(distance_bins), bin_spacing)
        return calculate_structure_function(structure_function_type, x, u, edges, *args, backend=backend,
                                            output_type=output_type, distance_metric=distance_metric,
                                            count_eltype=count_eltype, verbose=verbose, show_progress=show_progress)
    if bin_spacing is not None:
        raise ArgumentError("bin_spacing only applies to an integer distance_bins (automatic binning)")
    ops, multi = _ops_of(structure_function_type)
    value_bins, ct = _split_args(args)
    if count_eltype is not None:
        ct = count_eltype
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    if not isinstance(backend, B200Backend):
        raise ArgumentError(f"backend {backend!r} is not a B200Backend")
    joint = value_bins is not None
    if joint and multi:
        raise ArgumentError("a joint (distance x value) histogram takes exactly one operator")
    if output_type is None:
        output_type = StructureFunction2DSumsAndCounts if joint else StructureFunction
    shape = validate_array_shape(x, u, distance_metric)
    assert_counts_representable(ct, _shape_of(x)[1])
    if shape.aux:
        return _aux_result(backend, ops, multi, shape, x, u, distance_bins, value_bins, distance_metric, ct,
                           output_type)
    sums, counts, plan, xcode, ucode = _run(backend, ops, x, u, distance_bins, value_bins, distance_metric)
    ot = _output_float_type(xcode, ucode)
    ct = np.dtype(ct)
    if joint:
        nd = len(distance_bins) - 1
        nv = len(value_bins) - 1
        s2 = sums.reshape((nd, nv), order="F").astype(ot)
        c2 = counts.reshape((nd, nv), order="F").astype(ct)
        raw = StructureFunction2DSumsAndCounts(ops[0], distance_bins, value_bins, s2, c2)
        if output_type is not StructureFunction2DSumsAndCounts:
            raise ArgumentError(f"Cannot produce a {getattr(output_type, '__name__', output_type)} from this "
                                f"calculation (got a StructureFunction2DSumsAndCounts). Check the `output_type` keyword.")
        return raw
    nb = len(distance_bins) - 1
    c1 = counts.astype(ct)
    results = []
    for k, o in enumerate(ops):
        raw = StructureFunctionSumsAndCounts(o, distance_bins, sums[k * nb:(k + 1) * nb].astype(ot), c1.copy())
        results.append(_finalize(raw, output_type))
    return tuple(results) if multi else results[0]


def _aux_result(backend, ops, multi, shape, x, u, distance_bins, value_bins, distance_metric, ct, output_type):
    """Auxiliary-axis results: sums and counts of shape (n_bins, aux...) for 1D histograms
    (src/Calculations/batch.jl:209-217) and (n_dist, n_val, aux...) for joint ones."""
    parts, xcode, ucode = _run_aux(backend, ops, shape, x, u, distance_bins, value_bins, distance_metric)
    ot = _output_float_type(xcode, ucode)
    ct = np.dtype(ct)
    aux = shape.aux
    if value_bins is not None:
        nd, nv = len(distance_bins) - 1, len(value_bins) - 1
        s = np.stack([p[0].reshape((nd, nv), order="F") for p in parts], axis=-1)
        c = np.stack([p[1].reshape((nd, nv), order="F") for p in parts], axis=-1)
        s = s.reshape((nd, nv) + aux, order="F").astype(ot)
        c = c.reshape((nd, nv) + aux, order="F").astype(ct)
        if output_type is not StructureFunction2DSumsAndCounts:
            raise ArgumentError(f"Cannot produce a {getattr(output_type, '__name__', output_type)} from this "
                                f"calculation (got a StructureFunction2DSumsAndCounts). Check the `output_type` keyword.")
        return StructureFunction2DSumsAndCounts(ops[0], distance_bins, value_bins, s, c)
    nb = len(distance_bins) - 1
    c = np.stack([p[1] for p in parts], axis=-1).reshape((nb,) + aux, order="F").astype(ct)
    results = []
    for k, o in enumerate(ops):
        s = np.stack([p[0][k * nb:(k + 1) * nb] for p in parts], axis=-1).reshape((nb,) + aux, order="F")
        results.append(_finalize(StructureFunctionSumsAndCounts(o, distance_bins, s.astype(ot), c.copy()), output_type))
    return tuple(results) if multi else results[0]


def _finalize(raw, output_type):
    """_finalize (src/Calculations/dispatch.jl:20-29)."""
    if output_type is StructureFunctionSumsAndCounts:
        return raw
    if output_type is StructureFunction:
        return StructureFunction(raw.operator, raw.distance, bin_average(raw.sums, raw.counts))
    raise ArgumentError(f"Cannot produce a {getattr(output_type, '__name__', output_type)} from this calculation "
                        f"(got a {type(raw).__name__}). Check the `output_type` keyword.")


def calculate_structure_function_inplace(sums, counts, structure_function_type, x, u, distance_bins,
                                         value_bins=None, *, backend=None, distance_metric=None, verbose=False,
                                         show_progress=False):
    """The reference's mutating `calculate_structure_function!` (src/Calculations/dispatch.jl:346-373):
    adds this call's sums and counts into the caller's arrays."""
    if isinstance(x, tuple) or isinstance(u, tuple):
        raise ArgumentError("tuple-of-component-vector inputs are not part of the stabilized public API; "
                            "pass arrays with shape (D, N) or (D, N, auxiliary...) instead")
    ops, multi = _ops_of(structure_function_type)
    if multi:
        raise ArgumentError("the mutating entry takes one operator")
    distance_metric = Euclidean() if distance_metric is None else distance_metric
    backend = default_backend() if backend is None else backend
    shape = validate_array_shape(x, u, distance_metric)
    counts_arr = np.asarray(counts)
    assert_counts_representable(counts_arr.dtype, _shape_of(x)[1])
    if shape.aux:
        # auxiliary axes (the reference's auxiliary_structure_function! / auxiliary_joint2d!,
        # src/Calculations/dispatch.jl:380-386, 455-461): per-slice histograms added in place
        raw = _aux_result(backend, ops, False, shape, x, u, distance_bins, value_bins, distance_metric,
                          np.uint64, StructureFunction2DSumsAndCounts if value_bins is not None
                          else StructureFunctionSumsAndCounts)
        if sums.shape != raw.sums.shape or counts_arr.shape != raw.counts.shape:
            raise DimensionMismatch(f"sums/counts must have shape {raw.sums.shape}; got {sums.shape} and "
                                    f"{counts_arr.shape}")
        sums += raw.sums.astype(sums.dtype)
        counts += raw.counts.astype(counts_arr.dtype)
        return None
    s, c, plan, _, _ = _run(backend, ops, x, u, distance_bins, value_bins, distance_metric)
    if value_bins is not None:
        nd, nv = len(distance_bins) - 1, len(value_bins) - 1
        s = s.reshape((nd, nv), order="F")
        c = c.reshape((nd, nv), order="F")
    if sums.shape != s.shape or counts_arr.shape != c.shape:
        raise DimensionMismatch(f"sums/counts must have shape {s.shape}; got {sums.shape} and {counts_arr.shape}")
    sums += s.astype(sums.dtype)
    counts += c.astype(counts_arr.dtype)
    return None


def last_stats(backend=None):
    """Statistics of the most recent run of each cached plan of `backend`."""
    backend = default_backend() if backend is None else backend
    return [p.stats() for p in backend._plans.values()]
