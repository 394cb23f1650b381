"""
    StructureFunctionsB200

Julia glue for the B200 pair-histogram library (`libsfb200.so`, C ABI in `include/sfb200.h`).

Adds a `B200Backend` execution backend to jbphyswx/StructureFunctions.jl and the
`_dispatch_execution_backend[!]` methods that route `calculate_structure_function[!]` to it, beside
the package's own `GPUBackend` methods (src/Calculations/dispatch.jl:399-404, 537-544, 576-583).
Validation (`_validate_array_shape`, `_assert_counts_representable`) has already run in the public
entry (dispatch.jl:64-91, 108-136, 346-373) when these methods are reached; bin tables are built
here with the package's own functions (`squared_digitize_plan`, `BinEdges`), so the library bins
with exactly the reference's tables. There is no CPU fallback: unsupported shapes, metrics,
operators and bin types throw `ArgumentError`.

Load with `include("StructureFunctionsB200.jl")` after `using StructureFunctions`; set
`ENV["SFB200_LIB"]` to the path of `libsfb200.so` if it is not next to this package.
"""
module StructureFunctionsB200

using StructureFunctions: StructureFunctions as SF
using StructureFunctions: Calculations as SFC, StructureFunctionTypes as SFT,
    StructureFunctionObjects as SFO, HelperFunctions as SFH
using ComputationalBackends: ComputationalBackends as CB
using Distances: Distances as DI

export B200Backend, B200Server, submit!, start!, stop!, fetch_result

const LIB = Ref{String}("")
libpath() = isempty(LIB[]) ? get(ENV, "SFB200_LIB", joinpath(@__DIR__, "..", "libsfb200.so")) : LIB[]

"""
    B200Backend(; device = 0, precision = :mixed)

Run the O(N^2) pair loop on a B200. `precision`:
- `:mixed` (default): FP64 point differences, squared distance (the bin, exactly the reference's)
  and projection numerators; FP32 normalisation, operator powers and per-lane accumulation; FP64
  merge. Sums within 1e-6 of each bin's sum of |value|.
- `:fp64`: every pair in FP64 (the plain form).
- `:fp32`: FP32 pair arithmetic from (hi, lo) records with an FP64 recheck of the pairs near a bin
  edge; counts exact, sums within 2e-5 of each bin's sum of |value|.
Plans (bin tables, operator mapping, device workspace) are cached per call shape, so repeated
calls with the same operators, bins, metric and element types reuse them. Not an
`AbstractGPUBackend`, so no KernelAbstractions route captures it; `AutoBackend` never selects it.
"""
struct B200Backend <: CB.AbstractExecutionBackend
    device::Int
    precision::Symbol
end
B200Backend(; device::Integer = 0, precision::Symbol = :mixed) =
    precision in (:mixed, :fp64, :fp32) ? B200Backend(Int(device), precision) :
    throw(ArgumentError("precision must be :mixed, :fp64 or :fp32"))

c_precision(p::Symbol) = p === :fp64 ? Int32(0) : p === :mixed ? Int32(1) : Int32(2)

# ---------------------------------------------------------------------- C structs (sfb200.h)

struct COperator
    kind::Int32
    nl::Int32
    nt::Int32
    nf::Int32
end

struct CBins
    kind::Int32
    n_edges::Int32
    edges::Ptr{Float64}
    first::Float64
    last::Float64
    inv_step::Float64
    step::Float64
end

struct CPlanDesc
    geometry::Int32
    dim::Int32
    angle_unit::Int32
    radius::Float64
    n_ops::Int32
    ops::NTuple{8, COperator}
    distance::CBins
    joint::Int32
    value::CBins
    precision::Int32
    x_dtype::Int32
    u_dtype::Int32
end

const OK = 0
const ERR_INVALID_ARG = -1
const ERR_UNSUPPORTED = -2
const ERR_DIMENSION = -7
const RUN_ACCUMULATE = UInt32(0x4)

# ---------------------------------------------------------------------- mapping

c_op(::SFT.ProjectedStructureFunctionType{NL, NT}) where {NL, NT} = COperator(0, NL, NT, 0)
c_op(::SFT.SecondOrderStructureFunctionType) = COperator(1, 0, 0, 0)
c_op(::SFT.ThirdOrderStructureFunctionType) = COperator(2, 0, 0, 0)
c_op(::SFT.FullVectorStructureFunctionType{NF}) where {NF} = COperator(3, 0, 0, NF)
c_op(::SFT.TransverseComponentSecondOrderStructureFunctionType) = COperator(4, 0, 0, 0)
c_op(::SFT.LongitudinalTransverseComponentThirdOrderStructureFunctionType) = COperator(5, 0, 0, 0)
c_op(sf) = throw(ArgumentError("B200Backend does not support operator $(typeof(sf))"))

const NO_OP = COperator(0, 0, 0, 0)
const NO_BINS = CBins(0, 0, C_NULL, 0.0, 0.0, 0.0, 0.0)

c_dtype(::Type{Float64}) = Int32(0)
c_dtype(::Type{Float32}) = Int32(1)
c_dtype(T) = throw(ArgumentError("B200Backend takes Float32 or Float64 inputs; got $T"))

geometry_of(::DI.Euclidean, D) = (Int32(0), Int32(0), 1.0)
geometry_of(m::DI.Haversine, D) = (Int32(1), Int32(0), Float64(m.radius))
geometry_of(::DI.SphericalAngle, D) = (Int32(1), Int32(1), 1.0)
geometry_of(m, D) = SFH.pair_geometry_for(m, Val(D))  # throws the reference's ArgumentError

linear_bins(be::SF.LinearBinEdges) =
    CBins(2, length(be), C_NULL, Float64(be.first_edge), Float64(be.last_edge), Float64(be.inv_step),
          Float64(be.step_val))

# Distance axis. Euclidean: the reference's own squared-distance plan (src/BinEdges.jl:447-469) -> its
# squared table, or the LinearBinEdges parameters of a SquaredLinearPlan. Sphere: digitize(r, edges).
function distance_bins_of(keep, metric::DI.Euclidean, distance_bins)
    plan = SF.squared_digitize_plan(SF.BinEdges(distance_bins))
    plan isa SF.SquaredLinearPlan && return linear_bins(plan.edges)
    plan isa SF.SquaredInfPaddedPlan && throw(ArgumentError("InfPaddedBinEdges are not supported by B200Backend"))
    sq = Float64.(collect(plan.sqedges))
    push!(keep, sq)
    return CBins(1, length(sq), pointer(sq), 0.0, 0.0, 0.0, 0.0)
end

function distance_bins_of(keep, metric, distance_bins)
    be = SF.BinEdges(distance_bins)
    be isa SF.LinearBinEdges && return linear_bins(be)
    be isa SF.BinEdges || throw(ArgumentError("B200Backend supports vector or range distance bins off the Euclidean path; got $(typeof(be))"))
    e = Float64.(collect(be.edges))
    push!(keep, e)
    return CBins(0, length(e), pointer(e), 0.0, 0.0, 0.0, 0.0)
end

function value_bins_of(keep, value_bins)
    be = SF.BinEdges(value_bins)
    be isa SF.LinearBinEdges && return linear_bins(be)
    be isa SF.BinEdges || throw(ArgumentError("B200Backend supports vector or range value bins; got $(typeof(be))"))
    e = Float64.(collect(be.edges))
    push!(keep, e)
    return CBins(0, length(e), pointer(e), 0.0, 0.0, 0.0, 0.0)
end

# ---------------------------------------------------------------------- context / errors

const CONTEXTS = Dict{Int, Ptr{Cvoid}}()

function context(device::Int)
    get!(CONTEXTS, device) do
        ctx = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:sfb200_ctx_create, libpath()), Cint, (Cint, Ref{Ptr{Cvoid}}), device, ctx)
        rc == OK || error("sfb200_ctx_create(device=$device) failed with status $rc")
        ctx[]
    end
end

function check(rc, ctx)
    rc == OK && return nothing
    msg = unsafe_string(ccall((:sfb200_last_error, libpath()), Cstring, (Ptr{Cvoid},), ctx))
    rc in (ERR_INVALID_ARG, ERR_UNSUPPORTED) && throw(ArgumentError(msg))
    rc == ERR_DIMENSION && throw(DimensionMismatch(msg))
    error("sfb200 status $rc: $msg")
end

# ---------------------------------------------------------------------- core call

# Plan description of a call; `keep` holds the tables the description points to (the library copies
# them when the plan is created). xs, us: the inputs as contiguous column-major (W, N) / (D, N).
function plan_desc(precision::Int32, sfs::Tuple, xs::Matrix, us::Matrix, distance_bins, value_bins, metric)
    D = size(us, 1)
    geom, unit, radius = geometry_of(metric, D)
    keep = Any[]
    ops = ntuple(k -> k <= length(sfs) ? c_op(sfs[k]) : NO_OP, 8)
    desc = CPlanDesc(geom, D, unit, radius, length(sfs), ops, distance_bins_of(keep, metric, distance_bins),
                     value_bins === nothing ? Int32(0) : Int32(1),
                     value_bins === nothing ? NO_BINS : value_bins_of(keep, value_bins),
                     precision, c_dtype(eltype(xs)), c_dtype(eltype(us)))
    return desc, keep
end

# Plans cached per call shape: (device, precision, operator types, D, metric, bins, element types).
# A plan owns its device workspace and serves one call at a time (the reference's workspace rule,
# src/Calculations/workspace.jl:44), so calls on one backend from several tasks are serialised by
# PLAN_LOCK around the run.
const PLANS = Dict{Any, Ptr{Cvoid}}()
const PLAN_LOCK = ReentrantLock()

function cached_plan(b::B200Backend, sfs::Tuple, xs::Matrix, us::Matrix, distance_bins, value_bins, metric)
    key = (b.device, b.precision, map(typeof, sfs), sfs, size(us, 1), metric, collect(distance_bins),
           value_bins === nothing ? nothing : collect(value_bins), eltype(xs), eltype(us))
    ctx = context(b.device)
    plan = get!(PLANS, key) do
        desc, keep = plan_desc(c_precision(b.precision), sfs, xs, us, distance_bins, value_bins, metric)
        p = Ref{Ptr{Cvoid}}(C_NULL)
        GC.@preserve keep begin
            check(ccall((:sfb200_plan_create, libpath()), Cint, (Ptr{Cvoid}, Ref{CPlanDesc}, Ref{Ptr{Cvoid}}),
                        ctx, desc, p), ctx)
        end
        p[]
    end
    return plan, ctx
end

"""Destroy every cached plan (they are rebuilt on the next call)."""
function clear_plans!()
    lock(PLAN_LOCK) do
        for p in values(PLANS)
            ccall((:sfb200_plan_destroy, libpath()), Cint, (Ptr{Cvoid},), p)
        end
        empty!(PLANS)
    end
    return nothing
end

# Runs the pair loop into `sums` / `counts` (Float64 / UInt64, contiguous). flags: RUN_ACCUMULATE adds
# into them (the mutating API), 0 overwrites them.
function run_pairs(b::B200Backend, sfs::Tuple, x::AbstractMatrix, u::AbstractMatrix, distance_bins,
                   value_bins, metric, sums::Array{Float64}, counts::Array{UInt64}, flags::UInt32)
    xs = x isa Matrix ? x : Matrix(x)   # contiguous column-major (W, N)
    us = u isa Matrix ? u : Matrix(u)
    lock(PLAN_LOCK) do
        plan, ctx = cached_plan(b, sfs, xs, us, distance_bins, value_bins, metric)
        GC.@preserve xs us sums counts begin
            check(ccall((:sfb200_run, libpath()), Cint,
                        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, UInt32, Ptr{Float64}, Ptr{UInt64}, Ptr{Cvoid}),
                        plan, xs, us, size(xs, 2), flags, sums, counts, C_NULL), ctx)
        end
    end
    return nothing
end

out_type(x, u) = promote_type(float(eltype(x)), float(eltype(u)))

# ---------------------------------------------------------------------- dispatch methods

# 1D, non-mutating (beside dispatch.jl:537-544)
function SFC._dispatch_execution_backend(
    b::B200Backend, shape::SFC.PointField{D}, sf::SFT.AbstractPairwiseStructureFunctionType, x, u,
    distance_bins, count_eltype::Type{CT} = UInt32; distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
) where {D, CT}
    nb = length(distance_bins) - 1
    sums = zeros(Float64, nb)
    counts = zeros(UInt64, nb)
    run_pairs(b, (sf,), x, u, distance_bins, nothing, distance_metric, sums, counts, UInt32(0))
    return SFO.StructureFunctionSumsAndCounts(sf, distance_bins, out_type(x, u).(sums), CT.(counts))
end

# joint, non-mutating (beside dispatch.jl:576-583)
function SFC._dispatch_execution_backend(
    b::B200Backend, shape::SFC.PointField{D}, sf::SFT.AbstractPairwiseStructureFunctionType, x, u,
    distance_bins, value_bins::AbstractVector; distance_metric::DI.PreMetric = DI.Euclidean(),
    count_eltype::Type{CT} = UInt32, kwargs...,
) where {D, CT}
    nd, nv = length(distance_bins) - 1, length(value_bins) - 1
    sums = zeros(Float64, nd * nv)
    counts = zeros(UInt64, nd * nv)
    run_pairs(b, (sf,), x, u, distance_bins, value_bins, distance_metric, sums, counts, UInt32(0))
    return SFO.StructureFunction2DSumsAndCounts(sf, distance_bins, value_bins,
        reshape(out_type(x, u).(sums), nd, nv), reshape(CT.(counts), nd, nv))
end

# mutating: add into the caller's buffers (beside dispatch.jl:399-404). Float64 sums and UInt64 counts
# in contiguous arrays are accumulated into by the library itself (SFB200_RUN_ACCUMULATE); other
# element types go through library-typed buffers and a conversion.
function accumulate_into!(b, sfs, x, u, distance_bins, value_bins, metric, sums::AbstractArray, counts::AbstractArray)
    if sums isa Array{Float64} && counts isa Array{UInt64}
        run_pairs(b, sfs, x, u, distance_bins, value_bins, metric, sums, counts, RUN_ACCUMULATE)
    else
        s = zeros(Float64, length(sums))
        c = zeros(UInt64, length(counts))
        run_pairs(b, sfs, x, u, distance_bins, value_bins, metric, s, c, UInt32(0))
        sums .+= reshape(s, size(sums))
        counts .+= reshape(c, size(counts))
    end
    return nothing
end

function SFC._dispatch_execution_backend!(
    b::B200Backend, shape::SFC.PointField, sums::AbstractVector, counts::AbstractVector,
    sf::SFT.AbstractPairwiseStructureFunctionType, x, u, distance_bins;
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    accumulate_into!(b, (sf,), x, u, distance_bins, nothing, distance_metric, sums, counts)
end

function SFC._dispatch_execution_backend!(
    b::B200Backend, shape::SFC.PointField, sums_2d::AbstractMatrix, counts_2d::AbstractMatrix,
    sf::SFT.AbstractPairwiseStructureFunctionType, x, u, distance_bins, value_bins::AbstractVector;
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    accumulate_into!(b, (sf,), x, u, distance_bins, value_bins, distance_metric, sums_2d, counts_2d)
end

# ---------------------------------------------------------------------- six-invariant single pass
#
# calculate_structure_functions_single_pass[!] (src/Calculations/serial_single_pass.jl:408-421, 663-693)
# route here through _dispatch_single_pass[!]. One fused pass accumulates S2, L2, S3, L3 (operator
# list {S2, L2, S3, L3}); rows T2 = S2 - L2 and L1T2 = S3 - L3 and the shared count row are filled
# by the reference's own _sp1d_derive_rows! (serial_single_pass.jl:209-219).

const SP_ACCUMULATED = (SFT.SecondOrderStructureFunctionType(), SFT.LongitudinalSecondOrderStructureFunctionType(),
                        SFT.ThirdOrderStructureFunctionType(), SFT.DiagonalConsistentThirdOrderStructureFunctionType())
const SP_ROWS = (1, 2, 4, 5)

# Adds the four accumulated rows of one pass into `sums` / `counts` ((6, n_bins)); derives the rest.
function single_pass_into!(b::B200Backend, sums::AbstractMatrix, counts::AbstractMatrix, x, u, distance_bins,
                           metric)
    nb = length(distance_bins) - 1
    size(sums) == (SFC.SINGLE_PASS_N, nb) ||
        throw(DimensionMismatch("sums must have shape ($(SFC.SINGLE_PASS_N), n_bins); got $(size(sums))"))
    size(counts) == size(sums) || throw(DimensionMismatch("counts must have shape $(size(sums))"))
    s = zeros(Float64, 4 * nb)
    c = zeros(UInt64, nb)
    run_pairs(b, SP_ACCUMULATED, x, u, distance_bins, nothing, metric, s, c, UInt32(0))
    for (k, row) in enumerate(SP_ROWS)
        @views sums[row, :] .+= s[(k - 1) * nb + 1:k * nb]
    end
    @views counts[1, :] .+= c
    SFC._sp1d_derive_rows!(sums, counts)
    return sums, counts
end

function SFC._dispatch_single_pass(
    b::B200Backend, ::SFC.PointField, x::AbstractMatrix{FT1}, u::AbstractMatrix{FT2}, distance_bins::AbstractVector;
    count_eltype::Type{CT} = UInt32, distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
) where {FT1, FT2, CT}
    OT = promote_type(float(FT1), float(FT2))
    nb = length(distance_bins) - 1
    sums = zeros(OT, SFC.SINGLE_PASS_N, nb)
    counts = zeros(CT, SFC.SINGLE_PASS_N, nb)
    single_pass_into!(b, sums, counts, x, u, distance_bins, distance_metric)
    return (sums = sums, counts = counts)
end

function SFC._dispatch_single_pass!(
    b::B200Backend, sums::AbstractMatrix, counts::AbstractMatrix, x::AbstractMatrix, u::AbstractMatrix,
    distance_bins::AbstractVector; distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    return single_pass_into!(b, sums, counts, x, u, distance_bins, distance_metric)
end

# ---------------------------------------------------------------------- two-dimensional single pass
#
# calculate_structure_functions_single_pass_2d[!] (src/Calculations/serial_single_pass.jl:712-728,
# 1161-1181) route here through _dispatch_single_pass_2d[!]. Row t of the (6, n_dist, n_val)
# accumulator is the joint histogram of invariant t (S2, L2, T2, S3, L3, L1T2), computed on the device
# with the pass's own formulas (operator kind SFB200_OP_SP2D, nl = t - 1; flat du_L = (du . dx) *
# inv(sqrt(r2)), serial_single_pass.jl:889-893) and binned on that row's value edges as the reference's
# scatter digitizes them (:852-864): a LinearBinEdges by its FMA search, any other vector or range by
# searchsortedfirst over its elements.

struct SP2DRow <: SFT.AbstractPairwiseStructureFunctionType
    t::Int
end
c_op(r::SP2DRow) = COperator(6, r.t - 1, 0, 0)

# a row's value axis cut to its first n_val + 1 edges (bins above n_val are dropped by the scatter)
function sp2d_row_bins(vb, n_val::Int)
    vb isa SF.LinearBinEdges && length(vb) == n_val + 1 && return vb
    vb isa SF.LinearBinEdges && throw(ArgumentError("B200Backend needs a LinearBinEdges value axis of exactly n_val + 1 edges"))
    vb isa SF.InfPaddedBinEdges && throw(ArgumentError("InfPaddedBinEdges are not supported by B200Backend"))
    return Float64.(collect(vb))[1:n_val + 1]
end

# Adds the six rows of one point set into `sums` / `counts` ((6, n_dist, n_val)).
# Rows per joint run: on flat (Euclidean) geometry with one value axis shared by the six rows, as many
# consecutive rows as the shared-memory cell budget holds (one FP64 launch forms each pair's arithmetic
# once for all of them; sfb200.h, SFB200_OP_SP2D); one otherwise.
const SP2D_ROW_CELL_BYTES = 196 * 1024
function sp2d_rows_per_run(value_bins, nd::Int, n_val::Int, metric)
    (value_bins isa Tuple || !(metric isa DI.Euclidean)) && return 1
    return clamp(SP2D_ROW_CELL_BYTES ÷ max(1, 12 * nd * n_val), 1, SFC.SINGLE_PASS_N)
end

function single_pass_2d_into!(b::B200Backend, sums::AbstractArray, counts::AbstractArray, x, u, distance_bins,
                              value_bins, metric)
    nd, n_val = size(sums, 2), size(sums, 3)
    SFC._validate_value_bins!(value_bins, n_val)
    k = sp2d_rows_per_run(value_bins, nd, n_val, metric)
    m = nd * n_val
    s = zeros(Float64, k * m)
    c = zeros(UInt64, k * m)
    for t0 in 1:k:SFC.SINGLE_PASS_N
        rows = t0:min(SFC.SINGLE_PASS_N, t0 + k - 1)
        vb = sp2d_row_bins(value_bins isa Tuple ? value_bins[t0] : value_bins, n_val)
        run_pairs(b, Tuple(SP2DRow(t) for t in rows), x, u, distance_bins, vb, metric, s, c, UInt32(0))
        for (g, t) in enumerate(rows)
            @views sums[t, :, :] .+= reshape(s[(g - 1) * m + 1:g * m], nd, n_val)
            @views counts[t, :, :] .+= reshape(c[(g - 1) * m + 1:g * m], nd, n_val)
        end
    end
    return sums, counts
end

function SFC._dispatch_single_pass_2d(
    b::B200Backend, ::SFC.PointField, x::AbstractMatrix{FT1}, u::AbstractMatrix{FT2}, distance_bins::AbstractVector,
    value_bins::SFC.SinglePass2DValueBins; count_eltype::Type{CT} = UInt32,
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
) where {FT1, FT2, CT}
    OT = promote_type(float(FT1), float(FT2))
    nd = length(distance_bins) - 1
    n_val = length(value_bins isa Tuple ? value_bins[1] : value_bins) - 1
    sums = zeros(OT, SFC.SINGLE_PASS_N, nd, n_val)
    counts = zeros(CT, SFC.SINGLE_PASS_N, nd, n_val)
    single_pass_2d_into!(b, sums, counts, x, u, distance_bins, value_bins, distance_metric)
    return (sums = sums, counts = counts)
end

function SFC._dispatch_single_pass_2d(
    b::B200Backend, shape::Union{SFC.SharedPositionField, SFC.VaryingPositionField}, x::AbstractArray{FT1},
    u::AbstractArray{FT2}, distance_bins::AbstractVector, value_bins::SFC.SinglePass2DValueBins;
    count_eltype::Type{CT} = UInt32, distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
) where {FT1, FT2, CT}
    OT = promote_type(float(FT1), float(FT2))
    nd = length(distance_bins) - 1
    n_val = length(value_bins isa Tuple ? value_bins[1] : value_bins) - 1
    aux = size(u)[3:end]
    sums = zeros(OT, SFC.SINGLE_PASS_N, nd, n_val, aux...)
    counts = zeros(CT, SFC.SINGLE_PASS_N, nd, n_val, aux...)
    for (k, (xb, ub)) in zip(CartesianIndices(aux), aux_slices(x, u))
        single_pass_2d_into!(b, view(sums, :, :, :, k), view(counts, :, :, :, k), xb, ub, distance_bins,
                             value_bins, distance_metric)
    end
    return (sums = sums, counts = counts)
end

function SFC._dispatch_single_pass_2d!(
    b::B200Backend, sums_3d::AbstractArray, counts_3d::AbstractArray, x::AbstractMatrix, u::AbstractMatrix,
    distance_bins::AbstractVector, value_bins::SFC.SinglePass2DValueBins;
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    return single_pass_2d_into!(b, sums_3d, counts_3d, x, u, distance_bins, value_bins, distance_metric)
end

# auxiliary-axis shapes (src/Calculations/shapes.jl:19-20): one pair pass per auxiliary slice, results
# of shape (n_bins, aux...) / (n_dist, n_val, aux...) as the reference's batch drivers return them
# (src/Calculations/batch.jl:209-217)
aux_slices(x, u) = (ndims(x) == 2 ? (x, view(u, :, :, k)) : (view(x, :, :, k), view(u, :, :, k))
                    for k in CartesianIndices(size(u)[3:end]))

function SFC._dispatch_execution_backend(
    b::B200Backend, shape::SFC.AbstractFieldShape, sf::SFT.AbstractPairwiseStructureFunctionType, x, u,
    distance_bins, count_eltype::Type{CT} = UInt32; distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
) where {CT}
    nb = length(distance_bins) - 1
    aux = size(u)[3:end]
    sums = zeros(out_type(x, u), nb, aux...)
    counts = zeros(CT, nb, aux...)
    s = zeros(Float64, nb)
    c = zeros(UInt64, nb)
    for (k, (xb, ub)) in zip(CartesianIndices(aux), aux_slices(x, u))
        run_pairs(b, (sf,), xb, ub, distance_bins, nothing, distance_metric, s, c, UInt32(0))
        @views sums[:, k] .= s
        @views counts[:, k] .= c
    end
    return SFO.StructureFunctionSumsAndCounts(sf, distance_bins, sums, counts)
end

function SFC._dispatch_execution_backend(
    b::B200Backend, shape::SFC.AbstractFieldShape, sf::SFT.AbstractPairwiseStructureFunctionType, x, u,
    distance_bins, value_bins::AbstractVector; distance_metric::DI.PreMetric = DI.Euclidean(),
    count_eltype::Type{CT} = UInt32, kwargs...,
) where {CT}
    nd, nv = length(distance_bins) - 1, length(value_bins) - 1
    aux = size(u)[3:end]
    sums = zeros(out_type(x, u), nd, nv, aux...)
    counts = zeros(CT, nd, nv, aux...)
    s = zeros(Float64, nd * nv)
    c = zeros(UInt64, nd * nv)
    for (k, (xb, ub)) in zip(CartesianIndices(aux), aux_slices(x, u))
        run_pairs(b, (sf,), xb, ub, distance_bins, value_bins, distance_metric, s, c, UInt32(0))
        @views sums[:, :, k] .= reshape(s, nd, nv)
        @views counts[:, :, k] .= reshape(c, nd, nv)
    end
    return SFO.StructureFunction2DSumsAndCounts(sf, distance_bins, value_bins, sums, counts)
end

function SFC._dispatch_execution_backend!(
    b::B200Backend, shape::SFC.AbstractFieldShape, sums, counts, sf::SFT.AbstractPairwiseStructureFunctionType,
    x, u, distance_bins, value_bins::AbstractVector...; distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    for (k, (xb, ub)) in zip(CartesianIndices(size(u)[3:end]), aux_slices(x, u))
        if isempty(value_bins)
            accumulate_into!(b, (sf,), xb, ub, distance_bins, nothing, distance_metric, view(sums, :, k), view(counts, :, k))
        else
            accumulate_into!(b, (sf,), xb, ub, distance_bins, value_bins[1], distance_metric, view(sums, :, :, k),
                             view(counts, :, :, k))
        end
    end
    return nothing
end

# ---------------------------------------------------------------------- serving (many requests)
#
# No counterpart in the reference, which computes one call at a time. A `B200Server` keeps requests
# resident on the device as slices and runs their pairs together: a loop task admits requests in
# arrival order while a slot is free and the device has room (sfb200_device_memory), gives every
# active slice at least one tile pair per round and the rest of the round's pair budget
# shortest-remaining-first, queues each round as one batched launch per kernel variant
# (sfb200_batch_run; two rounds in flight, sfb200_batch_wait_oldest), and completes a request with its
# own result container once all its tile pairs have run. The same loop as `sfb200.serving.Server` in
# the Python mirror, which the test suite drives on the GPU.

struct CSliceInfo
    n_points::Int64
    pairs::Int64
    tile_pairs::Int64
    device_bytes::Int64
end

struct B200Request
    sf::Any
    x::Matrix
    u::Matrix
    distance_bins::Any
    value_bins::Any
    metric::Any
    count_eltype::Type
end

mutable struct B200Ticket
    request::B200Request
    t_submit::Float64
    t_done::Float64
    result::Any
    error::Any
    done::Base.Event
end

mutable struct ActiveSlice
    ticket::B200Ticket
    slice::Ptr{Cvoid}
    plan::Ptr{Cvoid}
    n_sums::Int64
    n_counts::Int64
    units::Int64          # tile pairs in total
    issued::Int64         # tile pairs queued so far (a prefix)
    done::Int64           # tile pairs completed (a prefix)
    pairs_per_unit::Float64
end

mutable struct B200Server
    device::Int
    max_slots::Int
    memory_reserve::Int64
    round_pairs::Float64
    min_units::Int
    max_wait::Float64     # seconds after which a waiting request is admitted before smaller ones
    pending::Vector{B200Ticket}
    active::Vector{ActiveSlice}
    plans::Dict{Any, Ptr{Cvoid}}
    lock::ReentrantLock
    stopping::Bool
    failed::Any           # the error that ended the loop (nothing while it runs)
    task::Union{Nothing, Task}
    rounds::Int
end

"""
    B200Server(; device = 0, max_slots = 256, memory_reserve = 1 << 30, round_pairs = 6e9, min_units = 1)

A request loop over one device (mixed precision). `start!` it, `submit!` requests (the arguments of
`calculate_structure_function`), `fetch_result` a ticket, `stop!` it when done.
"""
B200Server(; device::Integer = 0, max_slots::Integer = 256, memory_reserve::Integer = 1 << 30,
           round_pairs::Real = 6e9, min_units::Integer = 1, max_wait::Real = 1.0) =
    B200Server(Int(device), Int(max_slots), Int64(memory_reserve), Float64(round_pairs), Int(min_units),
               Float64(max_wait), B200Ticket[], ActiveSlice[], Dict{Any, Ptr{Cvoid}}(), ReentrantLock(), false,
               nothing, nothing, 0)

"""
    submit!(srv, sf, x, u, distance_bins[, value_bins]; distance_metric, count_eltype = UInt32)

Queue one request. The count guard of the public entry runs here (`_assert_counts_representable`,
src/Calculations/serial.jl:111-120): counts of `count_eltype` must hold N(N-1)/2. A request submitted
after the loop has failed fails at once with the loop's error.
"""
function submit!(srv::B200Server, sf, x::AbstractMatrix, u::AbstractMatrix, distance_bins, value_bins = nothing;
                 distance_metric::DI.PreMetric = DI.Euclidean(), count_eltype::Type = UInt32)
    SFC._assert_counts_representable(count_eltype, size(x, 2))
    t = B200Ticket(B200Request(sf, Matrix(x), Matrix(u), distance_bins, value_bins, distance_metric, count_eltype),
                   time(), NaN, nothing, nothing, Base.Event())
    err = lock(srv.lock) do
        srv.failed === nothing && push!(srv.pending, t)
        srv.failed
    end
    err === nothing || fail!(t, err)
    return t
end

"""The request's result container (`StructureFunctionSumsAndCounts` or `...2DSumsAndCounts`)."""
function fetch_result(t::B200Ticket)
    wait(t.done)
    t.error === nothing || throw(t.error)
    return t.result
end

start!(srv::B200Server) = (srv.task = Threads.@spawn serve_loop(srv); srv)

function stop!(srv::B200Server)
    lock(() -> (srv.stopping = true), srv.lock)
    try
        srv.task === nothing || wait(srv.task)  # rethrows the loop's failure, if any
    finally
        for plan in values(srv.plans)
            ccall((:sfb200_plan_destroy, libpath()), Cint, (Ptr{Cvoid},), plan)
        end
        empty!(srv.plans)
    end
    return nothing
end

function fail!(t::B200Ticket, err)
    t.error = err
    t.t_done = time()
    notify(t.done)
end

function free_bytes(ctx)
    f = Ref{Int64}(0)
    total = Ref{Int64}(0)
    check(ccall((:sfb200_device_memory, libpath()), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), ctx, f, total), ctx)
    return f[]
end

# device bytes of a slice: raw and packed points, ordering keys and the histogram (an estimate)
estimate_bytes(r::B200Request) = Int64(size(r.x, 2)) * (8 * (size(r.x, 1) + 2 * size(r.u, 1)) + 136) + (1 << 20)

function create_slice(srv::B200Server, ctx, t::B200Ticket)
    r = t.request
    key = (typeof(r.sf), r.sf, size(r.u, 1), r.metric, collect(r.distance_bins),
           r.value_bins === nothing ? nothing : collect(r.value_bins), eltype(r.x), eltype(r.u))
    plan = get!(srv.plans, key) do
        desc, keep = plan_desc(Int32(1), (r.sf,), r.x, r.u, r.distance_bins, r.value_bins, r.metric)
        p = Ref{Ptr{Cvoid}}(C_NULL)
        GC.@preserve keep begin
            check(ccall((:sfb200_plan_create, libpath()), Cint, (Ptr{Cvoid}, Ref{CPlanDesc}, Ref{Ptr{Cvoid}}),
                        ctx, desc, p), ctx)
        end
        p[]
    end
    ns, nc = Ref{Int64}(0), Ref{Int64}(0)
    check(ccall((:sfb200_plan_output_sizes, libpath()), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int64}), plan, ns, nc), ctx)
    sl = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve r begin
        check(ccall((:sfb200_slice_create, libpath()), Cint,
                    (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, UInt32, Ptr{Cvoid}, Ref{Ptr{Cvoid}}),
                    plan, r.x, r.u, size(r.x, 2), UInt32(0), C_NULL, sl), ctx)
    end
    info = Ref(CSliceInfo(0, 0, 0, 0))
    try
        check(ccall((:sfb200_slice_get_info, libpath()), Cint, (Ptr{Cvoid}, Ref{CSliceInfo}), sl[], info), ctx)
    catch
        ccall((:sfb200_slice_destroy, libpath()), Cint, (Ptr{Cvoid},), sl[])  # the slice exists: free it
        rethrow()
    end
    units = info[].tile_pairs
    return ActiveSlice(t, sl[], plan, ns[], nc[], units, 0, 0, max(1.0, info[].pairs / max(1, units)))
end

function complete!(ctx, a::ActiveSlice)
    t = a.ticket
    r = t.request
    try
        sums = zeros(Float64, a.n_sums)
        counts = zeros(UInt64, a.n_counts)
        check(ccall((:sfb200_slice_read, libpath()), Cint,
                    (Ptr{Cvoid}, Ptr{Float64}, Ptr{UInt64}, UInt32, Ptr{Cvoid}), a.slice, sums, counts, UInt32(0),
                    C_NULL), ctx)
        T = out_type(r.x, r.u)
        CT = r.count_eltype
        if r.value_bins === nothing
            t.result = SFO.StructureFunctionSumsAndCounts(r.sf, r.distance_bins, T.(sums), CT.(counts))
        else
            nd, nv = length(r.distance_bins) - 1, length(r.value_bins) - 1
            t.result = SFO.StructureFunction2DSumsAndCounts(r.sf, r.distance_bins, r.value_bins,
                reshape(T.(sums), nd, nv), reshape(CT.(counts), nd, nv))
        end
    catch err
        t.error = err
    finally
        ccall((:sfb200_slice_destroy, libpath()), Cint, (Ptr{Cvoid},), a.slice)
    end
    t.t_done = time()
    notify(t.done)
end

# The waiting request to admit next: the oldest once it has waited max_wait seconds, else the one with
# the fewest pairs (a small request arriving while the slots hold large ones waits for one slot, not
# for the whole queue).
function next_pending(srv::B200Server)
    oldest = srv.pending[1]
    (length(srv.pending) == 1 || time() - oldest.t_submit > srv.max_wait) && return 1
    return argmin([size(t.request.x, 2) for t in srv.pending])
end

function admit!(srv::B200Server, ctx)
    while true
        t = lock(srv.lock) do
            (isempty(srv.pending) || length(srv.active) >= srv.max_slots) && return nothing
            k = next_pending(srv)
            head = srv.pending[k]
            if !isempty(srv.active) && free_bytes(ctx) - estimate_bytes(head.request) < srv.memory_reserve
                return nothing  # wait for a slice to finish and free its memory
            end
            popat!(srv.pending, k)
        end
        t === nothing && return nothing
        try
            a = create_slice(srv, ctx, t)
            a.units == 0 ? complete!(ctx, a) : push!(srv.active, a)
        catch err
            fail!(t, err)
        end
    end
end

remaining(a::ActiveSlice) = a.units - a.issued

function plan_round(srv::B200Server)
    ready = filter(a -> remaining(a) > 0, srv.active)
    give = Dict{ActiveSlice, Int64}(a => min(remaining(a), srv.min_units) for a in ready)
    budget = srv.round_pairs - sum((give[a] * a.pairs_per_unit for a in ready); init = 0.0)
    for a in sort(ready; by = a -> remaining(a) * a.pairs_per_unit)
        budget <= 0 && break
        extra = min(remaining(a) - give[a], floor(Int64, budget / a.pairs_per_unit) + 1)
        if extra > 0
            give[a] += extra
            budget -= extra * a.pairs_per_unit
        end
    end
    return [(a, a.issued, a.issued + give[a]) for a in ready if give[a] > 0]
end

function serve_loop(srv::B200Server)
    ctx = context(srv.device)
    inflight = Vector{Vector{Tuple{ActiveSlice, Int64, Int64}}}()
    try
        while true
            admit!(srv, ctx)
            if length(inflight) < 2 && any(a -> remaining(a) > 0, srv.active)
                work = plan_round(srv)
                slices = Ptr{Cvoid}[w[1].slice for w in work]
                lo = Int64[w[2] for w in work]
                hi = Int64[w[3] for w in work]
                check(ccall((:sfb200_batch_run, libpath()), Cint,
                            (Ptr{Cvoid}, Int32, Ptr{Ptr{Cvoid}}, Ptr{Int64}, Ptr{Int64}, Ptr{Cvoid}),
                            ctx, length(work), slices, lo, hi, C_NULL), ctx)
                for (a, _, e) in work
                    a.issued = e
                end
                push!(inflight, work)
                srv.rounds += 1
                continue
            end
            if !isempty(inflight)
                check(ccall((:sfb200_batch_wait_oldest, libpath()), Cint, (Ptr{Cvoid}, Ptr{Int64}), ctx, C_NULL), ctx)
                for (a, _, e) in popfirst!(inflight)
                    a.done = e
                    if a.done >= a.units
                        filter!(b -> b !== a, srv.active)
                        complete!(ctx, a)
                    end
                end
                continue
            end
            idle = lock(() -> (isempty(srv.pending), srv.stopping), srv.lock)
            idle[1] && idle[2] && return nothing
            sleep(0.001)
        end
    catch err
        # a failed round fails every request the loop holds, instead of leaving it waiting
        ccall((:sfb200_batch_wait, libpath()), Cint, (Ptr{Cvoid},), ctx)
        for a in srv.active
            ccall((:sfb200_slice_destroy, libpath()), Cint, (Ptr{Cvoid},), a.slice)
            fail!(a.ticket, err)
        end
        empty!(srv.active)
        # under the lock: mark the loop failed and take what is pending, so that a later submit!
        # fails its ticket at once instead of queueing it for a loop that no longer runs
        waiting = lock(srv.lock) do
            srv.failed = err
            splice!(srv.pending, 1:length(srv.pending))
        end
        for t in waiting
            fail!(t, err)
        end
        rethrow()
    end
end

end # module
