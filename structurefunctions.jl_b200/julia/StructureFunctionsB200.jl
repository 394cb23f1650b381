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

export B200Backend

const LIB = Ref{String}("")
libpath() = isempty(LIB[]) ? get(ENV, "SFB200_LIB", joinpath(@__DIR__, "..", "libsfb200.so")) : LIB[]

"""
    B200Backend(; device = 0, precision = :mixed)

Run the O(N^2) pair loop on a B200. `precision = :mixed` (FP32 pair arithmetic, FP64 recheck of
pairs near a bin edge, FP64 merge) or `:fp64` (every pair in FP64). Not an `AbstractGPUBackend`, so
no KernelAbstractions route captures it; `AutoBackend` never selects it.
"""
struct B200Backend <: CB.AbstractExecutionBackend
    device::Int
    precision::Symbol
end
B200Backend(; device::Integer = 0, precision::Symbol = :mixed) =
    precision in (:mixed, :fp64) ? B200Backend(Int(device), precision) :
    throw(ArgumentError("precision must be :mixed or :fp64"))

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

function run_pairs(b::B200Backend, sfs::Tuple, x::AbstractMatrix, u::AbstractMatrix, distance_bins,
                   value_bins, metric, sums::Vector{Float64}, counts::Vector{UInt64}, flags::UInt32)
    D = size(u, 1)
    geom, unit, radius = geometry_of(metric, D)
    keep = Any[]
    xs = Matrix(x)   # contiguous column-major (W, N)
    us = Matrix(u)
    ops = ntuple(k -> k <= length(sfs) ? c_op(sfs[k]) : NO_OP, 8)
    desc = CPlanDesc(geom, D, unit, radius, length(sfs), ops, distance_bins_of(keep, metric, distance_bins),
                     value_bins === nothing ? Int32(0) : Int32(1),
                     value_bins === nothing ? NO_BINS : value_bins_of(keep, value_bins),
                     b.precision === :mixed ? Int32(1) : Int32(0), c_dtype(eltype(xs)), c_dtype(eltype(us)))
    ctx = context(b.device)
    plan = Ref{Ptr{Cvoid}}(C_NULL)
    GC.@preserve keep begin
        check(ccall((:sfb200_plan_create, libpath()), Cint, (Ptr{Cvoid}, Ref{CPlanDesc}, Ref{Ptr{Cvoid}}),
                    ctx, desc, plan), ctx)
    end
    try
        GC.@preserve xs us sums counts begin
            check(ccall((:sfb200_run, libpath()), Cint,
                        (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int64, UInt32, Ptr{Float64}, Ptr{UInt64}, Ptr{Cvoid}),
                        plan[], xs, us, size(xs, 2), flags, sums, counts, C_NULL), ctx)
        end
    finally
        ccall((:sfb200_plan_destroy, libpath()), Cint, (Ptr{Cvoid},), plan[])
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

# mutating: add into the caller's buffers (beside dispatch.jl:399-404)
function SFC._dispatch_execution_backend!(
    b::B200Backend, shape::SFC.PointField, sums::AbstractVector, counts::AbstractVector,
    sf::SFT.AbstractPairwiseStructureFunctionType, x, u, distance_bins;
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    s = zeros(Float64, length(sums))
    c = zeros(UInt64, length(counts))
    run_pairs(b, (sf,), x, u, distance_bins, nothing, distance_metric, s, c, UInt32(0))
    sums .+= s
    counts .+= c
    return nothing
end

function SFC._dispatch_execution_backend!(
    b::B200Backend, shape::SFC.PointField, sums_2d::AbstractMatrix, counts_2d::AbstractMatrix,
    sf::SFT.AbstractPairwiseStructureFunctionType, x, u, distance_bins, value_bins::AbstractVector;
    distance_metric::DI.PreMetric = DI.Euclidean(), kwargs...,
)
    s = zeros(Float64, length(sums_2d))
    c = zeros(UInt64, length(counts_2d))
    run_pairs(b, (sf,), x, u, distance_bins, value_bins, distance_metric, s, c, UInt32(0))
    sums_2d .+= reshape(s, size(sums_2d))
    counts_2d .+= reshape(c, size(counts_2d))
    return nothing
end

# auxiliary-axis shapes are not on this path (as the GPU in-place route, dispatch.jl:406-410)
SFC._dispatch_execution_backend(b::B200Backend, shape::SFC.AbstractFieldShape, args...; kwargs...) =
    throw(ArgumentError("auxiliary-axis inputs are not implemented for B200Backend"))
SFC._dispatch_execution_backend!(b::B200Backend, shape::SFC.AbstractFieldShape, args...; kwargs...) =
    throw(ArgumentError("in-place auxiliary-axis calculate_structure_function! is not implemented for B200Backend"))

end # module
