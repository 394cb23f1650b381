"""CPU tests of the Python host mirror: validation and error behaviour of the reference's public
entry (raised before any GPU work), bin-table construction, result containers."""
import math

import numpy as np
import pytest

import sfb200 as SF
from sfb200 import _abi
from sfb200.api import plan_description


def test_dimension_mismatch_like_reference():
    # src/Calculations/shapes.jl:67-105
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((2, 8)), np.zeros((4, 8)), SF.Euclidean())   # D not in {2,3}
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((3, 8)), np.zeros((2, 8)), SF.Euclidean())   # W != D (flat)
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((2, 8)), np.zeros((2, 9)), SF.Euclidean())   # N differ
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros(8), np.zeros((2, 8)), SF.Euclidean())        # ndims(x) < 2
    # the sphere locates a point with 2 coordinates for D = 2 and D = 3 (test/test_spherical_geometry.jl:226-233)
    SF.validate_array_shape(np.zeros((2, 8)), np.zeros((3, 8)), SF.Haversine(6.371e6))
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((3, 8)), np.zeros((3, 8)), SF.Haversine(6.371e6))
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((2, 8, 3)), np.zeros((2, 8, 4)), SF.Euclidean())


def test_auxiliary_axes_shapes_and_unknown_metrics():
    # src/Calculations/shapes.jl:17-20, 67-105: shared positions (x (W,N), u (D,N,aux...)) and varying
    # positions (matching auxiliary axes)
    sh = SF.validate_array_shape(np.zeros((2, 8)), np.zeros((2, 8, 3, 2)), SF.Euclidean())
    assert isinstance(sh, SF.api.SharedPositionField) and sh.aux == (3, 2) and sh.D == 2
    vh = SF.validate_array_shape(np.zeros((3, 8, 4)), np.zeros((3, 8, 4)), SF.Euclidean())
    assert isinstance(vh, SF.api.VaryingPositionField) and vh.aux == (4,)
    with pytest.raises(SF.DimensionMismatch):
        SF.validate_array_shape(np.zeros((2, 8, 4)), np.zeros((2, 8, 4, 1)), SF.Euclidean())
    with pytest.raises(SF.ArgumentError):
        SF.pair_geometry_for(SF.PreMetric(), 2)


def test_public_entry_validation_before_gpu():
    x = np.zeros((2, 100_000), dtype=np.float32)
    bins = np.linspace(0, 2, 9).astype(np.float32)
    # count guard fires at the boundary, before any pair work (test/test_core_correctness.jl:236-240)
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_function(SF.L2SF, x, x, bins)
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_function_inplace(np.zeros(8, np.float32), np.zeros(8, np.uint32), SF.L2SF, x, x, bins)
    # derived quantities are not pair operators (src/Calculations/dispatch.jl:7-13)
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_function(SF.RotationalSecondOrderStructureFunction, np.zeros((2, 4)),
                                        np.zeros((2, 4)), bins)
    # tuple inputs are rejected (src/Calculations/shapes.jl:42-49)
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_function(SF.L2SF, (np.zeros(4), np.zeros(4)), (np.zeros(4), np.zeros(4)), bins)
    # a joint histogram takes one operator
    with pytest.raises(SF.ArgumentError):
        SF.calculate_structure_function((SF.L2SF, SF.T2SF), np.zeros((2, 4)), np.zeros((2, 4)), bins,
                                        np.linspace(0, 1, 5))


def test_squared_edge_tables_follow_the_reference_rounding():
    # _sq_edges(T, v) = T(big(v)^2) (src/BinEdges.jl:440)
    e64 = np.array([0.1, 0.3, 0.7, 1.1])
    keep = []
    b = SF.BinEdges(e64).distance_abi(_abi.GEOM_FLAT, keep)
    assert b.kind == _abi.BINS_SQTABLE
    assert [b.edges[k] for k in range(4)] == [float(v) * float(v) for v in e64]
    e32 = e64.astype(np.float32)
    b = SF.BinEdges(e32).distance_abi(_abi.GEOM_FLAT, keep)
    from fractions import Fraction
    for k, v in enumerate(e32):
        exact = Fraction(float(v)) ** 2
        assert b.edges[k] == float(np.float32(float(exact)))
    # off the Euclidean path the raw edges are searched
    b = SF.BinEdges(e64).distance_abi(_abi.GEOM_SPHERE, keep)
    assert b.kind == _abi.BINS_TABLE and b.edges[2] == 0.7


def test_linear_bin_edges_parameters():
    # Julia's range() may lift decimal end points to exact rationals (step 0.14 here); the mirror
    # uses the correctly rounded (last - first)/(n - 1). The Julia glue passes the reference's own
    # fields, so only Python callers see the ulp-level difference.
    lb = SF.LinearBinEdges(0.0, 1.4, 11)
    assert lb.first_edge == 0.0 and lb.last_edge == 1.4
    assert abs(lb.step_val - 0.14) <= math.ulp(0.14)
    assert lb.inv_step == 1.0 / lb.step_val
    abi = lb.distance_abi(_abi.GEOM_FLAT, [])
    assert abi.kind == _abi.BINS_LINEAR and abi.n_edges == 11


def test_unsorted_or_negative_euclidean_edges_rejected():
    with pytest.raises(SF.ArgumentError):
        SF.BinEdges([0.0, 2.0, 1.0]).distance_abi(_abi.GEOM_FLAT, [])
    with pytest.raises(SF.ArgumentError):
        SF.BinEdges([-1.0, 0.5, 1.0]).distance_abi(_abi.GEOM_FLAT, [])   # squares unsorted
    SF.BinEdges([-1.0, 0.5, 1.0]).distance_abi(_abi.GEOM_SPHERE, [])      # fine off the squared path


def test_plan_description_layout():
    desc, keep = plan_description((SF.L2SF, SF.T3SF), 3, np.linspace(0, 1, 5), None, None, "mixed")
    assert desc.geometry == _abi.GEOM_FLAT and desc.dim == 3 and desc.n_ops == 2
    assert (desc.ops[0].kind, desc.ops[0].nl, desc.ops[0].nt) == (_abi.OP_PROJECTED, 2, 0)
    assert (desc.ops[1].nl, desc.ops[1].nt) == (0, 3)
    assert desc.precision == _abi.PREC_MIXED and desc.joint == 0
    desc, keep = plan_description((SF.L2SF,), 2, [1.0, 10.0, 100.0], SF.LinearBinEdges(-1, 1, 5),
                                  SF.Haversine(6371.0), "fp64", np.float32, np.float32)
    assert desc.geometry == _abi.GEOM_SPHERE and desc.radius == 6371.0 and desc.angle_unit == _abi.ANGLE_DEG
    assert desc.joint == 1 and desc.value.kind == _abi.BINS_LINEAR
    assert desc.x_dtype == _abi.F32


def test_result_containers():
    # src/StructureFunctionObjects.jl:50-115, 246-279, 357-366; src/Calculations/serial.jl:132-141
    d = [0.0, 1.0, 2.0]
    a = SF.StructureFunctionSumsAndCounts(SF.L2SF, d, np.array([2.0, 0.0]), np.array([2, 0], np.uint32))
    b = SF.StructureFunctionSumsAndCounts(SF.L2SF, d, np.array([1.0, 3.0]), np.array([1, 1], np.uint32))
    c = a + b
    assert c.sums.tolist() == [3.0, 3.0] and c.counts.tolist() == [3, 1]
    with pytest.raises(SF.ArgumentError):
        a + SF.StructureFunctionSumsAndCounts(SF.T2SF, d, np.zeros(2), np.zeros(2, np.uint32))
    with pytest.raises(SF.DimensionMismatch):
        SF.StructureFunctionSumsAndCounts(SF.L2SF, d, np.zeros(3), np.zeros(3, np.uint32))
    avg = SF.bin_average(a.sums, a.counts)
    assert avg[0] == 1.0 and math.isnan(avg[1])
    j = SF.StructureFunction2DSumsAndCounts(SF.L2SF, d, [0.0, 1.0, 2.0, 3.0], np.ones((2, 3)),
                                            np.ones((2, 3), np.uint64))
    m = SF.marginalize(j)
    assert m.sums.tolist() == [3.0, 3.0] and m.counts.tolist() == [3, 3]
    with pytest.raises(SF.DimensionMismatch):
        SF.StructureFunction2DSumsAndCounts(SF.L2SF, d, [0.0, 1.0], np.ones((2, 3)), np.ones((2, 3)))


def test_operator_lookup():
    # src/StructureFunctionTypes.jl:348-402
    assert SF.get_structure_function_type("L2SF") == SF.L2SF
    assert SF.get_structure_function_type(3, "transverse") == SF.T3SF
    assert SF.get_structure_function_type(2, "scalar") == SF.S2SF
    assert SF.order(SF.L1T2SF) == 3 and SF.order(SF.FullVectorStructureFunctionType(4)) == 4
    with pytest.raises(KeyError):
        SF.get_structure_function_type(4, "longitudinal")
