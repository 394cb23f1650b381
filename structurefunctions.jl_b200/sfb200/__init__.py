"""sfb200: B200-native pair-histogram backend for structure functions.

Python host mirror of the reference's public API for the O(N^2) pair path
(`calculate_structure_function` / `calculate_structure_function!` of jbphyswx/StructureFunctions.jl),
running on libsfb200.so (hand-written sm_100a CUDA kernels behind the C ABI of include/sfb200.h).
"""
from . import _abi
from .api import (B200Backend, PointField, assert_counts_representable, auto_distance_bins,
                  calculate_structure_function, calculate_structure_function_inplace, default_backend,
                  distance_range, last_stats, validate_array_shape)
from .bins import AbstractBinEdges, BinEdges, LinearBinEdges, LogBinEdges, as_bin_edges, jl_range, n_histogram_bins
from .errors import ArgumentError, DeviceError, DimensionMismatch
from .metrics import Euclidean, Haversine, PreMetric, SphericalAngle, pair_geometry_for
from .operators import *  # noqa: F401,F403  (operator types and singletons)
from .operators import get_structure_function_type, order
from .results import (AbstractStructureFunction, StructureFunction, StructureFunction2DSumsAndCounts,
                      StructureFunctionSumsAndCounts, bin_average, marginalize)
from .single_pass import (SINGLE_PASS_OPERATORS, HelmholtzDecomposition2D, SinglePass2DRow,
                          calculate_structure_functions_single_pass, calculate_structure_functions_single_pass_2d,
                          calculate_structure_functions_single_pass_2d_inplace,
                          calculate_structure_functions_single_pass_inplace, helmholtz_decompose_2d)

__version__ = "0.1.0"
