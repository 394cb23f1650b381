"""Bin-edge types mirroring src/BinEdges.jl of the reference.

The GPU library takes the distance axis *as data* (`_abi.Bins`): for Euclidean geometry the
squared-edge table of src/BinEdges.jl:440 (`_sq_edges`, correctly rounded squares in the edges'
own precision) or the LinearBinEdges parameters; for the sphere the raw edges. These classes build
those descriptors, so the bin a pair lands in is decided by exactly the table the reference uses.
"""
from fractions import Fraction

import numpy as np

from . import _abi
from .errors import ArgumentError


class AbstractBinEdges:
    """Sorted bin edges; bins are right-inclusive (a, b] (src/BinEdges.jl:32)."""

    def __len__(self):
        return len(self.edges)

    def __getitem__(self, i):
        return self.edges[i]

    def __array__(self, dtype=None, copy=None):
        return np.asarray(self.edges, dtype=dtype)

    def __eq__(self, other):
        if not isinstance(other, AbstractBinEdges):
            other_edges = np.asarray(other)
        else:
            other_edges = other.edges
        return type(self) is type(other) and np.array_equal(self.edges, other_edges)

    def __hash__(self):
        return hash((type(self).__name__, self.edges.tobytes()))

    def n_histogram_bins(self):
        """len(edges) - 1 (src/BinEdges.jl:352)."""
        return len(self.edges) - 1


class BinEdges(AbstractBinEdges):
    """Generic sorted edge vector searched by binary search (src/BinEdges.jl:49-61)."""

    def __init__(self, edges):
        a = np.asarray(edges)
        if a.ndim != 1:
            raise ArgumentError("bin edges must be a 1-D vector")
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float64)
        self.dtype = a.dtype
        self.edges = np.ascontiguousarray(a, dtype=a.dtype)

    def distance_abi(self, geometry, keep):
        """Distance-axis descriptor. `keep` collects arrays that must outlive the descriptor."""
        e64 = self.edges.astype(np.float64)
        if geometry == _abi.GEOM_FLAT:
            # _sq_edges(T, v) = T(big(v)^2): the square is exact in binary64 for Float32 edges and
            # correctly rounded for Float64 edges; rounding to T then gives the reference's table.
            if self.dtype == np.float32:
                sq = (e64 * e64).astype(np.float32).astype(np.float64)
            else:
                sq = e64 * e64
            return _table(_abi.BINS_SQTABLE, sq, keep)
        return _table(_abi.BINS_TABLE, e64, keep)

    def value_abi(self, keep):
        return _table(_abi.BINS_TABLE, self.edges.astype(np.float64), keep)


class LinearBinEdges(AbstractBinEdges):
    """Uniform edges searched by the FMA formula of src/BinEdges.jl:114-131.

    Built like Julia's `range(first, last; length=n)`: first and last exact, step the correctly
    rounded (last - first)/(n - 1), inv_step = 1/step in binary64. Float64 only.
    """

    def __init__(self, first, last, length):
        n = int(length)
        if n < 2:
            raise ArgumentError("LinearBinEdges needs at least 2 edges")
        f, l = float(first), float(last)
        step = float((Fraction(l) - Fraction(f)) / (n - 1))
        self.first_edge = f
        self.last_edge = l
        self.step_val = step
        self.inv_step = 1.0 / step
        self.dtype = np.dtype(np.float64)
        self.edges = np.array([float(Fraction(f) + k * (Fraction(l) - Fraction(f)) / (n - 1)) for k in range(n)])
        self.edges[0], self.edges[-1] = f, l

    def _linear(self):
        return _abi.Bins(_abi.BINS_LINEAR, len(self.edges), None, self.first_edge, self.last_edge,
                         self.inv_step, self.step_val)

    def distance_abi(self, geometry, keep):
        return self._linear()

    def value_abi(self, keep):
        return self._linear()


def jl_range(first, last, length):
    """`range(first, last; length)`, which the reference normalizes to LinearBinEdges."""
    return LinearBinEdges(first, last, length)


class LogBinEdges(AbstractBinEdges):
    """Log-uniform edges (src/BinEdges.jl:171-185). On the Euclidean path the reference bins from
    the squared physical edges exp(log_edges[i])^2 (SquaredLogPlan, src/BinEdges.jl:447-453), which
    is what this descriptor passes. The log(q) search used off the Euclidean path is not offered."""

    def __init__(self, edges):
        a = np.asarray(edges, dtype=np.float64)
        if np.any(a <= 0):
            raise ArgumentError("Log-spaced bin edges must be strictly positive.")
        n = len(a)
        self.log_edges = np.array([float(Fraction(np.log(a[0])) + k * (Fraction(np.log(a[-1])) - Fraction(np.log(a[0]))) / (n - 1)) for k in range(n)])
        self.dtype = np.dtype(np.float64)
        self.edges = np.exp(self.log_edges)

    def distance_abi(self, geometry, keep):
        if geometry != _abi.GEOM_FLAT:
            raise ArgumentError("LogBinEdges with a non-Euclidean metric is not supported by B200Backend; "
                                "pass the physical edges as a vector")
        return _table(_abi.BINS_SQTABLE, self.edges * self.edges, keep)

    def value_abi(self, keep):
        raise ArgumentError("LogBinEdges value bins are not supported by B200Backend; pass a vector")


def _table(kind, values, keep):
    arr = np.ascontiguousarray(values, dtype=np.float64)
    keep.append(arr)
    if np.any(np.isnan(arr)) or np.any(np.diff(arr) < 0):
        raise ArgumentError("bin edges must be sorted (non-decreasing); for Euclidean distances the "
                            "edges must also be non-negative so that their squares stay sorted")
    ptr = arr.ctypes.data_as(_abi.C.POINTER(_abi.C.c_double))
    return _abi.Bins(kind, len(arr), ptr, 0.0, 0.0, 0.0, 0.0)


def as_bin_edges(edges):
    """BinEdges(edges) normalization (src/BinEdges.jl:362-363)."""
    if isinstance(edges, AbstractBinEdges):
        return edges
    return BinEdges(edges)


def n_histogram_bins(edges):
    return len(edges) - 1
