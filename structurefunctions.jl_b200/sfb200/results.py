"""Result containers mirroring src/StructureFunctionObjects.jl of the reference."""
import numpy as np

from .errors import ArgumentError, DimensionMismatch


def _n_leading(a):
    a = np.asarray(a)
    return a.shape[0] if a.ndim > 1 else a.size


def _edges_equal(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


class AbstractStructureFunction:
    """Root of the result containers (src/StructureFunctionObjects.jl:19)."""


class StructureFunction(AbstractStructureFunction):
    """Averaged result: per-bin mean values (src/StructureFunctionObjects.jl:30-42)."""

    def __init__(self, operator, distance, values):
        if len(distance) != _n_leading(values) + 1:
            raise DimensionMismatch(
                "Flat distance edges must have length one greater than the leading value-bin axis "
                f"(got edges={len(distance)}, value bins={_n_leading(values)})")
        self.operator = operator
        self.distance = distance
        self.values = np.asarray(values)

    def __getitem__(self, i):
        return self.values[i]

    def __len__(self):
        return len(self.values)

    def __iter__(self):
        return iter(self.values)


class StructureFunctionSumsAndCounts(AbstractStructureFunction):
    """Raw per-bin sums and integer pair counts (src/StructureFunctionObjects.jl:50-74)."""

    def __init__(self, operator, distance, sums, counts):
        sums = np.asarray(sums)
        counts = np.asarray(counts)
        if not (len(distance) == _n_leading(sums) + 1 and _n_leading(sums) == _n_leading(counts)
                and sums.shape == counts.shape):
            raise DimensionMismatch(
                "Flat distance edges must satisfy length(distance) == size(sums,1) + 1 and sums/counts "
                f"must match shape (got edges={len(distance)}, sums={sums.shape}, counts={counts.shape})")
        self.operator = operator
        self.distance = distance
        self.sums = sums
        self.counts = counts

    def __len__(self):
        return len(self.sums)

    def __add__(self, other):
        # src/StructureFunctionObjects.jl:246-255
        if self.operator != other.operator:
            raise ArgumentError(f"Cannot add results with different operators: got {self.operator} and {other.operator}")
        if not _edges_equal(self.distance, other.distance):
            raise ArgumentError("Cannot add results with different binning")
        return StructureFunctionSumsAndCounts(self.operator, self.distance, self.sums + other.sums,
                                              self.counts + other.counts)


class StructureFunction2DSumsAndCounts(AbstractStructureFunction):
    """Joint distance x value histogram of sums and counts (src/StructureFunctionObjects.jl:88-115)."""

    def __init__(self, operator, distance_bins, value_bins, sums, counts):
        sums = np.asarray(sums)
        counts = np.asarray(counts)
        if sums.shape != counts.shape:
            raise DimensionMismatch(
                f"Sums and counts matrices must have identical shape (got sums: {sums.shape}, counts: {counts.shape})")
        if sums.shape[0] != len(distance_bins) - 1:
            raise DimensionMismatch(
                f"distance_bins must have length size(sums,1)+1 (got {len(distance_bins)} edges, {sums.shape[0]} distance bins)")
        if sums.shape[1] != len(value_bins) - 1:
            raise DimensionMismatch(
                f"value_bins must have length size(sums,2)+1 (got {len(value_bins)} edges, {sums.shape[1]} value bins)")
        self.operator = operator
        self.distance_bins = distance_bins
        self.value_bins = value_bins
        self.sums = sums
        self.counts = counts

    def __len__(self):
        return len(self.distance_bins) - 1

    def __add__(self, other):
        # src/StructureFunctionObjects.jl:269-279
        if self.operator != other.operator:
            raise ArgumentError(f"Cannot add results with different operators: got {self.operator} and {other.operator}")
        if not _edges_equal(self.distance_bins, other.distance_bins):
            raise ArgumentError("Cannot add results with different distance binning")
        if not _edges_equal(self.value_bins, other.value_bins):
            raise ArgumentError("Cannot add results with different value binning")
        return StructureFunction2DSumsAndCounts(self.operator, self.distance_bins, self.value_bins,
                                                self.sums + other.sums, self.counts + other.counts)


def marginalize(sf2d):
    """Sum a joint histogram over the value axis (src/StructureFunctionObjects.jl:357-366)."""
    return StructureFunctionSumsAndCounts(sf2d.operator, sf2d.distance_bins, sf2d.sums.sum(axis=1),
                                          sf2d.counts.sum(axis=1))


def bin_average(sums, counts):
    """sums / counts with count == 0 -> NaN, keeping the sums' float type (src/Calculations/serial.jl:132-141)."""
    sums = np.asarray(sums)
    counts = np.asarray(counts)
    out = np.full(sums.shape, np.nan, dtype=sums.dtype)
    nz = counts != 0
    out[nz] = sums[nz] / counts[nz]
    return out
