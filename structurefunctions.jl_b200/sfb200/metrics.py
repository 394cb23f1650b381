"""Distance metrics and the geometry each implies (src/HelperFunctions.jl:390-417).

Mirrors the three Distances.jl metrics the reference gives a pair geometry: Euclidean (flat),
Haversine(radius) (sphere, degrees) and SphericalAngle (unit sphere, radians). Any other metric
raises ArgumentError, as pair_geometry_for does.
"""
from dataclasses import dataclass

from . import _abi
from .errors import ArgumentError


class PreMetric:
    """Any distance function (Distances.PreMetric)."""


@dataclass(frozen=True)
class Euclidean(PreMetric):
    pass


@dataclass(frozen=True)
class Haversine(PreMetric):
    """Great-circle distance on a sphere of `radius`; coordinates (lon, lat) in degrees."""

    radius: float = 6371000.0


@dataclass(frozen=True)
class SphericalAngle(PreMetric):
    """Central angle on the unit sphere; coordinates (lon, lat) in radians."""


@dataclass(frozen=True)
class Geometry:
    kind: int          # _abi.GEOM_*
    dim: int           # velocity components D
    angle_unit: int = _abi.ANGLE_DEG
    radius: float = 1.0

    def coordinate_width(self):
        """Coordinates per point (src/HelperFunctions.jl:235-236)."""
        return self.dim if self.kind == _abi.GEOM_FLAT else 2


def pair_geometry_for(metric, D):
    """Geometry implied by `metric` for velocity dimension D (src/HelperFunctions.jl:390-417)."""
    if isinstance(metric, Euclidean):
        return Geometry(_abi.GEOM_FLAT, D)
    if isinstance(metric, Haversine):
        return Geometry(_abi.GEOM_SPHERE, D, _abi.ANGLE_DEG, float(metric.radius))
    if isinstance(metric, SphericalAngle):
        return Geometry(_abi.GEOM_SPHERE, D, _abi.ANGLE_RAD, 1.0)
    raise ArgumentError(
        f"no pair geometry is defined for distance_metric={type(metric).__name__}. A distance function "
        "fixes which histogram bin a pair falls in, but it does not define the separation direction or "
        "how to compare velocities at two different points, so this package will not guess one. Define "
        "`pair_geometry_for` for it, plus a pair geometry."
    )
