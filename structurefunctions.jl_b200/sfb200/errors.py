"""Exception types matching the reference's Julia errors (ArgumentError, DimensionMismatch)."""


class ArgumentError(ValueError):
    """Julia ArgumentError: invalid argument, unsupported operator/metric/shape."""


class DimensionMismatch(ValueError):
    """Julia DimensionMismatch: array shapes do not agree."""


class DeviceError(RuntimeError):
    """A CUDA or library failure reported by the GPU library (Julia ErrorException)."""
