"""Structure-function operator types, mirroring src/StructureFunctionTypes.jl of the reference.

Each operator is an immutable value object; the reference's singleton functors (L2SF, T2SF, ...)
are module-level instances here. `as_abi()` gives the C-ABI descriptor the GPU library consumes.
"""
from dataclasses import dataclass

from . import _abi


class AbstractStructureFunctionType:
    """Root of operator types (src/StructureFunctionTypes.jl:6)."""

    def __call__(self):
        # Identity call: SFType() returns the singleton (src/StructureFunctionTypes.jl:11).
        return self


class AbstractPairwiseStructureFunctionType(AbstractStructureFunctionType):
    """An operator evaluated on every point pair (src/StructureFunctionTypes.jl:7)."""

    def as_abi(self):
        raise NotImplementedError

    def order(self):
        raise NotImplementedError


class AbstractDerivedStructureFunctionType(AbstractStructureFunctionType):
    """A quantity derived from binned results, not a pair operator (src/StructureFunctionTypes.jl:8)."""


@dataclass(frozen=True)
class ProjectedStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """du_L^NL times the transverse factor of power NT (src/StructureFunctionTypes.jl:43-89).

    NT == 2 uses the invariant transverse energy |du|^2 - du_L^2; other NT use the signed
    component along n-hat = z-hat x r-hat.
    """

    NL: int
    NT: int

    def __post_init__(self):
        if int(self.NL) < 0 or int(self.NT) < 0:
            raise ValueError("ProjectedStructureFunctionType powers must be >= 0")

    def as_abi(self):
        return _abi.Operator(_abi.OP_PROJECTED, int(self.NL), int(self.NT), 0)

    def order(self):
        return self.NL + self.NT


@dataclass(frozen=True)
class SecondOrderStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """S2 = |du|^2 (src/StructureFunctionTypes.jl:97, 120)."""

    def as_abi(self):
        return _abi.Operator(_abi.OP_S2, 0, 0, 0)

    def order(self):
        return 2


@dataclass(frozen=True)
class ThirdOrderStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """S3 = du_L |du|^2 (src/StructureFunctionTypes.jl:106, 122-123)."""

    def as_abi(self):
        return _abi.Operator(_abi.OP_S3, 0, 0, 0)

    def order(self):
        return 3


@dataclass(frozen=True)
class FullVectorStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """|du|^NF (src/StructureFunctionTypes.jl:114-128)."""

    NF: int

    def as_abi(self):
        return _abi.Operator(_abi.OP_FULLVEC, 0, 0, int(self.NF))

    def order(self):
        return self.NF


@dataclass(frozen=True)
class TransverseComponentSecondOrderStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """|du_t|^2 / (D - 1) (src/StructureFunctionTypes.jl:137, 147-148)."""

    def as_abi(self):
        return _abi.Operator(_abi.OP_T2C, 0, 0, 0)

    def order(self):
        return 2


@dataclass(frozen=True)
class LongitudinalTransverseComponentThirdOrderStructureFunctionType(AbstractPairwiseStructureFunctionType):
    """du_L |du_t|^2 / (D - 1) (src/StructureFunctionTypes.jl:145, 150-151)."""

    def as_abi(self):
        return _abi.Operator(_abi.OP_L1T2C, 0, 0, 0)

    def order(self):
        return 3


@dataclass(frozen=True)
class RotationalSecondOrderStructureFunctionType(AbstractDerivedStructureFunctionType):
    """Helmholtz-derived; not a pair operator (src/StructureFunctionTypes.jl:253)."""


@dataclass(frozen=True)
class DivergentSecondOrderStructureFunctionType(AbstractDerivedStructureFunctionType):
    """Helmholtz-derived; not a pair operator (src/StructureFunctionTypes.jl:262)."""


@dataclass(frozen=True)
class HelmholtzDecomposition2DType(AbstractDerivedStructureFunctionType):
    """Helmholtz decomposition; not a pair operator (src/StructureFunctionTypes.jl:270)."""


# Type aliases (src/StructureFunctionTypes.jl:157-180)
def LongitudinalSecondOrderStructureFunctionType():
    return ProjectedStructureFunctionType(2, 0)


def TransverseSecondOrderStructureFunctionType():
    return ProjectedStructureFunctionType(0, 2)


def DiagonalConsistentThirdOrderStructureFunctionType():
    return ProjectedStructureFunctionType(3, 0)


def DiagonalInconsistentThirdOrderStructureFunctionType():
    return ProjectedStructureFunctionType(2, 1)


def OffDiagonalInconsistentThirdOrderStructureFunctionType():
    return ProjectedStructureFunctionType(1, 2)


def OffDiagonalConsistentThirdOrderStructureFunctionType():
    return ProjectedStructureFunctionType(0, 3)


# Singleton functors (src/StructureFunctionTypes.jl:186-212)
SecondOrderStructureFunction = SecondOrderStructureFunctionType()
LongitudinalSecondOrderStructureFunction = ProjectedStructureFunctionType(2, 0)
TransverseSecondOrderStructureFunction = ProjectedStructureFunctionType(0, 2)
T2ComponentSF = TransverseComponentSecondOrderStructureFunctionType()
ThirdOrderStructureFunction = ThirdOrderStructureFunctionType()
DiagonalConsistentThirdOrderStructureFunction = ProjectedStructureFunctionType(3, 0)
DiagonalInconsistentThirdOrderStructureFunction = ProjectedStructureFunctionType(2, 1)
OffDiagonalInconsistentThirdOrderStructureFunction = ProjectedStructureFunctionType(1, 2)
OffDiagonalConsistentThirdOrderStructureFunction = ProjectedStructureFunctionType(0, 3)
L1T2ComponentSF = LongitudinalTransverseComponentThirdOrderStructureFunctionType()
RotationalSecondOrderStructureFunction = RotationalSecondOrderStructureFunctionType()
DivergentSecondOrderStructureFunction = DivergentSecondOrderStructureFunctionType()
HelmholtzDecomposition2DOperator = HelmholtzDecomposition2DType()

S2SF = SecondOrderStructureFunction
L2SF = LongitudinalSecondOrderStructureFunction
T2SF = TransverseSecondOrderStructureFunction
S3SF = ThirdOrderStructureFunction
L3SF = DiagonalConsistentThirdOrderStructureFunction
T3SF = OffDiagonalConsistentThirdOrderStructureFunction
L2T1SF = DiagonalInconsistentThirdOrderStructureFunction
L1T2SF = OffDiagonalInconsistentThirdOrderStructureFunction

SF_TYPE_MAP = {
    "SecondOrderStructureFunction": SecondOrderStructureFunction,
    "LongitudinalSecondOrderStructureFunction": LongitudinalSecondOrderStructureFunction,
    "TransverseSecondOrderStructureFunction": TransverseSecondOrderStructureFunction,
    "T2ComponentSF": T2ComponentSF,
    "RotationalSecondOrderStructureFunction": RotationalSecondOrderStructureFunction,
    "DivergentSecondOrderStructureFunction": DivergentSecondOrderStructureFunction,
    "HelmholtzDecomposition2D": HelmholtzDecomposition2DOperator,
    "ThirdOrderStructureFunction": ThirdOrderStructureFunction,
    "DiagonalConsistentThirdOrderStructureFunction": DiagonalConsistentThirdOrderStructureFunction,
    "DiagonalInconsistentThirdOrderStructureFunction": DiagonalInconsistentThirdOrderStructureFunction,
    "OffDiagonalInconsistentThirdOrderStructureFunction": OffDiagonalInconsistentThirdOrderStructureFunction,
    "OffDiagonalConsistentThirdOrderStructureFunction": OffDiagonalConsistentThirdOrderStructureFunction,
    "L2SF": L2SF,
    "T2SF": T2SF,
    "RotationalSF": RotationalSecondOrderStructureFunction,
    "DivergentSF": DivergentSecondOrderStructureFunction,
    "L3SF": L3SF,
    "S2SF": S2SF,
    "S3SF": S3SF,
    "T3SF": T3SF,
    "L2T1SF": L2T1SF,
    "L1T2SF": L1T2SF,
    "L1T2ComponentSF": L1T2ComponentSF,
}


def get_structure_function_type(x, mode=None):
    """Name or (order, mode) lookup (src/StructureFunctionTypes.jl:348-402)."""
    if mode is None:
        key = str(x)
        if key in SF_TYPE_MAP:
            return SF_TYPE_MAP[key]
        raise KeyError(f"Unknown structure function type symbol: {key}")
    order, mode = int(x), str(mode)
    if order == 2:
        if mode in ("longitudinal", "long", "L"):
            return LongitudinalSecondOrderStructureFunction
        if mode in ("transverse", "trans", "T"):
            return TransverseSecondOrderStructureFunction
        if mode in ("transverse_component", "trans_component", "Tcomponent"):
            return T2ComponentSF
        if mode in ("scalar", "total", "S", "full"):
            return SecondOrderStructureFunction
        if mode in ("rotational", "rot"):
            return RotationalSecondOrderStructureFunction
        if mode in ("divergent", "div"):
            return DivergentSecondOrderStructureFunction
    elif order == 3:
        if mode in ("longitudinal", "long", "L", "diagonal_consistent"):
            return DiagonalConsistentThirdOrderStructureFunction
        if mode in ("transverse", "trans", "T", "off_diagonal_consistent"):
            return OffDiagonalConsistentThirdOrderStructureFunction
        if mode in ("scalar", "total", "S", "full"):
            return ThirdOrderStructureFunction
        if mode == "diagonal_inconsistent":
            return DiagonalInconsistentThirdOrderStructureFunction
        if mode == "off_diagonal_inconsistent":
            return OffDiagonalInconsistentThirdOrderStructureFunction
        if mode in ("off_diagonal_inconsistent_component", "L1T2_component"):
            return L1T2ComponentSF
    raise KeyError(f"No mapping for order {order} and mode {mode}")


def order(sf):
    """Order of an operator (src/StructureFunctionTypes.jl:416-424)."""
    if isinstance(sf, (RotationalSecondOrderStructureFunctionType, DivergentSecondOrderStructureFunctionType,
                       HelmholtzDecomposition2DType)):
        return 2
    return sf.order()
