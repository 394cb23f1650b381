"""CPU checks of the C ABI library: it loads without a GPU and exports exactly what the header declares."""
import os
import re

import pytest

from conftest import ROOT
from sfb200 import _abi, _lib


def header_functions():
    text = open(os.path.join(ROOT, "include", "sfb200.h")).read()
    return sorted(set(re.findall(r"^SFB200_API\s+[\w\s\*]+?\b(sfb200_\w+)\s*\(", text, re.M)))


def test_header_lists_every_entry_point():
    assert header_functions() == sorted(_abi.EXPORTED_SYMBOLS)


def test_library_loads_and_exports_every_symbol():
    lib = _lib.load()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert lib.sfb200_abi_version() == _abi.ABI_VERSION


def test_struct_layout_matches_header():
    import ctypes as C

    # sizes and offsets of the POD structs as gcc lays out include/sfb200.h on x86-64
    assert C.sizeof(_abi.Operator) == 16
    assert C.sizeof(_abi.Bins) == 48
    assert C.sizeof(_abi.Stats) == 48
    assert _abi.PlanDesc.ops.offset == 28
    assert _abi.PlanDesc.distance.offset == 160
    assert _abi.PlanDesc.value.offset == 216
    assert _abi.PlanDesc.precision.offset == 264
    assert C.sizeof(_abi.PlanDesc) == 280


def test_context_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(Exception):
        _lib.Context(0)
