"""Loader for libsfb200.so (the C ABI of include/sfb200.h).

The library is built in-tree next to this package (structurefunctions.jl_b200/libsfb200.so). There
is no CPU fallback: if the library or a CUDA device is missing, every entry point raises.
"""
import ctypes as C
import os
import threading

from . import _abi
from .errors import ArgumentError, DeviceError, DimensionMismatch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libsfb200.so")

_lib = None
_lock = threading.Lock()


def load():
    """Load the library once (raises OSError with the path when it is not built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libsfb200.so is not built ({LIB_PATH}); run `make -C structurefunctions.jl_b200` "
                          "or __graft_entry__.build()")
        lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        lib.sfb200_abi_version.restype = C.c_int
        lib.sfb200_ctx_create.argtypes = [C.c_int, C.POINTER(P)]
        lib.sfb200_ctx_create.restype = C.c_int
        lib.sfb200_ctx_destroy.argtypes = [P]
        lib.sfb200_ctx_destroy.restype = C.c_int
        lib.sfb200_last_error.argtypes = [P]
        lib.sfb200_last_error.restype = C.c_char_p
        lib.sfb200_ctx_stream.argtypes = [P]
        lib.sfb200_ctx_stream.restype = P
        lib.sfb200_plan_create.argtypes = [P, C.POINTER(_abi.PlanDesc), C.POINTER(P)]
        lib.sfb200_plan_create.restype = C.c_int
        lib.sfb200_plan_destroy.argtypes = [P]
        lib.sfb200_plan_destroy.restype = C.c_int
        lib.sfb200_plan_output_sizes.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.sfb200_plan_output_sizes.restype = C.c_int
        lib.sfb200_run.argtypes = [P, P, P, C.c_int64, C.c_uint32, P, P, P]
        lib.sfb200_run.restype = C.c_int
        lib.sfb200_plan_last_stats.argtypes = [P, C.POINTER(_abi.Stats)]
        lib.sfb200_plan_last_stats.restype = C.c_int
        lib.sfb200_plan_set_launch.argtypes = [P, C.c_int, C.c_int, C.c_int]
        lib.sfb200_plan_set_launch.restype = C.c_int
        lib.sfb200_plan_set_option.argtypes = [P, C.c_int, C.c_int64]
        lib.sfb200_plan_set_option.restype = C.c_int
        if lib.sfb200_abi_version() != _abi.ABI_VERSION:
            raise OSError(f"libsfb200.so ABI {lib.sfb200_abi_version()} != {_abi.ABI_VERSION}")
        _lib = lib
        return lib


def check(rc, ctx_ptr=None, what=""):
    """Map a status code to the reference's exception types."""
    if rc == _abi.OK:
        return
    msg = ""
    if ctx_ptr:
        raw = load().sfb200_last_error(ctx_ptr)
        msg = raw.decode() if raw else ""
    text = f"{what}: {msg}" if what else msg
    if rc in (_abi.ERR_INVALID_ARG, _abi.ERR_UNSUPPORTED):
        raise ArgumentError(text)
    if rc == _abi.ERR_DIMENSION:
        raise DimensionMismatch(text)
    raise DeviceError(f"sfb200 status {rc}: {text}")


class Context:
    """A CUDA device context of the library (one stream, one workspace pool)."""

    def __init__(self, device=0):
        lib = load()
        ptr = C.c_void_p()
        rc = lib.sfb200_ctx_create(int(device), C.byref(ptr))
        if rc != _abi.OK:
            raise DeviceError(f"sfb200_ctx_create(device={device}) failed with status {rc} "
                              "(no CUDA device, or the device is unusable)")
        self.ptr = ptr
        self.device = int(device)

    @property
    def stream(self):
        return load().sfb200_ctx_stream(self.ptr)

    def close(self):
        if self.ptr:
            load().sfb200_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A validated plan: geometry, operators, bin tables and precision."""

    def __init__(self, ctx, desc, keep=()):
        lib = load()
        self.ctx = ctx
        self._keep = list(keep)
        ptr = C.c_void_p()
        check(lib.sfb200_plan_create(ctx.ptr, C.byref(desc), C.byref(ptr)), ctx.ptr, "plan")
        self.ptr = ptr
        ns, nc = C.c_int64(), C.c_int64()
        check(lib.sfb200_plan_output_sizes(ptr, C.byref(ns), C.byref(nc)), ctx.ptr)
        self.n_sums, self.n_counts = ns.value, nc.value

    def run(self, x_ptr, u_ptr, n, flags, sums_ptr, counts_ptr, stream=None):
        check(load().sfb200_run(self.ptr, x_ptr, u_ptr, int(n), int(flags), sums_ptr, counts_ptr, stream),
              self.ctx.ptr, "run")

    def stats(self):
        st = _abi.Stats()
        check(load().sfb200_plan_last_stats(self.ptr, C.byref(st)), self.ctx.ptr)
        return {k: getattr(st, k) for k, _ in _abi.Stats._fields_}

    def set_launch(self, tile=0, privatization=-1, blocks_per_sm=0):
        check(load().sfb200_plan_set_launch(self.ptr, tile, privatization, blocks_per_sm), self.ctx.ptr)

    def set_option(self, option, value):
        """sfb200_plan_set_option: `option` is _abi.OPT_POINT_ORDER or _abi.OPT_HIST_COLUMNS."""
        check(load().sfb200_plan_set_option(self.ptr, int(option), int(value)), self.ctx.ptr)

    def close(self):
        if self.ptr:
            load().sfb200_plan_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
