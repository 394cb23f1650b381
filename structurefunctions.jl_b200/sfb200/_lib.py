"""Loader for libsfb200.so (the C ABI of include/sfb200.h).

The library is built in-tree next to this package (structurefunctions.jl_b200/libsfb200.so). There
is no CPU fallback: if the library or a CUDA device is missing, every entry point raises.
"""
import ctypes as C
import os
import threading
import weakref

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
        lib.sfb200_slice_create.argtypes = [P, P, P, C.c_int64, C.c_uint32, P, C.POINTER(P)]
        lib.sfb200_slice_create.restype = C.c_int
        lib.sfb200_slice_get_info.argtypes = [P, C.POINTER(_abi.SliceInfo)]
        lib.sfb200_slice_get_info.restype = C.c_int
        lib.sfb200_batch_run.argtypes = [P, C.c_int32, C.POINTER(P), C.POINTER(C.c_int64), C.POINTER(C.c_int64), P]
        lib.sfb200_batch_run.restype = C.c_int
        lib.sfb200_slice_read.argtypes = [P, P, P, C.c_uint32, P]
        lib.sfb200_slice_read.restype = C.c_int
        lib.sfb200_slice_destroy.argtypes = [P]
        lib.sfb200_slice_destroy.restype = C.c_int
        lib.sfb200_device_memory.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.sfb200_device_memory.restype = C.c_int
        lib.sfb200_batch_wait.argtypes = [P]
        lib.sfb200_batch_wait.restype = C.c_int
        lib.sfb200_batch_query.argtypes = [P, C.POINTER(C.c_int32)]
        lib.sfb200_batch_query.restype = C.c_int
        lib.sfb200_batch_wait_oldest.argtypes = [P, C.POINTER(C.c_int64)]
        lib.sfb200_batch_wait_oldest.restype = C.c_int
        lib.sfb200_shard_bounds.argtypes = [C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int64)]
        lib.sfb200_shard_bounds.restype = C.c_int
        lib.sfb200_distance_range.argtypes = [P, P, P, C.c_int64, C.c_uint32, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double), P]
        lib.sfb200_distance_range.restype = C.c_int
        lib.sfb200_run_noalloc.argtypes = [P, P, P, C.c_int64, C.c_uint32, P, P, P]
        lib.sfb200_run_noalloc.restype = C.c_int
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
    """A CUDA device context of the library (one stream, one workspace pool).

    Plans and slices created on a context are released with it: closing the context first closes
    its slices, then its plans, so that no later finaliser reaches a destroyed context (objects in a
    reference cycle are finalised in no particular order).
    """

    def __init__(self, device=0):
        lib = load()
        ptr = C.c_void_p()
        rc = lib.sfb200_ctx_create(int(device), C.byref(ptr))
        if rc != _abi.OK:
            raise DeviceError(f"sfb200_ctx_create(device={device}) failed with status {rc} "
                              "(no CUDA device, or the device is unusable)")
        self.ptr = ptr
        self.device = int(device)
        self._children = weakref.WeakSet()

    @property
    def stream(self):
        return load().sfb200_ctx_stream(self.ptr)

    def _adopt(self, obj):
        self._children.add(obj)

    def close(self):
        if self.ptr:
            children = list(self._children)
            for obj in children:
                if isinstance(obj, Slice):
                    obj.close()
            for obj in children:
                obj.close()
            load().sfb200_ctx_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_memory(ctx):
    """(free, total) device bytes of the context's device."""
    f, t = C.c_int64(), C.c_int64()
    check(load().sfb200_device_memory(ctx.ptr, C.byref(f), C.byref(t)), ctx.ptr)
    return f.value, t.value


class Slice:
    """One point set resident on the device with its own histogram (sfb200_slice_*)."""

    def __init__(self, plan, x_ptr, u_ptr, n, flags=0, stream=None):
        self.plan = plan
        ptr = C.c_void_p()
        check(load().sfb200_slice_create(plan.ptr, x_ptr, u_ptr, int(n), int(flags), stream, C.byref(ptr)),
              plan.ctx.ptr, "slice")
        self.ptr = ptr
        plan.ctx._adopt(self)
        info = _abi.SliceInfo()
        check(load().sfb200_slice_get_info(ptr, C.byref(info)), plan.ctx.ptr)
        self.n_points, self.pairs = info.n_points, info.pairs
        self.tile_pairs, self.device_bytes = info.tile_pairs, info.device_bytes

    def read(self, sums_ptr, counts_ptr, flags=0, stream=None):
        check(load().sfb200_slice_read(self.ptr, sums_ptr, counts_ptr, int(flags), stream), self.plan.ctx.ptr, "read")

    def close(self):
        if self.ptr:
            if self.plan.ptr and self.plan.ctx.ptr:  # else released with its context
                load().sfb200_slice_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_run(ctx, slices, begins, ends, stream=None):
    """One round of sfb200_batch_run over (slice, [begin, end)) tile-pair ranges."""
    n = len(slices)
    arr = (C.c_void_p * max(n, 1))(*[s.ptr for s in slices])
    b = (C.c_int64 * max(n, 1))(*[int(v) for v in begins])
    e = (C.c_int64 * max(n, 1))(*[int(v) for v in ends])
    check(load().sfb200_batch_run(ctx.ptr, n, arr, b, e, stream), ctx.ptr, "batch")


def batch_wait(ctx):
    """Block until every queued round of the context has finished."""
    check(load().sfb200_batch_wait(ctx.ptr), ctx.ptr, "batch wait")


def batch_wait_oldest(ctx):
    """Block until the oldest unfinished round has finished; returns its number (0: none was)."""
    r = C.c_int64()
    check(load().sfb200_batch_wait_oldest(ctx.ptr, C.byref(r)), ctx.ptr, "batch wait")
    return int(r.value)


def batch_done(ctx):
    """True when every queued round of the context has finished (non-blocking)."""
    d = C.c_int32()
    check(load().sfb200_batch_query(ctx.ptr, C.byref(d)), ctx.ptr, "batch query")
    return bool(d.value)


class Plan:
    """A validated plan: geometry, operators, bin tables and precision."""

    def __init__(self, ctx, desc, keep=()):
        lib = load()
        self.ctx = ctx
        self._keep = list(keep)
        ptr = C.c_void_p()
        check(lib.sfb200_plan_create(ctx.ptr, C.byref(desc), C.byref(ptr)), ctx.ptr, "plan")
        self.ptr = ptr
        ctx._adopt(self)
        ns, nc = C.c_int64(), C.c_int64()
        check(lib.sfb200_plan_output_sizes(ptr, C.byref(ns), C.byref(nc)), ctx.ptr)
        self.n_sums, self.n_counts = ns.value, nc.value

    def run(self, x_ptr, u_ptr, n, flags, sums_ptr, counts_ptr, stream=None):
        check(load().sfb200_run(self.ptr, x_ptr, u_ptr, int(n), int(flags), sums_ptr, counts_ptr, stream),
              self.ctx.ptr, "run")

    def distance_range(self, x_ptr, u_ptr, n, flags=0, stream=None):
        """(min, max) pair distance over all pairs (sfb200_distance_range)."""
        lo, hi = C.c_double(), C.c_double()
        check(load().sfb200_distance_range(self.ptr, x_ptr, u_ptr, int(n), int(flags), C.byref(lo), C.byref(hi),
                                           stream), self.ctx.ptr, "distance range")
        return lo.value, hi.value

    def stats(self):
        st = _abi.Stats()
        check(load().sfb200_plan_last_stats(self.ptr, C.byref(st)), self.ctx.ptr)
        return {k: getattr(st, k) for k, _ in _abi.Stats._fields_}

    def set_launch(self, tile=0, privatization=-1, blocks_per_sm=0):
        check(load().sfb200_plan_set_launch(self.ptr, tile, privatization, blocks_per_sm), self.ctx.ptr)

    def set_option(self, option, value):
        """sfb200_plan_set_option: `option` is one of the _abi.OPT_* values."""
        check(load().sfb200_plan_set_option(self.ptr, int(option), int(value)), self.ctx.ptr)

    def close(self):
        if self.ptr:
            if self.ctx.ptr:  # else released with its context
                load().sfb200_plan_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
