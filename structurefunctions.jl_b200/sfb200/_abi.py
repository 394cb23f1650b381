"""ctypes mirror of include/sfb200.h (structs, enums, status codes).

Pure data definitions: no library is loaded here, so the oracle wrapper and the tests can build
plan descriptions without a GPU library present.
"""
import ctypes as C

ABI_VERSION = 1
MAX_OPS = 8

# sfb200_status
OK = 0
ERR_INVALID_ARG = -1
ERR_UNSUPPORTED = -2
ERR_OOM = -3
ERR_CUDA = -4
ERR_TIMEOUT = -5
ERR_QUEUE_FULL = -6
ERR_DIMENSION = -7

GEOM_FLAT = 0
GEOM_SPHERE = 1
ANGLE_DEG = 0
ANGLE_RAD = 1

OP_PROJECTED = 0
OP_S2 = 1
OP_S3 = 2
OP_FULLVEC = 3
OP_T2C = 4
OP_L1T2C = 5
OP_SP2D = 6  # row nl of the two-dimensional single pass (S2, L2, T2, S3, L3, L1T2)

BINS_TABLE = 0
BINS_SQTABLE = 1
BINS_LINEAR = 2

PREC_FP64 = 0
PREC_MIXED = 1
PREC_FP32 = 2
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED, "fp32": PREC_FP32}

F64 = 0
F32 = 1

RUN_DEVICE_INPUT = 0x1
RUN_DEVICE_OUTPUT = 0x2
RUN_ACCUMULATE = 0x4


class Operator(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nl", C.c_int32), ("nt", C.c_int32), ("nf", C.c_int32)]


class Bins(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("n_edges", C.c_int32),
        ("edges", C.POINTER(C.c_double)),
        ("first", C.c_double),
        ("last", C.c_double),
        ("inv_step", C.c_double),
        ("step", C.c_double),
    ]


class PlanDesc(C.Structure):
    _fields_ = [
        ("geometry", C.c_int32),
        ("dim", C.c_int32),
        ("angle_unit", C.c_int32),
        ("radius", C.c_double),
        ("n_ops", C.c_int32),
        ("ops", Operator * MAX_OPS),
        ("distance", Bins),
        ("joint", C.c_int32),
        ("value", Bins),
        ("precision", C.c_int32),
        ("x_dtype", C.c_int32),
        ("u_dtype", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("pairs", C.c_int64),
        ("rechecked", C.c_int64),
        ("kernel_ms", C.c_double),
        ("tile", C.c_int32),
        ("blocks", C.c_int32),
        ("threads", C.c_int32),
        ("kernel_launches", C.c_int32),
        ("privatization", C.c_int32),
    ]


class SliceInfo(C.Structure):
    _fields_ = [
        ("n_points", C.c_int64),
        ("pairs", C.c_int64),
        ("tile_pairs", C.c_int64),
        ("device_bytes", C.c_int64),
    ]


# Every symbol include/sfb200.h declares (checked by the CPU test suite against the built library).
EXPORTED_SYMBOLS = (
    "sfb200_abi_version",
    "sfb200_ctx_create",
    "sfb200_ctx_destroy",
    "sfb200_last_error",
    "sfb200_ctx_stream",
    "sfb200_plan_create",
    "sfb200_plan_destroy",
    "sfb200_plan_output_sizes",
    "sfb200_run",
    "sfb200_plan_last_stats",
    "sfb200_plan_set_launch",
    "sfb200_plan_set_option",
    "sfb200_shard_bounds",
    "sfb200_distance_range",
    "sfb200_slice_create",
    "sfb200_slice_get_info",
    "sfb200_batch_run",
    "sfb200_slice_read",
    "sfb200_slice_destroy",
    "sfb200_device_memory",
    "sfb200_batch_wait",
    "sfb200_batch_query",
    "sfb200_batch_wait_oldest",
    "sfb200_run_noalloc",
)

# sfb200_option
OPT_POINT_ORDER = 1
OPT_HIST_COLUMNS = 2
OPT_SHARD = 3
OPT_TILE_SORT = 4
OPT_FORMULATION = 5
