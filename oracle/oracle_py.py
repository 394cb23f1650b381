"""ctypes wrapper of the CPU oracle (liboracle_sf.so). TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product.
`run(desc, x, u)` returns (sums, counts) with the same layout as sfb200_run. Inputs are widened to
float64 before the call (the oracle's "FP64 on widened inputs" semantics).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_sf.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        P = C.c_void_p
        lib.oracle_run.argtypes = [P, P, P, C.c_int64, C.c_int64, C.c_int64, P, P, P]
        lib.oracle_run.restype = C.c_int
        lib.oracle_run_threaded.argtypes = [P, P, P, C.c_int64, C.c_int, P, P]
        lib.oracle_run_threaded.restype = C.c_int
        lib.oracle_searchsortedfirst_vec.argtypes = [P, C.c_int64, C.c_double]
        lib.oracle_searchsortedfirst_vec.restype = C.c_int64
        lib.oracle_searchsortedfirst_linear.argtypes = [C.c_double] * 4 + [C.c_int64, C.c_double]
        lib.oracle_searchsortedfirst_linear.restype = C.c_int64
        lib.oracle_digitize.argtypes = [P, C.c_double]
        lib.oracle_digitize.restype = C.c_int64
        lib.oracle_sf_functor.argtypes = [P, C.c_int, P, P]
        lib.oracle_sf_functor.restype = C.c_double
        lib.oracle_sf_raw.argtypes = [P, C.c_int, P, P, C.c_double]
        lib.oracle_sf_raw.restype = C.c_double
        lib.oracle_sphere_point.argtypes = [C.c_double, C.c_double, C.c_int, P]
        lib.oracle_sphere_frame.argtypes = [P, P, C.c_double, P, P, P]
        lib.oracle_sphere_frame.restype = C.c_int
        lib.oracle_sincosd.argtypes = [C.c_double, P, P]
        lib.oracle_sincos.argtypes = [C.c_double, P, P]
        lib.oracle_atan2.argtypes = [C.c_double, C.c_double]
        lib.oracle_atan2.restype = C.c_double
        lib.oracle_threads_available.restype = C.c_int
        lib.oracle_run_single_pass.argtypes = [P, P, P, C.c_int64, C.c_int64, C.c_int64, P, P, P]
        lib.oracle_run_single_pass.restype = C.c_int
        lib.oracle_single_pass_derive.argtypes = [P, P, C.c_int64]
        _lib = lib
    return _lib


def _colmajor64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def out_sizes(desc):
    nd = desc.distance.n_edges - 1
    if desc.joint:  # several operators: consecutive single-pass 2D rows, one (nd, nv) matrix each
        nv = desc.value.n_edges - 1
        return nd * nv * desc.n_ops, nd * nv * desc.n_ops
    return nd * desc.n_ops, nd


def run(desc, x, u, threads=0, i0=0, istep=1, with_abs=False):
    """Oracle sums/counts for plan description `desc` (an sfb200 _abi.PlanDesc); with `with_abs`
    also the per-bin sum of |value| (serial only)."""
    lib = load()
    xa, ua = _colmajor64(x), _colmajor64(u)
    n = xa.shape[1]
    ns, nc = out_sizes(desc)
    sums = np.zeros(ns, dtype=np.float64)
    counts = np.zeros(nc, dtype=np.uint64)
    abss = np.zeros(ns, dtype=np.float64)
    if threads and threads > 1 and not with_abs:
        rc = lib.oracle_run_threaded(C.addressof(desc), xa.ctypes.data, ua.ctypes.data, n, int(threads),
                                     sums.ctypes.data, counts.ctypes.data)
    else:
        rc = lib.oracle_run(C.addressof(desc), xa.ctypes.data, ua.ctypes.data, n, int(i0), int(istep),
                            sums.ctypes.data, counts.ctypes.data, abss.ctypes.data if with_abs else None)
    if rc != 0:
        raise RuntimeError("oracle failed")
    if with_abs:
        return sums, counts, abss
    return sums, counts


def run_single_pass(desc, x, u, i0=0, istep=1, derive=True):
    """Six-invariant single pass (rows S2, L2, T2, S3, L3, L1T2) as (sums, counts, abs_sums), each
    (6, nb) column-major like the reference's accumulator. `abs_sums` holds the per-bin sums of
    |value| of the accumulated rows and, for the derived rows, |S2| + |L2| and |S3| + |L3| sums (the
    scale of a difference). With derive=False (partial rows of a split run) the derived rows are left
    for the caller to fill once the partial results are added."""
    lib = load()
    xa, ua = _colmajor64(x), _colmajor64(u)
    n = xa.shape[1]
    nb = desc.distance.n_edges - 1
    sums = np.zeros((6, nb), order="F")
    counts = np.zeros((6, nb), dtype=np.uint64, order="F")
    abss = np.zeros((6, nb), order="F")
    rc = lib.oracle_run_single_pass(C.addressof(desc), xa.ctypes.data, ua.ctypes.data, n, int(i0), int(istep),
                                    sums.ctypes.data, counts.ctypes.data, abss.ctypes.data)
    if rc != 0:
        raise RuntimeError("oracle failed")
    if derive:
        single_pass_derive(sums, counts, abss)
    return sums, counts, abss


def single_pass_derive(sums, counts, abss=None):
    """Fill the derived rows (T2 = S2 - L2, L1T2 = S3 - L3, counts of row S2 everywhere) in place."""
    nb = sums.shape[1]
    load().oracle_single_pass_derive(sums.ctypes.data, counts.ctypes.data, nb)
    if abss is not None:
        abss[2] = abss[0] + abss[1]
        abss[5] = abss[3] + abss[4]


def threads_available():
    return load().oracle_threads_available()


def sincosd(x):
    s, c = C.c_double(), C.c_double()
    load().oracle_sincosd(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


def sincos(x):
    s, c = C.c_double(), C.c_double()
    load().oracle_sincos(float(x), C.byref(s), C.byref(c))
    return s.value, c.value


def atan2(y, x):
    return load().oracle_atan2(float(y), float(x))


def sphere_point(lon, lat, unit=0):
    out = np.zeros(9)
    load().oracle_sphere_point(float(lon), float(lat), int(unit), out.ctypes.data)
    return out


def sphere_frame(A, B, radius):
    """(ok, r, tA, tB) for two 9-vectors from sphere_point."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    r = C.c_double()
    tA = np.zeros(2)
    tB = np.zeros(2)
    ok = load().oracle_sphere_frame(A.ctypes.data, B.ctypes.data, float(radius), C.byref(r), tA.ctypes.data,
                                    tB.ctypes.data)
    return bool(ok), r.value, tA, tB


def sf_functor(op_abi, du, rhat):
    du = np.ascontiguousarray(du, dtype=np.float64)
    rhat = np.ascontiguousarray(rhat, dtype=np.float64)
    return load().oracle_sf_functor(C.addressof(op_abi), len(du), du.ctypes.data, rhat.ctypes.data)


def digitize(bins_abi, x):
    return load().oracle_digitize(C.addressof(bins_abi), float(x))


def searchsortedfirst(v, x):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return load().oracle_searchsortedfirst_vec(v.ctypes.data, len(v), float(x))
