"""Launch autotuner: per plan shape, time the launch candidates once and keep the fastest.

A plan's launch has three knobs (sfb200_plan_set_launch / sfb200_plan_set_option): the tile (points
per tile = threads per block), the histogram privatisation mode, and the point order. Which
combination is fastest depends on the dimension, the number of bins and operators, the geometry and
the point count (tile-pair count against SM count; table footprint against shared memory; how often
a lane's bin changes). The tuner runs the plan on the caller's own inputs under each candidate,
reads the pair kernel's CUDA-event time, applies the fastest and remembers it per shape key:

    key = (geometry, D, operators, distance bins, value bins, precision, dtypes, log2(N) class)

so later plans of the same shape start from the tuned launch without timing anything. The cache can
be saved to and loaded from a JSON file.
"""
import json
import math
import threading

from . import _abi

# (tile, privatisation, point order); privatisation -1 = the library's default; order -1 = automatic
CANDIDATES_1D = tuple((t, p, o) for t in (128, 256) for p in (6, 3, 2, 0) for o in (-1, 0))
CANDIDATES_JOINT = tuple((t, -1, o) for t in (256, 512, 768) for o in (-1, 0))

_cache = {}
_lock = threading.Lock()


def shape_key(desc, n):
    """Cache key of a plan description (an _abi.PlanDesc) and a point count."""
    ops = tuple((desc.ops[k].kind, desc.ops[k].nl, desc.ops[k].nt, desc.ops[k].nf) for k in range(desc.n_ops))

    def bins(b):
        return (b.kind, b.n_edges)

    return (desc.geometry, desc.dim, ops, bins(desc.distance), bins(desc.value) if desc.joint else None,
            desc.precision, desc.x_dtype, desc.u_dtype, int(math.log2(max(n, 2))))


def lookup(key):
    with _lock:
        return _cache.get(key)


def apply(plan, choice):
    tile, priv, order = choice
    plan.set_launch(tile, priv, 0)
    plan.set_option(_abi.OPT_POINT_ORDER, order)


def tune(plan, desc, run, n, repeats=2, candidates=None):
    """Time `candidates` on `plan` and apply the fastest.

    `run()` runs the plan once on the caller's inputs (any flags); the time of a candidate is the
    smallest pair-kernel time (plan.stats()["kernel_ms"]) over `repeats` runs after one warm-up run.
    Returns {"choice": (tile, priv, order), "ms": ..., "timings": {candidate: ms}}; the choice is
    cached under shape_key(desc, n). Candidates the library refuses for this plan are skipped.
    """
    if candidates is None:
        candidates = CANDIDATES_JOINT if desc.joint else CANDIDATES_1D
    timings = {}
    for cand in candidates:
        try:
            apply(plan, cand)
            run()
            best = float("inf")
            for _ in range(max(1, repeats)):
                run()
                best = min(best, float(plan.stats()["kernel_ms"]))
            timings[cand] = best
        except Exception:  # a combination this plan cannot launch (shared memory, counters)
            continue
    if not timings:
        apply(plan, (0, -1, -1))
        return {"choice": (0, -1, -1), "ms": None, "timings": {}}
    choice = min(timings, key=timings.get)
    apply(plan, choice)
    with _lock:
        _cache[shape_key(desc, n)] = choice
    return {"choice": choice, "ms": timings[choice], "timings": timings}


def save(path):
    with _lock:
        items = [{"key": repr(k), "choice": list(v)} for k, v in _cache.items()]
    with open(path, "w") as f:
        json.dump(items, f)


def load(path):
    import ast

    with open(path) as f:
        items = json.load(f)
    with _lock:
        for it in items:
            _cache[ast.literal_eval(it["key"])] = tuple(it["choice"])


def clear():
    with _lock:
        _cache.clear()
