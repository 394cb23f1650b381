"""Oracle results of the full-size benchmark workloads (c1, c2, c3), cached by input hash.

TEST INFRASTRUCTURE ONLY. The FP64 oracle (oracle/sf_oracle.c, the restated SerialBackend) is run on
the exact seeded inputs of `sfb200.synthetic.config(name)` and its per-bin sums, counts and sums of
|value| are stored in tests/golden/full_oracle.npz together with a SHA-256 of the inputs. A test that
finds the same hash for its regenerated inputs uses the stored result; a different hash (the inputs
come from NumPy's transcendental and BLAS kernels, which may round differently on another CPU) makes
`oracle_for` compute the result on the spot instead, so a stale cache can never pass a test.

Regenerate with `python tests/golden/full_oracle.py [c1 c2 c3]` (c2, 2e10 sphere pairs, takes about
half an hour on 8 cores).
"""
import hashlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _p in (os.path.join(ROOT, "structurefunctions.jl_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

CACHE = os.path.join(HERE, "full_oracle.npz")
CONFIGS = ("c1", "c2", "c3")


def input_hash(w):
    h = hashlib.sha256()
    for a in (w.x, w.u):
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def _desc(w):
    from sfb200.api import plan_description

    return plan_description(w.ops, w.u.shape[0], w.distance_bins, w.value_bins, w.metric, "fp64",
                            w.x.dtype, w.u.dtype)


def _rows(args):
    """Worker (spawned process): the oracle over rows i0, i0 + step, ... of workload `name`."""
    name, i0, step = args
    import oracle_py
    from sfb200 import synthetic

    w = synthetic.config(name)
    desc, _keep = _desc(w)
    return oracle_py.run(desc, w.x, w.u, i0=i0, istep=step, with_abs=True)


def compute(name, workers=None):
    """(sums, counts, abs_sums) of the oracle on the full workload `name`, computed now with a
    process pool (spawned, so it is safe after CUDA initialisation)."""
    workers = workers or os.cpu_count() or 1
    step = 8 * workers  # interleaved rows balance the triangular loop across tasks
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        parts = pool.map(_rows, [(name, k, step) for k in range(step)], chunksize=1)
    sums = sum(p[0] for p in parts)
    counts = sum(p[1] for p in parts).astype(np.uint64)
    abss = sum(p[2] for p in parts)
    return sums, counts, abss


def load_cache():
    if not os.path.exists(CACHE):
        return {}
    z = np.load(CACHE)
    return {k: z[k] for k in z.files}


def oracle_for(name, w=None):
    """Oracle result of workload `name`: the cached one when the input hash matches, else computed.
    Returns (sums, counts, abs_sums, source) with source "cache" or "computed"."""
    from sfb200 import synthetic

    w = w if w is not None else synthetic.config(name)
    h = input_hash(w)
    z = load_cache()
    if z.get(name + "_hash") is not None and str(z[name + "_hash"]) == h:
        return z[name + "_sums"], z[name + "_counts"].astype(np.uint64), z[name + "_abs"], "cache"
    s, c, a = compute(name)
    return s, c, a, "computed"


def main(names):
    from sfb200 import synthetic

    z = load_cache()
    for name in names:
        t0 = time.time()
        w = synthetic.config(name)
        s, c, a = compute(name)
        z[name + "_hash"] = np.array(input_hash(w))
        z[name + "_sums"] = s
        z[name + "_counts"] = c
        z[name + "_abs"] = a
        print(f"{name}: {w.pairs} pairs, {int(c.sum())} in range, {time.time() - t0:.1f} s", flush=True)
        np.savez_compressed(CACHE, **z)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CONFIGS))
