"""Writes the golden fixtures under tests/golden/.

reference_kats.json
    Known-answer cases transcribed from the reference's own test files (jbphyswx/StructureFunctions.jl
    v0.4.0, cited per case). The reference is Julia and cannot run here, so these answers, which its
    authors wrote into their tests, are the pin for the oracle.
oracle_small.npz
    Oracle outputs on small seeded inputs for every geometry/operator family, frozen so that a change
    of the oracle (or of the GPU library) against the pinned version shows up as a diff. Regenerate with
    `python tests/golden/make_golden.py` after an intended change and review the diff.
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "structurefunctions.jl_b200"), os.path.join(ROOT, "oracle")]

KATS = [
    {"name": "two points L2 mean 1.0", "cite": "test/baseline_correctness.jl:6-22; test/test_core_correctness.jl:41-57",
     "op": ["PROJECTED", 2, 0], "x": [[0.0, 1.0], [0.0, 0.0]], "u": [[1.0, 2.0], [0.0, 0.0]], "bins": [0.0, 2.0],
     "mean": [1.0], "counts": [1]},
    {"name": "three points L2 mean 4/3", "cite": "test/test_core_correctness.jl:59-81",
     "op": ["PROJECTED", 2, 0], "x": [[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]], "u": [[0.0, 1.0, 0.0], [0.0, 0.0, 1.0]],
     "bins": [0.0, 2.0], "mean": [4.0 / 3.0], "sums": [4.0], "counts": [3]},
    {"name": "N=3 pair count", "cite": "test/test_core_correctness.jl:23-32",
     "op": ["S2"], "x": [[0.0, 1.0, 2.0], [0.0, 0.0, 0.0]], "u": [[0.0, 0.0, 0.0], [0.0, 0.0, 0.0]],
     "bins": [0.0, 3.0], "counts": [3]},
    {"name": "N=4 pair count", "cite": "test/test_core_correctness.jl:34-38",
     "op": ["S2"], "x": [[0.0, 1.0, 2.0, 3.0], [0.0, 0.0, 0.0, 0.0]], "u": [[0.0] * 4, [0.0] * 4],
     "bins": [0.0, 3.0], "counts": [6]},
]
for name, op, val in [("L2 of transverse du", ["PROJECTED", 2, 0], 0.0),
                      ("T2 of transverse du", ["PROJECTED", 0, 2], 1.0),
                      ("L3 of transverse du", ["PROJECTED", 3, 0], 0.0),
                      ("T3 of transverse du (n-hat = z x r-hat)", ["PROJECTED", 0, 3], 1.0),
                      ("L1T2 of transverse du", ["PROJECTED", 1, 2], 0.0)]:
    KATS.append({"name": name, "cite": "test/test_core_correctness.jl:83-140", "op": op,
                 "x": [[0.0, 1.0], [0.0, 0.0]], "u": [[0.0, 0.0], [1.0, 2.0]], "bins": [0.0, 2.0], "mean": [val],
                 "counts": [1]})

FUNCTOR_KATS = [
    # du, r_hat, operator, value   (test/test_core_correctness.jl:142-177, test/test_helpers.jl:62-117)
    {"cite": "test/test_core_correctness.jl:145-155", "du": [2.0, 3.0, 4.0], "rhat": [1.0, 0.0, 0.0],
     "values": {"L2": 4.0, "T2": 25.0, "T2C": 12.5, "L3": 8.0, "L1T2": 50.0, "L1T2C": 25.0, "S2": 29.0,
                "S3": 58.0, "FULLVEC3": 29.0 ** 1.5}},
    {"cite": "test/test_core_correctness.jl:157-165", "du": [2.0, 3.0], "rhat": [1.0, 0.0],
     "values": {"L2T1": 12.0, "T3": 27.0, "L2": 4.0, "T2": 9.0}},
]

DIGITIZE_KATS = [
    {"cite": "test/test_helpers.jl:7-26", "edges": [0.0, 1.0, 2.0, 5.0],
     "queries": [0.5, 1.5, 4.0, 0.0, 5.0, 6.0], "bins": [1, 2, 3, 0, 3, 4]},
    {"cite": "test/test_bin_edges.jl:9-30 (searchsortedfirst)", "edges": [1.0, 2.5, 5.0, 10.0],
     "queries": [0.5, 1.0, 2.0, 2.5, 8.0, 10.0, 12.0], "ssf": [1, 1, 2, 2, 4, 4, 5]},
]

NHAT_KATS = [
    {"cite": "test/test_helpers.jl:36-40", "rhat": [1.0, 0.0], "nhat": [-0.0, 1.0]},
    {"cite": "test/test_helpers.jl:43-54", "rhat": [0.0, 1.0, 0.0], "nhat": [-1.0, 0.0, 0.0]},
    {"cite": "test/test_helpers.jl:56-59", "rhat": [1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0)],
     "nhat": [-1.0 / math.sqrt(2.0), 1.0 / math.sqrt(2.0)]},
]

COUNT_GUARD = {"cite": "test/test_core_correctness.jl:225-249",
               "ok": [["uint32", 92682], ["uint64", 1000000], ["int64", 1000000]], "fail": [["uint32", 92683]]}


def oracle_small():
    import oracle_py
    import sfb200 as SF
    from sfb200 import synthetic
    from sfb200.api import plan_description

    out = {}
    cases = []
    rng = np.random.default_rng(2024)
    for D in (2, 3):
        x = rng.random((D, 300))
        u = rng.standard_normal((D, 300))
        bins = synthetic.log_edges(1e-2, math.sqrt(D), 12)
        ops = (SF.L2SF, SF.T2SF, SF.L3SF, SF.T3SF, SF.S3SF, SF.L1T2SF)
        cases.append((f"flat{D}", ops, x, u, bins, None, None))
    w = synthetic.config("c2", n=400)
    cases.append(("sphere2", (SF.L2SF, SF.T2SF, SF.L3SF), w.x, w.u, w.distance_bins, w.metric, None))
    w = synthetic.config("c3", n=400)
    cases.append(("joint2", w.ops, w.x, w.u, w.distance_bins, None, w.value_bins))
    for name, ops, x, u, bins, metric, vb in cases:
        desc, keep = plan_description(ops, u.shape[0], bins, vb, metric, "fp64", x.dtype, u.dtype)
        s, c = oracle_py.run(desc, x, u)
        out[name + "_x"] = x
        out[name + "_u"] = u
        out[name + "_sums"] = s
        out[name + "_counts"] = c
    return out


def main():
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump({"kats": KATS, "functor": FUNCTOR_KATS, "digitize": DIGITIZE_KATS, "nhat": NHAT_KATS,
                   "count_guard": COUNT_GUARD}, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **oracle_small())
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
