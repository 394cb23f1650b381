"""Batched serving on the GPU: every request's result is the same alone and in the mix.

A mix of requests (2D / 3D planar, spherical, 1D and joint histograms, several sizes) goes through
the continuous-batching loop at once; each result is compared with the same request run alone
(sfb200_run through its plan) and with the CPU oracle: counts identical, sums within the mixed
tolerance of the oracle's per-bin sum |v|.
"""
import math

import numpy as np
import pytest

import oracle_py
import sfb200 as SF
from helpers import TOL_MIXED, compare
from sfb200 import _lib, synthetic
from sfb200.api import plan_description
from sfb200.serving import GpuExecutor, Request, Server

pytestmark = pytest.mark.gpu


def make_requests(seed=21, count=18):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(count):
        n = int(rng.integers(300, 3500))
        kind = k % 3
        joint = k % 2 == 1
        ops = (SF.L2SF,) if rng.random() < 0.5 else (SF.L3SF,)
        nb = int(rng.integers(24, 40))
        if kind == 0:
            x = rng.random((2, n))
            u = synthetic.planar_field(x, 32, 64.0, rng, 0.01)
            edges, metric = synthetic.log_edges(1e-3, math.sqrt(2.0), nb), None
        elif kind == 1:
            x = rng.random((3, n))
            u = synthetic.solenoidal_field(x, 64, 128.0, rng)
            edges, metric = synthetic.log_edges(1e-4, math.sqrt(3.0), nb), None
        else:
            x = synthetic.sphere_points(n, rng).astype(np.float32)
            u = synthetic.sphere_field(x.astype(np.float64), 48, 200, rng).astype(np.float32)
            edges, metric = synthetic.log_edges(1.0, 20000.0, nb), SF.Haversine(6371.0)
        vb = None
        if joint:
            ops = (SF.ProjectedStructureFunctionType(1, 0),)
            sigma = math.sqrt(2.0) * float(np.std(u.astype(np.float64)))
            vb = SF.LinearBinEdges(-5.0 * sigma, 5.0 * sigma, 65)
        reqs.append(Request(ops, x, u, edges, vb, metric, tag=k))
    return reqs


def oracle_of(r):
    desc, keep = plan_description(r.ops, r.u.shape[0], r.distance_bins, r.value_bins, r.metric, "fp64",
                                  r.x.dtype, r.u.dtype)
    return oracle_py.run(desc, r.x, r.u, with_abs=True)


@pytest.mark.parametrize("depth", [1, 2])
def test_results_same_alone_and_in_the_mix(depth):
    reqs = make_requests()
    ex = GpuExecutor(0)
    try:
        # small rounds: many interleavings; depth 2 queues the next round while one runs
        srv = Server(ex, max_slots=12, round_pairs=2e6, depth=depth).start()
        tickets = [srv.submit(r) for r in reqs]
        srv.stop()
        assert srv.rounds > 1
        for r, t in zip(reqs, tickets):
            mix_s, mix_c = t.wait(60)
            # alone: the same plan through sfb200_run
            desc, keep = plan_description(r.ops, r.u.shape[0], r.distance_bins, r.value_bins, r.metric, "mixed",
                                          r.x.dtype, r.u.dtype)
            plan = _lib.Plan(ex.ctx, desc, keep)
            s = np.zeros(plan.n_sums)
            c = np.zeros(plan.n_counts, dtype=np.uint64)
            xa, ua = np.asfortranarray(r.x), np.asfortranarray(r.u)
            plan.run(xa.ctypes.data, ua.ctypes.data, r.n, 0, s.ctypes.data, c.ctypes.data)
            plan.close()
            assert np.array_equal(mix_c, c), f"request {r.tag}: counts differ between the mix and alone"
            rs, rc, ra = oracle_of(r)
            if r.value_bins is None:
                compare(mix_s, mix_c, rs, rc, ra, TOL_MIXED)
                compare(s, c, rs, rc, ra, TOL_MIXED)
            else:
                compare(mix_s, mix_c, rs, rc, ra, TOL_MIXED)
                compare(s, c, rs, rc, ra, TOL_MIXED)
            # alone vs mix: only the summation order differs
            scale = np.maximum(ra, 1e-300)
            assert float(np.max(np.abs(mix_s - s) / scale)) <= 2 * TOL_MIXED
    finally:
        ex.close()


def test_round_graph_replay_and_ranges_split_across_rounds():
    """One request split into many rounds gives the single-launch result (tile-pair coverage)."""
    r = make_requests(seed=5, count=1)[0]
    ex = GpuExecutor(0)
    try:
        srv = Server(ex, max_slots=4, round_pairs=1.0, min_units=1)  # one tile pair per round
        t = srv.submit(r)
        srv.run_until_idle()
        s, c = t.wait(60)
        assert t.rounds == srv.rounds and t.rounds > 3
        rs, rc, ra = oracle_of(r)
        compare(s, c, rs, rc, ra, TOL_MIXED)
    finally:
        ex.close()


def test_queued_rounds_on_one_slice_complete_in_order():
    """Three rounds over one slice queued back to back: queuing the third waits for the first (two
    buffers), the other two finish oldest first, the slice's result covers every tile pair once, and
    the slice memory is released without a host wait and counted free again."""
    import torch

    r = make_requests(seed=9, count=1)[0]
    ex = GpuExecutor(0)
    try:
        h = ex.create(r)
        units = h.tile_pairs
        assert units >= 3
        cuts = [0, units // 3, 2 * units // 3, units]
        for b, e in zip(cuts, cuts[1:]):
            _lib.batch_run(ex.ctx, [h.slice], [b], [e])
        assert _lib.batch_wait_oldest(ex.ctx) == 2  # rounds are numbered from 1 per context
        assert _lib.batch_wait_oldest(ex.ctx) == 3
        assert _lib.batch_wait_oldest(ex.ctx) == 0 and _lib.batch_done(ex.ctx)
        s, c = ex.read(h)
        rs, rc, ra = oracle_of(r)
        compare(s, c, rs, rc, ra, TOL_MIXED)
        free_before = ex.free_bytes()
        ex.destroy(h)
        torch.cuda.synchronize()
        assert ex.free_bytes() >= free_before + h.device_bytes - (2 << 20)
    finally:
        ex.close()


def test_arrivals_during_rounds_same_alone_and_in_the_mix():
    """Continuous batching proper: a large request is submitted first and, while its rounds are on the
    device (small rounds, two in flight), a feeder thread submits the others one by one; they are
    admitted and join rounds that still hold the first. Each result equals the request run alone
    (counts identical, sums within the mixed tolerance)."""
    import threading
    import time

    rng = np.random.default_rng(34)
    big_x = rng.random((2, 40000))
    big = Request((SF.L2SF,), big_x, synthetic.planar_field(big_x, 32, 64.0, rng, 0.01),
                  synthetic.log_edges(1e-3, math.sqrt(2.0), 32), tag="big")
    reqs = [big] + make_requests(seed=33, count=20)
    ex = GpuExecutor(0)
    try:
        srv = Server(ex, max_slots=32, round_pairs=3e6, depth=2).start()
        tickets = [srv.submit(big)]

        def feeder():
            for r in reqs[1:]:
                tickets.append(srv.submit(r))
                time.sleep(0.0005)

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        srv.stop()
        # the first request (8e8 pairs in rounds of 3e6) was still running when later ones were admitted,
        # and rounds held several slices at once
        first = tickets[0]
        assert first.rounds > 20
        assert sum(t.t_admit < first.t_done for t in tickets[1:]) >= 1
        assert max(n for n, _ in srv.round_log) > 1
        for r, t in zip(reqs, tickets):
            mix_s, mix_c = t.wait(120)
            desc, keep = plan_description(r.ops, r.u.shape[0], r.distance_bins, r.value_bins, r.metric, "mixed",
                                          r.x.dtype, r.u.dtype)
            plan = _lib.Plan(ex.ctx, desc, keep)
            s = np.zeros(plan.n_sums)
            c = np.zeros(plan.n_counts, dtype=np.uint64)
            xa, ua = np.asfortranarray(r.x), np.asfortranarray(r.u)
            plan.run(xa.ctypes.data, ua.ctypes.data, r.n, 0, s.ctypes.data, c.ctypes.data)
            plan.close()
            assert np.array_equal(mix_c, c), f"request {r.tag}: counts differ between the mix and alone"
            if r.tag != "big":  # the oracle of the small ones (the big one: alone = mix suffices)
                rs, rc, ra = oracle_of(r)
                compare(mix_s, mix_c, rs, rc, ra, TOL_MIXED)
                scale = np.maximum(ra, 1e-300)
            else:
                scale = np.maximum(np.abs(s), 1e-300)
            assert float(np.max(np.abs(mix_s - s) / scale)) <= 2 * TOL_MIXED
    finally:
        ex.close()
