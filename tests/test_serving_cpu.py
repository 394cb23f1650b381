"""The continuous-batching loop (sfb200.serving.Server) driven by a simulated executor, on the CPU.

The executor mirrors the library's slice / round contract: a request becomes `tile_pairs` units of
work (256-point tiles), a round runs tile-pair ranges of several slices, and a slice's result is
readable once every unit ran. The simulation records every range, so the tests can check the
invariants the GPU path relies on: each tile pair of each request runs exactly once, in order;
admission honours the slot count and the memory reserve; every admitted slice progresses in every
round; short requests are not held behind long ones, in the rounds and at admission (the smallest
waiting request is admitted first, the oldest once it has waited max_wait); a bad request fails alone; with pipelined
rounds, no more than `depth` rounds are queued at once, rounds complete oldest first, and a slice is
read only after every round that touched it has completed. Each invariant holds with slices prepared
on the loop thread and on a preparation thread (prepare_threads 0 and 1).
"""
import collections
import threading

import numpy as np
import pytest

from sfb200.serving import Request, Server

T = 256


class FakeHandle:
    def __init__(self, req, nbytes):
        nt = (req.n + T - 1) // T
        self.tile_pairs = nt * (nt + 1) // 2 if req.n >= 2 else 0
        self.pairs = req.n * (req.n - 1) // 2
        self.device_bytes = nbytes
        self.req = req
        self.ranges = []


class FakeExecutor:
    def __init__(self, memory=10_000_000, bytes_per_point=100, fail_n=None):
        self.memory = memory
        self.used = 0
        self.bpp = bytes_per_point
        self.fail_n = fail_n
        self.rounds = []
        self.inflight = collections.deque()
        self.max_inflight = 0
        self.live = 0
        self.max_live = 0
        self.admissions = []  # (slices live before, free bytes after)
        self.lock = threading.Lock()  # create runs on the preparation thread, destroy on the loop

    def estimate_bytes(self, req):
        return req.n * self.bpp

    def free_bytes(self):
        return self.memory - self.used

    def create(self, req):
        if self.fail_n is not None and req.n == self.fail_n:
            raise ValueError("rejected")
        h = FakeHandle(req, self.estimate_bytes(req))
        with self.lock:
            before = self.live
            self.used += h.device_bytes
            self.live += 1
            self.max_live = max(self.max_live, self.live)
            self.admissions.append((before, self.free_bytes()))
        return h

    def run_round(self, work):
        self.rounds.append([(h, b, e) for h, b, e in work])
        self.inflight.append(self.rounds[-1])
        self.max_inflight = max(self.max_inflight, len(self.inflight))
        for h, b, e in work:
            h.ranges.append((b, e))

    def wait_round(self):
        self.inflight.clear()

    def wait_oldest(self):
        self.inflight.popleft()

    def read(self, h):
        assert all(h is not g for r in self.inflight for g, _, _ in r), "read while a round is queued"
        # the "histogram": how many times each tile pair ran (must be all ones)
        cover = np.zeros(h.tile_pairs, dtype=np.int64)
        for b, e in h.ranges:
            cover[b:e] += 1
        return cover.astype(np.float64), np.array([h.req.n], dtype=np.uint64)

    def destroy(self, h):
        with self.lock:
            self.used -= h.device_bytes
            self.live -= 1


def req(n, tag=None):
    x = np.zeros((2, n))
    return Request((), x, x, [0.0, 1.0], tag=tag)


@pytest.mark.parametrize("prep", [0, 1])
def test_every_tile_pair_runs_exactly_once_in_order(prep):
    ex = FakeExecutor()
    srv = Server(ex, max_slots=4, round_pairs=5e5, memory_reserve=0, prepare_threads=prep)
    sizes = [1, 2, 300, 1000, 5000, 20000, 700, 2, 256, 257]
    tickets = [srv.submit(req(n)) for n in sizes]
    srv.run_until_idle()
    for t, n in zip(tickets, sizes):
        sums, counts = t.wait(0)
        assert int(counts[0]) == n
        assert np.all(sums == 1.0)  # every unit exactly once
    handles = {}
    for r in ex.rounds:
        for h, b, e in r:
            assert 0 <= b < e <= h.tile_pairs
            handles[id(h)] = h
    for h in handles.values():  # a slice's ranges are contiguous and increasing
        ends = [0] + [e for _, e in h.ranges]
        assert [b for b, _ in h.ranges] == ends[:-1]
    assert ex.live == 0 and ex.used == 0


@pytest.mark.parametrize("prep", [0, 1])
def test_slots_bound_concurrency(prep):
    ex = FakeExecutor()
    srv = Server(ex, max_slots=3, round_pairs=1e5, memory_reserve=0, prepare_threads=prep)
    for n in [3000] * 10:
        srv.submit(req(n))
    srv.run_until_idle()
    assert ex.max_live <= 3
    assert max(len(r) for r in ex.rounds) <= 3


@pytest.mark.parametrize("prep", [0, 1])
def test_memory_reserve_bounds_admission(prep):
    ex = FakeExecutor(memory=2_000_000, bytes_per_point=100)
    srv = Server(ex, max_slots=64, round_pairs=1e5, memory_reserve=500_000,
                 prepare_threads=prep)
    ts = [srv.submit(req(5000)) for _ in range(8)]  # 500 kB each
    srv.run_until_idle()
    assert all(t.done() for t in ts)
    # an admission next to live slices never pushed free memory below the reserve (an idle device
    # admits the head request regardless, so that a request larger than the reserve still runs)
    assert all(free >= 500_000 for before, free in ex.admissions if before > 0)
    assert ex.max_live == 3


@pytest.mark.parametrize("prep", [0, 1])
def test_every_active_slice_progresses_each_round(prep):
    ex = FakeExecutor()
    srv = Server(ex, max_slots=8, round_pairs=1.0, min_units=2, memory_reserve=0,  # budget ~ nothing extra
                 prepare_threads=prep)
    for n in [4000, 6000, 8000]:
        srv.submit(req(n))
    srv.run_until_idle()
    # from the round a slice first joins until it is done, every round advances it by the minimum
    # share (2 units, or what is left): no active slice is skipped
    seen = {}
    for k, rnd in enumerate(ex.rounds):
        for h, b, e in rnd:
            seen.setdefault(id(h), (h, k))
            assert e - b == min(2, h.tile_pairs - b)
    for h, k0 in seen.values():
        k_last = max(k for k, rnd in enumerate(ex.rounds) if any(g is h for g, _, _ in rnd))
        for k in range(k0, k_last + 1):
            assert any(g is h for g, _, _ in ex.rounds[k]), "an active slice sat out a round"
    if prep == 0:
        assert len(ex.rounds[0]) == 3


def test_short_request_overtakes_long_one():
    # the scheduling policy alone: slices prepared on the loop thread (with a preparation thread the
    # simulated rounds, which take no time, could finish the long request before the short one is ready)
    ex = FakeExecutor()
    srv = Server(ex, max_slots=8, round_pairs=2e6, memory_reserve=0, prepare_threads=0)
    big = srv.submit(req(60000))
    small = srv.submit(req(500))
    srv.run_until_idle()
    assert small.rounds == 1
    assert big.rounds > 1
    assert small.t_done <= big.t_done


@pytest.mark.parametrize("prep", [0, 1])
def test_invalid_request_fails_alone(prep):
    ex = FakeExecutor(fail_n=777)
    srv = Server(ex, max_slots=4, round_pairs=1e6, memory_reserve=0, prepare_threads=prep)
    good = srv.submit(req(1000))
    bad = srv.submit(req(777))
    also = srv.submit(req(2000))
    srv.run_until_idle()
    with pytest.raises(ValueError):
        bad.wait(0)
    assert good.wait(0)[1][0] == 1000
    assert also.wait(0)[1][0] == 2000


@pytest.mark.parametrize("prep", [0, 1])
def test_threaded_arrivals_complete(prep):
    ex = FakeExecutor()
    srv = Server(ex, max_slots=5, round_pairs=3e5, memory_reserve=0, prepare_threads=prep).start()
    rng = np.random.default_rng(4)
    sizes = rng.integers(2, 9000, 60)
    tickets = []

    def feeder():
        for n in sizes:
            tickets.append(srv.submit(req(int(n))))

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    srv.stop()
    assert len(tickets) == len(sizes)
    for t, n in zip(tickets, sizes):
        sums, counts = t.wait(5)
        assert int(counts[0]) == n and np.all(sums == 1.0)
        assert t.latency >= 0


class SerialExecutor(FakeExecutor):
    """An executor that can only wait for all queued rounds: the loop runs one round at a time."""

    def __getattribute__(self, name):
        if name == "wait_oldest":
            raise AttributeError(name)
        return super().__getattribute__(name)


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_pipelined_rounds_stay_within_depth(depth):
    ex = FakeExecutor()
    srv = Server(ex, max_slots=6, round_pairs=2e5, memory_reserve=0, depth=depth)
    sizes = [9000, 300, 4000, 12000, 2, 700, 5000, 256]
    tickets = [srv.submit(req(n)) for n in sizes]
    srv.run_until_idle()
    assert ex.max_inflight == depth
    assert not ex.inflight
    for t, n in zip(tickets, sizes):
        sums, counts = t.wait(0)
        assert int(counts[0]) == n and np.all(sums == 1.0)
    assert ex.live == 0


def test_executor_without_wait_oldest_runs_one_round_at_a_time():
    ex = SerialExecutor()
    srv = Server(ex, max_slots=4, round_pairs=2e5, memory_reserve=0, depth=2)
    assert srv.depth == 1
    ts = [srv.submit(req(n)) for n in (3000, 5000, 100)]
    srv.run_until_idle()
    assert ex.max_inflight == 1
    assert all(np.all(t.wait(0)[0] == 1.0) for t in ts)


class FailingExecutor(FakeExecutor):
    """Raises from the third round on, as a device error would."""

    def run_round(self, work):
        if len(self.rounds) >= 2:
            raise RuntimeError("device error")
        super().run_round(work)


@pytest.mark.parametrize("prep", [0, 1])
def test_loop_failure_fails_every_ticket(prep):
    ex = FailingExecutor()
    srv = Server(ex, max_slots=2, round_pairs=1e5, memory_reserve=0, prepare_threads=prep).start()
    tickets = [srv.submit(req(n)) for n in (6000, 7000, 8000, 9000)]
    for t in tickets:
        with pytest.raises(RuntimeError, match="device error"):
            t.wait(5)
    late = srv.submit(req(100))
    with pytest.raises(RuntimeError, match="device error"):
        late.wait(1)
    srv.stop()
    assert ex.live == 0


def test_smallest_waiting_request_is_admitted_first():
    # one slot: a small request submitted after two large ones is admitted before them
    ex = FakeExecutor()
    srv = Server(ex, max_slots=1, round_pairs=1e5, memory_reserve=0, prepare_threads=0)
    big = [srv.submit(req(8000)) for _ in range(2)]
    small = srv.submit(req(400))
    srv.run_until_idle()
    assert small.t_admit < min(t.t_admit for t in big)
    assert small.t_done < min(t.t_admit for t in big)  # one slot: the small request ran alone first


def test_long_waiting_request_is_admitted_before_smaller_ones():
    # a simulated clock: every reading advances one second, so the oldest waiting request has waited
    # longer than max_wait by the time its slot frees and goes before a smaller, newer one
    now = [0.0]

    def clock():
        now[0] += 1.0
        return now[0]

    ex = FakeExecutor()
    srv = Server(ex, max_slots=1, round_pairs=1e5, memory_reserve=0, prepare_threads=0, clock=clock,
                 max_wait=2.5)
    old = srv.submit(req(8000))
    srv.submit(req(7000))
    small = srv.submit(req(400))
    srv.run_until_idle()
    assert old.t_admit < small.t_admit


def test_fifo_admission_keeps_arrival_order():
    ex = FakeExecutor()
    srv = Server(ex, max_slots=1, round_pairs=1e5, memory_reserve=0, prepare_threads=0, admission="fifo")
    ts = [srv.submit(req(n)) for n in (6000, 8000, 400)]
    srv.run_until_idle()
    assert ts[0].t_admit < ts[1].t_admit < ts[2].t_admit
