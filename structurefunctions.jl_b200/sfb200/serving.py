"""Continuous-batching request loop for many point sets on one device.

The reference computes one call at a time. For a stream of requests of uneven size (time slices or
fields; 2D/3D, planar or spherical; with or without the joint histogram) this loop keeps the device
busy with all of them at once:

- Admission. A request is admitted when a slot is free and the device has room for it (free memory
  minus a reserve, checked against an estimate of the request's footprint before its buffers are
  created). Among the waiting requests the one with the fewest pairs goes first ("shortest"), so that
  a small request arriving while the slots hold large ones waits for one slot, not for the whole
  queue; a request that has waited longer than `max_wait` seconds goes first whatever its size, so a
  large one is not passed over forever. `admission="fifo"` admits in arrival order.
- Residency. An admitted request becomes a slice: its points are packed on the device and its
  histogram lives there until the request completes. Slices are prepared (host-to-device copy,
  ordering, packing) on `prepare_threads` worker threads, so that preparing arrivals never holds up
  the loop that keeps the device fed; a slice joins the rounds once it is prepared, in arrival order.
- Rounds. Work is cut into tile pairs (independent units of up to 256 x 256 pairs). Each round gives
  every slice at least `min_units` of its remaining tile pairs, then hands out the rest of the
  round's pair budget shortest-remaining-first, and runs all of it as one batched launch (one
  persistent kernel per kernel variant, replayed from a CUDA graph). Requests that arrive while a
  round runs join the next one: continuous batching, not a queue in front of one-at-a-time launches.
- Pipelining. Up to `depth` rounds are queued at once (the library double-buffers them): while one
  runs on the device the next is already queued behind it, so the device does not idle while the
  host completes, admits and plans between rounds.
- Completion. A slice whose tile pairs are all done is read back, its ticket completed with the
  latency (arrival to result) and the slice released.

`Server` is the loop; an executor does the device work. `GpuExecutor` drives libsfb200.so;
`tests/test_serving_cpu.py` drives the same loop with a simulated executor.
"""
import collections
import concurrent.futures
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .api import plan_description
from .errors import ArgumentError


def _host_layout(a):
    """(W, N) host array as column-major Float32 / Float64 memory."""
    arr = np.asarray(a)
    if arr.dtype not in (np.float32, np.float64):
        if arr.dtype.kind not in "iu":
            raise ArgumentError(f"inputs must be Float32 or Float64; got {arr.dtype}")
        arr = arr.astype(np.float64)
    return np.asfortranarray(arr)


@dataclass(eq=False)
class Request:
    """One structure-function request: the arguments of calculate_structure_function."""
    ops: tuple
    x: np.ndarray
    u: np.ndarray
    distance_bins: object
    value_bins: object = None
    metric: object = None
    tag: object = None

    @property
    def n(self):
        return int(self.x.shape[1])

    @property
    def pairs(self):
        return self.n * (self.n - 1) // 2


@dataclass(eq=False)
class Ticket:
    request: Request
    t_submit: float
    t_admit: float = float("nan")
    t_done: float = float("nan")
    sums: np.ndarray = None
    counts: np.ndarray = None
    error: BaseException = None
    rounds: int = 0
    _event: threading.Event = field(default_factory=threading.Event)

    def done(self):
        return self._event.is_set()

    def wait(self, timeout=None):
        if not self._event.wait(timeout):
            raise TimeoutError("request not completed in time")
        if self.error is not None:
            raise self.error
        return self.sums, self.counts

    @property
    def latency(self):
        return self.t_done - self.t_submit


@dataclass(eq=False)
class _Active:
    ticket: Ticket
    handle: object
    units: int          # tile pairs in total
    done: int = 0       # tile pairs completed (always a prefix [0, done))
    pairs_per_unit: float = 1.0
    issued: int = 0     # tile pairs queued in rounds so far (a prefix [0, issued), issued >= done)

    @property
    def remaining(self):
        return self.units - self.issued


class Server:
    """Continuous-batching loop over an executor (see the module documentation)."""

    def __init__(self, executor, max_slots=256, memory_reserve=1 << 30, round_pairs=6e9, min_units=1,
                 depth=2, prepare_threads=1, clock=time.perf_counter, admission="shortest", max_wait=1.0):
        if admission not in ("shortest", "fifo"):
            raise ArgumentError(f"admission must be 'shortest' or 'fifo'; got {admission!r}")
        self.admission = admission
        self.max_wait = float(max_wait)
        self.ex = executor
        self.depth = max(1, int(depth)) if hasattr(executor, "wait_oldest") else 1
        self._prep = (concurrent.futures.ThreadPoolExecutor(int(prepare_threads), thread_name_prefix="sfb200-prep")
                      if prepare_threads else None)
        self._preparing = collections.deque()  # (ticket, future, bytes), in admission order
        self._prep_bytes = 0
        self.failed = None  # the exception that stopped the loop, if any
        self.max_slots = int(max_slots)
        self.memory_reserve = int(memory_reserve)
        self.round_pairs = float(round_pairs)
        self.min_units = int(min_units)
        self.clock = clock
        self._pending = collections.deque()
        self._active = []
        self._cv = threading.Condition()
        self._stop = False
        self._thread = None
        self.rounds = 0
        self.round_log = []  # (n_slices, pairs) per round

    # ------------------------------------------------------------------ public
    def submit(self, request):
        t = Ticket(request, self.clock())
        with self._cv:
            failed = self.failed
            if failed is None:
                self._pending.append(t)
                self._cv.notify()
        if failed is not None:  # the loop has stopped on an error
            self._fail(t, failed)
        return t

    def start(self):
        self._thread = threading.Thread(target=self._loop, name="sfb200-server", daemon=True)
        self._thread.start()
        return self

    def stop(self, drain=True):
        with self._cv:
            self._stop = True
            self._drain = drain
            self._cv.notify()
        if self._thread:
            self._thread.join()
        if self._prep:
            self._prep.shutdown(wait=True)

    def run_until_idle(self):
        """Run the loop on the calling thread until nothing is pending or active."""
        self._stop = True
        self._drain = True
        self._loop(reraise=True)

    # ------------------------------------------------------------------ loop
    def _activate(self, t, h):
        t.t_admit = self.clock()
        a = _Active(t, h, int(h.tile_pairs), 0, max(1.0, h.pairs / max(1, h.tile_pairs)))
        if a.units == 0:
            self._complete(a)
        else:
            self._active.append(a)

    def _fail(self, t, e):  # invalid request: fail the ticket, keep serving
        t.error = e
        t.t_done = self.clock()
        t._event.set()

    def _harvest(self, block=False):
        """Move prepared slices into the rounds (in admission order)."""
        while self._preparing:
            t, fut, need = self._preparing[0]
            if not fut.done():
                if not block:
                    return
                concurrent.futures.wait([fut], timeout=0.005)
                if not fut.done():
                    return
            self._preparing.popleft()
            self._prep_bytes -= need
            try:
                h = fut.result()
            except BaseException as e:
                self._fail(t, e)
                continue
            self._activate(t, h)
            block = False

    def _next_pending(self):
        """The waiting ticket to admit next (called under the lock, with something pending): the
        oldest once it has waited `max_wait` seconds, else the one with the fewest pairs."""
        oldest = self._pending[0]
        if self.admission == "fifo" or len(self._pending) == 1 or self.clock() - oldest.t_submit > self.max_wait:
            return oldest
        return min(self._pending, key=lambda t: t.request.pairs)

    def _admit(self):
        self._harvest()
        while True:
            with self._cv:
                busy = len(self._active) + len(self._preparing)
                if not self._pending or busy >= self.max_slots:
                    return
                t = self._next_pending()
                need = self.ex.estimate_bytes(t.request)
                if busy and self.ex.free_bytes() - self._prep_bytes - need < self.memory_reserve:
                    return  # wait for a slice to finish and free its memory
                self._pending.remove(t)
            if self._prep is not None:
                self._preparing.append((t, self._prep.submit(self.ex.create, t.request), need))
                self._prep_bytes += need
                continue
            try:
                h = self.ex.create(t.request)
            except BaseException as e:
                self._fail(t, e)
                continue
            self._activate(t, h)

    def _plan_round(self):
        """Tile-pair ranges of this round: min_units each, then shortest remaining first (over the
        slices with tile pairs not yet queued)."""
        budget = self.round_pairs
        ready = [a for a in self._active if a.remaining > 0]
        give = {id(a): 0 for a in ready}
        for a in ready:
            k = min(a.remaining, self.min_units)
            give[id(a)] = k
            budget -= k * a.pairs_per_unit
        for a in sorted(ready, key=lambda a: a.remaining * a.pairs_per_unit):
            if budget <= 0:
                break
            extra = min(a.remaining - give[id(a)], int(budget // a.pairs_per_unit) + 1)
            if extra > 0:
                give[id(a)] += extra
                budget -= extra * a.pairs_per_unit
        return [(a, a.issued, a.issued + give[id(a)]) for a in ready if give[id(a)] > 0]

    def _complete(self, a):
        t = a.ticket
        try:
            t.sums, t.counts = self.ex.read(a.handle)
        except BaseException as e:
            t.error = e
        finally:
            self.ex.destroy(a.handle)
        t.t_done = self.clock()
        t._event.set()

    def _loop(self, reraise=False):
        try:
            self._run_loop()
        except BaseException as e:
            self._abort(e)  # every ticket now carries the error; the loop thread ends quietly
            if reraise:
                raise

    def _abort(self, e):
        """The loop failed (a device error): fail every ticket it holds instead of leaving it waiting."""
        with self._cv:
            self.failed = e  # from here on, submit fails new tickets itself
        try:
            self.ex.wait_round()
        except BaseException:
            pass
        tickets = [a.ticket for a in self._active]
        for a in self._active:
            try:
                self.ex.destroy(a.handle)
            except BaseException:
                pass
        self._active.clear()
        for t, fut, _ in self._preparing:
            tickets.append(t)
            try:
                self.ex.destroy(fut.result())
            except BaseException:
                pass
        self._preparing.clear()
        with self._cv:
            tickets.extend(self._pending)
            self._pending.clear()
            self._stop = True
        for t in tickets:
            if not t.done():
                self._fail(t, e)

    def _run_loop(self):
        inflight = collections.deque()  # queued rounds, oldest first: lists of (active, begin, end)
        while True:
            self._admit()
            if len(inflight) < self.depth and any(a.remaining > 0 for a in self._active):
                plan = self._plan_round()
                self.ex.run_round([(a.handle, b, e) for a, b, e in plan])
                for a, b, e in plan:
                    a.issued = e
                inflight.append(plan)
                self.rounds += 1
                self.round_log.append((len(plan), sum((e - b) * a.pairs_per_unit for a, b, e in plan)))
                continue
            if inflight:
                # admit arrivals while the queued rounds run (their preparation overlaps them)
                self._admit()
                if self.depth > 1:
                    self.ex.wait_oldest()
                else:
                    self.ex.wait_round()
                plan = inflight.popleft()
                finished = []
                for a, b, e in plan:
                    a.done = e
                    a.ticket.rounds += 1
                    if a.done >= a.units:
                        finished.append(a)
                for a in finished:
                    self._active.remove(a)
                    self._complete(a)
                continue
            if self._preparing:
                self._harvest(block=True)  # nothing to run until a prepared slice arrives
                continue
            with self._cv:
                if self._pending:
                    continue
                if self._stop:
                    return
                self._cv.wait(timeout=0.005)


# ---------------------------------------------------------------------------------- GPU executor

class _Handle:
    __slots__ = ("slice", "plan", "keep", "tile_pairs", "pairs", "device_bytes", "host", "n_sums", "n_counts",
                 "variant")


class GpuExecutor:
    """Executor over libsfb200.so: one context, plans cached per request shape, mixed precision."""

    def __init__(self, device=0, precision="mixed"):
        self.ctx = _lib.Context(device)
        self.precision = precision
        self._plans = {}
        self.launches = 0  # kernel launches issued by the rounds (one per kernel variant per round)

    def _plan(self, req, xd, ud):
        key = (tuple(repr(o) for o in req.ops), req.u.shape[0], repr(req.metric), xd.dtype.str, ud.dtype.str,
               np.asarray(getattr(req.distance_bins, "edges", req.distance_bins), dtype=np.float64).tobytes(),
               None if req.value_bins is None else repr(req.value_bins))
        p = self._plans.get(key)
        if p is None:
            desc, keep = plan_description(req.ops, req.u.shape[0], req.distance_bins, req.value_bins, req.metric,
                                          self.precision, xd.dtype, ud.dtype)
            p = (_lib.Plan(self.ctx, desc, keep), keep)
            self._plans[key] = p
        return p

    def estimate_bytes(self, req):
        sphere = req.x.shape[0] == 2 and req.metric is not None and type(req.metric).__name__ != "Euclidean"
        D = req.u.shape[0]
        per_point = 8 * (req.x.shape[0] + D) + 8 * ((8 if sphere else D) + D) + (80 if sphere else 0) + 48
        return int(req.n * per_point + (1 << 20))

    def free_bytes(self):
        return _lib.device_memory(self.ctx)[0]

    def create(self, req):
        xd, ud = _host_layout(req.x), _host_layout(req.u)
        plan, keep = self._plan(req, xd, ud)
        h = _Handle()
        h.host = (xd, ud)  # kept until the slice is released (the copy is asynchronous)
        h.plan = plan
        h.keep = keep
        h.slice = _lib.Slice(plan, xd.ctypes.data, ud.ctypes.data, req.n)
        h.tile_pairs, h.pairs, h.device_bytes = h.slice.tile_pairs, h.slice.pairs, h.slice.device_bytes
        h.n_sums, h.n_counts = plan.n_sums, plan.n_counts
        h.variant = (req.x.shape[0], req.u.shape[0], type(req.metric).__name__, req.value_bins is not None,
                     tuple(repr(o) for o in req.ops))
        return h

    def run_round(self, work):
        _lib.batch_run(self.ctx, [h.slice for h, _, _ in work], [b for _, b, _ in work], [e for _, _, e in work])
        self.launches += len({h.variant for h, _, _ in work})

    def wait_round(self):
        _lib.batch_wait(self.ctx)

    def wait_oldest(self):
        _lib.batch_wait_oldest(self.ctx)

    def read(self, h):
        sums = np.zeros(h.n_sums)
        counts = np.zeros(h.n_counts, dtype=np.uint64)
        h.slice.read(sums.ctypes.data, counts.ctypes.data)
        return sums, counts

    def destroy(self, h):
        h.slice.close()
        h.host = None

    def close(self):
        for p, _ in self._plans.values():
            p.close()
        self._plans.clear()
        self.ctx.close()
