"""Serving loop: continuous admission of simulation requests under an HBM
budget (no reference counterpart; SPHERA runs one case per process).

A request is a case to run to its end time t_end.  The server keeps every
admitted simulation resident on the device and advances it with CUDA-graph
launches on its group's own stream; it never waits for one group to let
another make progress:

* arrivals queue FIFO;
* admission: the head of the queue is admitted when the device bytes of the
  admitted groups plus its own (``memory_required``, computed on the host
  before any allocation) stay within the budget.  All queued requests that
  fit together (and share dim and precision) are admitted as one group, a
  ``Batch`` whose members advance in the same launches; a request larger
  than the whole budget is rejected;
* progress: each group runs ``chunk`` steps per enqueue; when its stream is
  idle (``idle()`` never waits) the server reads the members' status in one
  read-back, downloads each member that reached t_end (its result), and
  enqueues the next chunk.  Frozen members do no further work;
* a group whose members have all finished is destroyed and its bytes return
  to the budget, which may admit the next group.

Failures stay with their request.  The reference's only failure path is
fatal (``diagnostic`` ends with ``stop``, src/Memory_I_O/diagnostic.f90) and
its only clean stop is the kill file (time_step_loop.f90:485-487); here:

* a member whose device status turns fatal (for example its share of the
  boundary-data pool overflowing, diagnostic 8/2) freezes on the device at
  the end of that step; the server reports it failed with the code, and the
  other members of its group run on, unchanged;
* ``cancel(rid)`` withdraws a queued request or freezes a running one
  (``sph_batch_cancel``); it is reported cancelled;
* a group whose creation or upload fails on the device (for example an
  allocation the budget did not foresee) reports its requests failed with
  that code and returns their bytes.

Several GPUs (``devices``): each has its own budget; a group is formed for,
and built on, the device with the most free bytes (the head of the queue
waits only while it fits on none), so requests spread over the node's GPUs
as memory frees up.  A handle keeps its device (every library call runs
there), so one host thread drives all of them.

Every kernel treats each member of a group independently, so a request's
result does not depend on what else is admitted: it equals the same
request run alone, bit for bit.

The device side is reached only through a factory of group objects (the
``Batch`` class by default), so the scheduling logic is testable without a
device.
"""
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

CANCELLED = 7          # SPH_CANCELLED


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float = float("nan")
    finished: float = float("nan")
    n: int = 0
    steps: int = 0
    sim_time: float = 0.0
    state: object = None
    rejected: bool = False
    failed: bool = False
    cancelled: bool = False
    status: int = 0
    group: int = -1
    device: object = None

    @property
    def time_to_result(self):
        return self.finished - self.arrival

    @property
    def completed(self):
        return not (self.rejected or self.failed or self.cancelled)


@dataclass
class _Group:
    gid: int
    batch: object
    requests: list
    bytes: int
    done: list = field(default_factory=list)
    device: object = None


def _kind(case):
    prm = getattr(case, "params", None)
    return (getattr(prm, "dim", 0), getattr(prm, "precision", 0))


def _default_sizer(cases):
    from . import memory_required
    return memory_required(cases)


def _default_factory(cases, device=None):
    from . import Batch
    return Batch(cases, device=device)


class Server:
    """Admits requests by HBM budget and advances them concurrently.

    hbm_budget: bytes of device memory the admitted groups may hold, per
        device.
    devices: the GPUs to serve on (default: the thread's current one); the
        factory is then called as factory(cases, device).
    chunk: steps enqueued per group between two status reads.
    keep_state: download each result's state (the request's answer).
    """

    def __init__(self, hbm_budget, chunk=32, keep_state=True, sizer=None, factory=None, clock=None,
                 devices=None):
        self.budget = int(hbm_budget)
        self.devices = list(devices) if devices else [None]
        self.chunk = int(chunk)
        self.keep_state = keep_state
        self.sizer = sizer or _default_sizer
        self.factory = factory or _default_factory
        self.clock = clock or time.perf_counter
        self.used_by = {d: 0 for d in self.devices}
        self.peak_by = {d: 0 for d in self.devices}
        self.groups_formed = 0
        self.max_concurrent = 0
        self._cancel = set()

    @property
    def used(self):
        """Bytes the admitted groups hold, over all devices."""
        return sum(self.used_by.values())

    @property
    def peak_used(self):
        """The largest bytes any one device held at once."""
        return max(self.peak_by.values())

    def cancel(self, rid):
        """Withdraws request `rid`: taken out of the queue if it waits, frozen
        on the device (and its result reported cancelled) if it runs."""
        self._cancel.add(rid)

    def _admit(self, waiting, now, results):
        """Forms one group from the head of the queue (FIFO, no overtaking)
        for the device with the most free bytes."""
        dev = min(self.devices, key=lambda d: (self.used_by[d], self.devices.index(d)))
        used = self.used_by[dev]
        group, need = [], 0
        while waiting:
            if group and _kind(waiting[0].case) != _kind(group[0].case):
                break                  # a batch holds one dim and precision
            cand = group + [waiting[0]]
            b = self.sizer([r.case for r in cand])
            if used + b > self.budget:
                if not group and b > self.budget:
                    # larger than a whole device's budget: it can never run
                    r = waiting.popleft()
                    results[r.rid].rejected = True
                    continue
                break
            group, need = cand, b
            waiting.popleft()
        if not group:
            return None
        gid = self.groups_formed
        self.groups_formed += 1
        try:
            cases = [r.case for r in group]
            batch = self.factory(cases) if self.devices == [None] else self.factory(cases, dev)
        except RuntimeError as e:
            self._fail_group(group, gid, getattr(e, "code", -1), now, results)
            return None
        try:
            try:
                batch.upload([r.case.state for r in group])
            except RuntimeError:
                # the upload returns the first member's fatal status; when
                # members hold one, they alone failed (their IC pass): the
                # status poll reports them and the others run
                if not any(batch.status()[3]):
                    raise
            for i, r in enumerate(group):
                batch.set_end_time(i, r.t_end)
        except RuntimeError as e:
            batch.close()
            self._fail_group(group, gid, getattr(e, "code", -1), now, results)
            return None
        for r in group:
            results[r.rid].admitted = now
            results[r.rid].group = gid
            results[r.rid].device = dev
        self.used_by[dev] += need
        self.peak_by[dev] = max(self.peak_by[dev], self.used_by[dev])
        g = _Group(gid, batch, group, need, [False] * len(group), dev)
        batch.step_async(self.chunk)
        return g

    @staticmethod
    def _fail_group(group, gid, code, now, results):
        for r in group:
            res = results[r.rid]
            res.admitted = res.finished = now
            res.group = gid
            res.failed = True
            res.status = int(code)

    def _apply_cancels(self, waiting, active, now, results):
        for rid in list(self._cancel):
            for r in list(waiting):
                if r.rid == rid:
                    waiting.remove(r)
                    res = results[rid]
                    res.cancelled = True
                    res.status = CANCELLED
                    res.finished = now
                    self._cancel.discard(rid)
            for g in active:
                for i, r in enumerate(g.requests):
                    if r.rid == rid and not g.done[i]:
                        g.batch.cancel(i)   # takes effect from the next launch on
                        self._cancel.discard(rid)

    def run(self, requests, poll=2e-4, cancel_at=None):
        """Serves `requests` (arrival times in seconds from the start) in real
        time and returns {rid: Result}.  cancel_at: {rid: time} of cancels
        to issue during the run (as cancel() would from another thread)."""
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        results = {r.rid: Result(r.rid, r.arrival) for r in requests}
        cancels = sorted((t, rid) for rid, t in (cancel_at or {}).items())
        waiting = deque()
        active = []
        t0 = self.clock()
        while pending or waiting or active:
            now = self.clock() - t0
            while cancels and cancels[0][0] <= now:
                self.cancel(cancels.pop(0)[1])
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            if self._cancel:
                self._apply_cancels(waiting, active, now, results)
            while waiting:
                g = self._admit(waiting, now, results)
                if g is None:
                    break
                active.append(g)
            self.max_concurrent = max(self.max_concurrent, sum(len(g.requests) - sum(g.done) for g in active))
            progressed = False
            for g in list(active):
                if not g.batch.idle():
                    continue
                progressed = True
                frozen, t, steps, status = g.batch.status()
                for i, r in enumerate(g.requests):
                    if g.done[i] or not (frozen[i] or status[i]):
                        continue
                    g.done[i] = True
                    res = results[r.rid]
                    res.steps = int(steps[i])
                    res.sim_time = float(t[i])
                    res.status = int(status[i])
                    if status[i] == CANCELLED:
                        res.cancelled = True
                    elif status[i]:
                        res.failed = True
                    elif self.keep_state:
                        res.state = g.batch.download(i)
                        res.n = res.state.n
                    else:
                        res.n = r.case.n
                    res.finished = self.clock() - t0
                if all(g.done):
                    g.batch.close()
                    self.used_by[g.device] -= g.bytes
                    active.remove(g)
                else:
                    g.batch.step_async(self.chunk)
            if not progressed:
                nxt = pending[0].arrival - (self.clock() - t0) if pending and not waiting else poll
                if cancels:
                    nxt = min(nxt, cancels[0][0] - (self.clock() - t0))
                time.sleep(max(0.0, min(poll, nxt)))
        self.wall = self.clock() - t0
        return results


def summarize(results, wall):
    """p50/p99 time-to-result and aggregate particle-steps/s of a run (over
    the completed requests; failed, cancelled and rejected ones counted)."""
    done = [r for r in results.values() if r.completed]
    ttr = np.array([r.time_to_result for r in done])
    work = float(sum(r.n * r.steps for r in done))
    return dict(
        requests=len(results), completed=len(done), rejected=sum(r.rejected for r in results.values()),
        failed=sum(r.failed for r in results.values()), cancelled=sum(r.cancelled for r in results.values()),
        p50_s=float(np.percentile(ttr, 50)) if len(ttr) else None,
        p99_s=float(np.percentile(ttr, 99)) if len(ttr) else None,
        mean_queue_s=float(np.mean([r.admitted - r.arrival for r in done])) if done else None,
        particle_steps=work, wall_s=wall,
        particle_steps_per_s=work / wall if wall > 0 else None)
