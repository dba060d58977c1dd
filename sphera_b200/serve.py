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
    group: int = -1

    @property
    def time_to_result(self):
        return self.finished - self.arrival


@dataclass
class _Group:
    gid: int
    batch: object
    requests: list
    bytes: int
    done: list = field(default_factory=list)


def _kind(case):
    prm = getattr(case, "params", None)
    return (getattr(prm, "dim", 0), getattr(prm, "precision", 0))


def _default_sizer(cases):
    from . import memory_required
    return memory_required(cases)


def _default_factory(cases):
    from . import Batch
    return Batch(cases)


class Server:
    """Admits requests by HBM budget and advances them concurrently.

    hbm_budget: bytes of device memory the admitted groups may hold.
    chunk: steps enqueued per group between two status reads.
    keep_state: download each result's state (the request's answer).
    """

    def __init__(self, hbm_budget, chunk=32, keep_state=True, sizer=None, factory=None, clock=None):
        self.budget = int(hbm_budget)
        self.chunk = int(chunk)
        self.keep_state = keep_state
        self.sizer = sizer or _default_sizer
        self.factory = factory or _default_factory
        self.clock = clock or time.perf_counter
        self.used = 0
        self.peak_used = 0
        self.groups_formed = 0
        self.max_concurrent = 0

    def _admit(self, waiting, now, results):
        """Forms one group from the head of the queue (FIFO, no overtaking)."""
        group, need = [], 0
        while waiting:
            if group and _kind(waiting[0].case) != _kind(group[0].case):
                break                  # a batch holds one dim and precision
            cand = group + [waiting[0]]
            b = self.sizer([r.case for r in cand])
            if self.used + b > self.budget:
                if not group and self.used == 0:
                    # larger than the whole budget: it can never run
                    r = waiting.popleft()
                    results[r.rid].rejected = True
                    continue
                break
            group, need = cand, b
            waiting.popleft()
        if not group:
            return None
        batch = self.factory([r.case for r in group])
        batch.upload([r.case.state for r in group])
        for i, r in enumerate(group):
            batch.set_end_time(i, r.t_end)
            results[r.rid].admitted = now
            results[r.rid].group = self.groups_formed
        self.used += need
        self.peak_used = max(self.peak_used, self.used)
        g = _Group(self.groups_formed, batch, group, need, [False] * len(group))
        self.groups_formed += 1
        batch.step_async(self.chunk)
        return g

    def run(self, requests, poll=2e-4):
        """Serves `requests` (arrival times in seconds from the start) in real
        time and returns {rid: Result}."""
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        results = {r.rid: Result(r.rid, r.arrival) for r in requests}
        waiting = deque()
        active = []
        t0 = self.clock()
        while pending or waiting or active:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
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
                frozen, t, steps = g.batch.status()
                now = self.clock() - t0
                for i, r in enumerate(g.requests):
                    if frozen[i] and not g.done[i]:
                        g.done[i] = True
                        res = results[r.rid]
                        if self.keep_state:
                            res.state = g.batch.download(i)
                            res.n = res.state.n
                        else:
                            res.n = r.case.n
                        res.finished = self.clock() - t0
                        res.steps = int(steps[i])
                        res.sim_time = float(t[i])
                if all(g.done):
                    g.batch.close()
                    self.used -= g.bytes
                    active.remove(g)
                else:
                    g.batch.step_async(self.chunk)
            if not progressed:
                nxt = pending[0].arrival - (self.clock() - t0) if pending and not waiting else poll
                time.sleep(max(0.0, min(poll, nxt)))
        self.wall = self.clock() - t0
        return results


def summarize(results, wall):
    """p50/p99 time-to-result and aggregate particle-steps/s of a run."""
    done = [r for r in results.values() if not r.rejected]
    ttr = np.array([r.time_to_result for r in done])
    work = float(sum(r.n * r.steps for r in done))
    return dict(
        requests=len(results), completed=len(done), rejected=sum(r.rejected for r in results.values()),
        p50_s=float(np.percentile(ttr, 50)) if len(ttr) else None,
        p99_s=float(np.percentile(ttr, 99)) if len(ttr) else None,
        mean_queue_s=float(np.mean([r.admitted - r.arrival for r in done])) if done else None,
        particle_steps=work, wall_s=wall,
        particle_steps_per_s=work / wall if wall > 0 else None)
