"""Scheduling logic of the serving loop, driven on the CPU by a stand-in for
the device batches (every request here is synthetic bookkeeping: a size in
bytes, a time step and an end time)."""
import math
from dataclasses import dataclass

import pytest

from sphera_b200.serve import Server, summarize


@dataclass
class FakeCase:
    n: int
    dt: float
    nbytes: int
    state: object = None


@dataclass
class FakeReq:
    rid: int
    arrival: float
    case: FakeCase
    t_end: float


class FakeClock:
    def __init__(self, tick=1e-3):
        self.t = 0.0
        self.tick = tick

    def __call__(self):
        self.t += self.tick
        return self.t


class FakeBatch:
    live = []

    def __init__(self, cases):
        self.cases = cases
        self.t = [0.0] * len(cases)
        self.steps = [0] * len(cases)
        self.t_end = [0.0] * len(cases)
        self.closed = False
        FakeBatch.live.append(self)

    def upload(self, states):
        assert len(states) == len(self.cases)

    def set_end_time(self, i, t):
        self.t_end[i] = t

    def step_async(self, k):
        for i, c in enumerate(self.cases):
            for _ in range(k):
                if self.t[i] >= self.t_end[i]:
                    break
                self.t[i] += c.dt
                self.steps[i] += 1

    def idle(self):
        return True

    def status(self):
        fr = [self.t[i] >= self.t_end[i] for i in range(len(self.cases))]
        return fr, list(self.t), list(self.steps)

    def download(self, i):
        return None

    def close(self):
        self.closed = True


def _server(budget, peak_log):
    def sizer(cases):
        return sum(c.nbytes for c in cases)

    def factory(cases):
        b = FakeBatch(cases)
        return b

    srv = Server(budget, chunk=4, keep_state=False, sizer=sizer, factory=factory, clock=FakeClock())
    return srv


def _requests():
    sizes = [300, 500, 200, 800, 100, 400]
    # time steps and end times are binary fractions, so the step counts are exact
    return [FakeReq(i, 0.001 * i, FakeCase(n=10 * (i + 1), dt=(1 + i % 3) / 64.0, nbytes=s), 0.25)
            for i, s in enumerate(sizes)]


def test_all_requests_complete_within_budget():
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    res = srv.run(reqs, poll=0.0)
    assert all(not r.rejected for r in res.values())
    assert srv.peak_used <= 1000
    assert srv.used == 0
    assert all(b.closed for b in FakeBatch.live)
    for q in reqs:
        r = res[q.rid]
        assert r.steps == math.ceil(q.t_end / q.case.dt)
        assert r.admitted >= q.arrival
        assert r.finished > r.admitted


def test_admission_is_fifo_and_groups_what_fits():
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    for q in reqs:
        q.arrival = 0.0            # all queued at once
    res = srv.run(reqs, poll=0.0)
    order = sorted(res.values(), key=lambda r: (r.admitted, r.rid))
    assert [r.rid for r in order] == list(range(len(reqs)))
    # the first group takes the head requests while they fit: 300 + 500 + 200
    assert [res[i].group for i in range(3)] == [0, 0, 0]
    assert res[3].group != 0


def test_oversize_request_is_rejected():
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    reqs[1].case.nbytes = 5000
    res = srv.run(reqs, poll=0.0)
    assert res[1].rejected
    assert all(not res[i].rejected for i in range(len(reqs)) if i != 1)
    s = summarize(res, srv.wall)
    assert s["rejected"] == 1 and s["completed"] == len(reqs) - 1
    assert s["p50_s"] <= s["p99_s"]


@pytest.mark.parametrize("budget", [800, 1300, 10_000])
def test_budget_bounds_resident_bytes(budget):
    FakeBatch.live = []
    srv = _server(budget, None)
    srv.run(_requests(), poll=0.0)
    assert srv.peak_used <= budget
