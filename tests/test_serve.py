"""Scheduling logic of the serving loop, driven on the CPU by a stand-in for
the device batches (every request here is synthetic bookkeeping: a size in
bytes, a time step and an end time)."""
import math
from dataclasses import dataclass

import pytest

from sphera_b200.serve import Server, summarize


CANCELLED = 7            # SPH_CANCELLED
BDT_OVERFLOW = 802       # SPH_ERR_BDT_OVERFLOW
ALLOC = 400              # SPH_ERR_ALLOC


@dataclass
class FakeCase:
    n: int
    dt: float
    nbytes: int
    state: object = None
    fail_after: object = None     # steps after which the member reports fail_code
    fail_code: int = BDT_OVERFLOW
    oom: bool = False             # creating a batch that holds it fails (allocation)


class FakeSphError(RuntimeError):
    def __init__(self, code):
        self.code = code
        super().__init__(f"status {code}")


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
        self.code = [0] * len(cases)
        self.closed = False
        FakeBatch.live.append(self)

    def upload(self, states):
        assert len(states) == len(self.cases)

    def set_end_time(self, i, t):
        self.t_end[i] = t

    def step_async(self, k):
        for i, c in enumerate(self.cases):
            for _ in range(k):
                if self.t[i] >= self.t_end[i] or self.code[i]:
                    break
                self.t[i] += c.dt
                self.steps[i] += 1

    def idle(self):
        return True

    def status(self):
        for i, c in enumerate(self.cases):
            # host-side injection of a device failure: the member reports a
            # fatal code once it has run `fail_after` steps, and freezes
            if c.fail_after is not None and self.steps[i] >= c.fail_after and not self.code[i]:
                self.code[i] = c.fail_code
        fr = [self.t[i] >= self.t_end[i] or self.code[i] != 0 for i in range(len(self.cases))]
        return fr, list(self.t), list(self.steps), list(self.code)

    def cancel(self, i):
        if not (self.t[i] >= self.t_end[i] or self.code[i]):
            self.code[i] = CANCELLED

    def download(self, i):
        return None

    def close(self):
        self.closed = True


def _server(budget, peak_log):
    def sizer(cases):
        return sum(c.nbytes for c in cases)

    def factory(cases):
        if any(c.oom for c in cases):
            raise FakeSphError(ALLOC)
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


def _steps_alone(q):
    return math.ceil(q.t_end / q.case.dt)


def test_a_failed_member_is_reported_and_the_others_finish():
    """Host-side injection of a device failure: request 1 reports
    diagnostic 8/2 after 3 steps; it is reported failed with that code, its
    group mates finish with the step counts they have alone, and every
    group's bytes are returned."""
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    for q in reqs:
        q.arrival = 0.0
    reqs[1].case.fail_after = 3
    res = srv.run(reqs, poll=0.0)
    assert res[1].failed and res[1].status == BDT_OVERFLOW and not res[1].completed
    assert res[1].steps < _steps_alone(reqs[1])
    for q in reqs:
        if q.rid != 1:
            assert res[q.rid].completed and res[q.rid].steps == _steps_alone(q)
    assert res[0].group == res[1].group == res[2].group
    assert srv.used == 0 and all(b.closed for b in FakeBatch.live)
    s = summarize(res, srv.wall)
    assert s["failed"] == 1 and s["completed"] == len(reqs) - 1


def test_admission_oom_fails_the_group_and_frees_its_bytes():
    """A batch whose allocation fails on the device although the budget
    admitted it (injected: the factory raises diagnostic 4): its requests
    are reported failed, its bytes are never held, later requests run."""
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    for q in reqs:
        q.arrival = 0.0
    reqs[0].case.oom = True            # the first group: requests 0, 1, 2
    res = srv.run(reqs, poll=0.0)
    for rid in (0, 1, 2):
        assert res[rid].failed and res[rid].status == ALLOC
    for rid in (3, 4, 5):
        assert res[rid].completed
    assert srv.used == 0


def test_cancel_while_queued_and_while_running():
    """cancel() withdraws a queued request at once and freezes a running
    one from its next chunk on; both are reported cancelled and the others
    finish as alone."""
    FakeBatch.live = []
    srv = _server(1000, None)
    reqs = _requests()
    for q in reqs:
        q.arrival = 0.0
    # request 0 runs in the first group; request 5 waits for memory
    res = srv.run(reqs, poll=0.0, cancel_at={0: 0.0025, 5: 0.0025})
    assert res[0].cancelled and res[0].status == CANCELLED
    assert 0 < res[0].steps < _steps_alone(reqs[0])
    assert res[5].cancelled and res[5].steps == 0 and res[5].group == -1
    for rid in (1, 2, 3, 4):
        assert res[rid].completed and res[rid].steps == _steps_alone(reqs[rid])
    assert srv.used == 0


def _server_on(devices, budget):
    made = []

    def sizer(cases):
        return sum(c.nbytes for c in cases)

    def factory(cases, device):
        b = FakeBatch(cases)
        b.device = device
        made.append(b)
        return b

    srv = Server(budget, chunk=4, keep_state=False, sizer=sizer, factory=factory, clock=FakeClock(),
                 devices=devices)
    return srv, made


def test_requests_spread_over_devices_by_free_bytes():
    """Two GPUs with a budget each: a group goes to the device with the
    most free bytes, each device stays within its budget, both are used,
    and every request finishes with the steps it takes alone."""
    FakeBatch.live = []
    srv, made = _server_on(["gpu0", "gpu1"], 1000)
    reqs = _requests()
    for q in reqs:
        q.arrival = 0.0
    res = srv.run(reqs, poll=0.0)
    assert all(r.completed for r in res.values())
    for q in reqs:
        assert res[q.rid].steps == _steps_alone(q)
        assert res[q.rid].device == next(b.device for b in made if q.case in b.cases)
    # 300 + 500 + 200 fill gpu0; 800 + 100 go to the empty gpu1 at once
    assert res[0].device == res[1].device == res[2].device == "gpu0"
    assert res[3].device == res[4].device == "gpu1"
    assert res[3].admitted == res[0].admitted
    assert {b.device for b in made} == {"gpu0", "gpu1"}
    assert srv.peak_by["gpu0"] <= 1000 and srv.peak_by["gpu1"] <= 1000
    assert srv.used == 0 and all(b.closed for b in made)


def test_request_larger_than_one_device_is_rejected():
    FakeBatch.live = []
    srv, _ = _server_on(["gpu0", "gpu1"], 1000)
    reqs = _requests()
    reqs[2].case.nbytes = 1500        # fits in the two budgets together, in neither alone
    res = srv.run(reqs, poll=0.0)
    assert res[2].rejected
    assert all(res[i].completed for i in range(len(reqs)) if i != 2)
