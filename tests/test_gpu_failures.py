"""Failure isolation on the device, through the C ABI: a batch member that
meets a fatal condition (here its own share of the boundary-data pool
overflowing, diagnostic 8/2, injected by a deliberately small
SphParams.bdt_capacity) freezes and reports its code while its group mates
go on bit for bit as alone; sph_batch_cancel freezes a member the same
way; the serving loop reports both and returns the group's bytes.  Every
failure here is a status word the host reads: no device fault."""
import numpy as np
import pytest

from sphera_b200 import Batch, SphError, abi, cases
from sphera_b200.serve import Server, summarize

pytestmark = pytest.mark.gpu

T_END = 0.02


def _alone(case, t_end, chunk=16):
    b = Batch([case])
    b.upload()
    b.set_end_time(0, t_end)
    while True:
        b.step(chunk)
        info, frozen = b.info(0)
        if frozen:
            break
    st = b.download(0)
    b.close()
    return st, info.step


def _cases(precision=abi.SPH_PREC_FP32C):
    a = cases.dam_break_3d(dx=0.04, seed=1, precision=precision)
    bad = cases.dam_break_3d(dx=0.04, seed=2, precision=precision)
    bad.params.bdt_capacity = 8          # far below the wall-near particles' entries
    c = cases.sloshing_3d(dx=0.04, period=0.8, seed=3, precision=precision)
    return [a, bad, c]


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_failed_member_freezes_and_the_others_match_alone(precision):
    cs = _cases(precision)
    b = Batch(cs)
    with pytest.raises(SphError) as e:
        b.upload()                       # the IC boundary pass already overflows
    assert e.value.code == abi.SPH_ERR_BDT_OVERFLOW
    for i, c in enumerate(cs):
        b.set_end_time(i, T_END)
    for _ in range(40):
        b.step_async(16)
        fr, t, steps, code = b.status()
        if fr[0] and fr[2]:
            break
    assert code.tolist() == [0, abi.SPH_ERR_BDT_OVERFLOW, 0]
    assert fr.all() and steps[1] <= 1
    for i in (0, 2):
        st, nsteps = _alone(cs[i], T_END)
        assert steps[i] == nsteps
        got = b.download(i)
        assert np.array_equal(got.x, st.x)
        assert np.array_equal(got.v, st.v)
        assert np.array_equal(got.rho, st.rho)
    b.close()


def test_cancel_freezes_one_member():
    cs = [cases.dam_break_3d(dx=0.04, seed=1, precision=abi.SPH_PREC_FP32C),
          cases.dam_break_3d(dx=0.04, seed=5, precision=abi.SPH_PREC_FP32C)]
    b = Batch(cs)
    b.upload()
    for i in range(2):
        b.set_end_time(i, T_END)
    b.step(10)
    b.cancel(1)
    b.step_async(10)
    fr, t, steps, code = b.status()
    assert code.tolist() == [0, abi.SPH_CANCELLED]
    assert steps.tolist() == [20, 10] and fr[1]
    while not b.status()[0][0]:
        b.step_async(16)
    st, nsteps = _alone(cs[0], T_END)
    assert np.array_equal(b.download(0).x, st.x)
    b.close()


def test_serving_reports_failures_and_cancels():
    """Four requests: one fails on the device (diagnostic 8/2), one is
    cancelled while it runs; the two others equal their runs alone and the
    server ends holding no bytes."""
    P = abi.SPH_PREC_FP32C
    bad = cases.dam_break_3d(dx=0.04, seed=2, precision=P)
    bad.params.bdt_capacity = 8
    spec = [(0.000, cases.dam_break_3d(dx=0.04, seed=1, precision=P)),
            (0.000, bad),
            (0.001, cases.sloshing_3d(dx=0.04, period=0.8, seed=3, precision=P)),
            (0.002, cases.dam_break_3d(dx=0.04, seed=4, precision=P))]
    reqs = [cases.Request(i, t, c, 0.05) for i, (t, c) in enumerate(spec)]
    srv = Server(8 << 30, chunk=8)
    res = srv.run(reqs, cancel_at={3: 0.05})
    assert res[1].failed and res[1].status == abi.SPH_ERR_BDT_OVERFLOW
    s = summarize(res, srv.wall)
    assert s["failed"] == 1 and srv.used == 0
    if res[3].cancelled:                 # cancelled while it ran (it may have finished first)
        assert res[3].status == abi.SPH_CANCELLED
    for rid in (0, 2):
        st, nsteps = _alone(reqs[rid].case, reqs[rid].t_end)
        assert res[rid].completed and res[rid].steps == nsteps
        assert np.array_equal(res[rid].state.x, st.x)
