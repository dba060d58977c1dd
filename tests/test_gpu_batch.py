"""Batched simulations (several independent cases advanced by the same
launches and CUDA graph) and the autotuner.

A simulation's result must not depend on its companions: every kernel
treats each particle of each simulation independently, so a case run in a
batch is bit-identical to the same case run alone, in both forms.
"""
import numpy as np
import pytest

from sphera_b200 import Batch, Simulation, abi, cases

pytestmark = pytest.mark.gpu


def _columns(precision):
    return [cases.dam_break_2d(dx=0.02, column=(w, hgt), seed=100 + i, precision=precision)
            for i, (w, hgt) in enumerate([(0.6, 1.0), (1.0, 2.0), (0.4, 0.6), (1.4, 1.2)])]


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_batch_member_equals_alone(precision):
    cs = _columns(precision)
    b = Batch(cs)
    b.upload()
    b.step(150)
    for i, c in enumerate(cs):
        alone = Simulation(c)
        alone.upload(c.state)
        alone.step(150)
        sa = alone.download()
        sb = b.download(i)
        assert np.array_equal(sa.x, sb.x)
        assert np.array_equal(sa.v, sb.v)
        assert np.array_equal(sa.rho, sb.rho)
        info, frozen = b.info(i)
        assert info.step == 150 and not frozen


def test_batch_end_times_freeze_members():
    cs = _columns(abi.SPH_PREC_FP32C)
    b = Batch(cs)
    b.upload()
    ends = [0.004, 0.008, 0.002, 0.006]
    for i, t in enumerate(ends):
        b.set_end_time(i, t)
    for _ in range(200):
        b.step(10)
        if all(b.info(i)[1] for i in range(len(cs))):
            break
    for i, c in enumerate(cs):
        info, frozen = b.info(i)
        assert frozen
        assert ends[i] <= info.time < ends[i] + 2 * info.dt
        # the frozen state equals the same case run alone for as many steps
        alone = Simulation(c)
        alone.upload(c.state)
        alone.step(info.step)
        assert np.array_equal(alone.download().x, b.download(i).x)


def test_autotune_keeps_results():
    c = cases.dam_break_3d(dx=0.02, precision=abi.SPH_PREC_FP32C)
    a = Simulation(c)
    a.upload(c.state)
    t = Simulation(c)
    t.upload(c.state)
    grids = t.autotune(reps=2)
    assert all(grids[k] > 0 for k in ("lists", "momentum", "continuity", "boundary", "integrals"))
    assert grids["momentum_shape"] in (0, 1, 2) and grids["continuity_shape"] in (0, 1, 2)
    a.step(20)
    t.step(20)
    assert np.array_equal(a.download().x, t.download().x)
