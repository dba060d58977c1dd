"""Launch shapes change no result: the FP32c pair loops' two shapes (lean,
and a list chunk's records loaded together) and any persistent grid give
the same state bit for bit, for a single simulation and for a batch."""
import numpy as np
import pytest

from sphera_b200 import Batch, Simulation, abi, cases

pytestmark = pytest.mark.gpu

SHAPES = [dict(momentum_shape=0, continuity_shape=0),
          dict(momentum_shape=1, continuity_shape=0),
          dict(momentum_shape=0, continuity_shape=1),
          dict(momentum_shape=1, continuity_shape=1, lists=148, momentum=296, continuity=592)]


@pytest.mark.parametrize("dim", [2, 3])
def test_pair_loop_shapes_give_identical_states(dim):
    make = (lambda: cases.dam_break_2d(dx=0.02, precision=abi.SPH_PREC_FP32C)) if dim == 2 else \
        (lambda: cases.dam_break_3d(dx=0.02, precision=abi.SPH_PREC_FP32C))
    ref = None
    for shape in SHAPES:
        case = make()
        sim = Simulation(case)
        sim.upload(case.state)
        sim.set_launch_shape(shape)
        sim.step(25)
        st = sim.download()
        if ref is None:
            ref = st
        else:
            assert np.array_equal(st.x, ref.x), shape
            assert np.array_equal(st.v, ref.v), shape
            assert np.array_equal(st.rho, ref.rho), shape


def test_autotune_reports_the_shapes_and_keeps_results():
    cs = cases.ensemble_2d(n_sims=6, dx=0.02, seed=7)
    a = Batch(cs)
    a.upload()
    got = a.autotune(reps=1)
    assert got["momentum_shape"] in (0, 1) and got["continuity_shape"] in (0, 1)
    a.step(20)
    b = Batch(cs)
    b.upload()
    b.step(20)
    for i in range(len(cs)):
        assert np.array_equal(a.download(i).x, b.download(i).x)
