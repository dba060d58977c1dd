"""Launch shapes change no result: the pair loops' shapes (lean, several
list entries' records loaded together, and in the FP32c form the
batched one on paired FP32 instructions) and any persistent grid give
the same state bit for bit, in both forms, for a single simulation and for
a batch; in the FP64 form every shape stays on the oracle."""
import numpy as np
import pytest

from sphera_b200 import Batch, Simulation, abi, cases

pytestmark = pytest.mark.gpu

SHAPES = [dict(momentum_shape=0, continuity_shape=0),
          dict(momentum_shape=1, continuity_shape=0),
          dict(momentum_shape=0, continuity_shape=1),
          dict(momentum_shape=1, continuity_shape=1, lists=148, momentum=296, continuity=592),
          dict(momentum_shape=2, continuity_shape=1),
          dict(momentum_shape=2, continuity_shape=2)]


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP32C, abi.SPH_PREC_FP64], ids=["fp32c", "fp64"])
@pytest.mark.parametrize("dim", [2, 3])
def test_pair_loop_shapes_give_identical_states(dim, precision):
    make = (lambda: cases.dam_break_2d(dx=0.02, precision=precision)) if dim == 2 else \
        (lambda: cases.dam_break_3d(dx=0.02, precision=precision))
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
    assert got["momentum_shape"] in (0, 1, 2) and got["continuity_shape"] in (0, 1, 2)
    a.step(20)
    b = Batch(cs)
    b.upload()
    b.step(20)
    for i in range(len(cs)):
        assert np.array_equal(a.download(i).x, b.download(i).x)


def test_fp64_batched_shapes_stay_on_the_oracle(oracle_lib):
    """The FP64 form's batched pair loops: rates on an identical state and
    the state after 20 steps bit for bit as the lean loops give them, and
    the rates within the parity bar of the oracle."""
    case = cases.dam_break_3d(dx=0.02)
    o = oracle_lib.Oracle(case)
    o.prepare()
    sims = []
    for shape in (dict(momentum_shape=0, continuity_shape=0), dict(momentum_shape=1, continuity_shape=1)):
        sim = Simulation(case)
        sim.upload(case.state)
        sim.set_launch_shape(shape)
        sims.append(sim)
    acc = [s.rhs_momentum() for s in sims]
    dden = [s.continuity() for s in sims]
    assert np.array_equal(acc[0], acc[1]) and np.array_equal(dden[0], dden[1])
    o.rhs_momentum()
    o.continuity()
    ref = o.get()
    for a, d in zip(acc, dden):
        assert np.linalg.norm(a - ref["acc"]) <= 1e-12 * np.linalg.norm(ref["acc"])
        assert np.linalg.norm(d - ref["dden"]) <= 1e-12 * np.linalg.norm(ref["dden"])
    for s in sims:
        s.step(20)
    a, b = sims[0].download(), sims[1].download()
    assert np.array_equal(a.x, b.x) and np.array_equal(a.v, b.v) and np.array_equal(a.rho, b.rho)
