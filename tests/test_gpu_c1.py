"""GPU parity of the 1st-order consistency form (C1_BE, C1_divu; 3D, FP64)
against the oracle, through the C ABI.

Bars: the renormalisation matrices and the rates bit-exact on the same
state (the FP64 form keeps the reference's operation order); positions
after fused steps within relative L2 1e-12."""
import numpy as np
import pytest

from sphera_b200 import Batch, SphError, Simulation, abi, cases

pytestmark = pytest.mark.gpu


def c1_case(dx=0.04, divu=1, thresh=1.0e-3, **kw):
    case = cases.dam_break_3d(dx=dx, **kw)
    case.params.c1_be = 1
    case.params.c1_divu = divu
    case.params.invb_det_thresh = thresh
    return case


def make_pair(case, oracle_lib):
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    return sim, o


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("divu", [0, 1])
def test_fluid_matrices_bit_exact(divu, oracle_lib):
    sim, o = make_pair(c1_case(divu=divu), oracle_lib)
    bg, bd = sim.dump_renormalisation(divu=bool(divu))
    og, od = o.get_c1()
    assert np.array_equal(bg, og)
    if divu:
        assert np.array_equal(bd, od)


def test_first_step_momentum_bit_exact(oracle_lib):
    """The momentum of step 1 completes B_ren_gradp with the frontiers and
    inverts it (AddBoundaryContributions_to_ME3D.f90:172-187, 314-317)."""
    sim, o = make_pair(c1_case(), oracle_lib)
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    assert np.array_equal(acc, o.get()["acc"])
    bg, _ = sim.dump_renormalisation()
    og, _ = o.get_c1()
    assert np.array_equal(bg, og)


@pytest.mark.parametrize("divu", [0, 1])
def test_continuity_bit_exact(divu, oracle_lib):
    sim, o = make_pair(c1_case(divu=divu), oracle_lib)
    dden = sim.continuity()
    o.continuity()
    assert np.array_equal(dden, o.get()["dden"])
    bg, bd = sim.dump_renormalisation(divu=bool(divu))
    og, od = o.get_c1()
    assert np.array_equal(bg, og)
    if divu:
        assert np.array_equal(bd, od)


@pytest.mark.parametrize("divu", [0, 1])
def test_fused_steps_match_oracle(divu, oracle_lib):
    case = c1_case(divu=divu)
    sim, o = make_pair(case, oracle_lib)
    sim.step(15)
    o.step(15)
    g, s = sim.download(), o.get()
    assert rel_l2(g.x, s["x"]) <= 1e-12
    assert rel_l2(g.rho, s["rho"]) <= 1e-12
    # the momentum of a later step uses the inverses the continuity pass left
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    assert rel_l2(acc, o.get()["acc"]) <= 1e-12


def test_renormalisation_changes_the_flow(oracle_lib):
    plain = cases.dam_break_3d(dx=0.04)
    ren = c1_case()
    a = Simulation(plain)
    a.upload(plain.state)
    b = Simulation(ren)
    b.upload(ren.state)
    a.step(10)
    b.step(10)
    assert not np.array_equal(a.download().x, b.download().x)


def test_minus_identity_fallback_equals_plain_form():
    plain = cases.dam_break_3d(dx=0.04)
    ren = c1_case(thresh=1.0e30)
    a = Simulation(plain)
    a.upload(plain.state)
    b = Simulation(ren)
    b.upload(ren.state)
    a.step(5)
    b.step(5)
    assert np.array_equal(a.download().x, b.download().x)
    assert np.array_equal(a.download().rho, b.download().rho)


def test_batch_mixes_c1_and_plain_members():
    a = c1_case(seed=1)
    p = cases.dam_break_3d(dx=0.04, seed=2)
    bt = Batch([a, p])
    bt.upload([a.state, p.state])
    bt.step(8)
    for case, k in ((a, 0), (p, 1)):
        alone = Simulation(case)
        alone.upload(case.state)
        alone.step(8)
        assert np.array_equal(bt.download(k).x, alone.download().x)


def test_autotune_keeps_the_matrices():
    case = c1_case()
    sim = Simulation(case)
    sim.upload(case.state)
    before = sim.dump_renormalisation()
    sim.autotune(reps=1)
    after = sim.dump_renormalisation()
    assert np.array_equal(before[0], after[0])
    assert np.array_equal(before[1], after[1])


def test_c1_in_2d_is_unsupported():
    case = cases.dam_break_2d(dx=0.04)
    case.params.c1_be = 1
    case.params.invb_det_thresh = 1.0e-3
    with pytest.raises(SphError) as e:
        Simulation(case)
    assert e.value.code == abi.SPH_ERR_UNSUPPORTED
