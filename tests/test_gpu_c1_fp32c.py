"""The 1st-order consistency form (C1_BE, C1_divu; 3D) in the FP32-
compensated form, against the FP64 oracle, through the C ABI.

The renormalisation matrices, their frontier terms and their inversion stay
FP64 (the same code as the FP64 form), so they are bit-exact; the pair sums
they renormalise are compensated FP32 sums, so the rates meet the FP32c
form's bar, relative L2 1e-5, and the fields after fused steps its 1e-3."""
import numpy as np
import pytest

from sphera_b200 import Batch, Simulation, abi, cases

pytestmark = pytest.mark.gpu

RATE_TOL = 1e-5


def c1_case(precision, dx=0.04, divu=1, thresh=1.0e-3, **kw):
    case = cases.dam_break_3d(dx=dx, precision=precision, **kw)
    case.params.c1_be = 1
    case.params.c1_divu = divu
    case.params.invb_det_thresh = thresh
    return case


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _pair(case, oracle_lib):
    sim = Simulation(case)
    sim.upload(case.state)
    ref = c1_case(abi.SPH_PREC_FP64, divu=case.params.c1_divu)
    o = oracle_lib.Oracle(ref)
    o.prepare()
    return sim, o


@pytest.mark.parametrize("divu", [0, 1])
def test_matrices_bit_exact_and_rates(divu, oracle_lib):
    sim, o = _pair(c1_case(abi.SPH_PREC_FP32C, divu=divu), oracle_lib)
    bg, bd = sim.dump_renormalisation(divu=bool(divu))
    og, od = o.get_c1()
    assert np.array_equal(bg, og)
    if divu:
        assert np.array_equal(bd, od)
    # step-1 momentum: frontiers complete B_ren_gradp, inverted (FP64, exact)
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    assert rel_l2(acc, o.get()["acc"]) <= RATE_TOL
    bg, _ = sim.dump_renormalisation(divu=False)
    og, _ = o.get_c1()
    assert np.array_equal(bg, og)
    dden = sim.continuity()
    o.continuity()
    assert rel_l2(dden, o.get()["dden"]) <= RATE_TOL
    bg, bd = sim.dump_renormalisation(divu=bool(divu))
    og, od = o.get_c1()
    assert np.array_equal(bg, og)
    if divu:
        assert np.array_equal(bd, od)


def test_fields_follow_oracle(oracle_lib):
    sim, o = _pair(c1_case(abi.SPH_PREC_FP32C), oracle_lib)
    sim.step(40)
    o.step(40)
    g, s = sim.download(), o.get()
    assert rel_l2(g.x, s["x"]) <= 1e-3
    assert rel_l2(g.v, s["v"]) <= 1e-3
    assert rel_l2(g.rho - 1000.0, s["rho"] - 1000.0) <= 1e-3


def test_batch_member_with_c1_equals_alone():
    """A batch mixing a C1 member and a plain one (the C1 kernels sum the
    plain member exactly as the plain kernels do)."""
    a = c1_case(abi.SPH_PREC_FP32C, seed=1)
    plain = cases.dam_break_3d(dx=0.04, seed=2, precision=abi.SPH_PREC_FP32C)
    bt = Batch([a, plain])
    bt.upload()
    bt.step(15)
    for i, c in enumerate((a, plain)):
        s = Simulation(c)
        s.upload(c.state)
        s.step(15)
        assert np.array_equal(bt.download(i).x, s.download().x)
