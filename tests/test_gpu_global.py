"""fluid_global_quantities.f90:59-72 on the device: FP64 sums of mass,
linear momentum, angular momentum about the origin and volume, against
the oracle's sequential sums in pg order and against exactly rounded sums
(math.fsum) of the same terms.  The device sums are compensated, so they
agree with the exact sums to a few ulps; the oracle's plain sequential sums
carry their own rounding, bounded here by 1e-12 of the sum of magnitudes."""
import math

import numpy as np
import pytest

from sphera_b200 import Batch, Simulation, abi, cases

pytestmark = pytest.mark.gpu


def terms(st):
    m = st.m
    x, v = st.x, st.v
    ang = np.stack([x[:, 1] * v[:, 2] - x[:, 2] * v[:, 1],
                    x[:, 2] * v[:, 0] - x[:, 0] * v[:, 2],
                    x[:, 0] * v[:, 1] - x[:, 1] * v[:, 0]], axis=1)
    cols = [m] + [m * v[:, d] for d in range(3)] + [m * ang[:, d] for d in range(3)] + [m / st.rho]
    return np.stack(cols, axis=1)


def exact_sums(st):
    t = terms(st)
    return np.array([math.fsum(t[:, k]) for k in range(8)]), np.abs(t).sum(axis=0)


@pytest.mark.parametrize("name,nsteps", [("dam_break_2d", 150), ("dam_break_3d", 40)])
@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_global_quantities(name, nsteps, precision, oracle_lib):
    case = (cases.dam_break_2d(precision=precision) if name == "dam_break_2d"
            else cases.dam_break_3d(dx=0.02, precision=precision))
    sim = Simulation(case)
    sim.upload(case.state)
    g0 = sim.global_quantities()
    ex0, mag0 = exact_sums(case.state)
    assert np.all(np.abs(g0 - ex0) <= 4e-16 * mag0 + 1e-300)
    sim.step(nsteps)
    st = sim.download()
    g = sim.global_quantities()
    ex, mag = exact_sums(st)
    assert np.all(np.abs(g - ex) <= 4e-16 * mag + 1e-300)
    # the oracle's sequential FP64 sums over the same state
    c2 = cases.Case(case.name, case.params, case.geometry, st)
    o = oracle_lib.Oracle(c2)
    ref = o.global_quantities()
    assert np.all(np.abs(g - ref) <= 1e-12 * mag + 1e-300)
    # mass is carried unchanged by every step
    assert g[0] == g0[0]
    # the fluid has started to fall: momentum along gravity is negative
    assert g[3] < 0.0


def test_global_quantities_of_batch_members_equal_alone():
    a = cases.dam_break_2d(dx=0.04, seed=1)
    b = cases.dam_break_2d(dx=0.04, seed=2, column=(0.6, 1.2))
    bt = Batch([a, b])
    bt.upload()
    bt.step(20)
    gb = bt.global_quantities()
    for i, c in enumerate((a, b)):
        s = Simulation(c)
        s.upload(c.state)
        s.step(20)
        assert np.array_equal(gb[i], s.global_quantities())
