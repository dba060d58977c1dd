"""Parity at full size, through the C ABI, FP64 form against the oracle:

  * the 3D dam break of the headline workload (tank 1.6 x 0.6 x 0.6 m,
    block 0.6 x 0.3 x 0.6 m, dx 0.005 m, 864,000 particles): pg%cella,
    Icont, NPartOrd and the neighbour lists bit-exact, drho/dt and dv/dt on
    the identical state within 1e-12 (relative L2);
  * a 1,000,000-particle slice of the neighbour-search microbenchmark
    (uniform random cube at mean spacing 0.01 m, rho = 1000 (1 + N(0, 1e-3)),
    v ~ N(0, 0.1) m/s): the same bars, and the FP32c form's neighbour sets
    identical to the FP64 form's.

These are the sizes where the FP32 screening band of the list pass meets
large grid extents and cell indices."""
import numpy as np
import pytest

from sphera_b200 import Simulation, abi, cases

pytestmark = pytest.mark.gpu

RATE_TOL = 1e-12


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _check_case(case, oracle_lib):
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    cella, icont, npo = sim.dump_grid()
    rc, ri, rn = o.grid()
    assert np.array_equal(cella, rc)
    assert np.array_equal(icont, ri)
    assert np.array_equal(npo, rn)
    del cella, icont, npo, rc, ri, rn
    nm = o.nmaxpartj
    gc, gl = sim.dump_neighbours(nm)
    oc, ol = o.neighbours(nm)
    assert np.array_equal(gc, oc)
    assert np.array_equal(gl, ol)
    del gl, ol
    acc = sim.rhs_momentum()
    dden = sim.continuity()
    o.rhs_momentum()
    o.continuity()
    s = o.get()
    assert rel_l2(acc, s["acc"]) <= RATE_TOL
    assert rel_l2(dden, s["dden"]) <= RATE_TOL
    sim.close()
    o.close()
    return gc


def test_full_size_dam_break_3d(oracle_lib):
    case = cases.dam_break_3d()
    assert case.n == 864000
    counts = _check_case(case, oracle_lib)
    assert counts.mean() > 60


def test_random_box_1m_slice(oracle_lib):
    case = cases.random_box(n=1_000_000, seed=0xC2)
    counts = _check_case(case, oracle_lib)
    assert 65 < counts.mean() < 85
    # the FP32c form screens with its FP32 copies: identical neighbour sets
    c32 = cases.random_box(n=1_000_000, seed=0xC2, precision=abi.SPH_PREC_FP32C)
    s32 = Simulation(c32)
    s32.upload(c32.state)
    s64 = Simulation(case)
    s64.upload(case.state)
    nm = s64.diagnostics().nmaxpartj
    a, la = s32.dump_neighbours(nm)
    b, lb = s64.dump_neighbours(nm)
    assert np.array_equal(a, b)
    assert np.array_equal(la, lb)
