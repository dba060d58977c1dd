"""Wall-near and diagnostic branches of the momentum pass against the oracle,
through the C ABI: the elastic wall reaction of
AddElasticBoundaryReaction_3D.f90:67-105 / _2D.f90:63-97 (a particle closer
than 0.25 dx to a wall and approaching it) and pg%laminar_flag of
inter_EqMoto.f90:269-283."""
import numpy as np
import pytest

from sphera_b200 import Simulation, abi, cases

pytestmark = pytest.mark.gpu

RATE_TOL = 1e-12


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _near_floor(case, k=3, frac=0.1, vz=-0.3):
    """Moves the k lowest particles to frac * dx above the floor (z = 0)
    with a downward velocity: inside the reaction band of the floor."""
    st = case.state
    x, v = st.x.copy(), st.v.copy()
    low = np.argsort(x[:, 2], kind="stable")[:k * 7:7]     # spread along the floor
    x[low, 2] = frac * case.params.dx
    v[low, 2] = vz
    new = abi.State(x, v, st.rho, st.p, st.m)
    return cases.Case(case.name, case.params, case.geometry, new), low


@pytest.mark.parametrize("name", ["dam_break_2d", "dam_break_3d"])
@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_elastic_reaction_follows_oracle(name, precision, oracle_lib):
    base = (cases.dam_break_2d(dx=0.04, precision=precision) if name == "dam_break_2d"
            else cases.dam_break_3d(dx=0.04, precision=precision))
    case, low = _near_floor(base)
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    ref = o.get()["acc"]
    # the reaction fired: c0^2 ln((h + zi - zimin) / h) / h is thousands of m/s^2
    assert np.all(ref[low, 2] > 1000.0)
    tol = RATE_TOL if precision == abi.SPH_PREC_FP64 else 1e-5
    assert rel_l2(acc, ref) <= tol
    assert rel_l2(acc[low], ref[low]) <= tol


def test_elastic_reaction_needs_an_approaching_particle(oracle_lib):
    """Receding (v . n > 0) inside the band: no reaction, as the reference's
    `vin < zero` test."""
    case, low = _near_floor(cases.dam_break_3d(dx=0.04), vz=+0.3)
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    ref = o.get()["acc"]
    assert np.all(np.abs(ref[low, 2]) < 1000.0)
    assert rel_l2(acc, ref) <= RATE_TOL


def _viscous_box(kin_visc):
    case = cases.random_box(n=20000, seed=11)
    case.params.kin_visc = kin_visc
    return case


def test_laminar_flag_matches_oracle(oracle_lib):
    """pg%laminar_flag: 1 where the Morris term exceeds 5% of the pressure
    term plus g.  The viscosity is chosen on the oracle so that both values
    occur; the device's flags must equal the oracle's one for one."""
    for nu in (1e-3, 3e-3, 1e-2, 3e-2, 1e-1):
        case = _viscous_box(nu)
        o = oracle_lib.Oracle(case)
        o.prepare()
        o.rhs_momentum()
        ref = o.laminar()
        if 0.05 < ref.mean() < 0.95:
            break
    assert 0.05 < ref.mean() < 0.95
    sim = Simulation(case)
    sim.upload(case.state)
    sim.rhs_momentum(want=False)
    assert np.array_equal(sim.dump_laminar(), ref)
    # the fused step's flags: the oracle after one whole step
    sim.step(1)
    o.step(1)
    assert np.array_equal(sim.dump_laminar(), o.laminar())


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_convex_edge_reaction_follows_oracle(precision, oracle_lib):
    """A block standing in the tank gives the boundary convex edges
    (FindBoundaryConvexEdges3D.f90); a particle just outside the first one,
    off both faces' projections and approaching it, gets the edge reaction
    of AddElasticBoundaryReaction_3D.f90:106-153."""
    from .test_convex_edges import edge_case
    case, i = edge_case(precision=precision)
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    acc = sim.rhs_momentum()
    o.rhs_momentum()
    ref = o.get()["acc"]
    assert ref[i, 2] > 1.0e4
    tol = RATE_TOL if precision == abi.SPH_PREC_FP64 else 1e-5
    assert rel_l2(acc, ref) <= tol
    assert rel_l2(acc[i], ref[i]) <= tol
    if precision == abi.SPH_PREC_FP64:
        # whole steps on the non-box geometry follow the oracle too
        sim.step(30)
        o.step(30)
        assert rel_l2(sim.download().x, o.get()["x"]) <= 1e-12
