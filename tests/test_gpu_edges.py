"""Edge cases of the path on the device, each against the oracle or the
reference's documented behaviour: particles outside the grid (OrdGrid1's
swap-with-last removal), the NMAXPARTJ cap (truncated lists and the
warning), an overflowing boundary-data pool (diagnostic 8/2), an empty
state and a batch member without particles."""
import numpy as np
import pytest

from sphera_b200 import Batch, SphError, Simulation, abi, cases

pytestmark = pytest.mark.gpu


def _with_outsiders(case, k=7, seed=3):
    """Moves k particles of the case far outside the grid."""
    rng = np.random.default_rng(seed)
    st = case.state
    x = st.x.copy()
    idx = rng.choice(len(x), size=k, replace=False)
    x[idx, 0] = case.params.domain_hi[0] + 5.0
    new = abi.State(x, st.v, st.rho, st.p, st.m)
    return cases.Case(case.name, case.params, case.geometry, new), np.sort(idx)


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
def test_out_of_grid_particles_are_removed_like_oracle(precision, oracle_lib):
    base = cases.dam_break_2d(dx=0.04, precision=precision)
    case, idx = _with_outsiders(base)
    sim = Simulation(case)
    sim.upload(case.state)
    d = sim.diagnostics()
    o = oracle_lib.Oracle(case)
    o.prepare()
    assert d.removed_out_of_grid == o.removed == len(idx)
    assert d.warnings & abi.SPH_WARN_PARTICLES_REMOVED
    g = sim.download()
    s = o.get()
    assert g.n == o.n == case.n - len(idx)
    # the survivors in the reference's swap-with-last order
    assert np.array_equal(g.x, s["x"])
    assert np.array_equal(g.m, s["m"])
    if precision == abi.SPH_PREC_FP64:
        sim.step(20)
        o.step(20)
        assert np.linalg.norm(sim.download().x - o.get()["x"]) <= 1e-12 * np.linalg.norm(o.get()["x"])


def test_neighbour_cap_truncates_like_oracle(oracle_lib):
    case = cases.dam_break_3d(dx=0.04)
    case.params.coef_nmaxpartj = 0.3        # NMAXPARTJ 43, below the ~78 accepted
    sim = Simulation(case)
    sim.upload(case.state)
    o = oracle_lib.Oracle(case)
    o.prepare()
    nm = o.nmaxpartj
    assert nm == sim.diagnostics().nmaxpartj < 78
    assert o.truncated > 0
    assert sim.diagnostics().warnings & abi.SPH_WARN_NEIGHBOURS_TRUNCATED
    gc, gl = sim.dump_neighbours(nm)
    oc, ol = o.neighbours(nm)
    assert np.array_equal(gc, oc)
    assert np.array_equal(gl, ol)


def test_boundary_pool_overflow_is_reported():
    case = cases.dam_break_3d(dx=0.04)
    case.params.bdt_capacity = 16
    sim = Simulation(case)
    with pytest.raises(SphError) as e:
        sim.upload(case.state)
    assert e.value.code == abi.SPH_ERR_BDT_OVERFLOW


def test_empty_state_steps():
    case = cases.dam_break_2d(dx=0.04)
    sim = Simulation(case)
    empty = abi.State.empty(0)
    sim.upload(empty)
    info = sim.step(3)
    assert info.n == 0
    assert sim.download().n == 0


def test_batch_with_an_empty_member():
    a = cases.dam_break_2d(dx=0.04, seed=1)
    b = cases.dam_break_2d(dx=0.04, seed=2)
    bt = Batch([a, b])
    bt.upload([a.state, abi.State.empty(0)])
    bt.step(10)
    alone = Simulation(a)
    alone.upload(a.state)
    alone.step(10)
    assert np.array_equal(bt.download(0).x, alone.download().x)
    assert bt.download(1).n == 0
