"""Checkpoint and resume on the device: a simulation saved between steps
(sph_download, sph_get_clock, sph_dump_laminar -> a snapshot file) and
loaded into a new handle (sph_upload, sph_set_clock) continues exactly as
the uninterrupted run, bit for bit, in both forms -- with the tank forcing,
whose body force depends on the clock, and with walls whose no-slip term
depends on the laminar flags the last momentum pass left."""
import numpy as np
import pytest

from sphera_b200 import Simulation, SphError, abi, cases, snapshot

pytestmark = pytest.mark.gpu


def laminar_walls(case):
    """No-slip walls that act only where the laminar flag is set, and a
    viscosity high enough (1e-2 m^2/s) for the Morris term to set it."""
    case.params.kin_visc = 1.0e-2
    z = abi.make_zone(slip=0.5, laminar_no_slip_check=1)
    if case.params.dim == 2:
        case.geometry = cases.tank_2d(*case.meta["tank"], zone=z)
    else:
        case.geometry = cases.tank_3d(*case.meta["tank"], zone=z)
    return case


CASES = {
    "dam_break_2d_fp64": lambda: laminar_walls(cases.dam_break_2d(dx=0.02)),
    "dam_break_3d_fp32c": lambda: laminar_walls(cases.dam_break_3d(dx=0.02, precision=abi.SPH_PREC_FP32C)),
    "sloshing_3d_fp64": lambda: cases.sloshing_3d(dx=0.04, amplitude=0.02, period=0.5),
}


@pytest.mark.parametrize("name", list(CASES))
def test_resume_continues_bit_for_bit(name, tmp_path):
    case = CASES[name]()
    first, second = 60, 40
    with Simulation(case) as a:
        a.upload(case.state)
        a.step(first)
        path = tmp_path / "ck.snap"
        snapshot.save(path, a)
        lam = a.dump_laminar()
        a.step(second)
        ref = a.download()
        ref_clock = a.clock()
    with snapshot.load(path) as b:
        assert b.clock()["step"] == first
        b.step(second)
        got = b.download()
        assert b.clock() == ref_clock
    for f in ("x", "v", "rho", "p"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    if name != "sloshing_3d_fp64":
        assert lam.any(), "no laminar flag set: the walls' no-slip term was not exercised"


def test_resume_rejects_c1_and_bad_clocks():
    case = cases.dam_break_3d(dx=0.04)
    case.params.c1_be = 1
    with Simulation(case) as s:
        s.upload(case.state)
        with pytest.raises(SphError) as e:
            s.set_clock({"time": 0.1, "dt": 1e-4, "dt_prev": 1e-4, "dt_average": 1e-4, "step": 10})
        assert e.value.code == abi.SPH_ERR_UNSUPPORTED
    case = cases.dam_break_2d(dx=0.05)
    with Simulation(case) as s:
        s.upload(case.state)
        with pytest.raises(SphError):
            s.set_clock({"time": 0.1, "dt": 0.0, "dt_prev": 1e-4, "dt_average": 1e-4, "step": 10})
