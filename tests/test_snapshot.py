"""Snapshot files on the CPU: what write() stores, read() gives back, array
for array and field for field; a file that is not a snapshot is refused."""
import numpy as np
import pytest

from sphera_b200 import abi, cases, snapshot


def test_round_trip(tmp_path):
    c = cases.dam_break_3d(dx=0.05)
    geo = cases.tank_with_block_3d(1.6, 0.6, 0.6, (1.0, 1.2, 0.1, 0.3, 0.1),
                                   zone=abi.make_zone(velocity=(0.1, 0.0, 0.0), slip=0.5, laminar_no_slip_check=1))
    rng = np.random.Generator(np.random.PCG64(3))
    lam = rng.integers(0, 2, c.n).astype(np.int32)
    clock = {"time": 0.0123456789, "dt": 2.5e-5, "dt_prev": 2.6e-5, "dt_average": 2.55e-5, "step": 421}
    path = tmp_path / "a.snap"
    snapshot.write(path, c.params, geo, c.state, clock, lam)
    d = snapshot.read(path)
    for f in ("x", "v", "rho", "p", "m"):
        assert np.array_equal(getattr(d["state"], f), getattr(c.state, f)), f
    assert np.array_equal(d["laminar"], lam)
    assert d["clock"] == clock
    for name, _ in abi.SphParams._fields_:
        a, b = getattr(d["params"], name), getattr(c.params, name)
        assert (list(a) == list(b)) if hasattr(a, "__len__") else a == b, name
    g = d["geometry"]
    assert np.array_equal(g.vertices, geo.vertices)
    assert np.array_equal(g.faces, geo.faces) and np.array_equal(g.face_zone, geo.face_zone)
    assert g.sides is None
    z0, z1 = g.zones[0], geo.zones[0]
    assert (z0.type, z0.slip_coefficient_mode, list(z0.velocity), z0.bc_shear_stress_input,
            z0.laminar_no_slip_check) == (z1.type, z1.slip_coefficient_mode, list(z1.velocity),
                                          z1.bc_shear_stress_input, z1.laminar_no_slip_check)


def test_2d_geometry_and_no_laminar(tmp_path):
    c = cases.dam_break_2d(dx=0.1)
    clock = {"time": 0.0, "dt": 1e-4, "dt_prev": 1e-4, "dt_average": 1e-4, "step": 0}
    path = tmp_path / "b.snap"
    snapshot.write(path, c.params, c.geometry, c.state, clock)
    d = snapshot.read(path)
    assert d["laminar"] is None
    assert np.array_equal(d["geometry"].sides, c.geometry.sides)
    assert d["geometry"].faces is None
    assert np.array_equal(d["state"].x, c.state.x)


def test_not_a_snapshot(tmp_path):
    p = tmp_path / "junk"
    p.write_bytes(b"NOTASNAP" + b"\0" * 64)
    with pytest.raises(ValueError):
        snapshot.read(p)
    c = cases.dam_break_2d(dx=0.1)
    clock = {"time": 0.0, "dt": 1e-4, "dt_prev": 1e-4, "dt_average": 1e-4, "step": 0}
    q = tmp_path / "t.snap"
    snapshot.write(q, c.params, c.geometry, c.state, clock)
    raw = q.read_bytes()
    q.write_bytes(raw[:-64])
    with pytest.raises(ValueError):
        snapshot.read(q)
