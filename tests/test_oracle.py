"""CPU tests of the oracle (the FP64 restatement the CUDA path is checked
against): known answers derived from the reference's own sources, an
independent O(N^2) cross-check and conservation properties."""
import numpy as np
import pytest
from scipy import integrate

from sphera_b200 import abi, cases
from tests import naive

KS3D = 0.31830989          # JdWsRn.f90
PI = 3.14159265358979


def _small_box(n=1500, seed=7, grav=(0.0, 0.0, 0.0), dim=3):
    c = cases.random_box(n=n, spacing=0.01, seed=seed)
    c.params.grav = abi._d3(*grav)
    return c


def test_bit2d_table_is_single_precision(oracle_lib):
    """SA_SPH_module.f90:29-54 stores default-REAL literals in a double
    array: the table must hold their float32 roundings."""
    o = oracle_lib.Oracle(cases.dam_break_2d())
    _, _, b2 = o.tables()
    lit = np.array([-9.900000E-02, 6.916001E-01, 5.671769E-01, 1.614238E+00, 7.329450E-01, 8.813822E-01])
    assert np.array_equal(b2[0], lit.astype(np.float32).astype(np.float64))
    assert not np.array_equal(b2[0], lit)
    assert np.all(np.diff(b2[:, 0]) > 0.0999) and np.all(np.diff(b2[:, 0]) < 0.1001)
    assert np.all(b2[-1, 1:] == 0.0)


def _f(q):        # cubic beta-spline shape, w.f90 with the exact 2/3 and 1/6
    return np.where(q < 1, 1 - 1.5 * q ** 2 + 0.75 * q ** 3, np.where(q < 2, 0.25 * (2 - q) ** 3, 0.0))


def _df(q):
    return np.where(q < 1, -3 * q + 2.25 * q ** 2, np.where(q < 2, -0.75 * (2 - q) ** 2, 0.0))


@pytest.mark.parametrize("ro", [0.0, 0.3, 0.77, 1.0, 1.25, 1.9, 2.0])
def test_kernel_table_closed_forms(oracle_lib, ro):
    """IWro2dro.f90 and JdWsRn.f90 are closed forms of the integrals that
    ComputeKernelTable.f90 documents; compare with quadrature."""
    L = oracle_lib.lib()
    ref1 = integrate.quad(lambda q: _f(q) * q * q, ro, 2.0, points=[1.0], epsabs=1e-15, epsrel=1e-14)[0] / PI
    assert L.ora_IWro2dro(ro) == pytest.approx(ref1, rel=1e-12, abs=1e-15)
    for n in (1, 2, 3):
        refn = KS3D * integrate.quad(lambda q: _df(q) * q ** n, ro, 2.0, points=[1.0], epsabs=1e-15,
                                     epsrel=1e-14)[0]
        # JdWsRn is defined as minus the integral from ro to 2 (it returns the
        # integral from 0 to ro minus the total) -- check both sign conventions
        got = L.ora_JdWsRn(ro, n)
        assert got == pytest.approx(-refn, rel=1e-9, abs=1e-12) or got == pytest.approx(refn, rel=1e-9, abs=1e-12)


def test_kernel_normalisation():
    """coefke (Gest_Input.f90:279-289) normalises the beta spline: the
    truncated literal 0.477464 ~ 1.5/pi and 0.682093 ~ 1.5 * 10/(7 pi)."""
    assert 0.477464 == pytest.approx(1.5 / np.pi, rel=2e-6)
    assert 0.682093 == pytest.approx(1.5 * 10 / (7 * np.pi), rel=2e-6)
    vol3 = integrate.quad(lambda q: _f(q) * 4 * np.pi * q * q, 0, 2, points=[1.0])[0] / np.pi
    assert vol3 == pytest.approx(1.0, rel=1e-12)


def test_neighbour_lists_match_bruteforce(oracle_lib):
    c = _small_box()
    o = oracle_lib.Oracle(c)
    o.prepare()
    counts, lists = o.neighbours()
    _, _, nb = naive.pair_rates(c.params, c.state.x, c.state.v, c.state.rho, c.state.p, c.state.m)
    for i in range(c.n):
        got = sorted(lists[i, :counts[i]] - 1)
        exp = list(np.nonzero(nb[i])[0])
        assert got == exp
    # symmetry j in N(i) <=> i in N(j)
    assert np.array_equal(nb, nb.T)


def test_grid_arrays(oracle_lib):
    c = cases.dam_break_2d()
    o = oracle_lib.Oracle(c)
    o.prepare()
    cella, icont, npo = o.grid()
    assert icont[0] == 1 and icont[-1] == c.n + 1
    cnt = np.diff(icont)
    assert np.array_equal(np.bincount(cella, minlength=len(icont))[1:len(icont)], cnt)
    # NPartOrd is a permutation, sorted by cell then by particle index
    assert np.array_equal(np.sort(npo), np.arange(1, c.n + 1))
    key = cella[npo - 1].astype(np.int64) * (c.n + 1) + npo
    assert np.all(np.diff(key) > 0)


@pytest.mark.parametrize("dim", [3])
def test_oracle_rates_match_naive(oracle_lib, dim):
    c = _small_box(grav=(0.0, 0.0, -9.81))
    o = oracle_lib.Oracle(c)
    o.prepare()
    o.rhs_momentum()
    o.continuity()
    s = o.get()
    dden, acc, _ = naive.pair_rates(c.params, c.state.x, c.state.v, c.state.rho, c.state.p, c.state.m)
    # summation-order tolerance, normwise
    assert np.linalg.norm(s["dden"] - dden) <= 1e-12 * np.linalg.norm(dden)
    assert np.linalg.norm(s["acc"] - acc) <= 1e-12 * np.linalg.norm(acc)


def test_momentum_conservation_without_walls(oracle_lib):
    """Pair forces are antisymmetric: sum m a = 0 without walls and gravity."""
    c = _small_box()
    o = oracle_lib.Oracle(c)
    o.prepare()
    o.rhs_momentum()
    s = o.get()
    tot = (s["m"][:, None] * s["acc"]).sum(0)
    scale = (s["m"][:, None] * np.abs(s["acc"])).sum(0)
    assert np.all(np.abs(tot) <= 1e-12 * scale.max())


def test_hydrostatic_column_interior_at_rest(oracle_lib):
    """A still column (dam break before release): in the interior the SPH
    pressure gradient carries most of the weight (without it every particle
    would accelerate at -g); the jitter of +-0.01 dx leaves a per-particle
    scatter of a few m/s^2 with the stiff EoS."""
    c = cases.dam_break_2d()
    o = oracle_lib.Oracle(c)
    o.prepare()
    o.rhs_momentum()
    o.continuity()
    s = o.get()
    x = s["x"]
    interior = (x[:, 0] > 0.1) & (x[:, 0] < 0.8) & (x[:, 2] > 0.1) & (x[:, 2] < 1.8)
    assert np.all(s["dden"] == 0.0)                 # at rest: no velocity divergence
    assert abs(np.mean(s["acc"][interior, 2])) < 0.25 * 9.81
    assert abs(np.mean(s["acc"][interior, 0])) < 0.25 * 9.81


def test_steps_advance_time(oracle_lib):
    c = cases.dam_break_2d()
    o = oracle_lib.Oracle(c)
    o.prepare()
    dt0 = o.dt
    assert dt0 == pytest.approx(0.1 * 2 * 0.026 / 40.0, rel=1e-12)   # CFL 2h / c at rest
    o.step(5)
    assert 0.98 * 5 * dt0 <= o.time <= 5 * dt0 * (1 + 1e-12)   # dt shrinks as the column starts to move
    s = o.get()
    assert np.all(np.isfinite(s["x"]))
    assert s["v"][:, 0].max() > 0.0


def test_tank_forcing_is_a_lateral_body_force(oracle_lib):
    """The sloshing tank's forcing adds A w^2 sin(w t) to the x acceleration
    of every particle (t: the end time of the step being computed, here the
    first step's) and leaves y and z untouched; zero amplitude is plain
    gravity."""
    A, T = 0.02, 0.8
    base = _small_box(grav=(0.0, 0.0, -9.81))
    forced = _small_box(grav=(0.0, 0.0, -9.81))
    forced.params.forcing_amplitude = A
    forced.params.forcing_period = T
    out = []
    for c in (base, forced):
        o = oracle_lib.Oracle(c)
        o.prepare()
        o.rhs_momentum()
        out.append((o.get()["acc"], o.dt))
    (a0, dt0), (a1, dt1) = out
    assert dt0 == dt1
    w = 2.0 * np.pi / T
    expect = A * w * w * np.sin(w * dt0)
    scale = np.abs(a0).max()
    assert np.all(np.abs((a1[:, 0] - a0[:, 0]) - expect) <= 1e-13 * scale)
    assert np.array_equal(a1[:, 1:], a0[:, 1:])


def test_forcing_sine_matches_libm(oracle_lib):
    """The forcing's own sine (range reduction by the nearest multiple of
    2 pi, Taylor series; the same IEEE sequence on host and device) against
    libm over phases well beyond what a run reaches."""
    x = np.concatenate([np.linspace(-200.0, 200.0, 40001), np.pi * np.arange(-64, 65) / 4.0])
    got = np.array([oracle_lib.forcing_sin(v) for v in x])
    assert np.all(np.abs(got - np.sin(x)) <= 1e-15 * (1.0 + np.abs(x)))


def test_velocity_smoothing_keeps_a_uniform_flow(oracle_lib):
    """Partial smoothing pulls each particle towards its neighbourhood mean:
    after one step of a box moving as a whole (no walls, no gravity, the
    density jitter the only disturbance) the pressure field has a smaller
    spread with TetaP = TetaV = 0.5 than without smoothing, and the mean
    velocity is kept."""
    c = _small_box(n=1500, grav=(0.0, 0.0, 0.0))
    c.state.v[:] = np.array([0.3, -0.1, 0.2])
    c.params.teta_v = 0.5
    c.params.teta_p = 0.5
    o = oracle_lib.Oracle(c)
    o.prepare()
    s0 = o.get()
    o.step(1)
    s1 = o.get()
    assert np.all(np.isfinite(s1["x"])) and np.all(np.isfinite(s1["p"]))
    # the pressure field is smoother after a smoothed step than after a plain one
    c2 = _small_box(n=1500, grav=(0.0, 0.0, 0.0))
    c2.state.v[:] = np.array([0.3, -0.1, 0.2])
    o2 = oracle_lib.Oracle(c2)
    o2.prepare()
    o2.step(1)
    s2 = o2.get()
    assert np.std(s1["p"]) < np.std(s2["p"])
    assert np.allclose(s1["v"].mean(0), s2["v"].mean(0), rtol=0, atol=1e-3)
    assert s0["p"].shape == s1["p"].shape


def test_smoothed_dam_break_runs(oracle_lib):
    """TetaP = TetaV = 0.2 (the tutorial decks' values) on the 2D dam break."""
    c = cases.dam_break_2d(dx=0.04)
    c.params.teta_v = 0.2
    c.params.teta_p = 0.2
    o = oracle_lib.Oracle(c)
    o.prepare()
    o.step(20)
    s = o.get()
    assert np.all(np.isfinite(s["x"])) and np.all(np.isfinite(s["v"]))
    assert s["v"][:, 0].max() > 0.0
