"""sph_step_download against sph_step followed by sph_download: the same
state, bit for bit, in both forms, including a step that removes a particle
leaving the grid (the count returned drops and the surviving rows match)."""
import numpy as np
import pytest

from sphera_b200 import Simulation, abi, cases

pytestmark = pytest.mark.gpu

FIELDS = ("x", "v", "rho", "p", "m")


def _pair(case):
    a = Simulation(case)
    a.upload(case.state)
    b = Simulation(case)
    b.upload(case.state)
    return a, b


def _same(sa, sb):
    assert sa.n == sb.n
    for f in FIELDS:
        assert np.array_equal(getattr(sa, f), getattr(sb, f)), f


@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C])
@pytest.mark.parametrize("dim", [2, 3])
def test_step_download_equals_step_then_download(dim, precision):
    case = (cases.dam_break_3d if dim == 3 else cases.dam_break_2d)(dx=0.04, precision=precision)
    a, b = _pair(case)
    for nsteps in (1, 4):
        a.step(nsteps)
        _same(a.download(), b.step_download(nsteps))


def test_step_download_zero_steps_is_a_download():
    case = cases.dam_break_2d(dx=0.04)
    a, b = _pair(case)
    _same(a.download(), b.step_download(0))


def test_step_download_through_a_removal():
    """A particle launched out of the grid: the step that removes it returns
    the lower count, and every surviving row equals the two-call path's."""
    base = cases.dam_break_2d(dx=0.04)
    st = base.state
    h = base.params.dx * base.params.trunc
    x, v = st.x.copy(), st.v.copy()
    x[0] = [base.params.domain_hi[0] + h, 0.0, 0.5 * base.params.domain_hi[2]]
    v[0] = [40.0, 0.0, 0.0]
    case = cases.Case(base.name, base.params, base.geometry, abi.State(x, v, st.rho, st.p, st.m))
    probe = Simulation(case)
    probe.upload(case.state)
    n0 = probe.n
    k = 0
    while k < 200:
        k += 1
        if probe.step(1).n < n0:
            break
    assert probe.step_download(0).n == n0 - 1, "the particle never left the grid"
    a, b = _pair(case)
    a.step(k)
    sa = a.download()
    sb = b.step_download(k)
    assert sb.n == n0 - 1
    _same(sa, sb)
