"""1st-order consistency (C1_BE / C1_divu) on the CPU: the oracle's
renormalisation matrices against their continuum values, the host-side
validation of the parameters, and the matrices' device memory."""
import numpy as np
import pytest

from sphera_b200 import SphError, abi, cases, memory_required


def c1_case(dx=0.04, divu=1, thresh=1.0e-3, **kw):
    case = cases.dam_break_3d(dx=dx, **kw)
    case.params.c1_be = 1
    case.params.c1_divu = divu
    case.params.invb_det_thresh = thresh
    return case


def interior(x, lo=(0.12, 0.1, 0.12), hi=(0.45, 0.2, 0.35)):
    return np.all((x > np.array(lo)) & (x < np.array(hi)), axis=1)


def test_oracle_fluid_matrices_are_minus_identity_inside(oracle_lib):
    """sum_j (x_j - x_i) grad W_ij V_j -> -I for a full kernel support."""
    case = c1_case(dx=0.02)
    o = oracle_lib.Oracle(case)
    o.prepare()
    bg, bd = o.get_c1()
    m = interior(o.get()["x"])
    assert m.sum() > 500
    eye = np.eye(3)
    # lattice sums of the two kernels at h = 1.3 dx: within a few per cent
    assert np.abs(bg[m] + eye).max() < 0.06
    assert np.abs(bd[m] + eye).max() < 0.03
    # symmetric on the lattice (up to rounding)
    assert np.abs(bg[m] - bg[m].transpose(0, 2, 1)).max() < 1e-10


def test_oracle_inverted_matrices_after_a_step(oracle_lib):
    case = c1_case(dx=0.02)
    o = oracle_lib.Oracle(case)
    o.prepare()
    raw_g, raw_d = o.get_c1()
    o.continuity()
    inv_g, inv_d = o.get_c1()
    m = interior(o.get()["x"])
    # the continuity pass leaves the inverses of the completed matrices;
    # inside, away from the walls, nothing is added to them
    prod = np.einsum("nij,njk->nik", inv_g[m], raw_g[m])
    assert np.abs(prod - np.eye(3)).max() < 1e-12
    prod = np.einsum("nij,njk->nik", inv_d[m], raw_d[m])
    assert np.abs(prod - np.eye(3)).max() < 1e-12


def test_oracle_singular_matrix_falls_back_to_minus_identity(oracle_lib):
    """|det| below invB_det_thresh gives -I (B_ren_gradp_inversion.f90)."""
    case = c1_case(dx=0.04, thresh=1.0e6)
    o = oracle_lib.Oracle(case)
    o.prepare()
    o.continuity()
    bg, bd = o.get_c1()
    assert np.array_equal(bg, np.broadcast_to(-np.eye(3), bg.shape))
    assert np.array_equal(bd, np.broadcast_to(-np.eye(3), bd.shape))


def test_oracle_minus_identity_fallback_equals_plain_form(oracle_lib):
    """With every matrix replaced by -I the renormalisation is the identity:
    the rates equal the plain form's bit for bit after the first step."""
    plain = cases.dam_break_3d(dx=0.04)
    ren = c1_case(dx=0.04, thresh=1.0e30)
    a = oracle_lib.Oracle(plain)
    b = oracle_lib.Oracle(ren)
    for o in (a, b):
        o.prepare()
        o.step(3)
    sa, sb = a.get(), b.get()
    assert np.array_equal(sa["x"], sb["x"])
    assert np.array_equal(sa["rho"], sb["rho"])


def c1_case_2d(dx=0.04, divu=1, thresh=1.0e-3, **kw):
    case = cases.dam_break_2d(dx=dx, **kw)
    case.params.c1_be = 1
    case.params.c1_divu = divu
    case.params.invb_det_thresh = thresh
    return case


def test_oracle_2d_matrices_are_singular_and_fall_back(oracle_lib):
    """2D: the x-z matrices (grad_W_sub's 2D factors 10/7 and 4/3) have a
    zero y row and column, so their determinant is zero and the inversion
    takes the -I fallback; renormalising with -I changes nothing, so the
    rates equal the plain form's."""
    case = c1_case_2d()
    o = oracle_lib.Oracle(case)
    o.prepare()
    bg, bd = o.get_c1()
    m = interior(o.get()["x"], lo=(0.15, -1.0, 0.15), hi=(0.85, 1.0, 1.85))
    assert m.sum() > 100
    # the fluid sums: y row and column zero, the x-z block near -I inside
    assert np.all(bg[:, 1, :] == 0.0) and np.all(bg[:, :, 1] == 0.0)
    sub = bg[m][:, ::2, ::2]
    assert np.abs(sub + np.eye(2)).max() < 0.15
    plain = cases.dam_break_2d(dx=0.04)
    p = oracle_lib.Oracle(plain)
    p.prepare()
    o.rhs_momentum()
    p.rhs_momentum()
    bg, _ = o.get_c1()
    assert np.all(bg == -np.eye(3))
    # the time loop's order: a search between the momentum and continuity
    # passes forms the fluid sums again, which the continuity pass completes
    # and inverts
    o.search()
    p.search()
    o.continuity()
    p.continuity()
    a, b = o.get(), p.get()
    assert np.array_equal(a["acc"], b["acc"])
    assert np.array_equal(a["dden"], b["dden"])
    bg, bd = o.get_c1()
    assert np.all(bg == -np.eye(3)) and np.all(bd == -np.eye(3))
    # whole steps from the IC (the time loop's order) equal the plain form's
    o2, p2 = oracle_lib.Oracle(case), oracle_lib.Oracle(plain)
    o2.prepare()
    p2.prepare()
    o2.step(20)
    p2.step(20)
    assert np.array_equal(o2.get()["x"], p2.get()["x"])
    assert np.array_equal(o2.get()["v"], p2.get()["v"])


def test_c1_in_2d_needs_a_positive_threshold():
    c2 = c1_case_2d(thresh=0.0)
    with pytest.raises(SphError) as e:
        memory_required([c2])
    assert e.value.code == abi.SPH_ERR_INVALID_ARGUMENT
    assert memory_required([c1_case_2d()]) > memory_required([cases.dam_break_2d(dx=0.04)])
    # both precision forms in 3D; the FP32c form with C1 holds three more
    # pair sums per particle
    c3 = c1_case(precision=abi.SPH_PREC_FP32C)
    plain = cases.dam_break_3d(dx=0.04, precision=abi.SPH_PREC_FP32C)
    assert memory_required([c3]) > memory_required([plain])


def test_c1_threshold_must_be_non_negative():
    case = c1_case(thresh=-1.0)
    with pytest.raises(SphError) as e:
        memory_required([case])
    assert e.value.code == abi.SPH_ERR_INVALID_ARGUMENT


def test_c1_matrices_memory():
    """9 doubles per slot for B_ren_gradp, 9 more with C1_divu; C1_divu
    alone does nothing (CalcVarLength.f90:285)."""
    base = memory_required([cases.dam_break_3d(dx=0.04)])
    g = memory_required([c1_case(divu=0)])
    gd = memory_required([c1_case(divu=1)])
    only_divu = cases.dam_break_3d(dx=0.04)
    only_divu.params.c1_divu = 1
    n = cases.dam_break_3d(dx=0.04).n
    slots = -(-n // 256) * 256
    assert g - base >= 72 * slots
    assert gd - g >= 72 * slots
    assert memory_required([only_divu]) == base


@pytest.mark.parametrize("thresh,blows_up", [(1.0e-3, True), (0.614, False)])
def test_oracle_dam_break_stability_depends_on_the_threshold(oracle_lib, thresh, blows_up):
    """The reference's input template warns that C1_BE is unstable when
    invB_det_thresh is too small; its tutorials with C1_BE use 0.614.  The 3D
    dam break at dx 0.02 shows both: at 1e-3 the time step collapses within
    300 steps (to about 5e-9 s), at 0.614 it stays at its initial size."""
    case = c1_case(dx=0.02, thresh=thresh)
    o = oracle_lib.Oracle(case, nthreads=8)
    o.prepare()
    dt0 = o.dt
    o.step(300)
    if blows_up:
        assert o.dt < 1.0e-3 * dt0
    else:
        assert o.dt > 0.5 * dt0 and o.removed == 0
