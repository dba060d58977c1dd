"""Convex boundary edges (FindBoundaryConvexEdges3D.f90 and the edge loop of
AddElasticBoundaryReaction_3D.f90:106-153) in the oracle, on the CPU: a box
tank with a block standing on its floor, and one particle placed just
outside the block's first convex edge, off both faces' projections."""
import numpy as np
import pytest

from sphera_b200 import abi, cases

SQ = 1.0 / np.sqrt(2.0)


def edge_case(speed=0.5, dist_frac=0.1, precision=abi.SPH_PREC_FP64):
    """The block tank plus a particle at dist_frac * dx from the block's
    edge y = 0.05, z = 0.1 (along x, between its top and its y = 0.05 side),
    diagonally outside it, moving toward the edge at `speed` (negative: away
    from it)."""
    base = cases.block_tank_3d(precision=precision)
    dx = base.params.dx
    d = dist_frac * dx
    xe = np.array([0.2, 0.05 - d * SQ, 0.1 + d * SQ])
    ve = speed * np.array([0.0, SQ, -SQ])
    st = base.state
    x = np.vstack([st.x, xe])
    v = np.vstack([st.v, ve])
    p, rho = cases._hydrostatic(np.append(st.x[:, 2], xe[2]), dx, base.params.den0, base.params.eps,
                                base.params.p_ref)
    p[:-1], rho[:-1] = st.p, st.rho
    m = np.append(st.m, st.m[0])
    new = abi.State(x, v, rho, p, m)
    return cases.Case(base.name, base.params, base.geometry, new), len(x) - 1


def test_block_tank_has_convex_edges(oracle_lib):
    case = cases.block_tank_3d()
    o = oracle_lib.Oracle(case)
    edges = o.convex_edges()
    # tank faces 1-6 meet at concave edges; the block's top (7) and sides
    # (8: y0, 9: y1, 10: x0, 11: x1) meet at convex ones, but the reference
    # records at most one edge per face, with the first later face that
    # shares one: top-y0, y0-x0, y1-x0
    assert edges.tolist() == [[7, 8], [8, 10], [9, 10]]


def test_edge_reaction_fires_for_an_approaching_particle(oracle_lib):
    case, i = edge_case(speed=0.5)
    o = oracle_lib.Oracle(case)
    o.prepare()
    o.rhs_momentum()
    acc = o.get()["acc"][i]
    # -c0^2 ln(zi / zimin) / zimin along the edge normal (-y, +z): thousands of m/s^2
    assert acc[2] > 1.0e4 and acc[1] < -1.0e4
    case2, i2 = edge_case(speed=-0.5)
    o2 = oracle_lib.Oracle(case2)
    o2.prepare()
    o2.rhs_momentum()
    acc2 = o2.get()["acc"][i2]
    assert abs(acc2[1]) < 1.0e3 and abs(acc2[2]) < 1.0e3
