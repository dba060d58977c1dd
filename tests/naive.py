"""An independent O(N^2) numpy statement of the fluid-fluid pair terms.

It uses no cells and no neighbour order: every particle pair within 2h is
visited through a dense distance matrix.  It checks the oracle's
restatement of CalcVarLength.f90:223-269 (kernel values),
Continuity_Equation.f90:123-235 and inter_EqMoto.f90:195-254 with
viscomon.f90 / viscomorris.f90 for configurations without walls, to a
summation-order tolerance.
"""
import numpy as np


def constants(prm):
    dim = prm.dim
    h = prm.dx * prm.trunc
    hp = h ** 3 if dim == 3 else h ** 2
    coefke = (0.477464 if dim == 3 else 0.682093) / hp
    coefkacl = (0.074603 if dim == 3 else 0.099472) / hp
    return dict(h=h, eta=1e-3 * h, eta2=1e-2 * h * h, ke=coefke / h, kacl=coefkacl / h,
                c=np.sqrt(prm.eps / prm.den0))


def pair_rates(prm, x, v, rho, p, m):
    """Returns (dden, acc, neighbour boolean matrix) without walls."""
    k = constants(prm)
    h = k["h"]
    d = x[:, None, :] - x[None, :, :]            # rag = x_i - x_j
    r2 = (d ** 2).sum(-1)
    nb = r2 <= (2 * h) ** 2
    r = np.sqrt(r2)
    q = r / h
    q2 = r2 / (h * h)
    denom = 1.0 / (r + k["eta"])
    inner = q < 1.0
    grad = np.where(inner, -2 * q + 1.5 * q2, 2 * q - 0.5 * q2 - 2.0)
    grad = np.where(q < 2.0, grad, 0.0)
    gwacl = np.where(q < 2.0, -12.0 - 3.0 * q2 + 12.0 * q, 0.0)
    PK1 = grad * k["ke"] * denom
    PK2 = PK1 / (r2 + k["eta2"])
    PK3 = gwacl * k["kacl"] * denom
    PK1 = np.where(nb, PK1, 0.0)
    PK2 = np.where(nb, PK2, 0.0)
    PK3 = np.where(nb, PK3, 0.0)
    np.fill_diagonal(PK1, 0.0)
    np.fill_diagonal(PK2, 0.0)
    np.fill_diagonal(PK3, 0.0)
    dv = v[None, :, :] - v[:, None, :]           # v_j - v_i
    ri, rj = rho[:, None], rho[None, :]
    pi, pj = p[:, None], p[None, :]
    mj = m[None, :]
    # continuity: drho_i/dt = - sum_j rho_i m_j/rho_j PK1 (dv . rag)
    dden = -(ri * (mj / rj) * PK1 * (dv * d).sum(-1)).sum(1)
    # pressure: symmetric sum of the two accumulators of inter_EqMoto
    coef = -(mj * ((pj - pi) / (ri * rj) + (pi * (rj / ri + 1) + pj * (ri / rj - 1)) / (ri * rj)) * PK3)
    tpres = (coef[..., None] * d).sum(1)
    vr = -(dv * d).sum(-1)
    term_mon = prm.alfa_mon * (2 * k["c"]) * h / (ri + rj)
    tdiss = ((mj * term_mon * vr * PK2)[..., None] * d).sum(1)
    nu = prm.kin_visc
    if nu > 1e-12:
        fact = mj * (4 * nu * nu) / (nu * ri + nu * rj + 1e-3)
        tvisc = (fact[..., None] * (-dv) * (PK2 * r2)[..., None]).sum(1)
    else:
        tvisc = np.zeros_like(tpres)
    acc = tpres + tdiss + tvisc + np.array(prm.grav[:])[None, :]
    return dden, acc, nb
