"""Seeded synthetic initial states for the workloads of this path.

The reference builds its initial lattice in src/IC (GeneratePart.f90,
SetParticleParameters.f90:55-131, SubCalcPreIdro.f90:98-196) with an
unseeded white-noise jitter (pos_plus_white_noise.f90:48-55).  These
generators restate the same conventions -- particle centres at (i+1/2)dx,
mass = dx**D * den0, hydrostatic pressure of type "pl" (level = highest
particle + dx/2) and density from the inverse linear EoS -- with a seeded
jitter so every run sees the identical state.

Workloads (all synthetic, no external dataset):
  * dam_break_2d:  4.0 x 3.0 m tank, 1.0 x 2.0 m column, dx 0.02 (5,000 particles)
  * dam_break_3d:  1.6 x 0.6 x 0.6 m tank, 0.6 x 0.3 x 0.6 m block, dx 0.005
                   (864,000 particles)
  * random_box:    N particles uniform in a cube at mean spacing 0.01 m,
                   rho = 1000 (1 + N(0, 1e-3)), v ~ N(0, 0.1), no walls
  * ensemble_2d:   dam breaks with column width U[0.5, 2.0] and height
                   U[0.5, 2.5] in the 2D tank at dx 0.01
  * sloshing_3d:   1.0 x 0.5 x 0.5 m tank, half filled, moved sideways as
                   x = A sin(2 pi t / T) (A = 0.02 m); the fluid is computed
                   in the tank frame with the body force
                   g + A (2 pi / T)^2 sin(2 pi t / T) along x
  * serving_requests: a seeded Poisson stream of dam-break and sloshing
                   requests, each run to t_end = 0.3 s
"""
from dataclasses import dataclass, field

import numpy as np

from . import abi

G = 9.81


@dataclass
class Case:
    name: str
    params: abi.SphParams
    geometry: abi.Geometry
    state: abi.State
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.state.n


def _params(dim, dx, lo, hi, cfl=0.1, precision=abi.SPH_PREC_FP64, **extra):
    den0 = 1000.0
    c0 = 40.0
    kw = dict(
        dim=dim, precision=precision, dx=dx, trunc=1.3, coef_nmaxpartj=2.0,
        max_close_bound_faces=100, dt_alfa_mon=0,
        domain_lo=lo, domain_hi=hi, den0=den0, eps=den0 * c0 * c0,
        alfa_mon=0.05, kin_visc=1.0e-6, p_ref=0.0,
        grav=(0.0, 0.0, -G), cfl=cfl, vsc_coeff=0.05, pesodt=0.0,
        density_thresholds=0, bdt_capacity=0, teta_p=0.0, teta_v=0.0)
    kw.update(extra)
    return abi.make_params(**kw)


def _hydrostatic(z, dx, den0, eps, p_ref, g=G):
    # SubCalcPreIdro.f90:182-196, pressure type "pl" (coshor = 1, senhor = 0)
    level = z.max() + dx / 2.0
    p = (level - z) * 1.0 * den0 * g + p_ref
    # EoS_barotropic_linear.f90:49-55, inverse form
    rho = den0 * (1.0 + (p - p_ref) / eps)
    return p, rho


def _box_faces(lx, ly, lz):
    """Six quads of the box [0,lx]x[0,ly]x[0,lz], each with its normal
    (V1-V4)x(V3-V4) pointing into the box (DefineLocalSystemVersors.f90)."""
    V = np.array([[0, 0, 0], [lx, 0, 0], [lx, ly, 0], [0, ly, 0],
                  [0, 0, lz], [lx, 0, lz], [lx, ly, lz], [0, ly, lz]], dtype=np.float64)
    quads = [(1, 2, 3, 4), (5, 8, 7, 6), (1, 5, 6, 2), (4, 3, 7, 8), (1, 4, 8, 5), (2, 6, 7, 3)]
    centre = V.mean(axis=0)
    faces = []
    for q in quads:
        a, b, c, d = (V[i - 1] for i in q)
        nrm = np.cross(a - d, c - d)
        fc = (a + b + c + d) / 4.0
        if np.dot(nrm, centre - fc) < 0:
            q = q[::-1]
        faces.append(q)
    return V, np.array(faces, dtype=np.int32)


def tank_3d(lx, ly, lz, zone=None):
    V, F = _box_faces(lx, ly, lz)
    z = zone or abi.make_zone()
    return abi.Geometry(V, [z], faces=F, face_zone=np.ones(len(F), dtype=np.int32))


def tank_with_block_3d(lx, ly, lz, block, zone=None):
    """The box tank plus a block standing on its floor, block = (x0, x1,
    y0, y1, z1): five more quads (top and four sides; the base lies on the
    floor) with normals pointing away from the block, into the fluid.  The
    block's top and side edges are convex edges of the boundary
    (FindBoundaryConvexEdges3D.f90)."""
    V, F = _box_faces(lx, ly, lz)
    x0, x1, y0, y1, z1 = block
    B = np.array([[x0, y0, 0], [x1, y0, 0], [x1, y1, 0], [x0, y1, 0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], dtype=np.float64)
    quads = [(5, 6, 7, 8), (1, 5, 6, 2), (4, 3, 7, 8), (1, 4, 8, 5), (2, 6, 7, 3)]
    centre = B.mean(axis=0)
    bf = []
    for q in quads:
        a, b, c, d = (B[i - 1] for i in q)
        nrm = np.cross(a - d, c - d)
        fc = (a + b + c + d) / 4.0
        if np.dot(nrm, fc - centre) < 0:
            q = q[::-1]
        bf.append(tuple(i + len(V) for i in q))
    V = np.vstack([V, B])
    F = np.vstack([F, np.array(bf, dtype=np.int32)])
    z = zone or abi.make_zone()
    return abi.Geometry(V, [z], faces=F, face_zone=np.ones(len(F), dtype=np.int32))


def tank_2d(lx, lz, zone=None):
    # counter-clockwise in the x-z plane: the side normal (-sz, sx) points inside
    V = np.array([[0, 0, 0], [lx, 0, 0], [lx, 0, lz], [0, 0, lz]], dtype=np.float64)
    S = np.array([[1, 2], [2, 3], [3, 4], [4, 1]], dtype=np.int32)
    z = zone or abi.make_zone()
    return abi.Geometry(V, [z], sides=S, side_zone=np.ones(len(S), dtype=np.int32))


def _jitter(rng, shape, dx, frac):
    return rng.uniform(-frac * dx, frac * dx, size=shape)


def dam_break_2d(dx=0.02, tank=(4.0, 3.0), column=(1.0, 2.0), jitter=0.01, seed=0xC0,
                 precision=abi.SPH_PREC_FP64, cfl=0.1):
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, nz = int(round(column[0] / dx)), int(round(column[1] / dx))
    i, k = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    x = np.zeros((nx * nz, 3))
    x[:, 0] = (i.ravel() + 0.5) * dx
    x[:, 2] = (k.ravel() + 0.5) * dx
    j = _jitter(rng, (nx * nz, 2), dx, jitter)
    x[:, 0] += j[:, 0]
    x[:, 2] += j[:, 1]
    prm = _params(2, dx, (0.0, 0.0, 0.0), (tank[0], 0.0, tank[1]), cfl=cfl, precision=precision)
    p, rho = _hydrostatic(x[:, 2], dx, prm.den0, prm.eps, prm.p_ref)
    m = np.full(len(p), dx * dx * prm.den0)
    st = abi.State(x, np.zeros_like(x), rho, p, m)
    return Case("dam_break_2d", prm, tank_2d(*tank), st,
                dict(dx=dx, tank=tank, column=column, seed=seed, t_end=1.0))


def dam_break_3d(dx=0.005, tank=(1.6, 0.6, 0.6), block=(0.6, 0.3, 0.6), jitter=0.01, seed=0xC1,
                 precision=abi.SPH_PREC_FP64, cfl=0.1):
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, ny, nz = (int(round(b / dx)) for b in block)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = np.stack([(i.ravel() + 0.5) * dx, (j.ravel() + 0.5) * dx, (k.ravel() + 0.5) * dx], axis=1)
    x += _jitter(rng, x.shape, dx, jitter)
    prm = _params(3, dx, (0.0, 0.0, 0.0), tank, cfl=cfl, precision=precision)
    p, rho = _hydrostatic(x[:, 2], dx, prm.den0, prm.eps, prm.p_ref)
    m = np.full(len(p), dx ** 3 * prm.den0)
    st = abi.State(x, np.zeros_like(x), rho, p, m)
    return Case("dam_break_3d", prm, tank_3d(*tank), st,
                dict(dx=dx, tank=tank, block=block, seed=seed, t_end=0.5))


def block_tank_3d(dx=0.02, tank=(0.4, 0.2, 0.3), block=(0.15, 0.25, 0.05, 0.15, 0.1), level=0.2, jitter=0.01,
                  seed=0xC6, precision=abi.SPH_PREC_FP64):
    """Still water to `level` in a box tank around a block standing on its
    floor (tank_with_block_3d): a geometry with convex edges.  Lattice points
    closer than dx / 2 to the block are left out."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, ny, nz = (int(round(v / dx)) for v in (tank[0], tank[1], level))
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = np.stack([(i.ravel() + 0.5) * dx, (j.ravel() + 0.5) * dx, (k.ravel() + 0.5) * dx], axis=1)
    x0, x1, y0, y1, z1 = block
    h = dx / 2
    inside = ((x[:, 0] > x0 - h) & (x[:, 0] < x1 + h) & (x[:, 1] > y0 - h) & (x[:, 1] < y1 + h)
              & (x[:, 2] < z1 + h))
    x = x[~inside]
    x += _jitter(rng, x.shape, dx, jitter)
    prm = _params(3, dx, (0.0, 0.0, 0.0), tank, precision=precision)
    p, rho = _hydrostatic(x[:, 2], dx, prm.den0, prm.eps, prm.p_ref)
    m = np.full(len(p), dx ** 3 * prm.den0)
    st = abi.State(x, np.zeros_like(x), rho, p, m)
    return Case("block_tank_3d", prm, tank_with_block_3d(*tank, block), st,
                dict(dx=dx, tank=tank, block=block, level=level, seed=seed))


def random_box(n=16_000_000, spacing=0.01, seed=0xC2, precision=abi.SPH_PREC_FP64):
    rng = np.random.Generator(np.random.PCG64(seed))
    L = (n * spacing ** 3) ** (1.0 / 3.0)
    x = rng.uniform(0.0, L, size=(n, 3))
    prm = _params(3, spacing, (0.0, 0.0, 0.0), (L, L, L), precision=precision)
    rho = prm.den0 * (1.0 + rng.normal(0.0, 1.0e-3, size=n))
    v = rng.normal(0.0, 0.1, size=(n, 3))
    p = prm.eps / prm.den0 * (rho - prm.den0) + prm.p_ref
    m = np.full(n, spacing ** 3 * prm.den0)
    geo = abi.Geometry(np.zeros((1, 3)), [abi.make_zone()])
    return Case("random_box", prm, geo, abi.State(x, v, rho, p, m),
                dict(spacing=spacing, side=L, seed=seed))


def ensemble_2d(n_sims=256, dx=0.01, seed=0xC3, precision=abi.SPH_PREC_FP32C):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for s in range(n_sims):
        w = rng.uniform(0.5, 2.0)
        hgt = rng.uniform(0.5, 2.5)
        w = round(w / dx) * dx
        hgt = round(hgt / dx) * dx
        out.append(dam_break_2d(dx=dx, column=(w, hgt), seed=int(rng.integers(1 << 31)),
                                precision=precision))
    return out


def sloshing_3d(dx=0.01, tank=(1.0, 0.5, 0.5), fill=0.5, amplitude=0.02, period=1.2, jitter=0.01, seed=0xC5,
                precision=abi.SPH_PREC_FP64, cfl=0.1):
    rng = np.random.Generator(np.random.PCG64(seed))
    nx, ny, nz = (int(round(v / dx)) for v in (tank[0], tank[1], tank[2] * fill))
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x = np.stack([(i.ravel() + 0.5) * dx, (j.ravel() + 0.5) * dx, (k.ravel() + 0.5) * dx], axis=1)
    x += _jitter(rng, x.shape, dx, jitter)
    prm = _params(3, dx, (0.0, 0.0, 0.0), tank, cfl=cfl, precision=precision,
                  forcing_amplitude=amplitude, forcing_period=period)
    p, rho = _hydrostatic(x[:, 2], dx, prm.den0, prm.eps, prm.p_ref)
    m = np.full(len(p), dx ** 3 * prm.den0)
    st = abi.State(x, np.zeros_like(x), rho, p, m)
    return Case("sloshing_3d", prm, tank_3d(*tank), st,
                dict(dx=dx, tank=tank, fill=fill, amplitude=amplitude, period=period, seed=seed, t_end=0.3))


@dataclass
class Request:
    """One simulation request of a serving stream: run `case` to `t_end`."""
    rid: int
    arrival: float          # seconds after the stream starts
    case: Case
    t_end: float


def serving_requests(n_requests=16, rate=20.0, seed=0xC4, t_end=0.3, dx_range=(0.005, 0.0125),
                     period_range=(0.8, 1.6), amplitude=0.02, precision=abi.SPH_PREC_FP32C):
    """Seeded Poisson arrivals (mean `rate` per second) of 3D dam-break and
    sloshing-tank requests, half of each on average.  dx is drawn
    log-uniformly from `dx_range`; at the default range the dam break holds
    55k-864k particles and the half-filled sloshing tank 64k-1M (a larger
    dx would fall under 50k particles with these geometries).  Sloshing
    periods are uniform in `period_range`."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    t = 0.0
    lo, hi = np.log(dx_range[0]), np.log(dx_range[1])
    for r in range(n_requests):
        t += rng.exponential(1.0 / rate)
        dx = float(np.exp(rng.uniform(lo, hi)))
        sub = int(rng.integers(1 << 31))
        if rng.random() < 0.5:
            case = dam_break_3d(dx=dx, seed=sub, precision=precision)
        else:
            case = sloshing_3d(dx=dx, amplitude=amplitude, period=float(rng.uniform(*period_range)),
                               seed=sub, precision=precision)
        out.append(Request(r, t, case, t_end))
    return out
