"""One simulation split into slabs along x (no reference counterpart: the
reference is one shared-memory process; this is the decomposition of a
single large simulation over several GPUs).

Each slab owns a contiguous range of the whole grid's x cells and holds, as
ghosts, the particles of one more cell layer on each side (the cells are at
least 2h wide, so that layer holds every neighbour of an owned particle).
A slab is a library handle over its cells of the whole grid
(``sph_create_slab``: same origin and cell size, so every particle lies in
the cell it has in the whole grid).  Every exchange rebuilds each slab's
particle set -- owned particles, migrants from its neighbours and fresh
ghosts -- in increasing order of the particles' index in the whole
simulation, which is the order OrdGrid1 ranks a cell's particles in
(OrdGrid1.f90:84-105).  An owned particle therefore meets the same
neighbours, in the same order, with the same values as in the undivided run,
and its FP64 arithmetic is bit for bit the same.

One step is the per-call sequence of time_step_loop.f90 with two exchanges:

  1. every slab: RHS_momentum_equation, Leapfrog_momentum and
     Leapfrog_trajectories (ghosts get meaningless rates: their
     neighbourhoods are incomplete; they are replaced before use);
  2. exchange: particles that crossed a slab edge migrate, ghosts are taken
     again from their owners (with the laminar flags the momentum pass just
     set); every slab runs OrdGrid1, CalcVarLength and
     ComputeBoundaryDataTab on its new set (``sph_replace_particles``);
  3. every slab: the continuity block, Leapfrog_continuity and the EoS;
  4. exchange: ghosts get their owners' new densities and pressures;
  5. dt: each slab closed the step with the CFL minimum over its own
     particles and ghosts (copies of other slabs' particles); the minimum
     over the slabs is the whole simulation's dt (pesodt = 0), set on all.

Two transports: ``SlabRun`` keeps all slabs in one process (on one device:
the exchanges gather on the host); ``DistributedSlabRun`` runs one slab per
rank of torch.distributed and trades only the edge layers and the migrants
with the two neighbouring ranks (send/recv, gloo or NCCL).  The engine of a
slab is reached through a small interface (``SlabEngine``), so the exchange
logic is testable without a device.
"""
import numpy as np

from . import abi

# record layout of an exchanged particle: global index, x(3), v(3), rho, p, m,
# pg%laminar_flag (the one value besides the state that a particle carries
# from one momentum pass to the next)
_REC = 11


def _torch(a):
    return type(a).__module__.startswith("torch")


def whole_grid(params):
    """CreaGrid.f90:51-74 restated on the host (the device's own sequence of
    IEEE operations): x-extent origin, cell count and cell size."""
    h = params.dx * params.trunc
    doubleh = 2.0 * h
    epsi = 0.01 * params.dx
    lo = params.domain_lo[0] - doubleh - epsi
    hi = params.domain_hi[0] + doubleh + epsi
    dextr = hi - lo
    ncd = int(np.floor(dextr / doubleh + 0.5))     # NINT, positive argument
    return lo, ncd, dextr / ncd


def cell_x(x, lo, dcd):
    """ParticleCellNumber.f90:52-62 in x: ceiling((x - extr) / dcd), on numpy
    arrays or torch tensors (the same correctly rounded FP64 operations)."""
    if _torch(x):
        import torch
        return torch.ceil((x[:, 0] - lo) / dcd).to(torch.int64)
    return np.ceil((x[:, 0] - lo) / dcd).astype(np.int64)


def split_cells(ncd, nslabs, weights=None):
    """Owned x-cell ranges [(a, b)] (1-based, inclusive) of nslabs slabs:
    equal cell counts, or cut where the cumulative weight per cell (e.g. the
    particle counts) reaches equal shares."""
    if weights is None:
        cuts = [round(ncd * k / nslabs) for k in range(nslabs + 1)]
    else:
        c = np.cumsum(weights)
        cuts = [0] + [int(np.searchsorted(c, c[-1] * k / nslabs)) + 1 for k in range(1, nslabs)] + [ncd]
    ranges = [(cuts[k] + 1, cuts[k + 1]) for k in range(nslabs)]
    if any(b < a for a, b in ranges):
        raise ValueError("a slab without cells: fewer slabs or another split")
    return ranges


def assemble(rec, ci, own, ncd):
    """The particle set of the slab owning x cells own = (a, b): its owned
    particles and the ghosts of cells a - 1 and b + 1, in increasing global
    index.  rec: (n, _REC) records, ci their x cells (numpy or torch).
    Returns the rows and the mask of owned rows."""
    a, b = own
    keep = (ci >= max(a - 1, 1)) & (ci <= min(b + 1, ncd))
    rows = rec[keep]
    if _torch(rows):
        import torch
        order = torch.argsort(rows[:, 0], stable=True)
    else:
        order = np.argsort(rows[:, 0], kind="stable")
    rows = rows[order]
    c = ci[keep][order]
    return rows, (c >= a) & (c <= b)


class DeviceState:
    """An SphState over torch tensors in the handle's device memory (the
    library's copies take their direction from the pointers)."""

    def __init__(self, x, v, rho, p, m):
        self.x, self.v, self.rho, self.p, self.m = (t.contiguous() for t in (x, v, rho, p, m))
        st = abi.SphState()
        st.n = int(self.rho.shape[0])
        for f in ("x", "v", "rho", "p", "m"):
            setattr(st, f, abi.C.cast(getattr(self, f).data_ptr(), abi.C.POINTER(abi.C.c_double)))
        self.struct = st

    @property
    def n(self):
        return int(self.rho.shape[0])


def records(gid, st, laminar=None):
    if _torch(st.x):
        import torch
        out = torch.empty((st.n, _REC), dtype=torch.float64, device=st.x.device)
    else:
        out = np.empty((st.n, _REC))
    out[:, 0] = gid
    out[:, 1:4] = st.x
    out[:, 4:7] = st.v
    out[:, 7] = st.rho
    out[:, 8] = st.p
    out[:, 9] = st.m
    out[:, 10] = 0.0 if laminar is None else laminar
    return out


def state_of(rows):
    if _torch(rows):
        return DeviceState(rows[:, 1:4], rows[:, 4:7], rows[:, 7], rows[:, 8], rows[:, 9])
    return abi.State(np.ascontiguousarray(rows[:, 1:4]), np.ascontiguousarray(rows[:, 4:7]),
                     np.ascontiguousarray(rows[:, 7]), np.ascontiguousarray(rows[:, 8]),
                     np.ascontiguousarray(rows[:, 9]))


def laminar_of(rows):
    if _torch(rows):
        import torch
        return rows[:, 10].to(torch.int32).contiguous()
    return np.ascontiguousarray(rows[:, 10], dtype=np.int32)


class SlabEngine:
    """The device side of one slab: a library handle over the slab's cells.
    With device=True its state crosses the C ABI as device tensors."""

    def __init__(self, case, cells, capacity, device=False):
        from . import Simulation
        self.sim = Simulation(params=case.params, geometry=case.geometry, capacity=capacity, cells=cells)
        self.device = device

    def _ready(self):
        # device tensors are written by torch on its own stream; the
        # library reads them on the handle's stream, so torch's work must
        # be complete first (the library synchronises its own stream before
        # it returns, so what it writes is complete for torch)
        if self.device:
            import torch
            torch.cuda.current_stream().synchronize()

    def upload(self, st):
        self._ready()
        self.sim.upload(st)

    def replace(self, st, laminar):
        self._ready()
        self.sim.replace_particles(st, laminar)

    def download(self):
        if not self.device:
            return self.sim.download()
        import torch
        n = self.sim.n
        dev = torch.device("cuda", torch.cuda.current_device())
        st = DeviceState(*(torch.empty(sh, dtype=torch.float64, device=dev)
                           for sh in ((n, 3), (n, 3), (n,), (n,), (n,))))
        self.sim.download_into(st)
        return st

    def laminar(self):
        if not self.device:
            return self.sim.dump_laminar()
        import torch
        f = torch.empty(self.sim.n, dtype=torch.int32, device=torch.device("cuda", torch.cuda.current_device()))
        self.sim.dump_laminar_into(f)
        return f

    def momentum(self):
        self.sim.rhs_momentum(want=False)
        self.sim.leapfrog_momentum()
        self.sim.leapfrog_trajectories()

    def continuity(self):
        self.sim.continuity(want=False)
        self.sim.leapfrog_continuity()
        self.sim.eos()

    def dt(self):
        return self.sim.time_step_duration()

    def set_dt(self, dt):
        self.sim.set_time_step(dt)

    def close(self):
        self.sim.close()


class SlabRun:
    """All slabs in one process; the exchanges gather the owned particles
    and rebuild every slab's set from them -- on the host, or with
    device=True as device tensors that cross the C ABI without a host copy."""

    def __init__(self, case, nslabs=2, ranges=None, engine=SlabEngine, capacity=None, device=False):
        self.case = case
        self.lo, self.ncd, self.dcd = whole_grid(case.params)
        st = case.state
        if ranges is None:
            ci = cell_x(st.x, self.lo, self.dcd)
            ranges = split_cells(self.ncd, nslabs, np.bincount(ci, minlength=self.ncd + 1)[1:])
        self.ranges = ranges
        cap = capacity or st.n
        kw = dict(device=True) if device else {}
        self.engines = [engine(case, (max(a - 1, 1), min(b + 1, self.ncd)), cap, **kw) for a, b in ranges]
        self.rec = records(np.arange(st.n, dtype=np.float64), st)
        if device:
            import torch
            self.rec = torch.from_numpy(self.rec).to(torch.device("cuda", torch.cuda.current_device()))
        self.n = st.n
        self.owned = [None] * len(ranges)
        sets = self._sets()
        for e, rows in zip(self.engines, sets):
            e.upload(state_of(rows))
        self._global_dt()

    def _sets(self):
        ci = cell_x(self.rec[:, 1:4], self.lo, self.dcd)
        if bool(((ci < 1) | (ci > self.ncd)).any()):
            raise RuntimeError("a particle left the grid: slab runs do not remove particles")
        out = []
        for k, own in enumerate(self.ranges):
            rows, mask = assemble(self.rec, ci, own, self.ncd)
            gid = rows[:, 0]
            gid = gid.long() if _torch(gid) else gid.astype(np.int64)
            self.owned[k] = (gid, mask)
            out.append(rows)
        return out

    def _gather(self):
        for e, (gid, mask) in zip(self.engines, self.owned):
            r = records(gid, e.download(), e.laminar())
            self.rec[gid[mask]] = r[mask]

    def _exchange(self):
        self._gather()
        for e, rows in zip(self.engines, self._sets()):
            e.replace(state_of(rows), laminar_of(rows))

    def _global_dt(self):
        dt = min(e.dt() for e in self.engines)
        for e in self.engines:
            e.set_dt(dt)
        return dt

    def step(self, nsteps=1):
        for _ in range(nsteps):
            for e in self.engines:
                e.momentum()
            self._exchange()
            for e in self.engines:
                e.continuity()
            self._exchange()
            self._global_dt()

    def _host_rec(self):
        self._gather()
        return self.rec.cpu().numpy() if _torch(self.rec) else self.rec

    def state(self):
        """The whole simulation's state in its original particle order (host arrays)."""
        return state_of(self._host_rec())

    def laminar(self):
        """pg%laminar_flag of the whole simulation, original particle order."""
        return laminar_of(self._host_rec())

    def counts(self):
        return [int(m.sum()) for _, m in self.owned], [int((~m).sum()) for _, m in self.owned]

    def close(self):
        for e in self.engines:
            e.close()


class DistributedSlabRun:
    """One slab per rank of an initialised torch.distributed group: rank r
    owns the r-th x-cell range.  The exchanges trade, with ranks r - 1 and
    r + 1 only, the owned particles in the cells next to the shared edge
    (the neighbour's ghosts) and those that crossed it (migrants); a step
    moves a particle far less than a cell, so no other rank is reached.  The
    dt is an all-reduce (min).  With device=True (an NCCL group, one GPU per
    rank) the records stay in device tensors: the slab's state is read and
    replaced through the C ABI with device pointers and the edge layers go
    rank to rank with NCCL send/recv, never through the host; otherwise
    (gloo) they are host arrays."""

    def __init__(self, case, ranges, engine=SlabEngine, capacity=None, device=False):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = dist.get_rank(), dist.get_world_size()
        if len(ranges) != self.size:
            raise ValueError("one x-cell range per rank")
        self.device = device
        self.lo, self.ncd, self.dcd = whole_grid(case.params)
        self.ranges = ranges
        self.own = ranges[self.rank]
        st = case.state
        all_rec = records(np.arange(st.n, dtype=np.float64), st)
        ci = cell_x(st.x, self.lo, self.dcd)
        rows, mask = assemble(all_rec, ci, self.own, self.ncd)
        a, b = self.own
        kw = dict(device=True) if device else {}
        self.engine = engine(case, (max(a - 1, 1), min(b + 1, self.ncd)), capacity or st.n, **kw)
        if device:
            import torch
            dev = torch.device("cuda", torch.cuda.current_device())
            rows, mask = torch.from_numpy(rows).to(dev), torch.from_numpy(mask).to(dev)
        self.rows, self.mask = rows, mask
        self.engine.upload(state_of(rows))
        self._global_dt()

    def _trade(self, peer, send):
        """Sends `send` rows to `peer` and returns the rows it sent back
        (tensors on the rows' device: NCCL moves device memory, gloo host)."""
        import torch
        dist = self.dist
        dev = send.device if _torch(send) else torch.device("cpu")
        payload = send if _torch(send) else torch.from_numpy(np.ascontiguousarray(send))
        cnt_out = torch.tensor([payload.shape[0]], dtype=torch.int64, device=dev)
        cnt_in = torch.zeros(1, dtype=torch.int64, device=dev)
        reqs = [dist.isend(cnt_out, peer), dist.irecv(cnt_in, peer)]
        for r in reqs:
            r.wait()
        m = int(cnt_in.item())
        buf_in = torch.empty((m, _REC), dtype=torch.float64, device=dev)
        reqs = []
        if payload.shape[0]:
            reqs.append(dist.isend(payload.contiguous(), peer))
        if m:
            reqs.append(dist.irecv(buf_in, peer))
        for r in reqs:
            r.wait()
        return buf_in if _torch(send) else buf_in.numpy()

    def _exchange(self):
        st = self.engine.download()
        mine = records(self.rows[:, 0], st, self.engine.laminar())[self.mask]   # my owned particles, updated
        ci = cell_x(mine[:, 1:4], self.lo, self.dcd)
        if bool(((ci < 1) | (ci > self.ncd)).any()):
            raise RuntimeError("a particle left the grid: slab runs do not remove particles")
        a, b = self.own
        got = [mine]
        # left neighbour: cells up to its edge + 1 (its ghosts and my emigrants);
        # right neighbour likewise; the same order of trades on every rank
        for peer, sel in ((self.rank - 1, ci <= a), (self.rank + 1, ci >= b)):
            if 0 <= peer < self.size:
                got.append(self._trade(peer, mine[sel]))
        if _torch(mine):
            import torch
            allrec = torch.cat(got)
        else:
            allrec = np.vstack(got)
        # the ranks own disjoint particle sets, so every row is a distinct
        # particle; assemble orders them by global index
        rows, mask = assemble(allrec, cell_x(allrec[:, 1:4], self.lo, self.dcd), self.own, self.ncd)
        self.rows, self.mask = rows, mask
        self.engine.replace(state_of(rows), laminar_of(rows))

    def _global_dt(self):
        import torch
        dev = torch.device("cuda", torch.cuda.current_device()) if self.device else torch.device("cpu")
        t = torch.tensor([self.engine.dt()], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN)
        dt = float(t.item())
        self.engine.set_dt(dt)
        return dt

    def step(self, nsteps=1):
        for _ in range(nsteps):
            self.engine.momentum()
            self._exchange()
            self.engine.continuity()
            self._exchange()
            self._global_dt()

    def owned_records(self):
        """(global index, x, v, rho, p, m, laminar) rows of the particles this
        rank owns (host array)."""
        st = self.engine.download()
        r = records(self.rows[:, 0], st, self.engine.laminar())[self.mask]
        return r.cpu().numpy() if _torch(r) else r

    def close(self):
        self.engine.close()
