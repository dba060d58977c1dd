"""The slab decomposition's host logic on the CPU: the whole grid restated on
the host against the oracle's CreaGrid, the split into x-cell ranges, the
ghost layers, and the exchanges of SlabRun (one process) and
DistributedSlabRun (gloo ranks, world sizes 2 and 3).

The device is replaced by FakeEngine: neighbour sums over the slab's own
particle set within 2h (the same radius as the SPH pair loops, so an owned
particle's sums are complete only if its slab holds every particle within
2h of it), summed in the set's order.  A slab run is then bit for bit the
undivided run if, and only if, every exchange gives every slab its owned
particles, its migrants and fresh ghosts, in increasing global index.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from sphera_b200 import abi, cases
from sphera_b200 import slab

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STEPS = 10


class FakeEngine:
    """A stand-in for a slab's device handle with the same call sequence."""

    def __init__(self, case, cells, capacity):
        self.h = case.params.dx * case.params.trunc
        self.r2 = (2.0 * self.h) ** 2
        self.cells = cells
        self.dt_cur = None
        self.st = None

    def _sums(self, f):
        x = self.st.x
        out = []
        for i in range(len(x)):
            d = x[i] - x
            r2 = np.einsum("ij,ij->i", d, d)
            nb = np.flatnonzero((r2 < self.r2) & (np.arange(len(x)) != i))   # increasing set order
            out.append(np.add.reduce(f(i, nb, d[nb], r2[nb]), axis=0) if len(nb) else f(i, nb, d[nb], r2[nb]).sum(0))
        return np.array(out)

    def _close(self):
        speed = np.sqrt(np.einsum("ij,ij->i", self.st.v, self.st.v))
        return float(np.min(0.02 / (1.0 + speed)))

    def upload(self, st):
        self.st = abi.State(st.x.copy(), st.v.copy(), st.rho.copy(), st.p.copy(), st.m.copy())
        self.lam = np.zeros(st.n, np.int32)
        self.dt_cur = self._close()

    def laminar(self):
        return self.lam.copy()

    def replace(self, st, laminar):
        self.st = abi.State(st.x.copy(), st.v.copy(), st.rho.copy(), st.p.copy(), st.m.copy())
        self.lam = laminar.copy()

    def download(self):
        s = self.st
        return abi.State(s.x.copy(), s.v.copy(), s.rho.copy(), s.p.copy(), s.m.copy())

    def momentum(self):
        # the flag set by the last pass scales this one's acceleration, as the
        # laminar flag switches the wall's no-slip term
        s = self.st
        acc = self._sums(lambda i, nb, d, r2: d * ((self.r2 - r2) * s.p[nb] / s.rho[nb])[:, None])
        acc = acc * (1.0 + 0.5 * self.lam)[:, None]
        self.lam = (np.abs(acc[:, 0]) > 2e-3).astype(np.int32)
        s.v[:] = s.v + self.dt_cur * 1e-3 * acc
        s.x[:] = s.x + self.dt_cur * s.v

    def continuity(self):
        s = self.st
        dd = self._sums(lambda i, nb, d, r2: s.m[nb] * (self.r2 - r2) * np.einsum("ij,ij->i", d, s.v[i] - s.v[nb]))
        s.rho[:] = s.rho + self.dt_cur * dd
        s.p[:] = 2.0 * s.rho
        self.dt_cur = self._close()

    def dt(self):
        return self.dt_cur

    def set_dt(self, dt):
        self.dt_cur = dt

    def close(self):
        pass


def moving_case():
    """dam_break_2d at dx = 0.05 with a velocity field that carries
    particles across the slab edges within a few steps."""
    case = cases.dam_break_2d(dx=0.05)
    rng = np.random.Generator(np.random.PCG64(7))
    st = case.state
    v = np.zeros_like(st.x)
    v[:, 0] = 3.0 + rng.uniform(-1.0, 1.0, st.n)
    v[:, 2] = rng.uniform(-0.5, 0.5, st.n)
    case.state = abi.State(st.x, v, st.rho, st.p, st.m)
    return case


def undivided(case, steps):
    e = FakeEngine(case, None, case.n)
    e.upload(case.state)
    for _ in range(steps):
        e.momentum()
        e.continuity()
    return slab.records(np.arange(case.n, dtype=np.float64), e.download(), e.laminar())


@pytest.mark.parametrize("name", ["dam_break_2d", "dam_break_3d_dx02", "random_box_5k"])
def test_whole_grid_matches_the_oracle(name, oracle_lib):
    case = {"dam_break_2d": lambda: cases.dam_break_2d(),
            "dam_break_3d_dx02": lambda: cases.dam_break_3d(dx=0.02),
            "random_box_5k": lambda: cases.random_box(n=5000, seed=3)}[name]()
    o = oracle_lib.Oracle(case)
    ncd, lo, dcd = o.grid_info()
    glo, gncd, gdcd = slab.whole_grid(case.params)
    assert gncd == ncd[0] and glo == lo[0] and gdcd == dcd[0]
    # every particle's x cell as CreaGrid/ParticleCellNumber give it
    o.prepare()
    cella, _, _ = o.grid()
    ci = slab.cell_x(case.state.x, glo, gdcd)
    # cella numbers cells ((k-1) nj + (j-1)) ni + i (CellNumber.f90:58)
    i_oracle = (np.asarray(cella) - 1) % ncd[0] + 1
    assert np.array_equal(ci, i_oracle)


def test_split_cells():
    assert slab.split_cells(10, 3) == [(1, 3), (4, 7), (8, 10)]
    w = np.zeros(20)
    w[4:8] = 10.0
    r = slab.split_cells(20, 2, w)
    assert r[0][0] == 1 and r[-1][1] == 20
    assert all(r[k][1] + 1 == r[k + 1][0] for k in range(len(r) - 1))
    assert w[: r[0][1]].sum() == 20.0          # the loaded cells 5..8 split in half
    with pytest.raises(ValueError):
        slab.split_cells(2, 3)


def test_assemble_layers_and_order():
    rng = np.random.Generator(np.random.PCG64(1))
    n, ncd = 200, 12
    ci = rng.integers(1, ncd + 1, n)
    rec = np.zeros((n, slab._REC))
    rec[:, 0] = rng.permutation(n)
    rows, mask = slab.assemble(rec, ci, (4, 7), ncd)
    assert np.all(np.diff(rows[:, 0]) > 0)
    got = {int(g) for g in rows[:, 0]}
    assert got == {int(rec[i, 0]) for i in range(n) if 3 <= ci[i] <= 8}
    owned = {int(g) for g in rows[mask, 0]}
    assert owned == {int(rec[i, 0]) for i in range(n) if 4 <= ci[i] <= 7}
    # at the grid's ends there is no outer layer
    rows, mask = slab.assemble(rec, ci, (1, 3), ncd)
    assert set(rows[:, 0].astype(int)) == {int(rec[i, 0]) for i in range(n) if ci[i] <= 4}


@pytest.mark.parametrize("nslabs", [2, 3])
def test_slab_run_is_the_undivided_run(nslabs):
    case = moving_case()
    ref = undivided(case, STEPS)
    run = slab.SlabRun(case, nslabs=nslabs, engine=FakeEngine)
    owned0, _ = run.counts()
    run.step(STEPS)
    owned1, ghosts = run.counts()
    st = run.state()
    assert owned0 != owned1, "no particle crossed a slab edge"
    assert sum(owned1) == case.n and min(ghosts) > 0
    got = slab.records(np.arange(case.n, dtype=np.float64), st, run.laminar())
    assert 0 < ref[:, 10].sum() < case.n, "the flags took one value only"
    assert np.array_equal(got, ref)


def test_torch_records_and_sets_equal_numpy():
    """The device path's record handling (torch tensors; here on the CPU)
    gives the numpy path's cells, sets, order and state columns exactly."""
    import torch
    case = moving_case()
    lo, ncd, dcd = slab.whole_grid(case.params)
    rng = np.random.Generator(np.random.PCG64(4))
    lam = rng.integers(0, 2, case.n).astype(np.int32)
    rec = slab.records(np.arange(case.n, dtype=np.float64), case.state, lam)
    trec = torch.from_numpy(rec.copy())
    ci, tci = slab.cell_x(rec[:, 1:4], lo, dcd), slab.cell_x(trec[:, 1:4], lo, dcd)
    assert np.array_equal(ci, tci.numpy())
    for own in slab.split_cells(ncd, 3, np.bincount(ci, minlength=ncd + 1)[1:]):
        rows, mask = slab.assemble(rec, ci, own, ncd)
        trows, tmask = slab.assemble(trec, tci, own, ncd)
        assert np.array_equal(rows, trows.numpy()) and np.array_equal(mask, tmask.numpy())
        st, tst = slab.state_of(rows), slab.state_of(trows)
        for f in ("x", "v", "rho", "p", "m"):
            assert np.array_equal(getattr(st, f), getattr(tst, f).numpy()), f
        assert tst.struct.n == st.n
        assert np.array_equal(slab.laminar_of(rows), slab.laminar_of(trows).numpy())
    back = slab.records(trec[:, 0], slab.DeviceState(trec[:, 1:4], trec[:, 4:7], trec[:, 7], trec[:, 8],
                                                      trec[:, 9]), trec[:, 10])
    assert np.array_equal(back.numpy(), rec)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    from tests.test_slab import FakeEngine, moving_case
    case = moving_case()
    lo, ncd, dcd = slab.whole_grid(case.params)
    ci = slab.cell_x(case.state.x, lo, dcd)
    ranges = slab.split_cells(ncd, ws, np.bincount(ci, minlength=ncd + 1)[1:])
    run = slab.DistributedSlabRun(case, ranges, engine=FakeEngine)
    run.step(STEPS)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), run.owned_records())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("ws", [2, 3])
def test_distributed_slab_run_gloo(ws, tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, ws, port, str(tmp_path))) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(200)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    case = moving_case()
    ref = undivided(case, STEPS)
    parts = [np.load(os.path.join(tmp_path, f"r{r}.npy")) for r in range(ws)]
    got = np.vstack(parts)
    got = got[np.argsort(got[:, 0])]
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)
