"""A simulation split into slabs along x (sph_create_slab,
sph_replace_particles, sph_set_time_step and the host exchanges of
sphera_b200.slab) against the undivided simulation, bit for bit.

The cases get a velocity field that carries particles across the slab
edges within the steps run (the dam break alone barely moves in a few
dozen steps), so migrations, ghost refreshes and the global dt are all
exercised.  Both arithmetic forms: every owned particle meets the same
neighbours in the same order with the same values (and, in the FP32
screening copies, the same cell origins), so FP32c too is bit-identical.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from sphera_b200 import Simulation, abi, cases, slab

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def moving(case, seed=5, u=3.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    st = case.state
    v = np.zeros_like(st.x)
    v[:, 0] = u + rng.uniform(-1.0, 1.0, st.n)
    v[:, 2] = rng.uniform(-0.5, 0.5, st.n)
    case.state = abi.State(st.x, v, st.rho, st.p, st.m)
    return case


def make(name, precision):
    if name == "dam_break_2d":
        return moving(cases.dam_break_2d(dx=0.02, precision=precision))
    if name == "dam_break_2d_laminar":
        # no-slip walls that act only where pg%laminar_flag is set, and a
        # viscosity high enough for the Morris term to set it: the flags a
        # momentum pass leaves must travel with the particles
        case = moving(cases.dam_break_2d(dx=0.02, precision=precision))
        case.params.kin_visc = 1.0e-2
        case.geometry = cases.tank_2d(*case.meta["tank"], zone=abi.make_zone(slip=0.5, laminar_no_slip_check=1))
        return case
    return moving(cases.dam_break_3d(dx=0.02, precision=precision), u=6.0)


def undivided(case, steps):
    with Simulation(case) as sim:
        sim.upload(case.state)
        for _ in range(steps):
            sim.step(1)
        return sim.download(), sim.diagnostics()


@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
@pytest.mark.parametrize("precision", [abi.SPH_PREC_FP64, abi.SPH_PREC_FP32C], ids=["fp64", "fp32c"])
@pytest.mark.parametrize("name,nslabs,steps", [("dam_break_2d", 2, 60), ("dam_break_2d", 3, 60),
                                               ("dam_break_2d_laminar", 2, 60), ("dam_break_3d", 2, 60)])
def test_slabs_are_the_undivided_run(name, nslabs, steps, precision, device):
    """host: the exchanges go through host arrays; device: the records stay
    in device tensors and cross the C ABI as device pointers."""
    case = make(name, precision)
    ref, _ = undivided(case, steps)
    run = slab.SlabRun(case, nslabs=nslabs, device=device)
    try:
        owned0, _ = run.counts()
        run.step(steps)
        owned1, ghosts = run.counts()
        got = run.state()
        dts = {e.dt() for e in run.engines}
    finally:
        run.close()
    assert owned0 != owned1, "no particle crossed a slab edge"
    assert sum(owned1) == case.n and min(ghosts) > 0
    assert len(dts) == 1
    for f in ("x", "v", "rho", "p", "m"):
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f


def test_slab_rejects_what_it_does_not_exchange():
    case = cases.dam_break_3d(dx=0.02)
    case.params.c1_be = 1
    with pytest.raises(Exception):
        Simulation(params=case.params, geometry=case.geometry, capacity=case.n, cells=(3, 9))
    case = cases.dam_break_3d(dx=0.02)
    case.params.pesodt = 0.5
    with pytest.raises(Exception):
        Simulation(params=case.params, geometry=case.geometry, capacity=case.n, cells=(3, 9))
    case = cases.dam_break_3d(dx=0.02)
    _, ncd, _ = slab.whole_grid(case.params)
    with pytest.raises(Exception):
        Simulation(params=case.params, geometry=case.geometry, capacity=case.n, cells=(3, ncd + 1))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out_dir, steps):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
    from tests.test_gpu_slab import make
    case = make("dam_break_2d", abi.SPH_PREC_FP64)
    lo, ncd, dcd = slab.whole_grid(case.params)
    ci = slab.cell_x(case.state.x, lo, dcd)
    ranges = slab.split_cells(ncd, ws, np.bincount(ci, minlength=ncd + 1)[1:])
    run = slab.DistributedSlabRun(case, ranges)
    run.step(steps)
    np.save(os.path.join(out_dir, f"r{rank}.npy"), run.owned_records())
    run.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_distributed_slabs_gloo(tmp_path):
    """Two ranks, one slab each, exchanging over gloo (both on the one
    device this test has; their kernels never wait on each other, the
    exchanges are host-side)."""
    ws, steps = 2, 40
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, ws, port, str(tmp_path), steps)) for r in range(ws)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(280)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    case = make("dam_break_2d", abi.SPH_PREC_FP64)
    ref, _ = undivided(case, steps)
    got = np.vstack([np.load(os.path.join(tmp_path, f"r{r}.npy")) for r in range(ws)])
    got = got[np.argsort(got[:, 0])]
    assert np.array_equal(got[:, 0], np.arange(case.n))
    assert np.array_equal(got[:, 1:4], ref.x)
    assert np.array_equal(got[:, 4:7], ref.v)
    assert np.array_equal(got[:, 7], ref.rho)
    assert np.array_equal(got[:, 8], ref.p)
