"""The allocation-free entry point sph_ord_grid_static.

It serves callers that cannot let a library allocate device memory (a host
whose device arrays all come from its own pool allocator, or a loop that
must not meet cudaMalloc's implicit synchronisation): the caller passes
device buffers for inputs and outputs and the library works inside a fixed
device array.  Its output must equal the grid arrays of the regular path
(sph_dump_grid) exactly, on two calls in a row -- the second call runs on a
scratch array that still holds the first call's contents.
"""
import ctypes as C

import numpy as np
import pytest

from sphera_b200 import Simulation, abi, cases, lib

pytestmark = pytest.mark.gpu


def _static(params, x_dev, n, cella, icont, npo, stream):
    L = lib()
    f = L.sph_ord_grid_static
    f.argtypes = [C.POINTER(abi.SphParams), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f(C.byref(params), n, x_dev.data_ptr(), cella.data_ptr(), icont.data_ptr(), npo.data_ptr(), stream)


@pytest.mark.parametrize("make", [lambda: cases.dam_break_3d(dx=0.01), lambda: cases.dam_break_2d()])
def test_static_ord_grid_matches_regular_path(make):
    import torch
    case = make()
    sim = Simulation(case)
    sim.upload(case.state)
    ref_cella, ref_icont, ref_npo = sim.dump_grid()
    n = case.n
    x = torch.tensor(case.state.x, dtype=torch.float64, device="cuda")
    cella = torch.empty(n, dtype=torch.int32, device="cuda")
    icont = torch.empty(len(ref_icont), dtype=torch.int32, device="cuda")
    npo = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        cella.fill_(-7)
        icont.fill_(-7)
        npo.fill_(-7)
        rc = _static(case.params, x, n, cella, icont, npo, stream)
        torch.cuda.synchronize()
        assert rc == abi.SPH_OK
        assert np.array_equal(cella.cpu().numpy(), ref_cella)
        assert np.array_equal(icont.cpu().numpy(), ref_icont)
        assert np.array_equal(npo.cpu().numpy(), ref_npo)


def test_static_ord_grid_with_particles_outside_the_grid():
    """Particles outside the grid get cella 0 and stay out of NPartOrd; the
    rest is OrdGrid1 of the particles inside, with their own indices (the
    static call removes nothing, unlike the regular path)."""
    import torch
    base = cases.dam_break_2d(dx=0.04)
    x = base.state.x.copy()
    out = np.array([3, 50, 51, 400])
    x[out, 0] = base.params.domain_hi[0] + 5.0
    keep = np.setdiff1d(np.arange(base.n), out)
    st = base.state
    inside = abi.State(x[keep], st.v[keep], st.rho[keep], st.p[keep], st.m[keep])
    sim = Simulation(cases.Case(base.name, base.params, base.geometry, inside))
    sim.upload(inside)
    sub_cella, sub_icont, sub_npo = sim.dump_grid()
    n = base.n
    want_cella = np.zeros(n, np.int32)
    want_cella[keep] = sub_cella
    want_npo = (keep[sub_npo - 1] + 1).astype(np.int32)
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    cella = torch.empty(n, dtype=torch.int32, device="cuda")
    icont = torch.empty(len(sub_icont), dtype=torch.int32, device="cuda")
    npo = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        cella.fill_(-7)
        icont.fill_(-7)
        npo.fill_(-7)
        rc = _static(base.params, xd, n, cella, icont, npo, stream)
        torch.cuda.synchronize()
        assert rc == abi.SPH_OK
        assert np.array_equal(cella.cpu().numpy(), want_cella)
        assert np.array_equal(icont.cpu().numpy(), sub_icont)
        assert np.array_equal(npo.cpu().numpy()[:len(keep)], want_npo)


def test_static_ord_grid_rejects_oversize():
    import torch
    case = cases.dam_break_2d()
    big = (1 << 20) + 1
    x = torch.zeros((1, 3), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = _static(case.params, x, big, out, out, out, None)
    assert rc == abi.SPH_ERR_INVALID_ARGUMENT
