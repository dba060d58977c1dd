"""sphera_b200 -- B200 (sm_100a) implementation of SPHERA's per-step particle path.

Python host mirror of the C ABI declared in include/sphera_b200.h.  The
method names follow the reference subroutines each call replaces
(src/Main_algorithm/time_step_loop.f90), so a test reads like the
reference's time loop:

    sim = Simulation(case)            # CreaGrid + IC tables, device memory
    sim.upload(case.state)            # OrdGrid1 + CalcVarLength + ComputeBoundaryDataTab + dt
    sim.step(100)                     # whole leapfrog steps (CUDA graph)
    st = sim.download()

The compute runs only in libsphera_b200.so; if the library is missing the
import of the CUDA path fails loudly (there is no CPU fallback).
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsphera_b200.so")
_lib = None


class SphError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__(f"{what}: status {code} ({abi.STATUS_NAMES.get(code, 'unknown')})")


def lib():
    """Loads libsphera_b200.so (built by sphera_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python sphera_b200/build.py` "
                          "(the CUDA library is the only implementation)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    hp = C.POINTER(vp)
    sig = {
        "sph_create": ([C.POINTER(abi.SphParams), C.POINTER(abi.SphGeometry), C.c_int32, hp], C.c_int),
        "sph_batch_create": ([C.c_int32, C.POINTER(abi.SphParams), C.POINTER(abi.SphGeometry), ip, hp], C.c_int),
        "sph_destroy": ([vp], None),
        "sph_upload": ([vp, C.POINTER(abi.SphState)], C.c_int),
        "sph_batch_upload": ([vp, C.c_int32, C.POINTER(abi.SphState)], C.c_int),
        "sph_download": ([vp, C.POINTER(abi.SphState)], C.c_int),
        "sph_batch_download": ([vp, C.c_int32, C.POINTER(abi.SphState)], C.c_int),
        "sph_batch_set_end_time": ([vp, C.c_int32, C.c_double], C.c_int),
        "sph_batch_info": ([vp, C.c_int32, C.POINTER(abi.SphStepInfo), ip], C.c_int),
        "sph_step": ([vp, C.c_int32, C.POINTER(abi.SphStepInfo)], C.c_int),
        "sph_step_async": ([vp, C.c_int32], C.c_int),
        "sph_step_download": ([vp, C.c_int32, C.POINTER(abi.SphState)], C.c_int),
        "sph_sync": ([vp], C.c_int),
        "sph_stream": ([vp], vp),
        "sph_get_diagnostics": ([vp, C.POINTER(abi.SphDiagnostics)], C.c_int),
        "sph_time_step_duration": ([vp, dp], C.c_int),
        "sph_rhs_momentum": ([vp, dp], C.c_int),
        "sph_leapfrog_momentum": ([vp], C.c_int),
        "sph_leapfrog_trajectories": ([vp], C.c_int),
        "sph_ord_grid": ([vp], C.c_int),
        "sph_boundary_data_tab": ([vp], C.c_int),
        "sph_continuity": ([vp, dp], C.c_int),
        "sph_leapfrog_continuity": ([vp], C.c_int),
        "sph_eos": ([vp], C.c_int),
        "sph_dump_grid": ([vp, ip, ip, ip], C.c_int),
        "sph_dump_neighbours": ([vp, C.c_int32, ip, ip], C.c_int),
        "sph_dump_boundary": ([vp, C.c_int32, ip, ip, dp], C.c_int),
        "sph_dump_renormalisation": ([vp, dp, dp], C.c_int),
        "sph_profile_phases": ([vp, C.c_int32, dp], C.c_int),
        "sph_get_counters": ([vp, C.POINTER(C.c_uint64), C.c_int32], C.c_int),
        "sph_measure_fp64_peak": ([dp], C.c_int),
        "sph_measure_fma_peak": ([C.c_int32, dp], C.c_int),
        "sph_check_division": ([C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64), dp], C.c_int),
        "sph_autotune": ([vp, C.c_int32, ip], C.c_int),
        "sph_batch_status": ([vp, ip, dp, ip, ip], C.c_int),
        "sph_batch_cancel": ([vp, C.c_int32], C.c_int),
        "sph_memory_required": ([C.c_int32, C.POINTER(abi.SphParams), C.POINTER(abi.SphGeometry), ip,
                                 C.POINTER(C.c_uint64)], C.c_int),
        "sph_idle": ([vp, ip], C.c_int),
        "sph_global_quantities": ([vp, C.c_int32, dp], C.c_int),
        "sph_dump_laminar": ([vp, ip], C.c_int),
        "sph_set_launch_shape": ([vp, ip], C.c_int),
        "sph_create_slab": ([C.POINTER(abi.SphParams), C.POINTER(abi.SphGeometry), C.c_int32, C.c_int32,
                             C.c_int32, hp], C.c_int),
        "sph_replace_particles": ([vp, C.POINTER(abi.SphState), ip], C.c_int),
        "sph_set_time_step": ([vp, C.c_double], C.c_int),
        "sph_get_clock": ([vp, C.POINTER(abi.SphClock)], C.c_int),
        "sph_select_device": ([C.c_int32], C.c_int),
        "sph_set_clock": ([vp, C.POINTER(abi.SphClock), ip], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _chk(code, what):
    if code != abi.SPH_OK:
        raise SphError(code, what)


_SHAPE_KEYS = ("lists", "momentum", "continuity", "boundary", "integrals", "momentum_shape", "continuity_shape")


def _autotune(h, reps):
    g = np.zeros(7, np.int32)
    _chk(lib().sph_autotune(h, int(reps), abi.iptr(g)), "sph_autotune")
    return dict(zip(_SHAPE_KEYS, g.tolist()))


def _set_launch_shape(h, shape):
    g = np.array([int(shape.get(k, 0)) for k in _SHAPE_KEYS], np.int32)
    _chk(lib().sph_set_launch_shape(h, abi.iptr(g)), "sph_set_launch_shape")


def _int_ptr(a):
    """int32* of a numpy array or of a torch tensor (host or device), or NULL."""
    if a is None:
        return C.POINTER(C.c_int32)()
    if type(a).__module__.startswith("torch"):
        assert str(a.dtype) == "torch.int32" and a.is_contiguous()
        return C.cast(a.data_ptr(), C.POINTER(C.c_int32))
    return abi.iptr(np.ascontiguousarray(a, dtype=np.int32))


class Simulation:
    """One simulation on the device (a one-entry batch of the C ABI)."""

    def __init__(self, case=None, params=None, geometry=None, capacity=None, cells=None):
        """cells = (lo, hi): a slab of the simulation, its x cells lo..hi
        (1-based, inclusive) of the whole grid (sph_create_slab)."""
        if case is not None:
            params, geometry = case.params, case.geometry
            capacity = capacity or case.n
        self.params = params
        self.geometry = geometry
        self.capacity = int(capacity)
        self._h = C.c_void_p()
        if cells is None:
            _chk(lib().sph_create(C.byref(params), C.byref(geometry.struct), self.capacity, C.byref(self._h)),
                 "sph_create")
        else:
            _chk(lib().sph_create_slab(C.byref(params), C.byref(geometry.struct), self.capacity, int(cells[0]),
                                       int(cells[1]), C.byref(self._h)), "sph_create_slab")
        self.n = 0

    def replace_particles(self, state, laminar=None):
        """A new particle set (and its laminar flags), the clock kept; the
        search runs on it.  state and laminar may be host arrays or, for a
        host that keeps them on the device, device tensors."""
        _chk(lib().sph_replace_particles(self._h, C.byref(state.struct), _int_ptr(laminar)), "sph_replace_particles")
        self.n = state.n

    def set_time_step(self, dt):
        _chk(lib().sph_set_time_step(self._h, float(dt)), "sph_set_time_step")

    def clock(self):
        """time, dt, dt_prev, dt_average and step between steps (sph_get_clock)."""
        c = abi.SphClock()
        _chk(lib().sph_get_clock(self._h, C.byref(c)), "sph_get_clock")
        return {"time": c.time, "dt": c.dt, "dt_prev": c.dt_prev, "dt_average": c.dt_average, "step": c.step}

    def set_clock(self, clock, laminar=None):
        """Resume after upload(): the saved clock and laminar flags (sph_set_clock)."""
        c = abi.SphClock()
        c.time, c.dt, c.dt_prev = float(clock["time"]), float(clock["dt"]), float(clock["dt_prev"])
        c.dt_average, c.step = float(clock["dt_average"]), int(clock["step"])
        lam = None if laminar is None else np.ascontiguousarray(laminar, dtype=np.int32)
        _chk(lib().sph_set_clock(self._h, C.byref(c), abi.iptr(lam)), "sph_set_clock")

    def close(self):
        if self._h:
            lib().sph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ----------------------------------------------------------------- state
    def upload(self, state):
        _chk(lib().sph_upload(self._h, C.byref(state.struct)), "sph_upload")
        self.n = state.n

    def download(self):
        info = self.diagnostics()
        n = self.n
        st = abi.State.empty(n)
        _chk(lib().sph_download(self._h, C.byref(st.struct)), "sph_download")
        n2 = st.struct.n
        if n2 != n:
            st = abi.State(st.x[:n2], st.v[:n2], st.rho[:n2], st.p[:n2], st.m[:n2])
            self.n = n2
        del info
        return st

    def step(self, nsteps=1):
        info = abi.SphStepInfo()
        _chk(lib().sph_step(self._h, int(nsteps), C.byref(info)), "sph_step")
        self.n = info.n
        return info

    def step_async(self, nsteps=1):
        _chk(lib().sph_step_async(self._h, int(nsteps)), "sph_step_async")

    def step_download(self, nsteps=1):
        """step(nsteps) then download(), the last step's x, v, m copied to
        the host while that step finishes (sph_step_download).  The buffers
        here are pageable numpy arrays, so the results are the same but the
        copy does not overlap the step; a caller that wants the overlap
        passes page-locked buffers to the C ABI (as bench.py's e2e leg does)."""
        n = self.n
        st = abi.State.empty(n)
        _chk(lib().sph_step_download(self._h, int(nsteps), C.byref(st.struct)), "sph_step_download")
        n2 = st.struct.n
        if n2 != n:
            st = abi.State(st.x[:n2], st.v[:n2], st.rho[:n2], st.p[:n2], st.m[:n2])
            self.n = n2
        return st

    def sync(self):
        _chk(lib().sph_sync(self._h), "sph_sync")

    def idle(self):
        """True when the work enqueued by step_async has finished (never waits)."""
        v = C.c_int32()
        _chk(lib().sph_idle(self._h, C.byref(v)), "sph_idle")
        return bool(v.value)

    @property
    def stream(self):
        return lib().sph_stream(self._h)

    def diagnostics(self):
        d = abi.SphDiagnostics()
        _chk(lib().sph_get_diagnostics(self._h, C.byref(d)), "sph_get_diagnostics")
        return d

    # ------------------------------------------- one call per Fortran call site
    def time_step_duration(self):
        dt = C.c_double()
        _chk(lib().sph_time_step_duration(self._h, C.byref(dt)), "sph_time_step_duration")
        return dt.value

    def rhs_momentum(self, want=True):
        acc = np.zeros((self.n, 3)) if want else None
        _chk(lib().sph_rhs_momentum(self._h, abi.dptr(acc)), "sph_rhs_momentum")
        return acc

    def leapfrog_momentum(self):
        _chk(lib().sph_leapfrog_momentum(self._h), "sph_leapfrog_momentum")

    def leapfrog_trajectories(self):
        _chk(lib().sph_leapfrog_trajectories(self._h), "sph_leapfrog_trajectories")

    def ord_grid(self):
        _chk(lib().sph_ord_grid(self._h), "sph_ord_grid")

    def boundary_data_tab(self):
        _chk(lib().sph_boundary_data_tab(self._h), "sph_boundary_data_tab")

    def continuity(self, want=True):
        dden = np.zeros(self.n) if want else None
        _chk(lib().sph_continuity(self._h, abi.dptr(dden)), "sph_continuity")
        return dden

    def leapfrog_continuity(self):
        _chk(lib().sph_leapfrog_continuity(self._h), "sph_leapfrog_continuity")

    def eos(self):
        _chk(lib().sph_eos(self._h), "sph_eos")

    def global_quantities(self):
        """fluid_global_quantities: [mass, linear momentum (3), angular
        momentum about the origin (3), volume], FP64 sums on the device."""
        out = np.zeros(8)
        _chk(lib().sph_global_quantities(self._h, 0, abi.dptr(out)), "sph_global_quantities")
        return out

    # ------------------------------------------------------------ autotuner
    def autotune(self, reps=3):
        """Sizes the persistent grids of the pair, list and boundary kernels
        and picks the pair loops' shapes (0 lean, 1 batched record loads,
        2 in the FP32c form: batched with paired FP32 arithmetic)."""
        return _autotune(self._h, reps)

    def set_launch_shape(self, shape):
        """Applies a launch configuration (autotune's dict; missing keys 0)."""
        _set_launch_shape(self._h, shape)

    # ------------------------------------------------------------ profiling
    PHASES = ("momentum", "ord_grid", "boundary_data_tab", "neighbour_lists", "continuity", "time_step")

    def profile_phases(self, nsteps):
        ms = np.zeros(6)
        _chk(lib().sph_profile_phases(self._h, int(nsteps), abi.dptr(ms)), "sph_profile_phases")
        return dict(zip(self.PHASES, ms))

    def counters(self, reset=False):
        c = (C.c_uint64 * 4)()
        _chk(lib().sph_get_counters(self._h, c, int(bool(reset))), "sph_get_counters")
        return dict(candidates=c[0], pairs=c[1])

    # --------------------------------------------------------- verification
    def dump_grid(self):
        d = self.diagnostics()
        cella = np.zeros(self.n, np.int32)
        icont = np.zeros(d.n_cells + 1, np.int32)
        npo = np.zeros(self.n, np.int32)
        _chk(lib().sph_dump_grid(self._h, abi.iptr(cella), abi.iptr(icont), abi.iptr(npo)), "sph_dump_grid")
        return cella, icont, npo

    def dump_neighbours(self, nmaxj=None):
        nmaxj = nmaxj or self.diagnostics().nmaxpartj
        counts = np.zeros(self.n, np.int32)
        lists = np.zeros((self.n, nmaxj), np.int32)
        _chk(lib().sph_dump_neighbours(self._h, nmaxj, abi.iptr(counts), abi.iptr(lists)), "sph_dump_neighbours")
        return counts, lists

    def dump_boundary(self, max_per=4):
        ncb = np.zeros(self.n, np.int32)
        clob = np.zeros((self.n, max_per), np.int32)
        vals = np.zeros((self.n, max_per, 20))
        _chk(lib().sph_dump_boundary(self._h, max_per, abi.iptr(ncb), abi.iptr(clob), abi.dptr(vals)),
             "sph_dump_boundary")
        return ncb, clob, vals

    def dump_laminar(self):
        """pg%laminar_flag of the last momentum pass, caller order."""
        f = np.zeros(self.n, np.int32)
        _chk(lib().sph_dump_laminar(self._h, abi.iptr(f)), "sph_dump_laminar")
        return f

    def dump_laminar_into(self, flags):
        """dump_laminar into a caller's int32 array or device tensor of n entries."""
        _chk(lib().sph_dump_laminar(self._h, _int_ptr(flags)), "sph_dump_laminar")

    def download_into(self, state):
        """download() into a caller's state (abi.State or a state of device
        tensors, n rows); returns the particle count."""
        _chk(lib().sph_download(self._h, C.byref(state.struct)), "sph_download")
        return state.struct.n

    def dump_renormalisation(self, divu=True):
        """B_ren_gradp and (divu) B_ren_divu in caller order, (n, 3, 3)."""
        bg = np.zeros((self.n, 3, 3))
        bd = np.zeros((self.n, 3, 3)) if divu else None
        _chk(lib().sph_dump_renormalisation(self._h, abi.dptr(bg), abi.dptr(bd)),
             "sph_dump_renormalisation")
        return bg, bd


def memory_required(cases):
    """Device bytes a batch of these cases would allocate (one case: a
    Simulation), computed on the host; no device is needed."""
    cases = list(cases)
    n = len(cases)
    prm = (abi.SphParams * n)(*[c.params for c in cases])
    geo = (abi.SphGeometry * n)(*[c.geometry.struct for c in cases])
    caps = np.array([c.n for c in cases], np.int32)
    b = C.c_uint64()
    _chk(lib().sph_memory_required(n, prm, geo, abi.iptr(caps), C.byref(b)), "sph_memory_required")
    return int(b.value)


def measure_fp64_peak():
    """Dense FP64 FMA throughput of the current device, TFLOP/s."""
    t = C.c_double()
    _chk(lib().sph_measure_fp64_peak(C.byref(t)), "sph_measure_fp64_peak")
    return t.value


def measure_fp32_peak():
    """Dense FP32 FMA throughput of the current device, TFLOP/s."""
    t = C.c_double()
    _chk(lib().sph_measure_fma_peak(1, C.byref(t)), "sph_measure_fma_peak")
    return t.value


def check_division(count, seed=0x5EED):
    """The kernels' exact FP64 division against the IEEE a / b on count
    generated operand pairs (sph_check_division): (mismatches, (a, b) of one
    mismatch or None)."""
    n = C.c_uint64()
    first = (C.c_double * 2)()
    _chk(lib().sph_check_division(int(count), int(seed), C.byref(n), first), "sph_check_division")
    return int(n.value), ((first[0], first[1]) if n.value else None)


def select_device(device):
    """The device the next Simulation / Batch of this thread is built on
    (sph_select_device); a handle keeps its device afterwards."""
    _chk(lib().sph_select_device(int(device)), "sph_select_device")


class Batch:
    """Several independent simulations advanced by the same launches;
    device: the GPU to build it on (default: the thread's current one)."""

    def __init__(self, cases, device=None):
        if device is not None:
            select_device(device)
        self.device = device
        self.cases = list(cases)
        n = len(self.cases)
        self._params = (abi.SphParams * n)(*[c.params for c in self.cases])
        self._geoms = (abi.SphGeometry * n)(*[c.geometry.struct for c in self.cases])
        self._caps = np.array([c.n for c in self.cases], np.int32)
        self._h = C.c_void_p()
        _chk(lib().sph_batch_create(n, self._params, self._geoms, abi.iptr(self._caps), C.byref(self._h)),
             "sph_batch_create")

    def close(self):
        if self._h:
            lib().sph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, states=None):
        states = states or [c.state for c in self.cases]
        arr = (abi.SphState * len(states))(*[s.struct for s in states])
        _chk(lib().sph_batch_upload(self._h, len(states), arr), "sph_batch_upload")

    def set_end_time(self, sim, t_end):
        _chk(lib().sph_batch_set_end_time(self._h, int(sim), float(t_end)), "sph_batch_set_end_time")

    def step(self, nsteps=1):
        info = abi.SphStepInfo()
        _chk(lib().sph_step(self._h, int(nsteps), C.byref(info)), "sph_step")

    def step_async(self, nsteps=1):
        _chk(lib().sph_step_async(self._h, int(nsteps)), "sph_step_async")

    def sync(self):
        _chk(lib().sph_sync(self._h), "sph_sync")

    def idle(self):
        """True when the work enqueued by step_async has finished (never waits)."""
        v = C.c_int32()
        _chk(lib().sph_idle(self._h, C.byref(v)), "sph_idle")
        return bool(v.value)

    def autotune(self, reps=3):
        return _autotune(self._h, reps)

    def set_launch_shape(self, shape):
        _set_launch_shape(self._h, shape)

    def info(self, sim):
        info = abi.SphStepInfo()
        fr = C.c_int32()
        _chk(lib().sph_batch_info(self._h, int(sim), C.byref(info), C.byref(fr)), "sph_batch_info")
        return info, bool(fr.value)

    def status(self):
        """(frozen, time, steps, status) arrays of all simulations, one
        read-back; status holds each member's fatal code (0: none)."""
        n = len(self.cases)
        fr = np.zeros(n, np.int32)
        t = np.zeros(n)
        st = np.zeros(n, np.int32)
        code = np.zeros(n, np.int32)
        _chk(lib().sph_batch_status(self._h, abi.iptr(fr), abi.dptr(t), abi.iptr(st), abi.iptr(code)),
             "sph_batch_status")
        return fr.astype(bool), t, st, code

    def cancel(self, sim):
        """Freezes member `sim` from the next launch on (SPH_CANCELLED)."""
        _chk(lib().sph_batch_cancel(self._h, int(sim)), "sph_batch_cancel")

    def global_quantities(self):
        """fluid_global_quantities of every simulation, (nsims, 8)."""
        out = np.zeros((len(self.cases), 8))
        _chk(lib().sph_global_quantities(self._h, -1, abi.dptr(out)), "sph_global_quantities")
        return out

    def download(self, sim):
        n = self.cases[sim].n
        st = abi.State.empty(n)
        _chk(lib().sph_batch_download(self._h, int(sim), C.byref(st.struct)), "sph_batch_download")
        n2 = st.struct.n
        return abi.State(st.x[:n2], st.v[:n2], st.rho[:n2], st.p[:n2], st.m[:n2])
