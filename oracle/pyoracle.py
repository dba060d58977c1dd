"""ctypes wrapper of the oracle (oracle/liboracle.so) -- test infrastructure.

Only the tests, the smoke check and bench.py's CPU-baseline leg use this
module; the product never imports it.  The oracle is the FP64 C++/OpenMP
restatement in oracle/sph_oracle.cpp; parity is unpinned by reference
outputs (the reference is Fortran and cannot be built here), see that
file's header.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from sphera_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        L.ora_create.restype = vp
        L.ora_create.argtypes = [C.POINTER(abi.SphParams), C.POINTER(abi.SphGeometry), C.c_int,
                                 dp, dp, dp, dp, dp, C.c_int]
        L.ora_destroy.argtypes = [vp]
        for f in ("ora_nmaxpartj", "ora_n", "ora_nmax", "ora_truncated", "ora_removed",
                  "ora_ncbf_max", "ora_prepare", "ora_search", "ora_rhs_momentum",
                  "ora_continuity", "ora_time_step_duration", "ora_step_index"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = C.c_int
        L.ora_step.argtypes = [vp, C.c_int]
        L.ora_dt.argtypes = [vp]
        L.ora_dt.restype = C.c_double
        L.ora_time.argtypes = [vp]
        L.ora_time.restype = C.c_double
        L.ora_get.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp]
        L.ora_get_c1.argtypes = [vp, dp, dp]
        L.ora_global_quantities.argtypes = [vp, dp]
        L.ora_laminar.argtypes = [vp, ip]
        L.ora_convex_edges.argtypes = [vp, ip]
        L.ora_convex_edges.restype = C.c_int
        L.ora_grid.argtypes = [vp, ip, ip, ip]
        L.ora_grid_info.argtypes = [vp, ip, dp, dp]
        L.ora_neighbours.argtypes = [vp, C.c_int, ip, ip]
        L.ora_pair_data.argtypes = [vp, C.c_int, dp]
        L.ora_boundary.argtypes = [vp, C.c_int, ip, ip, dp]
        L.ora_tables.argtypes = [vp, dp, dp, dp]
        for f in ("ora_IWro2dro", "ora_J2Wro2"):
            getattr(L, f).argtypes = [C.c_double]
            getattr(L, f).restype = C.c_double
        L.ora_JdWsRn.argtypes = [C.c_double, C.c_int]
        L.ora_JdWsRn.restype = C.c_double
        L.ora_WIntegr.argtypes = [C.c_double, C.c_double]
        L.ora_WIntegr.restype = C.c_double
        L.ora_w.argtypes = [C.c_double, C.c_double, C.c_double]
        L.ora_w.restype = C.c_double
        L.ora_forcing_sin.argtypes = [C.c_double]
        L.ora_forcing_sin.restype = C.c_double
        _lib = L
    return _lib


def forcing_sin(x):
    """The sine used by the tank forcing (an extension, not in the reference)."""
    return lib().ora_forcing_sin(float(x))


class Oracle:
    """One simulation held by the oracle, in the reference's particle order."""

    def __init__(self, case, nthreads=0):
        L = lib()
        self.case = case
        st = case.state
        self._h = L.ora_create(C.byref(case.params), C.byref(case.geometry.struct), st.n,
                               abi.dptr(st.x), abi.dptr(st.v), abi.dptr(st.rho), abi.dptr(st.p),
                               abi.dptr(st.m), int(nthreads))
        self.dim = case.params.dim

    def close(self):
        if self._h:
            lib().ora_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, what):
        if st != 0:
            raise RuntimeError(f"oracle {what}: status {st} ({abi.STATUS_NAMES.get(st, '?')})")

    @property
    def n(self):
        return lib().ora_n(self._h)

    @property
    def nmaxpartj(self):
        return lib().ora_nmaxpartj(self._h)

    @property
    def nmax(self):
        return lib().ora_nmax(self._h)

    @property
    def dt(self):
        return lib().ora_dt(self._h)

    @property
    def time(self):
        return lib().ora_time(self._h)

    @property
    def truncated(self):
        return lib().ora_truncated(self._h)

    @property
    def removed(self):
        return lib().ora_removed(self._h)

    @property
    def ncbf_max(self):
        return lib().ora_ncbf_max(self._h)

    def prepare(self):
        self._chk(lib().ora_prepare(self._h), "prepare")

    def search(self):
        self._chk(lib().ora_search(self._h), "search")

    def rhs_momentum(self):
        self._chk(lib().ora_rhs_momentum(self._h), "rhs_momentum")

    def continuity(self):
        self._chk(lib().ora_continuity(self._h), "continuity")

    def time_step_duration(self):
        lib().ora_time_step_duration(self._h)

    def step(self, nsteps=1):
        self._chk(lib().ora_step(self._h, int(nsteps)), "step")

    def get(self):
        n = self.n
        out = {k: np.zeros((n, 3)) for k in ("x", "v", "acc")}
        out.update({k: np.zeros(n) for k in ("rho", "p", "m", "dden")})
        lib().ora_get(self._h, *(abi.dptr(out[k]) for k in ("x", "v", "rho", "p", "m", "acc", "dden")))
        return out

    def global_quantities(self):
        """fluid_global_quantities: [mass, linear momentum (3), angular
        momentum (3), volume], FP64 sums in pg order."""
        out = np.zeros(8)
        lib().ora_global_quantities(self._h, abi.dptr(out))
        return out

    def convex_edges(self):
        """(n_edges, 2) face ids of the convex edges, in the order found."""
        n = lib().ora_convex_edges(self._h, None)
        f = np.zeros((max(n, 1), 2), np.int32)
        lib().ora_convex_edges(self._h, abi.iptr(f))
        return f[:n]

    def laminar(self):
        """pg%laminar_flag as the last momentum evaluation set it."""
        f = np.zeros(self.n, np.int32)
        lib().ora_laminar(self._h, abi.iptr(f))
        return f

    def get_c1(self):
        """B_ren_gradp and B_ren_divu, (n, 3, 3) each."""
        bg = np.zeros((self.n, 3, 3))
        bd = np.zeros((self.n, 3, 3))
        lib().ora_get_c1(self._h, abi.dptr(bg), abi.dptr(bd))
        return bg, bd

    def grid(self):
        n = self.n
        cella = np.zeros(n, np.int32)
        icont = np.zeros(self.nmax + 1, np.int32)
        npo = np.zeros(n, np.int32)
        lib().ora_grid(self._h, abi.iptr(cella), abi.iptr(icont), abi.iptr(npo))
        return cella, icont, npo

    def grid_info(self):
        ncd = np.zeros(3, np.int32)
        lo = np.zeros(3)
        dcd = np.zeros(3)
        lib().ora_grid_info(self._h, abi.iptr(ncd), abi.dptr(lo), abi.dptr(dcd))
        return ncd, lo, dcd

    def neighbours(self, nmaxj=None):
        nmaxj = nmaxj or self.nmaxpartj
        counts = np.zeros(self.n, np.int32)
        lists = np.zeros((self.n, nmaxj), np.int32)
        lib().ora_neighbours(self._h, nmaxj, abi.iptr(counts), abi.iptr(lists))
        return counts, lists

    def pair_data(self, nmaxj):
        out = np.zeros((self.n, nmaxj, 7))
        lib().ora_pair_data(self._h, nmaxj, abi.dptr(out))
        return out

    def boundary(self, max_per=4):
        n = self.n
        ncb = np.zeros(n, np.int32)
        clob = np.zeros((n, max_per), np.int32)
        vals = np.zeros((n, max_per, 20))
        lib().ora_boundary(self._h, max_per, abi.iptr(ncb), abi.iptr(clob), abi.dptr(vals))
        return ncb, clob, vals

    def tables(self):
        kt = np.zeros((41, 5))
        bit = np.zeros((256, 7))
        b2 = np.zeros((22, 6))
        lib().ora_tables(self._h, abi.dptr(kt), abi.dptr(bit), abi.dptr(b2))
        return kt, bit, b2
