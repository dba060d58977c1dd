"""ctypes mirror of the C ABI structs declared in include/sphera_b200.h.

The field order and types match the header exactly; `make_params`,
`make_geometry` and `make_state` build them from Python values / numpy
arrays and keep the backing arrays alive on the returned object.
"""
import ctypes as C

import numpy as np

SPH_OK = 0
SPH_ERR_INVALID_ARGUMENT = 1
SPH_ERR_UNSUPPORTED = 2
SPH_ERR_CUDA = 3
SPH_ERR_NO_DEVICE = 5
SPH_ERR_TIMEOUT = 6
SPH_CANCELLED = 7
SPH_ERR_ALLOC = 400
SPH_ERR_BDT_OVERFLOW = 802
SPH_ERR_CLOSE_FACES = 807
SPH_ERR_CLOSE_SIDES = 808
SPH_ERR_NCBF_MAX = 904

SPH_WARN_NEIGHBOURS_TRUNCATED = 0x1
SPH_WARN_PARTICLES_REMOVED = 0x2

SPH_PREC_FP64 = 0
SPH_PREC_FP32C = 1

SPH_ZONE_FIXE = 1
SPH_ZONE_TAPI = 2

STATUS_NAMES = {
    SPH_OK: "ok",
    SPH_ERR_INVALID_ARGUMENT: "invalid argument",
    SPH_ERR_UNSUPPORTED: "unsupported feature",
    SPH_ERR_CUDA: "CUDA runtime error",
    SPH_ERR_NO_DEVICE: "no sm_100 device",
    SPH_ERR_TIMEOUT: "bounded device wait timed out",
    SPH_CANCELLED: "cancelled by the host",
    SPH_ERR_ALLOC: "allocation failure (diagnostic 4)",
    SPH_ERR_BDT_OVERFLOW: "BoundaryDataTab overflow (diagnostic 8/2)",
    SPH_ERR_CLOSE_FACES: "too many close boundary faces (diagnostic 8/7)",
    SPH_ERR_CLOSE_SIDES: "too many close boundary sides (diagnostic 8/8)",
    SPH_ERR_NCBF_MAX: "Ncbf_Max > MAXCLOSEBOUNDFACES (diagnostic 9/4)",
}

_d3 = C.c_double * 3
_i3 = C.c_int32 * 3


class SphParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32),
        ("precision", C.c_int32),
        ("dx", C.c_double),
        ("trunc", C.c_double),
        ("coef_nmaxpartj", C.c_double),
        ("max_close_bound_faces", C.c_int32),
        ("dt_alfa_mon", C.c_int32),
        ("domain_lo", _d3),
        ("domain_hi", _d3),
        ("den0", C.c_double),
        ("eps", C.c_double),
        ("alfa_mon", C.c_double),
        ("kin_visc", C.c_double),
        ("p_ref", C.c_double),
        ("grav", _d3),
        ("cfl", C.c_double),
        ("vsc_coeff", C.c_double),
        ("pesodt", C.c_double),
        ("density_thresholds", C.c_int32),
        ("bdt_capacity", C.c_int32),
        ("teta_p", C.c_double),
        ("teta_v", C.c_double),
        ("forcing_amplitude", C.c_double),
        ("forcing_period", C.c_double),
        ("c1_be", C.c_int32),
        ("c1_divu", C.c_int32),
        ("invb_det_thresh", C.c_double),
    ]


class SphZone(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("slip_coefficient_mode", C.c_int32),
        ("velocity", _d3),
        ("bc_shear_stress_input", C.c_double),
        ("laminar_no_slip_check", C.c_int32),
        ("reserved", C.c_int32),
    ]


class SphGeometry(C.Structure):
    _fields_ = [
        ("n_vertices", C.c_int32),
        ("vertices", C.POINTER(C.c_double)),
        ("n_zones", C.c_int32),
        ("zones", C.POINTER(SphZone)),
        ("n_faces", C.c_int32),
        ("face_nodes", C.POINTER(C.c_int32)),
        ("face_zone", C.POINTER(C.c_int32)),
        ("n_sides", C.c_int32),
        ("side_vertices", C.POINTER(C.c_int32)),
        ("side_zone", C.POINTER(C.c_int32)),
    ]


class SphState(C.Structure):
    _fields_ = [
        ("n", C.c_int32),
        ("x", C.POINTER(C.c_double)),
        ("v", C.POINTER(C.c_double)),
        ("rho", C.POINTER(C.c_double)),
        ("p", C.POINTER(C.c_double)),
        ("m", C.POINTER(C.c_double)),
    ]


class SphStepInfo(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("step", C.c_int32),
        ("n", C.c_int32),
        ("warnings", C.c_int32),
        ("max_neighbours", C.c_int32),
    ]


class SphClock(C.Structure):
    _fields_ = [
        ("time", C.c_double),
        ("dt", C.c_double),
        ("dt_prev", C.c_double),
        ("dt_average", C.c_double),
        ("step", C.c_int32),
        ("reserved", C.c_int32),
    ]


class SphDiagnostics(C.Structure):
    _fields_ = [
        ("warnings", C.c_int32),
        ("status", C.c_int32),
        ("removed_out_of_grid", C.c_int32),
        ("ncbf_max", C.c_int32),
        ("bdt_entries", C.c_int32),
        ("nmaxpartj", C.c_int32),
        ("grid_ncd", _i3),
        ("n_cells", C.c_int32),
    ]


def dptr(a):
    """double* of a C-contiguous float64 array (or NULL for None)."""
    if a is None:
        return C.POINTER(C.c_double)()
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    """int32* of a C-contiguous int32 array (or NULL for None)."""
    if a is None:
        return C.POINTER(C.c_int32)()
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def make_params(**kw):
    p = SphParams()
    for k, v in kw.items():
        if k in ("domain_lo", "domain_hi", "grav"):
            setattr(p, k, _d3(*[float(t) for t in v]))
        else:
            setattr(p, k, v)
    return p


class Geometry:
    """Owns the arrays behind an SphGeometry struct."""

    def __init__(self, vertices, zones, faces=None, face_zone=None, sides=None, side_zone=None):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
        self.zones = list(zones)
        self.faces = None if faces is None else np.ascontiguousarray(faces, dtype=np.int32).reshape(-1, 4)
        self.face_zone = None if face_zone is None else np.ascontiguousarray(face_zone, dtype=np.int32)
        self.sides = None if sides is None else np.ascontiguousarray(sides, dtype=np.int32).reshape(-1, 2)
        self.side_zone = None if side_zone is None else np.ascontiguousarray(side_zone, dtype=np.int32)
        self._zone_arr = (SphZone * max(1, len(self.zones)))()
        for i, z in enumerate(self.zones):
            self._zone_arr[i] = z
        g = SphGeometry()
        g.n_vertices = len(self.vertices)
        g.vertices = dptr(self.vertices)
        g.n_zones = len(self.zones)
        g.zones = C.cast(self._zone_arr, C.POINTER(SphZone))
        g.n_faces = 0 if self.faces is None else len(self.faces)
        g.face_nodes = iptr(self.faces)
        g.face_zone = iptr(self.face_zone)
        g.n_sides = 0 if self.sides is None else len(self.sides)
        g.side_vertices = iptr(self.sides)
        g.side_zone = iptr(self.side_zone)
        self.struct = g


def make_zone(type=SPH_ZONE_FIXE, velocity=(0.0, 0.0, 0.0), slip=0.0, laminar_no_slip_check=0):
    z = SphZone()
    z.type = type
    z.slip_coefficient_mode = 1
    z.velocity = _d3(*velocity)
    z.bc_shear_stress_input = slip
    z.laminar_no_slip_check = laminar_no_slip_check
    return z


class State:
    """Owns the arrays behind an SphState struct (caller order)."""

    def __init__(self, x, v, rho, p, m):
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        self.v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self.rho = np.ascontiguousarray(rho, dtype=np.float64)
        self.p = np.ascontiguousarray(p, dtype=np.float64)
        self.m = np.ascontiguousarray(m, dtype=np.float64)
        s = SphState()
        s.n = len(self.rho)
        s.x = dptr(self.x)
        s.v = dptr(self.v)
        s.rho = dptr(self.rho)
        s.p = dptr(self.p)
        s.m = dptr(self.m)
        self.struct = s

    @property
    def n(self):
        return len(self.rho)

    @staticmethod
    def empty(n):
        return State(np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n), np.zeros(n), np.zeros(n))
