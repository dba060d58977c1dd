"""Checkpoint files of one simulation: the state part of a restart.

SPHERA's restart (Memo_Results.f90, read back by ReadRestartFile.f90)
writes the clock (it, simulation_time, dt) and pg(1:nag) as Fortran
unformatted records.  A snapshot here holds the same things for the device
path -- parameters, geometry, the SoA state in caller order, the clock
(sph_get_clock) and pg%laminar_flag, the one per-particle value a step
carries into the next besides the state -- so that load() and the steps
after it continue exactly as the uninterrupted run.

File layout, all little-endian:

    8 bytes   b"SPHSNAP1"
    8 bytes   uint64, length H of the header
    H bytes   UTF-8 JSON: {"format": 1, "params": {...}, "zones": [...],
              "clock": {...}, "arrays": {name: {"dtype", "shape", "offset",
              "nbytes"}}}
    ...       the arrays, each at its offset (16-byte aligned) from the end
              of the header
"""
import json
import struct

import numpy as np

from . import abi

MAGIC = b"SPHSNAP1"
_ALIGN = 16


def _params_dict(p):
    out = {}
    for name, _ in abi.SphParams._fields_:
        v = getattr(p, name)
        out[name] = list(v) if hasattr(v, "__len__") else v
    return out


def _zone_dict(z):
    return {"type": z.type, "slip_coefficient_mode": z.slip_coefficient_mode, "velocity": list(z.velocity),
            "bc_shear_stress_input": z.bc_shear_stress_input, "laminar_no_slip_check": z.laminar_no_slip_check}


def _zone(d):
    z = abi.make_zone(type=d["type"], velocity=d["velocity"], slip=d["bc_shear_stress_input"],
                      laminar_no_slip_check=d["laminar_no_slip_check"])
    z.slip_coefficient_mode = d["slip_coefficient_mode"]
    return z


def write(path, params, geometry, state, clock, laminar=None):
    """Writes a snapshot from host data (no device needed)."""
    arrays = {"x": state.x, "v": state.v, "rho": state.rho, "p": state.p, "m": state.m,
              "vertices": geometry.vertices}
    if laminar is not None:
        arrays["laminar"] = np.ascontiguousarray(laminar, dtype=np.int32)
    for name in ("faces", "face_zone", "sides", "side_zone"):
        a = getattr(geometry, name)
        if a is not None:
            arrays[name] = a
    meta, blobs, off = {}, [], 0
    for name, a in arrays.items():
        a = np.ascontiguousarray(a)
        le = a.astype(a.dtype.newbyteorder("<"), copy=False)
        meta[name] = {"dtype": le.dtype.str, "shape": list(a.shape), "offset": off, "nbytes": le.nbytes}
        pad = (-le.nbytes) % _ALIGN
        blobs.append(le.tobytes() + b"\0" * pad)
        off += le.nbytes + pad
    header = {"format": 1, "params": _params_dict(params), "zones": [_zone_dict(z) for z in geometry.zones],
              "clock": {k: clock[k] for k in ("time", "dt", "dt_prev", "dt_average", "step")}, "arrays": meta}
    hb = json.dumps(header).encode("utf-8")
    hb += b" " * ((-len(hb)) % _ALIGN)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(hb)))
        f.write(hb)
        for b in blobs:
            f.write(b)


def read(path):
    """The snapshot's contents on the host: dict with params (SphParams),
    geometry (abi.Geometry), state (abi.State), clock (dict), laminar."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a snapshot file")
        (hlen,) = struct.unpack("<Q", f.read(8))
        header = json.loads(f.read(hlen).decode("utf-8"))
        blob = f.read()
    if header.get("format") != 1:
        raise ValueError(f"{path}: unknown snapshot format {header.get('format')}")
    arr = {}
    for name, m in header["arrays"].items():
        if m["offset"] + m["nbytes"] > len(blob):
            raise ValueError(f"{path}: truncated array {name}")
        a = np.frombuffer(blob, dtype=np.dtype(m["dtype"]), count=int(np.prod(m["shape"], dtype=np.int64)),
                          offset=m["offset"]).reshape(m["shape"])
        arr[name] = a.astype(a.dtype.newbyteorder("="))
    params = abi.make_params(**header["params"])
    geometry = abi.Geometry(arr["vertices"], [_zone(z) for z in header["zones"]], arr.get("faces"),
                            arr.get("face_zone"), arr.get("sides"), arr.get("side_zone"))
    state = abi.State(arr["x"], arr["v"], arr["rho"], arr["p"], arr["m"])
    return {"params": params, "geometry": geometry, "state": state, "clock": header["clock"],
            "laminar": arr.get("laminar")}


def save(path, sim):
    """Checkpoints a Simulation between steps."""
    write(path, sim.params, sim.geometry, sim.download(), sim.clock(), sim.dump_laminar())


def load(path, capacity=None):
    """A new Simulation resumed from a snapshot (sph_upload + sph_set_clock)."""
    from . import Simulation
    d = read(path)
    sim = Simulation(params=d["params"], geometry=d["geometry"], capacity=capacity or d["state"].n)
    sim.upload(d["state"])
    sim.set_clock(d["clock"], d["laminar"])
    return sim
