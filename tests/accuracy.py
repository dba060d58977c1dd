"""Accuracy study of the device forms against the FP64 oracle on the
3D dam break: fields compared every 0.05 s
up to 0.5 s of physical time.

Three device runs start from the oracle's initial state:

  * fp64       the plain FP64 form (the reference's arithmetic and order);
  * fp64_pert  the same form from positions perturbed by 1e-12 relative
               (seeded): a control that shows how far any run that does not
               reproduce the oracle's floating-point sums bit for bit drifts
               from it;
  * fp64_ic32  the same form from the initial state rounded to FP32 (x, v,
               rho, p, m as an FP32 code would hold them): a control of the
               size of the differences FP32 arithmetic brings, made once;
  * fp32c      the FP32-compensated form.

The time step is adaptive (CFL on the largest speed), so the runs' clocks
drift apart once their fastest particles differ.  Every run is therefore
compared at the same physical times: each one (the oracle too) is stepped
until its clock passes t = 0.05 k, and its state is interpolated linearly
between the last step before and the first step after t (an error of order
dt^2 |a|, far below the differences measured).  Per field: relative L2 of
rho - rho0 (the density variation, the demanding measure), rho, p, v and x;
the FP64 global sums (fluid_global_quantities) of each run at its step
after t; and the position of the water front (largest x of the oracle's
particles).  Test infrastructure: only the tests use it.
"""
import time

import numpy as np

from sphera_b200 import Simulation, abi, cases

FIELDS = ("x", "v", "rho", "p")


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _with_precision(case, precision, state=None):
    prm = abi.make_params(**{f: getattr(case.params, f) for f, _ in abi.SphParams._fields_})
    prm.precision = precision
    return cases.Case(case.name, prm, case.geometry, state or case.state)


def _lerp(a, b, ta, tb, t):
    w = (t - ta) / (tb - ta) if tb > ta else 1.0
    return {k: a[k] + w * (b[k] - a[k]) for k in FIELDS}


def _errors(g, ref, den0):
    return {"rho_dev": rel_l2(g["rho"] - den0, ref["rho"] - den0), "rho": rel_l2(g["rho"], ref["rho"]),
            "p": rel_l2(g["p"], ref["p"]), "v": rel_l2(g["v"], ref["v"]), "x": rel_l2(g["x"], ref["x"])}


def _oracle_snaps(oracle_mod, case, targets, threads):
    o = oracle_mod.Oracle(case, nthreads=threads)
    o.prepare()
    snaps, steps = [], 0
    prev, t_prev = None, 0.0
    for t in targets:
        while o.time < t - 1e-12:
            if o.time + 1.5 * o.dt >= t:
                prev, t_prev = o.get(), o.time
            o.step(1)
            steps += 1
        cur = o.get()
        state = _lerp(prev, cur, t_prev, o.time, t) if prev is not None else cur
        snaps.append(dict(t=t, step=steps, t_after=o.time, state=state, gq=o.global_quantities(),
                          front_x=float(cur["x"][:, 0].max())))
    o.close()
    return snaps


def _device_snaps(case, targets):
    sim = Simulation(case)
    sim.upload(case.state)
    out = []
    t_now, dt_last, steps = 0.0, sim.time_step_duration(), 0
    prev, t_prev = None, 0.0

    def grab():
        st = sim.download()
        return {"x": st.x, "v": st.v, "rho": st.rho, "p": st.p}

    for t in targets:
        while t_now < t - 1e-12:
            if t_now + 1.5 * dt_last >= t:
                prev, t_prev = grab(), t_now
            info = sim.step(1)
            steps += 1
            t_now, dt_last = info.time, info.dt
        cur = grab()
        state = _lerp(prev, cur, t_prev, t_now, t) if prev is not None else cur
        out.append(dict(t=t, step=steps, t_after=t_now, state=state, gq=sim.global_quantities(),
                        n=sim.n))
    sim.close()
    return out


def study(oracle_mod, dx, t_end=0.5, every=0.05, threads=0, perturb=1e-12, seed=0xACC, pre_impact=0.10):
    case = cases.dam_break_3d(dx=dx)
    den0 = case.params.den0
    targets = [every * (k + 1) for k in range(int(round(t_end / every)))]
    t_wall = time.perf_counter()
    snaps = _oracle_snaps(oracle_mod, case, targets, threads)
    oracle_s = time.perf_counter() - t_wall
    rng = np.random.default_rng(seed)
    x = case.state.x
    xp = x * (1.0 + perturb * rng.uniform(-1.0, 1.0, size=x.shape))
    st = case.state
    r32 = lambda a: a.astype(np.float32).astype(np.float64)
    runs = {
        "fp64": _with_precision(case, abi.SPH_PREC_FP64),
        "fp64_pert": _with_precision(case, abi.SPH_PREC_FP64, abi.State(xp, st.v, st.rho, st.p, st.m)),
        "fp64_ic32": _with_precision(case, abi.SPH_PREC_FP64,
                                     abi.State(r32(st.x), r32(st.v), r32(st.rho), r32(st.p), r32(st.m))),
        "fp32c": _with_precision(case, abi.SPH_PREC_FP32C),
    }
    out = {"dx": dx, "particles": case.n, "t_end": t_end, "every": every, "oracle_seconds": oracle_s,
           "perturbation": perturb, "pre_impact_t": pre_impact, "tank_length": 1.6,
           "front_x": [s["front_x"] for s in snaps], "forms": {}}
    for name, c in runs.items():
        rows = []
        for sn, g in zip(snaps, _device_snaps(c, targets)):
            ref = sn["state"]
            if g["n"] != ref["x"].shape[0]:
                rows.append({"t": sn["t"], "particles_differ": [g["n"], ref["x"].shape[0]]})
                continue
            rows.append({"t": sn["t"], "step_oracle": sn["step"], "step_form": g["step"],
                         "errors": _errors(g["state"], ref, den0),
                         "global": g["gq"].tolist(), "global_oracle": sn["gq"].tolist(),
                         "global_rel": (np.abs(g["gq"] - sn["gq"])
                                        / np.maximum(np.abs(sn["gq"]), 1e-300)).tolist()})
        out["forms"][name] = rows
    # per form and field: the largest error before the divergence time and
    # over the whole run
    summ = {}
    for name, rows in out["forms"].items():
        ok = [r for r in rows if "errors" in r]
        s = {}
        for f in ("rho_dev", "rho", "p", "v", "x"):
            s[f] = {"max": max(r["errors"][f] for r in ok),
                    "max_pre_impact": max((r["errors"][f] for r in ok if r["t"] <= pre_impact + 1e-9), default=None)}
        s["mass_drift"] = max(abs(r["global"][0] - ok[0]["global"][0]) / ok[0]["global"][0] for r in ok)
        s["volume_rel_max"] = max(r["global_rel"][7] for r in ok)
        summ[name] = s
    out["summary"] = summ
    return out
