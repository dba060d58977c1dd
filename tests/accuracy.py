"""Accuracy study of the device forms against the FP64 oracle on the
3D dam break, on the north star's schedule: fields compared every 0.05 s
up to 0.5 s of physical time.

Three device runs start from the oracle's initial state:

  * fp64       the plain FP64 form (the reference's arithmetic and order);
  * fp64_pert  the same form from positions perturbed by 1e-12 relative
               (seeded): a control that shows how far any run that does not
               reproduce the oracle's summation bit for bit drifts from it;
  * fp32c      the FP32-compensated form.

The time step is adaptive (CFL), so the forms' clocks differ slightly; each
comparison is made at the oracle's first step at or past t = 0.05 k, with
every device run stopped at that same step count (the clock offset is
recorded).  Per field: relative L2 of rho - rho0 (the density variation,
the demanding measure), rho, p, v and x; and the FP64 global sums
(fluid_global_quantities) of each run.  Test infrastructure: only the tests
use it.
"""
import time

import numpy as np

from sphera_b200 import Simulation, abi, cases


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def _with_precision(case, precision, state=None):
    prm = abi.make_params(**{f: getattr(case.params, f) for f, _ in abi.SphParams._fields_})
    prm.precision = precision
    return cases.Case(case.name, prm, case.geometry, state or case.state)


def _errors(g, ref, den0):
    return {"rho_dev": rel_l2(g.rho - den0, ref["rho"] - den0), "rho": rel_l2(g.rho, ref["rho"]),
            "p": rel_l2(g.p, ref["p"]), "v": rel_l2(g.v, ref["v"]), "x": rel_l2(g.x, ref["x"])}


def study(oracle_mod, dx, t_end=0.5, every=0.05, threads=0, perturb=1e-12, seed=0xACC):
    case = cases.dam_break_3d(dx=dx)
    den0 = case.params.den0
    t_wall = time.perf_counter()
    o = oracle_mod.Oracle(case, nthreads=threads)
    o.prepare()
    targets = [every * (k + 1) for k in range(int(round(t_end / every)))]
    snaps = []
    steps = 0
    for t in targets:
        while o.time < t - 1e-12:
            o.step(1)
            steps += 1
        snaps.append(dict(t_target=t, step=steps, t_oracle=o.time, ref=o.get(), gq=o.global_quantities()))
    oracle_s = time.perf_counter() - t_wall
    o.close()
    rng = np.random.default_rng(seed)
    x = case.state.x
    xp = x * (1.0 + perturb * rng.uniform(-1.0, 1.0, size=x.shape))
    st = case.state
    runs = {
        "fp64": _with_precision(case, abi.SPH_PREC_FP64),
        "fp64_pert": _with_precision(case, abi.SPH_PREC_FP64, abi.State(xp, st.v, st.rho, st.p, st.m)),
        "fp32c": _with_precision(case, abi.SPH_PREC_FP32C),
    }
    out = {"dx": dx, "particles": case.n, "t_end": t_end, "every": every, "oracle_seconds": oracle_s,
           "perturbation": perturb, "forms": {}}
    for name, c in runs.items():
        sim = Simulation(c)
        sim.upload(c.state)
        cur = 0
        rows = []
        for sn in snaps:
            info = sim.step(sn["step"] - cur)
            cur = sn["step"]
            g = sim.download()
            if g.n != sn["ref"]["x"].shape[0]:
                rows.append({"t": sn["t_target"], "particles_differ": [g.n, sn["ref"]["x"].shape[0]]})
                continue
            gq = sim.global_quantities()
            err = _errors(g, sn["ref"], den0)
            rows.append({"t": sn["t_target"], "step": sn["step"], "t_oracle": sn["t_oracle"],
                         "t_form": info.time, "errors": err,
                         "global": gq.tolist(), "global_oracle": sn["gq"].tolist(),
                         "global_rel": (np.abs(gq - sn["gq"]) / np.maximum(np.abs(sn["gq"]), 1e-300)).tolist()})
        sim.close()
        out["forms"][name] = rows
    # per form and field: the largest error over the schedule, before the
    # front reaches the far wall (t <= 0.15 s) and over the whole run
    summ = {}
    for name, rows in out["forms"].items():
        ok = [r for r in rows if "errors" in r]
        s = {}
        for f in ("rho_dev", "rho", "p", "v", "x"):
            s[f] = {"max": max(r["errors"][f] for r in ok),
                    "max_pre_impact": max((r["errors"][f] for r in ok if r["t"] <= 0.15 + 1e-9), default=None)}
        s["mass_drift"] = max(abs(r["global"][0] - ok[0]["global"][0]) / ok[0]["global"][0] for r in ok)
        summ[name] = s
    out["summary"] = summ
    return out
