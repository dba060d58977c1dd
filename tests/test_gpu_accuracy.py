"""The FP32-compensated form against the FP64 oracle on the north star's
schedule: the 3D dam break compared every 0.05 s up to 0.5 s of physical
time (tests/accuracy.py), with an FP64 run from a 1e-12-perturbed state as
the control.

The dam-break flow is chaotic: any difference in the floating-point sums
grows by about three orders of magnitude every 0.05 s once the front is
well under way.  The perturbed FP64 control (1e-12 at t = 0) reaches
velocity errors of ~1e-3 near t = 0.2 s; the FP32c form, whose rates differ
from the FP64 ones by ~1e-6 every step, gets there about 0.05 s sooner;
beyond that both wander equally far from the oracle (the plain FP64 form
too, once a single rounding differs).  No form that does not reproduce the
oracle's sums bit for bit can meet 1e-3 on the velocity field at 0.5 s.
The bars therefore are:

  * before the divergence (t <= 0.10 s): every field of the FP32c form
    within 1e-3 relative L2 of the oracle;
  * over the whole run: every FP32c field within a small factor of the
    larger drift of the two FP64 runs (the control and the plain form),
    i.e. no worse than rounding-level noise in the reference's own
    arithmetic;
  * the FP64 global sums: the mass exactly conserved by every form, and the
    FP32c volume within the same factor of the FP64 runs' drift.

The default case is dx = 0.02 m (13,500 particles).  The full-size study of
the north star, dx = 0.01 m (108,000 particles, about six minutes of the
oracle on 16 host threads), runs when SPH_ACCURACY_FULL=1; either writes its
record as JSON to $SPH_ACCURACY_OUT when that is set.
"""
import json
import os

import pytest

from . import accuracy

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-3
CONTROL_FACTOR = 3.0
FIELDS = ("rho_dev", "rho", "p", "v", "x")


def _record(out):
    path = os.environ.get("SPH_ACCURACY_OUT")
    if path:
        with open(path, "w") as f:
            json.dump(out, f, indent=1)


def _check(out):
    s32 = out["summary"]["fp32c"]
    ctl = [out["summary"]["fp64_pert"], out["summary"]["fp64"]]
    for f in FIELDS:
        assert s32[f]["max_pre_impact"] <= FIELD_TOL, (f, s32[f])
    for f in FIELDS:
        drift = max(c[f]["max"] for c in ctl)
        assert s32[f]["max"] <= CONTROL_FACTOR * max(drift, 1e-6), (f, s32[f], drift)
    for name in ("fp64", "fp64_pert", "fp32c"):
        assert out["summary"][name]["mass_drift"] == 0.0
    vol = max(c["volume_rel_max"] for c in ctl)
    assert s32["volume_rel_max"] <= CONTROL_FACTOR * max(vol, 1e-7)


def test_fp32c_schedule_dam_break_3d_dx002(oracle_lib):
    out = accuracy.study(oracle_lib, dx=0.02)
    _record(out)
    _check(out)


@pytest.mark.skipif(os.environ.get("SPH_ACCURACY_FULL") != "1",
                    reason="full-size study (dx 0.01 m, about 6 min of oracle time): set SPH_ACCURACY_FULL=1")
def test_fp32c_schedule_dam_break_3d_dx001(oracle_lib):
    out = accuracy.study(oracle_lib, dx=0.01)
    _record(out)
    _check(out)
