"""The FP32-compensated form against the FP64 oracle on the accuracy
schedule: the 3D dam break compared every 0.05 s up to 0.5 s of physical
time (tests/accuracy.py), with three FP64 controls: the plain FP64 form,
the FP64 form from positions perturbed by 1e-12, and the FP64 form from the
initial state rounded to FP32.

The dam-break flow is chaotic: once the front is under way any difference
grows by about three orders of magnitude every 0.05 s.  The FP32c form's
pair sums differ from FP64 at the FP32 level every step, and from about
0.15 s on it drifts from the oracle about as far as the FP64 form started
from an FP32 copy of the initial state does (0.3 to 1.25 times that
control's error, field by field and time by time, at dx 0.01 and 0.02).
No form that does not reproduce the oracle's sums bit
for bit can meet 1e-3 on the velocity field at 0.5 s.  The bars therefore
are:

  * before the divergence (t <= 0.10 s): every field of the FP32c form
    within 1e-3 relative L2 of the oracle;
  * over the whole run: every FP32c field within a small factor of the
    largest drift of the FP64 controls, i.e. no worse than differences of
    FP32 size in the reference's own arithmetic;
  * the FP64 global sums: the mass exactly conserved by every run, and the
    FP32c volume within the same factor of the controls' drift.

The default case is dx = 0.02 m (13,500 particles).  The full-size study,
dx = 0.01 m (108,000 particles, about six minutes of the
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
    ctl = [out["summary"][k] for k in ("fp64_pert", "fp64", "fp64_ic32")]
    for f in FIELDS:
        assert s32[f]["max_pre_impact"] <= FIELD_TOL, (f, s32[f])
    for f in FIELDS:
        drift = max(c[f]["max"] for c in ctl)
        assert s32[f]["max"] <= CONTROL_FACTOR * max(drift, 1e-6), (f, s32[f], drift)
    for name in ("fp64", "fp64_pert", "fp64_ic32", "fp32c"):
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
