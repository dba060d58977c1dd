"""The C ABI without a device: the library loads, exports every entry point
include/sphera_b200.h declares, and the ctypes mirror of each struct has the
header's layout (checked against the C compiler's own sizeof/offsetof)."""
import ctypes as C
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import sphera_b200
from sphera_b200 import abi, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sphera_b200.h")

STRUCTS = [abi.SphParams, abi.SphZone, abi.SphGeometry, abi.SphState, abi.SphStepInfo, abi.SphDiagnostics,
           abi.SphClock]


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sph_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_entry_point():
    L = sphera_b200.lib()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_header_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "sphera_b200.h"', "int main(void) {"]
    for S in STRUCTS:
        name = S.__name__
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for f, _ in S._fields_:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    c_layout = {}
    for ln in out:
        if ln.strip():
            s, f, v = ln.split()
            c_layout[(s, f)] = int(v)
    for S in STRUCTS:
        name = S.__name__
        assert c_layout[(name, "sizeof")] == C.sizeof(S), name
        for f, _ in S._fields_:
            assert c_layout[(name, f)] == getattr(S, f).offset, (name, f)


def test_memory_required_needs_no_device():
    small = cases.dam_break_3d(dx=0.02)
    big = cases.dam_break_3d(dx=0.01)
    a = sphera_b200.memory_required([small])
    b = sphera_b200.memory_required([big])
    both = sphera_b200.memory_required([small, big])
    assert 0 < a < b
    # per-particle arrays dominate: about 2 kB a particle in 3D
    assert 1500 < b / big.n < 2600
    assert both >= a + b - (1 << 20)


def test_invalid_forcing_is_rejected():
    c = cases.sloshing_3d(dx=0.05, amplitude=0.02, period=0.0)
    with pytest.raises(sphera_b200.SphError) as e:
        sphera_b200.memory_required([c])
    assert e.value.code == abi.SPH_ERR_INVALID_ARGUMENT


def test_without_a_device_create_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    c = cases.dam_break_2d(dx=0.05)
    with pytest.raises(sphera_b200.SphError) as e:
        sphera_b200.Simulation(c)
    assert e.value.code in (abi.SPH_ERR_NO_DEVICE, abi.SPH_ERR_CUDA)


def test_batch_of_mixed_dims_is_rejected_before_allocation():
    a = cases.dam_break_2d(dx=0.05)
    b = cases.dam_break_3d(dx=0.05)
    with pytest.raises(sphera_b200.SphError) as e:
        sphera_b200.memory_required([a, b])
    assert e.value.code == abi.SPH_ERR_INVALID_ARGUMENT
    assert np.isfinite(a.state.x).all()
