"""Builds the CUDA library sphera_b200/libsphera_b200.so for sm_100a.

Every translation unit is built with --fmad=false: the FP64 path must not
contract a multiply and an add (the reference's arithmetic has no fused
multiply-add), and the compensated sums of the FP32-compensated form need
their additions rounded one by one.  Where the FP32c pair arithmetic wants a
fused multiply-add it writes fmaf / __ffma2_rn explicitly.  Host code is
built with -ffp-contract=off for the same reason.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsphera_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v"]
UNITS = [
    ("sph_kernels.cu", ["--fmad=false"]),
    ("sph_api.cu", ["--fmad=false"]),
    ("sph_static.cu", ["--fmad=false"]),
]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    hdr = os.path.join(os.path.dirname(HERE), "include", "sphera_b200.h")
    newest = max(os.path.getmtime(p) for p in srcs + [hdr, __file__])
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    nvcc = _nvcc()
    objs = []
    for unit, flags in UNITS:
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *COMMON, *flags, "-c", os.path.join(CSRC, unit), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {unit}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = OUT + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
