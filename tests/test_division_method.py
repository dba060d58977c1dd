"""The exact-division method of the FP64 kernels (div_rn, sph_kernels.cu),
restated on the CPU and compared with the IEEE quotient.

div_rn(a, b, y) with y = RN(1/b):
    q0 = RN(a y); r0 = RN(a - b q0); q1 = r0 ? RN(q0 + r0 y) : q0
    r1 = RN(a - b q1); q = r1 ? RN(q1 + r1 y) : q1
(each RN(x + y z) a single rounding: a fused multiply-add).  By Markstein's
theorem q = RN(a / b) when q1 is within one ulp of a/b and y within half an
ulp of 1/b.  Python's float division is the IEEE quotient; the fused
multiply-add is emulated exactly with fractions and one rounding to double
(int / int true division rounds correctly)."""
import random
import struct
from fractions import Fraction


def _fma(x, y, z):
    return float(Fraction(x) * Fraction(y) + Fraction(z))


def div_rn(a, b, y):
    q0 = a * y
    r0 = _fma(-b, q0, a)
    q1 = q0 if r0 == 0.0 else _fma(r0, y, q0)
    r1 = _fma(-b, q1, a)
    return q1 if r1 == 0.0 else _fma(r1, y, q1)


def _compose(frac, exp, sign):
    bits = ((sign & 1) << 63) | ((exp + 1023) << 52) | (frac & ((1 << 52) - 1))
    return struct.unpack("<d", struct.pack("<Q", bits))[0]


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _operands(n, seed):
    rng = random.Random(seed)
    for i in range(n):
        u1, u2 = rng.getrandbits(64), rng.getrandbits(64)
        e1, e2 = ((u1 >> 52) & 127) - 64, ((u2 >> 52) & 127) - 64
        kind = i % 5
        if kind == 0:
            yield _compose(u1, e1, u1 >> 63), _compose(u2, e2, u2 >> 63)
        elif kind == 1:
            yield _compose(u1, e1, u1 >> 63), _compose(((1 << 52) - 1) - (u2 & 255), e2 & 15, u2 >> 63)
        elif kind == 2:
            q = _compose(u1, e1 & 31, 0)
            half_ulp = _compose(0, (e1 & 31) - 53, 0)
            b = _compose(u2, e2 & 31, u2 >> 63)
            yield _fma(b, half_ulp, b * q), b
        elif kind == 3:
            yield (-0.0 if u1 & 1 else 0.0), _compose(u2, e2, u2 >> 63)
        else:
            yield _compose(u1, ((u1 >> 52) % 30) - 20, u1 >> 63), _compose(u2, ((u2 >> 52) % 21) - 10, 0)


def test_method_gives_the_ieee_quotient():
    bad = []
    for a, b in _operands(20000, 0xD1F1):
        q = div_rn(a, b, 1.0 / b)
        if _bits(q) != _bits(a / b):
            bad.append((a, b, q, a / b))
    assert not bad, bad[:5]


def test_one_correction_alone_is_not_always_enough():
    """Why div_rn corrects twice: RN(a RN(1/b)) alone can be more than half
    an ulp off, so it is not the quotient."""
    off = 0
    for a, b in _operands(20000, 0xD1F2):
        if _bits(a * (1.0 / b)) != _bits(a / b):
            off += 1
    assert off > 0
