"""The kernels' exact FP64 division (div_rn in sph_kernels.cu) against the
IEEE division on the device.

The FP64 passes divide by constants (h, h^2, the kernel-table step) and by
divisors a pair shares (|r|, rho_j in the renormalisation matrices) through
a correctly rounded reciprocal and two remainder corrections (Markstein's
method).  The bit-exact parity tests rest on these quotients being the IEEE
ones bit for bit; this checks that directly on 2^28 generated operand pairs
of five kinds (random; divisors with all-ones significands; quotients next
to a rounding midpoint; zero dividends of either sign; the kernels' own
ranges)."""
import pytest

import sphera_b200 as sb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 0xD1F1D3])
def test_division_is_ieee_bit_for_bit(seed):
    bad, first = sb.check_division(1 << 28, seed=seed)
    assert bad == 0, f"{bad} quotients differ from a / b, e.g. a, b = {first!r}"
