"""The AB3 update's division by 12 (``div12``: Markstein's correction step on RN(1/12), three
floating-point operations) against the IEEE division of the same build, bit for bit.

The fused steppers compute ``(dt * (23 k0 - 16 k1 + 5 k2)) / 12.0`` (ab3_w_advection.pyx:168-170) with
``div12``; bit parity with the reference needs every quotient to equal the division's.  Markstein's
theorem gives that for every x in the range it covers; this checks it on the device over random bit
patterns (every exponent, the special values), random values in the range the update sees, quotients
next to midpoints between doubles, and the edges of the range the correction step covers.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def check():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    from offline_particles_b200 import _lib

    lib = _lib.load()

    def run(x: "torch.Tensor") -> int:
        bad = torch.zeros(1, dtype=torch.int64, device="cuda")
        x = x.to(device="cuda", dtype=torch.float64).contiguous()
        _lib.call("opb_check_div12", x.data_ptr(), x.numel(), bad.data_ptr(), None)
        return int(bad.item())

    assert lib is not None
    return run


def test_div12_random_bit_patterns(check):
    import torch

    g = torch.Generator(device="cuda").manual_seed(12)
    for _ in range(8):
        bits = torch.randint(-(2**63), 2**63 - 1, (1 << 24,), dtype=torch.int64, device="cuda", generator=g)
        assert check(bits.view(torch.float64)) == 0


def test_div12_update_range_and_near_midpoints(check):
    import torch

    g = torch.Generator(device="cuda").manual_seed(13)
    for lo, hi in ((-12, 4), (-320, -300), (-960, -940), (300, 308)):
        e = torch.randint(lo, hi, (1 << 24,), device="cuda", generator=g).to(torch.float64)
        m = 1.0 + torch.rand(1 << 24, dtype=torch.float64, device="cuda", generator=g)
        s = torch.where(torch.rand(1 << 24, device="cuda", generator=g) < 0.5, -1.0, 1.0).to(torch.float64)
        assert check(s * m * torch.pow(2.0, e)) == 0
    # x = 12 (q + u/2 + j ulp-steps): quotients at and next to midpoints between consecutive doubles
    q = (1.0 + torch.rand(1 << 22, dtype=torch.float64, device="cuda", generator=g)) * torch.pow(
        2.0, torch.randint(-40, 40, (1 << 22,), device="cuda", generator=g).to(torch.float64))
    up = torch.nextafter(q, torch.full_like(q, float("inf")))
    for j in (-3, -2, -1, 0, 1, 2, 3):
        mid = q + (up - q) * 0.5
        x = 12.0 * mid
        for _ in range(abs(j)):
            x = torch.nextafter(x, torch.full_like(x, float("inf") if j > 0 else float("-inf")))
        assert check(x) == 0


def test_div12_special_values(check):
    import torch

    f = np.finfo(np.float64)
    vals = [0.0, -0.0, np.inf, -np.inf, np.nan, f.max, -f.max, f.tiny, -f.tiny, 5e-324, -5e-324, 2.0**-960,
            -(2.0**-960), np.nextafter(2.0**-960, 0.0), np.nextafter(2.0**-960, 1.0), 2.0**-1000, 12.0, -12.0, 3.0,
            1.0, 6.0, 24.0, 1.5, 1e-300, 1e300]
    x = np.array(vals, dtype=np.float64)
    x = np.concatenate([x, np.nextafter(x, np.inf), np.nextafter(x, -np.inf)])
    assert check(torch.from_numpy(x)) == 0


def test_check_entry_arguments(check):
    from offline_particles_b200 import _lib

    lib = _lib.load()
    assert lib.opb_check_div12(None, -1, None, None) == _lib.EINVAL
    assert lib.opb_check_div12(None, 0, None, None) == _lib.OK
