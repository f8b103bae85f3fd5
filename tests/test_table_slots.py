"""CPU check of kernels.table_slots: the spin-2 table slots the gather kernel
fills per sample -- restated here from its footprint setup (window rings of
the HEALPix RING scheme within reach of the footprint centre, per ring the
disc's longitude stretch with 2% margin rounded up to 2k + 1 slots, at most
the ring table's reservation for the table's reach) -- never exceed the
request for footprint centres anywhere in the disc-sizing range, and the
window's rings never exceed the header the kernel reserves for that request
(gather_impl.cuh ring_cap_for), so no sample loses its table to the
estimate."""

import math

import numpy as np
import pytest

from tod_generation_mapbased_beam_b200.kernels import table_slots


def _ring_z(n, i):
    if i < n:
        return 1 - i * i / (3.0 * n * n)
    if i <= 3 * n:
        return (2 * n - i) * 2.0 / (3.0 * n)
    j = 4 * n - i
    return -(1 - j * j / (3.0 * n * n))


def _ring_npix(n, i):
    return 4 * min(i, n, 4 * n - i)


def _ring_above(n, z):
    az = abs(z)
    if az > 2.0 / 3.0:
        ir = int(n * math.sqrt(3 * (1 - az)))
        return 4 * n - ir - 1 if z < 0 else ir
    return int(n * (2 - 1.5 * z))


def _slots_filled(n, reach_table, reach, theta_u):
    lo, hi = theta_u - reach, theta_u + reach
    ir_lo = 1 if lo <= 0 else _ring_above(n, math.cos(lo))
    ir_hi = 4 * n - 1 if hi >= math.pi else _ring_above(n, math.cos(hi)) + 1
    ir_lo, ir_hi = max(ir_lo, 1), min(ir_hi, 4 * n - 1)
    disc = reach < 0.05 and theta_u - reach > 0.1 and theta_u + reach < math.pi - 0.1
    total = 0
    for ir in range(ir_lo, ir_hi + 1):
        z = _ring_z(n, ir)
        ta, sth = math.acos(z), math.sqrt(max(0.0, 1 - z * z))
        npx = _ring_npix(n, ir)
        dphi = 2 * math.pi / npx
        cnt = npx
        if reach_table < ta and reach_table < math.pi - ta:
            x = math.sin(reach_table) / sth
            if x < 1:
                cnt = min(2 * math.ceil(math.asin(x) / dphi) + 5, npx)
        if disc:
            h2 = reach * reach - (ta - theta_u) ** 2
            k = math.ceil(1.02 * math.sqrt(h2) / sth / dphi) if h2 > 0 else 0
            cnt = min(cnt, 2 * k + 1)
        total += cnt
    return total, ir_hi - ir_lo + 1


def _ring_cap_for(requested):
    """Window rings the kernel's table header holds for a request (restated
    from gather_impl.cuh ring_cap_for)."""
    return 192 if requested <= 0 else min(192, math.ceil(3.0 * math.sqrt(requested / 3.2)) + 6)


@pytest.mark.parametrize("nside, reach", [(1024, 0.0143), (2048, 0.0146), (512, 0.02), (128, 0.045),
                                          (4096, 0.01)])
def test_request_covers_every_footprint(nside, reach):
    reach_table = math.ceil(reach / 1e-4) * 1e-4  # ring tables are built for the reach rounded up
    want = table_slots(nside, reach_table)
    centres = np.linspace(0.1 + reach + 1e-6, math.pi - 0.1 - reach - 1e-6, 601)
    filled = [_slots_filled(nside, reach_table, reach, t) for t in centres]
    worst = max(f[0] for f in filled)
    assert worst <= want
    assert want <= 1.3 * worst + 64  # and not far more (the rest of shared memory is L1)
    assert max(f[1] for f in filled) <= _ring_cap_for(want)
