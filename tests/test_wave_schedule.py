"""The ticket table of the one-launch symmetric sweep (k_gs_wave), on the CPU.

hpcgx_wave_schedule returns the table the library uploads for a level; no
device is needed.  The sweep's bounded waits rely on these properties:
  * every (stage, class plane) of the seven stages appears once, its tickets
    are contiguous and the tickets cover 0 .. total-1 without gaps;
  * stage s on plane z waits for stage s-1 on the planes z-1, z, z+1 that
    hold its class; all of those tickets are smaller than every ticket of
    (s, z), so a block only ever waits for tickets already taken by running
    blocks (the waits end whatever the number of co-resident blocks);
  * the sweep is unavailable (empty table) where a class has no line next to
    some plane (ny or nz below 2) or the lag is below 2.
"""
import ctypes as C

import pytest


def schedule(nx, ny, nz, lag, rows):
    from hpcg_b200 import _lib
    h = _lib.lib()
    count, total, lpi = C.c_int(), C.c_int(), C.c_int()
    ipp = (C.c_int * 4)()
    rc = h.hpcgx_wave_schedule(nx, ny, nz, lag, rows, 0, None, None, C.byref(count),
                               C.byref(total), C.byref(lpi), ipp)
    n = count.value
    if n == 0:
        assert rc == 0
        return [], 0, 0, list(ipp)
    assert rc == 1   # EINVAL: cap 0 is too small, count says how many
    codes, starts = (C.c_int * n)(), (C.c_int * n)()
    rc = h.hpcgx_wave_schedule(nx, ny, nz, lag, rows, n, codes, starts, C.byref(count),
                               C.byref(total), C.byref(lpi), ipp)
    assert rc == 0
    tab = [(codes[i] >> 16, codes[i] & 0xFFFF, starts[i]) for i in range(n)]
    return tab, total.value, lpi.value, list(ipp)


def stage_class(s):
    return s if s <= 3 else 6 - s


CASES = [(16, 16, 16, 4, 4096), (16, 16, 16, 2, 1), (24, 24, 24, 6, 2048), (16, 24, 32, 3, 64),
         (64, 32, 16, 9, 512), (32, 32, 64, 2, 1), (8, 6, 10, 2, 1), (5, 7, 9, 3, 16),
         (512, 512, 512, 6, 2048), (2, 2, 2, 2, 1), (3, 2, 3, 4, 1)]


@pytest.mark.parametrize("nx,ny,nz,lag,rows", CASES)
def test_every_wait_is_for_smaller_tickets(nx, ny, nz, lag, rows):
    tab, total, lpi, ipp = schedule(nx, ny, nz, lag, rows)
    assert tab, "the sweep is available on this level"
    nyq = [(ny - (q & 1) + 1) // 2 for q in range(4)]
    assert lpi >= 1 and all(ipp[q] == -(-nyq[q] // lpi) for q in range(4))
    # coverage: each (stage, class plane) once, contiguous tickets, no gaps
    seen = {}
    expect = 0
    for s, jz, start in tab:
        assert 0 <= s <= 6 and (s, jz) not in seen
        q = stage_class(s)
        assert (q >> 1) + 2 * jz < nz
        assert start == expect
        expect += ipp[q]
        seen[(s, jz)] = start
    assert expect == total
    for s in range(7):
        q = stage_class(s)
        planes = [jz for jz in range(nz) if (q >> 1) + 2 * jz < nz]
        assert all((s, jz) in seen for jz in planes)
    # dependencies: every ticket of (s-1, z') for z' in z-1..z+1 is below (s, z)'s first
    for (s, jz), start in seen.items():
        if s == 0:
            continue
        z = (stage_class(s) >> 1) + 2 * jz
        p = s - 1
        qp = stage_class(p)
        deps = [zz for zz in (z - 1, z, z + 1) if 0 <= zz < nz and (zz & 1) == (qp >> 1)]
        assert deps, "stage %d plane %d waits for no plane of stage %d" % (s, z, p)
        for zz in deps:
            dstart = seen[(p, (zz - (qp >> 1)) // 2)]
            assert dstart + ipp[qp] <= start


@pytest.mark.parametrize("nx,ny,nz,lag", [(16, 1, 16, 4), (16, 16, 1, 4), (2, 1, 1, 2),
                                          (16, 16, 16, 1), (16, 16, 16, 0)])
def test_unavailable_where_waits_would_not_order_the_stages(nx, ny, nz, lag):
    tab, total, _, _ = schedule(nx, ny, nz, lag, 2048)
    assert tab == [] and total == 0


def test_bad_arguments_are_rejected():
    from hpcg_b200 import _lib
    h = _lib.lib()
    count, total, lpi = C.c_int(), C.c_int(), C.c_int()
    ipp = (C.c_int * 4)()
    assert h.hpcgx_wave_schedule(0, 4, 4, 4, 64, 0, None, None, C.byref(count), C.byref(total),
                                 C.byref(lpi), ipp) == 1
    assert h.hpcgx_wave_schedule(4, 4, 4, 4, 64, 8, None, None, C.byref(count), C.byref(total),
                                 C.byref(lpi), ipp) == 1
