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
    some plane (ny or nz below 2) or the lag is below 2;
  * those waits suffice: the table's items, run one at a time in random orders
    that only respect the waits, reproduce the oracle's colour-ordered SYMGS
    bit for bit (and a weaker wait does not).
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


# ---------------------------------------------------------------------------
# Execution model: the items of the library's table run one at a time in a
# random order that only respects the sweep's waits.  Every such order must
# reproduce the oracle's colour-ordered SYMGS bit for bit; an order allowed by
# a weaker wait (stage s-1 on plane z only) must not.

def _gs_rows(lev, rows, r, x):
    """Reference GS update of independent rows (src/ComputeSYMGS_ref.cpp:67-81),
    vectorised; the slot order of each row is kept."""
    import numpy as np
    if rows.size == 0:
        return
    nnz = lev.nnz[rows].astype(np.int64)
    cols = lev.cols.reshape(-1, 27)[rows]
    vals = lev.vals.reshape(-1, 27)[rows]
    d = vals[np.arange(rows.size), lev.diag[rows]]
    s = r[rows].copy()
    for j in range(27):
        m = j < nnz
        s[m] = s[m] - vals[m, j] * x[cols[m, j]]
    s = s + x[rows] * d
    x[rows] = s / d


def _item_rows(nx, ny, q, jz, b, lpi, px):
    import numpy as np
    py, pz = q & 1, q >> 1
    nyq = (ny - py + 1) // 2
    j0 = jz * nyq + b * lpi
    j1 = min(j0 + lpi, (jz + 1) * nyq)
    iz = pz + 2 * jz
    out = []
    for j in range(j0, j1):
        iy = py + 2 * (j - jz * nyq)
        ix = np.arange(px, nx, 2)
        out.append((iz * ny + iy) * nx + ix)
    return np.concatenate(out) if out else np.zeros(0, np.int64)


def _run_item(lev, nx, ny, s, jz, b, lpi, r, x):
    q = stage_class(s)
    if s < 3:
        phases = [(q, 0), (q, 1)]
    elif s == 3:
        phases = [(3, 0), (3, 1), (3, 1), (3, 0)]   # 6 fwd, 7 fwd, 7 bwd, 6 bwd
    else:
        phases = [(q, 1), (q, 0)]
    for qq, px in phases:
        _gs_rows(lev, _item_rows(nx, ny, qq, jz, b, lpi, px), r, x)


def _random_order_sweep(lev, dims, tab, ipp, lpi, r, x, rng, weak=False):
    nx, ny, nz = dims
    items = [(s, jz, b) for s, jz, _ in tab for b in range(ipp[stage_class(s)])]
    done = {}
    pending = list(items)
    while pending:
        ready = []
        for k, (s, jz, b) in enumerate(pending):
            if s == 0:
                ready.append(k)
                continue
            z = (stage_class(s) >> 1) + 2 * jz
            qp = stage_class(s - 1)
            planes = (z,) if weak else (z - 1, z, z + 1)
            ok = all(done.get((s - 1, (zz - (qp >> 1)) // 2), 0) == ipp[qp]
                     for zz in planes if 0 <= zz < nz and (zz & 1) == (qp >> 1))
            if ok:
                ready.append(k)
        assert ready, "no item can run: the waits deadlock"
        k = ready[rng.integers(len(ready))]
        s, jz, b = pending.pop(k)
        _run_item(lev, nx, ny, s, jz, b, lpi, r, x)
        done[(s, jz)] = done.get((s, jz), 0) + 1
    return x


@pytest.mark.parametrize("dims,lag,rows", [((8, 8, 8), 2, 1), ((6, 4, 6), 3, 1),
                                           ((5, 6, 7), 2, 1), ((8, 6, 10), 4, 16)])
def test_any_order_the_waits_allow_reproduces_the_colour_sweep(dims, lag, rows, oracle):
    import numpy as np
    L, _, _, _ = oracle.hierarchy(*dims, levels=1)
    oracle.colour_order(L)
    lev = L[0]
    r = oracle.uniform(12, lev.nrow)
    x0 = oracle.uniform(13, lev.nrow)
    want = oracle.symgs(lev, r, x0, coloured=True)
    tab, total, lpi, ipp = schedule(*dims, lag, rows)
    rng = np.random.default_rng(7)
    for _ in range(6):
        got = _random_order_sweep(lev, dims, tab, ipp, lpi, r, x0.copy(), rng)
        assert (got == want).all()
    # control: waiting for the previous stage on plane z alone is not enough
    wrong = 0
    for _ in range(6):
        got = _random_order_sweep(lev, dims, tab, ipp, lpi, r, x0.copy(), rng, weak=True)
        wrong += not (got == want).all()
    assert wrong > 0
