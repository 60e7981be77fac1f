"""Gauge stencils without a GPU: the library's station cells and bilinear
weights against a restatement of the reference's compute_local_gauges /
compute_interp_weights (src/io/structured/rki_gauges.F90:208-336), including
stations left / right of the first / last cell centre (clamped), exactly on
centres and on the domain edge, and stations outside the domain (dropped)."""
import ctypes
import math

import numpy as np
import pytest

DP = ctypes.POINTER(ctypes.c_double)
IP = ctypes.POINTER(ctypes.c_int)


@pytest.fixture(scope="module")
def lib():
    from rakali_b200 import _lib
    return _lib.load()


def _stencils_ref(nx, ny, ng, dx, dy, xs, ys):
    """rki_gauges.F90:208-243 (which cells own a station) and :245-336 (the
    stencil and weights), 0-based array indices."""
    out = []
    for k, (gx, gy) in enumerate(zip(xs, ys)):
        ig = math.floor(gx / dx) + 1
        jg = math.floor(gy / dy) + 1
        if not (1 <= ig <= nx and 1 <= jg <= ny):
            continue
        ia, ja = ig + ng, jg + ng
        xc, yc = (ig - 0.5) * dx, (jg - 0.5) * dy

        def axis(g, c, i1, n, a, d):
            if g < c:
                return (a - 1, (g - (c - d)) / d) if i1 > 1 else (a, 0.0)
            return (a, (g - c) / d) if i1 < n else (a, 0.0)

        ix0, wx = axis(gx, xc, ig, nx, ia, dx)
        iy0, wy = axis(gy, yc, jg, ny, ja, dy)
        out.append((k, ix0 - 1, iy0 - 1, max(0.0, min(1.0, wx)), max(0.0, min(1.0, wy))))
    return out


@pytest.mark.parametrize("nx,ny,ng,dx,dy", [(40, 30, 2, 10.0, 7.5), (5, 3, 3, 2.0, 4.0)])
def test_stencils_match_the_reference_rules(lib, nx, ny, ng, dx, dy):
    rng = np.random.default_rng(nx)
    X, Y = nx * dx, ny * dy
    xs = list(rng.uniform(-0.1 * X, 1.1 * X, 200))
    ys = list(rng.uniform(-0.1 * Y, 1.1 * Y, 200))
    # edges and centres
    xs += [0.0, 0.5 * dx, 0.2 * dx, X - 0.2 * dx, X - 0.5 * dx, X, 1.5 * dx, X - 1e-9]
    ys += [0.0, 0.5 * dy, 0.2 * dy, Y - 0.2 * dy, Y - 0.5 * dy, Y, 1.5 * dy, Y - 1e-9]
    x = np.array(xs)
    y = np.array(ys)
    n = len(xs)
    st, i0, j0 = (np.zeros(n, dtype=np.int32) for _ in range(3))
    wx, wy = np.zeros(n), np.zeros(n)
    got_n = lib.rkb_gauge_stencils(nx, ny, ng, dx, dy, x.ctypes.data_as(DP), y.ctypes.data_as(DP),
                                   n, st.ctypes.data_as(IP), i0.ctypes.data_as(IP),
                                   j0.ctypes.data_as(IP), wx.ctypes.data_as(DP),
                                   wy.ctypes.data_as(DP))
    ref = _stencils_ref(nx, ny, ng, dx, dy, xs, ys)
    assert got_n == len(ref) > 0
    got = list(zip(st[:got_n].tolist(), i0[:got_n].tolist(), j0[:got_n].tolist(),
                   wx[:got_n].tolist(), wy[:got_n].tolist()))
    assert got == ref


def test_non_finite_and_huge_stations_are_dropped(lib):
    """NaN, infinite and out-of-range coordinates lie outside the domain:
    those stations get no stencil, and the finite ones around them keep
    theirs."""
    nx, ny, ng, dx, dy = 10, 8, 2, 5.0, 5.0
    xs = [np.nan, 12.0, np.inf, -np.inf, 1e300, -1e300, 21.0, 3.0e10]
    ys = [10.0, np.nan, 10.0, 10.0, 10.0, 10.0, 12.5, 10.0]
    x, y = np.array(xs), np.array(ys)
    n = len(xs)
    st, i0, j0 = (np.zeros(n, dtype=np.int32) for _ in range(3))
    wx, wy = np.zeros(n), np.zeros(n)
    got_n = lib.rkb_gauge_stencils(nx, ny, ng, dx, dy, x.ctypes.data_as(DP), y.ctypes.data_as(DP),
                                   n, st.ctypes.data_as(IP), i0.ctypes.data_as(IP),
                                   j0.ctypes.data_as(IP), wx.ctypes.data_as(DP),
                                   wy.ctypes.data_as(DP))
    ref = _stencils_ref(nx, ny, ng, dx, dy, [21.0], [12.5])
    assert got_n == 1
    assert (int(st[0]), int(i0[0]), int(j0[0]), float(wx[0]), float(wy[0])) == \
        (6,) + tuple(ref[0][1:])


def test_bad_arguments(lib):
    z = np.zeros(1)
    zi = np.zeros(1, dtype=np.int32)
    assert lib.rkb_gauge_stencils(0, 4, 2, 1.0, 1.0, z.ctypes.data_as(DP), z.ctypes.data_as(DP), 1,
                                  zi.ctypes.data_as(IP), zi.ctypes.data_as(IP),
                                  zi.ctypes.data_as(IP), z.ctypes.data_as(DP),
                                  z.ctypes.data_as(DP)) == -2
