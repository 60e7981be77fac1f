"""Reverse-mode face and cell derivatives against central differences (CPU).

The adjoint kernels are built from host+device functions; their host builds
are exported by librakali.so (rkb_test_*), so the derivative formulas of the
HLL / HLLC face with the Audusse reconstruction, the clamp / KP07 / Froude
backstop and Manning friction are checked here without a GPU.  Each check
compares <g_out, dF(x) d> computed by the adjoint with the central
difference (F(x + e d) - F(x - e d)) / 2e along random directions d, at
states that keep every branch fixed within +-e.
"""
import ctypes

import numpy as np
import pytest

DP = ctypes.POINTER(ctypes.c_double)


def _p(a):
    return a.ctypes.data_as(DP)


@pytest.fixture(scope="module")
def lib():
    from rakali_b200 import _lib
    return _lib.load()


def _face(lib, d, hllc, x):
    out = np.zeros(6)
    lib.rkb_test_face_flux(d, hllc, _p(np.ascontiguousarray(x)), _p(out))
    return out


def _face_adj(lib, d, hllc, x, gout):
    gin = np.zeros(8)
    lib.rkb_test_face_adj(d, hllc, _p(np.ascontiguousarray(x)), _p(np.ascontiguousarray(gout)),
                          _p(gin))
    return gin


def _states(rng, kind):
    """(eL, qxL, qyL, bL, eR, qxR, qyR, bR) for a few regimes."""
    bL, bR = rng.uniform(-10, -2, 2)
    if kind == "wet":
        eL, eR = rng.uniform(-0.5, 0.5, 2)
        q = rng.normal(0, 1.0, 4)
    elif kind == "step":  # bed step, both sides wet
        bL, bR = -8.0 + rng.uniform(-0.3, 0.3), -3.0 + rng.uniform(-0.3, 0.3)
        eL, eR = rng.uniform(-0.5, 0.5, 2)
        q = rng.normal(0, 0.5, 4)
    elif kind == "supercritical":
        eL, eR = rng.uniform(-0.5, 0.5, 2)
        q = np.array([60.0, 5.0, 55.0, -3.0]) * rng.uniform(0.9, 1.1, 4)
    elif kind == "wetdry":  # right side dry above the left surface
        bL, bR = -2.0 + rng.uniform(-0.3, 0.3), 1.0 + rng.uniform(-0.3, 0.3)
        eL, eR = rng.uniform(-0.2, 0.2), bR - 0.5
        q = np.array([rng.normal(0, 0.3), rng.normal(0, 0.3), 0.0, 0.0])
    else:
        raise ValueError(kind)
    return np.array([eL, q[0], q[1], bL, eR, q[2], q[3], bR])


@pytest.mark.parametrize("d", [0, 1])
@pytest.mark.parametrize("hllc", [0, 1])
@pytest.mark.parametrize("kind", ["wet", "step", "supercritical", "wetdry"])
def test_face_adjoint_matches_central_differences(lib, d, hllc, kind):
    rng = np.random.default_rng(100 * d + 10 * hllc + len(kind))
    for _ in range(6):
        x = _states(rng, kind)
        gout = rng.normal(0, 1, 6)
        gin = _face_adj(lib, d, hllc, x, gout)
        for _ in range(4):
            dirn = rng.normal(0, 1, 8)
            if kind == "wetdry":
                dirn[4:] = 0.0  # a dry side contributes nothing; keep it dry
                dirn[6] = 0.0
            eps = 1e-6
            fp = _face(lib, d, hllc, x + eps * dirn)
            fm = _face(lib, d, hllc, x - eps * dirn)
            fd = float(np.dot(gout, (fp - fm) / (2 * eps)))
            ad = float(np.dot(gin, dirn))
            assert abs(fd - ad) <= 1e-6 * max(1.0, abs(fd)), (kind, fd, ad)


def _cell(lib, x, dt):
    out = np.zeros(3)
    lib.rkb_test_cell(_p(np.ascontiguousarray(x)), dt, _p(out))
    return out


def _cell_adj(lib, x, dt, gout):
    gin = np.zeros(4)
    lib.rkb_test_cell_adj(_p(np.ascontiguousarray(x)), dt, _p(np.ascontiguousarray(gout)), _p(gin))
    return gin


@pytest.mark.parametrize("regime", ["deep", "thin_kp07", "froude"])
def test_cell_adjoint_matches_central_differences(lib, regime):
    rng = np.random.default_rng({"deep": 1, "thin_kp07": 2, "froude": 3}[regime])
    for _ in range(10):
        if regime == "deep":
            x = np.array([rng.uniform(0.5, 12.0), rng.normal(0, 2), rng.normal(0, 2),
                          rng.uniform(0.01, 0.05)])
        elif regime == "thin_kp07":  # h < 1.5e-4: KP07 velocity desingularisation
            x = np.array([rng.uniform(2e-5, 1.2e-4), rng.normal(0, 1e-6), rng.normal(0, 1e-6),
                          rng.uniform(0.01, 0.05)])
        else:  # |u| above 50 sqrt(g h): the Froude backstop scales the momentum
            h = rng.uniform(0.01, 0.05)
            x = np.array([h, 80.0 * h * np.sqrt(9.81 * h), 30.0 * h, rng.uniform(0.01, 0.05)])
        dt = 0.3
        gout = rng.normal(0, 1, 3)
        gin = _cell_adj(lib, x, dt, gout)
        for _ in range(4):
            dirn = rng.normal(0, 1, 4) * np.abs(x) + 1e-12
            eps = 1e-6
            fp = _cell(lib, x + eps * dirn, dt)
            fm = _cell(lib, x - eps * dirn, dt)
            fd = float(np.dot(gout, (fp - fm) / (2 * eps)))
            ad = float(np.dot(gin, dirn))
            assert abs(fd - ad) <= 1e-5 * max(1e-8, abs(fd)) + 1e-14, (regime, fd, ad)
