"""Shared builders for the parity tests: the same configuration through the
B200 library (``rakali_b200.Rakali``) and through the CPU oracle."""
from __future__ import annotations

import numpy as np

G = 9.80665


def gaussian_bed(nx, ny, dx, dy, n_bumps, seed, base=-10.0, amp=(-4.0, 12.0),
                 width=(50.0, 500.0)):
    """Bed = base + sum of seeded Gaussians (the config-2 family), interior (nx, ny)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(x, y, indexing="ij")
    b = np.full((nx, ny), base)
    A = rng.uniform(amp[0], amp[1], n_bumps)
    W = rng.uniform(width[0], width[1], n_bumps)
    cx = rng.uniform(0.0, nx * dx, n_bumps)
    cy = rng.uniform(0.0, ny * dy, n_bumps)
    for a, w, px, py in zip(A, W, cx, cy):
        b += a * np.exp(-((X - px) ** 2 + (Y - py) ** 2) / (2.0 * w * w))
    return np.asfortranarray(b)


def hump_depth(b, dx, dy, amp=0.5, width=200.0, eta0=0.0):
    nx, ny = b.shape
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dy
    X, Y = np.meshgrid(x, y, indexing="ij")
    eta = eta0 + amp * np.exp(-((X - nx * dx / 2) ** 2 + (Y - ny * dy / 2) ** 2) / (2 * width ** 2))
    return np.asfortranarray(np.maximum(eta - b, 0.0))


def pair(cfg: dict, bathymetry=None, initial_h=None):
    """(Rakali, OracleSim) built from the same kwargs and optional fields."""
    from oracle.oracle import OracleSim
    from rakali_b200 import Rakali

    defer = bathymetry is not None or initial_h is not None
    sim = Rakali(defer_init=defer, **cfg)
    if bathymetry is not None:
        sim.set_bathymetry(bathymetry)
    if initial_h is not None:
        sim.set_initial_h(initial_h)
    if defer:
        sim.finalize()
    orc = OracleSim.from_config(cfg, bathymetry=bathymetry, initial_h=initial_h)
    return sim, orc


def max_rel_diff(a, b, floor=1.0e-6):
    """Relative L-infinity error max|a - b| / max|b| (scale floored at `floor`)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.max(np.abs(b))), floor)
    return float(np.max(np.abs(a - b))) / scale


def compare_state(sim, orc, rtol=0.0, ghosts=True, fields=("h", "hu", "hv", "b")):
    """Return {field: max relative diff}; asserts each <= rtol."""
    out = {}
    for f in fields:
        a = getattr(sim, f)
        b = orc.arrays[f]
        if not ghosts:
            g = orc.ng
            a = a[g:-g, g:-g]
            b = b[g:-g, g:-g]
        d = max_rel_diff(a, b)
        out[f] = d
        assert d <= rtol, f"{f}: max relative difference {d:.3e} > {rtol:.1e}"
    return out
