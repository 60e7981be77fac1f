"""Seeded synthetic inputs with the shapes of the benchmark configurations.

The reference publishes no datasets for this path; these generators build the
bathymetry / initial depth families the benchmark configurations describe,
from ``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import numpy as np


def gaussian_bed(nx, ny, dx, dy, n_bumps, seed, base=-10.0, amp=(-4.0, 12.0),
                 width=(50.0, 500.0), chunk=256):
    """Interior bed (nx, ny), Fortran order: base + sum of seeded Gaussians.

    Amplitudes U[amp], widths U[width] (m), centres uniform over the domain.
    Evaluated in column chunks to bound temporary memory.
    """
    rng = np.random.default_rng(seed)
    A = rng.uniform(amp[0], amp[1], n_bumps)
    W = rng.uniform(width[0], width[1], n_bumps)
    cx = rng.uniform(0.0, nx * dx, n_bumps)
    cy = rng.uniform(0.0, ny * dy, n_bumps)
    x = (np.arange(nx) + 0.5) * dx
    b = np.empty((nx, ny), order="F")
    for j0 in range(0, ny, chunk):
        j1 = min(ny, j0 + chunk)
        y = (np.arange(j0, j1) + 0.5) * dy
        blk = np.full((nx, j1 - j0), base)
        for a, w, px, py in zip(A, W, cx, cy):
            gx = np.exp(-((x - px) ** 2) / (2.0 * w * w))
            gy = np.exp(-((y - py) ** 2) / (2.0 * w * w))
            blk += a * np.outer(gx, gy)
        b[:, j0:j1] = blk
    return b


def hump_depth(b, dx, dy, amp=0.5, width=200.0, eta0=0.0):
    """h = max(eta - b, 0) with eta = eta0 + a Gaussian hump at the centre."""
    nx, ny = b.shape
    x = (np.arange(nx) + 0.5) * dx - nx * dx / 2
    y = (np.arange(ny) + 0.5) * dy - ny * dy / 2
    gx = np.exp(-(x ** 2) / (2 * width ** 2))
    gy = np.exp(-(y ** 2) / (2 * width ** 2))
    eta = eta0 + amp * np.outer(gx, gy)
    return np.asfortranarray(np.maximum(eta - b, 0.0))


def config2(n=4096, dx=5.0, seed=2024, hump=True):
    """Single-instance wet/dry workload: 32-Gaussian bed, 0.5 m hump (or at rest)."""
    b = gaussian_bed(n, n, dx, dx, 32, seed)
    h = hump_depth(b, dx, dx, amp=0.5 if hump else 0.0, width=200.0)
    return b, h


CONFIG2_KW = dict(dx=5.0, dy=5.0, t_end=1.0e9, cfl=0.45, manning_n=0.025,
                  bc_west="wall", bc_east="wall", bc_south="wall", bc_north="wall")


M2_PERIOD = 44712.0  # s


def ensemble_members(n_inst=256, seed=7, size=(64, 1024), dx=10.0, manning_n=0.02):
    """Configurations of the batched ensemble: per member (nx, ny) uniform in
    [size[0], size[1]], a planar bed from -20 m at the west edge to +2 m at the
    east edge, still water at eta = 0 (the east part starts dry), a tidal west
    edge driven by one M2 constituent (amplitude U[0.5, 2] m, phase U[0, 2 pi)),
    walls elsewhere, Manning n = 0.02.

    Returns a list of dicts: ``kw`` (namelist keywords), ``b`` (interior bed),
    ``h`` (initial depth), ``tide`` ((amp,), (phase,), (omega,)).
    """
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_inst):
        nx, ny = (int(v) for v in rng.integers(size[0], size[1] + 1, 2))
        amp = float(rng.uniform(0.5, 2.0))
        phase = float(rng.uniform(0.0, 2.0 * np.pi))
        x = (np.arange(nx) + 0.5) / nx
        b = np.asfortranarray(np.repeat((-20.0 + 22.0 * x)[:, None], ny, axis=1))
        h = np.asfortranarray(np.maximum(0.0 - b, 0.0))
        kw = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1.0e9, cfl=0.45, manning_n=manning_n,
                  bc_west="tidal", bc_east="wall", bc_south="wall", bc_north="wall")
        out.append(dict(kw=kw, b=b, h=h,
                        tide=((amp,), (phase,), (2.0 * np.pi / M2_PERIOD,))))
    return out


def build_member(m, precision=64):
    """A finalised ``Rakali`` for one ``ensemble_members`` entry."""
    from .core import Rakali
    s = Rakali(defer_init=True, **m["kw"])
    s.set_bathymetry(m["b"])
    s.set_initial_h(m["h"])
    s.finalize()
    s.set_tidal_constituents(*m["tide"])
    if precision != 64:
        s.set_precision(precision)
    return s


def adjoint_problem(n=1024, steps=500, n_gauges=64, dx=10.0, seed=31):
    """The gradient workload: (nx = ny = n), bed of 16 seeded Gaussians on a
    -10 m base, a 0.5 m / 200 m hump at the centre on top of a 2-3 cm smooth
    surface undulation (so the water moves everywhere: a lake exactly at rest
    makes the limiter non-differentiable), Manning n = 0.025 as a field, 64
    seeded distinct gauge cells, and the smooth 0.2 m-amplitude bed noise
    whose forward run provides the observations.

    Returns dict(b, h, n, gauges, noise, dx, steps).
    """
    rng = np.random.default_rng(seed)
    b = gaussian_bed(n, n, dx, dx, 16, seed)
    x = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    L = n * dx
    surf = (0.02 * np.sin(2 * np.pi * X / (0.37 * L) + 0.3) * np.cos(2 * np.pi * Y / (0.23 * L) + 0.7)
            + 0.01 * np.sin(2 * np.pi * (X + 2 * Y) / (0.51 * L)))
    h = hump_depth(b, dx, dx, amp=0.5, width=200.0)
    h = np.asfortranarray(np.where(h > 0, np.maximum(h + surf, 0.0), 0.0))
    cells = rng.choice(n * n, size=n_gauges, replace=False)
    gauges = [(int(c % n), int(c // n)) for c in cells]
    noise = gaussian_bed(n, n, dx, dx, 24, seed + 1, base=0.0, amp=(-1.0, 1.0),
                         width=(100.0, 800.0))
    noise = np.asfortranarray(0.2 * noise / np.abs(noise).max())
    return dict(b=b, h=h, n=np.full((n, n), 0.025, order="F"), gauges=gauges, noise=noise,
                dx=dx, steps=steps)
