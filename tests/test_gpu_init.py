"""Initial conditions of src/core/rki_init.F90 on the device, against the oracle.

init_gaussian_hump (:60-129: h0 + A exp(-r^2 / 2 sigma^2) about the domain
centre plus the offsets; flat bed unless one was loaded) and
init_castro_dam_break (:131-174: a Gaussian-dimpled bed and a cylinder of
water, the Castro-Diaz benchmark) are built at finalize and then stepped:
the fields are compared with the oracle's restatement of the same routines,
bit for bit, right after finalize and after 40 steps.
"""
import numpy as np
import pytest

from helpers import gaussian_bed, pair

pytestmark = pytest.mark.gpu


def _same(sim, orc, names=("h", "hu", "hv", "b")):
    for name in names:
        got, want = getattr(sim, name), orc.arrays[name]
        assert np.array_equal(got, want), (name, float(np.max(np.abs(got - want))))


@pytest.mark.parametrize("hllc", [False, True])
def test_gaussian_hump_flat_bed(hllc):
    cfg = dict(nx=72, ny=50, dx=2.0, dy=3.0, nghost=2, t_end=1e6, cfl=0.45, use_hllc=hllc,
               init_condition="gaussian_hump", h0=1.5, hump_amplitude=0.3, hump_sigma=11.0,
               hump_x_offset=12.5, hump_y_offset=-7.0, manning_n=0.02)
    sim, orc = pair(cfg)
    with sim:
        _same(sim, orc)
        assert float(sim.h_phys.max()) > 1.7 and not np.any(sim.b_phys)
        sim.step(40)
        orc.step(40)
        assert sim.step_count == orc.step_count == 40
        _same(sim, orc)


def test_gaussian_hump_over_a_loaded_bed():
    """With a bed set before finalize the hump keeps it (the reference only
    zeroes the bed when none was loaded) and the depth is h0 + hump."""
    nx, ny = 64, 40
    b = gaussian_bed(nx, ny, 2.0, 2.0, 5, seed=9, base=-0.5, amp=(-0.3, 0.6), width=(5.0, 20.0))
    cfg = dict(nx=nx, ny=ny, dx=2.0, dy=2.0, nghost=3, t_end=1e6, cfl=0.45,
               init_condition="gaussian_hump", h0=1.0, hump_amplitude=0.2, hump_sigma=8.0)
    sim, orc = pair(cfg, bathymetry=b)
    with sim:
        _same(sim, orc)
        assert np.array_equal(sim.b_phys, b)
        sim.step(40)
        orc.step(40)
        _same(sim, orc)


@pytest.mark.parametrize("nghost", [2, 3])
def test_castro_dam_break(nghost):
    cfg = dict(nx=40, ny=40, dx=0.05, dy=0.05, nghost=nghost, t_end=1e6, cfl=0.45,
               init_condition="castro_dam_break")
    sim, orc = pair(cfg)
    with sim:
        _same(sim, orc)
        eta = sim.h_phys + sim.b_phys
        assert abs(float(eta.max()) - 3.0) < 1e-12 and abs(float(eta.min()) - 1.0) < 1e-12
        sim.step(40)
        orc.step(40)
        _same(sim, orc)
