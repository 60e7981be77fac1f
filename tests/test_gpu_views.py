"""Zero-copy field views and setters while the device holds the state.

The reference hands out pointers into its host arrays (rki_get_*_ptr,
src/api/rki_api.F90:502-700) after bringing every array home, and uploads
every array before the next step (ensure_host / ensure_device, :104-123).
This library moves only the field asked for: a pointer brings that field
home, and the next step uploads it again, so whatever the caller writes
through the view is what the step sees - checked here against the oracle
with the same writes - while the other fields never cross PCIe.  Setters
(rki_set_h/hu/hv, :926-1000) send the interior straight to the device.
"""
import numpy as np
import pytest

from helpers import gaussian_bed, hump_depth, pair

pytestmark = pytest.mark.gpu

NX, NY, DX = 96, 80, 5.0


def _pair(precision=64):
    b = gaussian_bed(NX, NY, DX, DX, 8, seed=3, width=(30.0, 120.0))
    h = hump_depth(b, DX, DX, width=60.0)
    cfg = dict(nx=NX, ny=NY, dx=DX, dy=DX, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    if precision == 32:
        sim.set_precision(32)
    return sim, orc


def _same_state(sim, orc):
    for name in ("h", "hu", "hv"):
        assert np.array_equal(getattr(sim, name), orc.arrays[name]), name


def test_write_through_view_is_seen_by_next_step():
    sim, orc = _pair()
    with sim:
        sim.step(5)
        orc.step(5)
        g = orc.ng
        hv = sim.hu_phys  # pointer to hu only
        hv[10:20, 30:40] += 0.05
        orc.arrays["hu"][g + 10:g + 20, g + 30:g + 40] += 0.05
        h = sim.h_phys
        h[40:50, 5:9] *= 1.01
        orc.arrays["h"][g + 40:g + 50, g + 5:g + 9] *= 1.01
        sim.step(7)
        orc.step(7)
        _same_state(sim, orc)


def test_setters_go_straight_to_the_device_and_views_see_them():
    sim, orc = _pair()
    rng = np.random.default_rng(4)
    with sim:
        sim.step(3)
        orc.step(3)
        g = orc.ng
        new_h = np.asfortranarray(orc.interior("h") * (1.0 + 1e-3 * rng.random((NX, NY))))
        new_hu = np.asfortranarray(orc.interior("hu") + 1e-3 * rng.standard_normal((NX, NY)))
        sim.set_h(new_h)
        sim.set_hu(new_hu)
        orc.arrays["h"][g:-g, g:-g] = new_h
        orc.arrays["hu"][g:-g, g:-g] = new_hu
        assert np.array_equal(sim.h_phys, new_h)  # brought home from the device
        sim.step(4)
        orc.step(4)
        _same_state(sim, orc)


def test_setter_after_a_view_then_a_write_through_it():
    """A view of hu is out when set_hu runs: the view shows the set values,
    and a write through it afterwards still reaches the next step."""
    sim, orc = _pair()
    with sim:
        sim.step(2)
        orc.step(2)
        g = orc.ng
        view = sim.hu_phys
        new_hu = np.asfortranarray(orc.interior("hu") * 0.5)
        sim.set_hu(new_hu)
        orc.arrays["hu"][g:-g, g:-g] = new_hu
        assert np.array_equal(view, new_hu)
        view[3:6, 3:6] = 0.01
        orc.arrays["hu"][g + 3:g + 6, g + 3:g + 6] = 0.01
        sim.step(3)
        orc.step(3)
        _same_state(sim, orc)


def test_bed_view_write_is_seen_in_both_forms():
    for precision in (64, 32):
        sim, orc = _pair(precision)
        with sim:
            sim.step(2)
            orc.step(2)
            g = orc.ng
            bview = sim.b_phys
            bview[20:30, 20:30] += 0.2
            orc.arrays["b"][g + 20:g + 30, g + 20:g + 30] += 0.2
            sim.step(3)
            orc.step(3)
            if precision == 64:
                _same_state(sim, orc)
                assert np.array_equal(sim.b, orc.arrays["b"])
            else:
                assert np.abs(sim.h_phys - orc.interior("h")).max() < 1e-5


def test_rk2_saves_and_state_readable_in_any_order():
    sim, orc = _pair()
    with sim:
        sim.step(4)
        orc.step(4)
        for name in ("h0", "hv", "hu0", "b", "h", "hv0", "hu"):
            got = getattr(sim, name)
            g = orc.ng
            want = orc.arrays[name]
            if name.endswith("0"):
                got, want = got[g:-g, g:-g], want[g:-g, g:-g]
            assert np.array_equal(got, want), name
        sim.step(1)
        orc.step(1)
        _same_state(sim, orc)
