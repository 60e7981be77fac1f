"""FP32 surface form of the step against the FP64 oracle (GPU, through the C ABI).

The FP32 form keeps eta = h + b, hu, hv in FP32 and the bed in FP64; every
difference against the bed, every wet/dry test and the mass sums are FP64.

Tolerances (free surface = depth difference, the bed being shared):

* lake at rest is exact: the FP32 state does not change at all;
* where the flow does not amplify perturbations (fixed dt, short horizons,
  the dam break) the surface is within ``ETA_TOL`` = 1e-5 m of the oracle
  and the momentum within ``MOM_RTOL`` = 1e-4 of the field's max |hu|, |hv|;
* over longer CFL-stepped runs the FP64 scheme itself amplifies round-off
  (dt follows the state, and the limiter / wave-speed switches respond to
  the last bits): the oracle started from h x (1 + 1e-7 noise), an FP32-sized
  perturbation, drifts from the unperturbed oracle by up to ~1e-4 m.  There
  the FP32 error is bounded by max(ETA_TOL, 2 x that drift), max and RMS
  separately (``_floor``);
* rain-fed films on dry land: an FP32 surface at +3 m resolves depth to
  ~2e-7 m, so a sub-millimetre film's momentum carries a relative error near
  1e-3 (``FILM_MOM_RTOL``) while the surface stays within ETA_TOL.

Both forms advance to the same time with their own CFL steps when dt is not
fixed (dt differs in the last bits), so the comparison is at equal time.
"""
import numpy as np
import pytest

from tests.helpers import gaussian_bed, hump_depth, max_rel_diff, pair

pytestmark = pytest.mark.gpu

ETA_TOL = 1.0e-5   # m
MOM_RTOL = 1.0e-4
FILM_MOM_RTOL = 2.0e-3


def _errors(sim, orc):
    """(max |h - h_ref| in m, relative L-inf of hu, of hv) over the interior."""
    dh = float(np.max(np.abs(sim.h_phys - orc.interior("h"))))
    du = max_rel_diff(sim.hu_phys, orc.interior("hu"), floor=1e-3)
    dv = max_rel_diff(sim.hv_phys, orc.interior("hv"), floor=1e-3)
    return dh, du, dv


def _floor(cfg, bathymetry, initial_h, target):
    """(max, rms) drift of the FP64 oracle when h is perturbed by 1e-7 relative noise."""
    from oracle.oracle import OracleSim
    rng = np.random.default_rng(99)
    a = OracleSim.from_config(cfg, bathymetry=bathymetry, initial_h=initial_h)
    hp = np.asfortranarray(initial_h * (1.0 + 1e-7 * rng.standard_normal(initial_h.shape)))
    c = OracleSim.from_config(cfg, bathymetry=bathymetry, initial_h=hp)
    a.advance(target)
    c.advance(target)
    d = np.abs(a.interior("h") - c.interior("h"))
    return float(d.max()), float(np.sqrt(np.mean(d * d)))


def _check_against_floor(sim, orc, cfg, b, h, target):
    dh = np.abs(sim.h_phys - orc.interior("h"))
    fmax, frms = _floor(cfg, b, h, target)
    assert dh.max() <= max(ETA_TOL, 2.0 * fmax), (dh.max(), fmax)
    assert np.sqrt(np.mean(dh * dh)) <= max(1e-6, 2.0 * frms), (np.sqrt(np.mean(dh * dh)), frms)


def _fp32_pair(cfg, bathymetry=None, initial_h=None):
    sim, orc = pair(cfg, bathymetry=bathymetry, initial_h=initial_h)
    sim.set_precision(32)
    assert sim.precision == 32
    return sim, orc


def test_lake_at_rest_is_exact_with_islands():
    """Flat surface (eta = 0) over a bed with dry islands: nothing moves, bit for bit."""
    nx, ny, dx = 160, 128, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=3, width=(20.0, 120.0))
    h = np.asfortranarray(np.maximum(0.0 - b, 0.0))
    assert (h == 0.0).sum() > 50
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, _ = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(300)
        assert np.array_equal(sim.h_phys, h)
        assert not np.any(sim.hu_phys) and not np.any(sim.hv_phys)


def test_lake_at_rest_unrepresentable_surface():
    """eta0 = 0.3 m (not an FP32 number): the stored surface never changes."""
    nx, ny, dx = 128, 96, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 16, seed=11, width=(20.0, 100.0))
    h = np.asfortranarray(np.maximum(0.3 - b, 0.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02, use_hllc=True)
    sim, _ = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(1)  # the first step uploads the state in the FP32 form
        h0 = sim.h_phys.copy()
        wet = h0 > 0.0
        assert np.abs((h0 + sim.b_phys)[wet] - 0.3).max() <= 2e-8  # f32(0.3)
        sim.step(200)
        assert np.array_equal(sim.h_phys, h0)
        assert not np.any(sim.hu_phys) and not np.any(sim.hv_phys)


@pytest.mark.parametrize("hllc", [False, True])
def test_wet_dry_hump_short_horizon(hllc):
    """Config-2 family at 192 x 160 (islands, hump, Manning 0.025), fixed dt, 12 steps:
    before any amplification the FP32 surface is within 1e-6 m."""
    nx, ny, dx = 192, 160, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=7, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=80.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025, use_hllc=hllc,
               dt_fixed=0.2)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(12)
        orc.step(12)
        dh, du, dv = _errors(sim, orc)
        assert dh <= 1e-6, dh
        assert du <= 1e-5 and dv <= 1e-5, (du, dv)


def test_wet_dry_hllc_fixed_dt_100_steps():
    """HLLC over islands with a fixed dt does not amplify round-off: 1e-5 m after 100 steps."""
    nx, ny, dx = 192, 160, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=7, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=80.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025, use_hllc=True,
               dt_fixed=0.2)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(100)
        orc.step(100)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= MOM_RTOL and dv <= MOM_RTOL, (du, dv)


@pytest.mark.parametrize("hllc", [False, True])
def test_wet_dry_hump_cfl_steps_at_conditioning_floor(hllc):
    """Same configuration, CFL steps to t = 20 s: within 2x the FP64 scheme's own drift."""
    nx, ny, dx = 192, 160, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=7, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=80.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025, use_hllc=hllc)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.advance(20.0)
        orc.advance(20.0)
        assert abs(sim.time - 20.0) < 1e-9 and abs(orc.time - 20.0) < 1e-9
        assert abs(sim.step_count - orc.step_count) <= 1
        _check_against_floor(sim, orc, cfg, b, h, 20.0)


def test_config1_dam_break():
    """200 x 100 dam break (HLLC, CFL 0.5, 60 s): within 1e-5 m."""
    cfg = dict(nx=200, ny=100, dx=10.0, dy=10.0, t_end=60.0, cfl=0.5, use_hllc=True)
    sim, orc = _fp32_pair(cfg)
    with sim:
        sim.advance(60.0)
        orc.advance(60.0)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= MOM_RTOL and dv <= MOM_RTOL, (du, dv)


def test_sweep_shape_does_not_change_results():
    """Columns per lane and the row partition of the sweep are invisible in the state (bitwise)."""
    nx, ny, dx = 300, 200, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 24, seed=5, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=100.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    out = []
    for cols, rows in ((0, 0), (2, 4), (2, 37), (4, 0), (4, 9)):
        sim, _ = _fp32_pair(cfg, bathymetry=b, initial_h=h)
        with sim:
            sim.set_sweep(cols, rows)
            sim.step(40)
            out.append((sim.h_phys.copy(), sim.hu_phys.copy(), sim.hv_phys.copy(), sim.time))
    for o in out[1:]:
        for a, c in zip(o, out[0]):
            assert np.array_equal(a, c)


BC_CASES = [
    dict(bc_west="tidal", tidal_amplitude=0.5, tidal_period=600.0),
    dict(bc_west="open", bc_east="open", bc_south="open", bc_north="open"),
    dict(bc_west="inflow", inflow_velocity=0.3, bc_east="open"),
    dict(bc_west="discharge", discharge_flux=0.5, bc_east="open"),
    dict(bc_west="clamped", clamped_elevation=0.2, bc_east="open"),
    dict(bc_west="chapman", bc_east="chapman", bc_south="chapman", bc_north="chapman"),
    dict(bc_west="sponge", bc_east="sponge", sponge_width=6, sponge_strength=0.05),
]


def _bc_setup(edges, **extra):
    nx, ny, dx = 96, 64, 10.0
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=2, base=-5.0, amp=(-1.0, 3.0), width=(40.0, 150.0))
    h = hump_depth(b, dx, dx, amp=0.3, width=120.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02, **edges, **extra)
    return cfg, b, h


@pytest.mark.parametrize("edges", BC_CASES, ids=[c["bc_west"] for c in BC_CASES])
def test_boundary_types_fixed_dt(edges):
    """Every boundary type, fixed dt, 60 steps: within 1e-5 m / 1e-4 relative momentum."""
    cfg, b, h = _bc_setup(edges, dt_fixed=0.5)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(60)
        orc.step(60)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= MOM_RTOL and dv <= MOM_RTOL, (du, dv)


@pytest.mark.parametrize("edges", BC_CASES, ids=[c["bc_west"] for c in BC_CASES])
def test_boundary_types_cfl_steps(edges):
    """Every boundary type, CFL steps to t = 25 s: within 2x the FP64 drift."""
    cfg, b, h = _bc_setup(edges)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.advance(25.0)
        orc.advance(25.0)
        _check_against_floor(sim, orc, cfg, b, h, 25.0)


def test_forcing_and_coriolis():
    """Wind stress, pressure gradient, rain and Coriolis (as the FP64 parity case)."""
    nx, ny, dx = 64, 48, 50.0
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.03,
               coriolis_f=1.0e-4, init_condition="still_water", eta_initial=0.0)
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=11, base=-5.0, amp=(-2.0, 6.0),
                     width=(100.0, 400.0))
    sim, orc = _fp32_pair(cfg, bathymetry=b)
    rng = np.random.default_rng(5)
    wx = rng.uniform(0.0, 0.3, (nx, ny))
    wy = rng.uniform(-0.1, 0.1, (nx, ny))
    p = rng.uniform(-50.0, 50.0, (nx, ny))
    rain = np.full((nx, ny), 1.0e-5)
    with sim:
        sim.set_wind(wx, wy)
        sim.set_atm_pressure(p)
        sim.set_precipitation(rain)
        g = orc.ng
        for name, arr in (("wind_x", wx), ("wind_y", wy), ("atm", p), ("precip", rain)):
            orc.arrays[name][g:-g, g:-g] = arr
        orc.s.forcing_active = 1
        sim.step(40)
        orc.step(40)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= FILM_MOM_RTOL and dv <= FILM_MOM_RTOL, (du, dv)


def test_forcing_switched_on_mid_run():
    """Steps without forcing (the sweep built without forcing terms, captured in
    the step graphs), then wind, pressure and rain set on the same handle: the
    next steps must run the forcing terms, as in the oracle."""
    nx, ny, dx = 64, 48, 50.0
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.03, dt_fixed=2.0,
               init_condition="still_water", eta_initial=0.0)
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=12, base=-5.0, amp=(-2.0, 6.0),
                     width=(100.0, 400.0))
    h = hump_depth(b, dx, dx, amp=0.3, width=300.0)
    sim, orc = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    rng = np.random.default_rng(6)
    wx = rng.uniform(0.0, 0.3, (nx, ny))
    wy = rng.uniform(-0.1, 0.1, (nx, ny))
    p = rng.uniform(-50.0, 50.0, (nx, ny))
    rain = np.full((nx, ny), 1.0e-5)
    with sim:
        sim.step(20)
        orc.step(20)
        sim.set_wind(wx, wy)
        sim.set_atm_pressure(p)
        sim.set_precipitation(rain)
        g = orc.ng
        for name, arr in (("wind_x", wx), ("wind_y", wy), ("atm", p), ("precip", rain)):
            orc.arrays[name][g:-g, g:-g] = arr
        orc.s.forcing_active = 1
        sim.step(20)
        orc.step(20)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= FILM_MOM_RTOL and dv <= FILM_MOM_RTOL, (du, dv)


def test_closed_basin_mass():
    """Walls, wet/dry hump: domain volume kept to FP32 round-off of the surface."""
    nx, ny, dx = 256, 192, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=21, width=(20.0, 150.0))
    h = hump_depth(b, dx, dx, amp=0.5, width=100.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, _ = _fp32_pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        m0 = float(sim.h_phys.sum())
        sim.step(400)
        m1 = float(sim.h_phys.sum())
        assert abs(m1 - m0) / m0 <= 1e-6, (m0, m1)


def test_switch_precision_mid_run():
    """FP64 -> FP32 -> FP64 on one handle: the state carries over both ways."""
    nx, ny, dx = 128, 128, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 16, seed=13, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=80.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025, dt_fixed=0.2)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(25)
        sim.set_precision(32)
        sim.step(25)
        sim.set_precision(64)
        assert sim.precision == 64
        sim.step(25)
        orc.step(75)
        dh, du, dv = _errors(sim, orc)
        assert dh <= ETA_TOL, dh
        assert du <= MOM_RTOL and dv <= MOM_RTOL, (du, dv)


def test_device_fields_refused_in_fp32():
    cfg = dict(nx=32, ny=16, dx=10.0, dy=10.0, t_end=10.0)
    from rakali_b200 import Rakali
    with Rakali(precision=32, **cfg) as sim:
        sim.step(2)
        with pytest.raises(RuntimeError, match="FP32"):
            sim.device_fields()
