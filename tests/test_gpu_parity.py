"""GPU parity of the B200 step against the CPU oracle, through the C ABI.

FP64 tolerance: the required bar is 1e-12 relative; these tests hold the
state to bit-identity.  The kernels keep the reference's operation order and
are built with --fmad=false, and the friction (h**(1/3)), tidal and Coriolis
(sin/cos) terms are evaluated correctly rounded on both sides, so every
field, the clock and dt match exactly.  Only the mass-budget diagnostics,
sums in a different order, carry a tolerance.
"""
import math

import numpy as np
import pytest

from tests.helpers import G, compare_state, gaussian_bed, hump_depth, max_rel_diff, pair

pytestmark = pytest.mark.gpu
RTOL = 0.0  # bit-identical: every transcendental is evaluated correctly rounded on both sides


def test_config1_dam_break_bit_exact():
    """200 x 100 dam break, dx = 10 m, HLLC, CFL 0.5, walls, 60 s."""
    cfg = dict(nx=200, ny=100, dx=10.0, dy=10.0, t_end=60.0, cfl=0.5, use_hllc=True,
               bc_west="wall", bc_east="wall", bc_south="wall", bc_north="wall")
    sim, orc = pair(cfg)
    with sim:
        sim.advance(60.0)
        orc.advance(60.0)
        assert sim.step_count == orc.step_count
        assert sim.time == orc.time
        assert sim.dt == orc.dt
        d = compare_state(sim, orc, rtol=0.0)
        compare_state(sim, orc, rtol=0.0, fields=("h0", "hu0", "hv0"))
        m0 = 0.5 * (2.0 + 1.0) * 200 * 100 * 100.0
        assert abs(sim.h_phys.sum() * 100.0 - m0) / m0 < 1e-12
        assert d["h"] == 0.0


@pytest.mark.parametrize("hllc", [False, True])
@pytest.mark.parametrize("nghost", [2, 3])
def test_wet_dry_islands_with_friction(hllc, nghost):
    """Config-2 family at 192 x 160: emergent islands, hump, Manning n = 0.025."""
    nx, ny, dx = 192, 160, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=7, width=(20.0, 120.0))
    h = hump_depth(b, dx, dx, width=80.0)
    assert (h == 0.0).sum() > 50  # dry islands present
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025,
               use_hllc=hllc, nghost=nghost)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(60)
        orc.step(60)
        assert sim.step_count == orc.step_count == 60
        assert abs(sim.time - orc.time) <= 1e-12 * orc.time
        compare_state(sim, orc, rtol=RTOL)


def test_lake_at_rest_emergent_island_1e13():
    """Flat surface over an irregular bed with dry islands stays at rest."""
    nx, ny, dx = 160, 128, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 32, seed=3, width=(20.0, 120.0))
    h = np.asfortranarray(np.maximum(0.0 - b, 0.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(200)
        hp = sim.h_phys
        wet = hp > 0.0
        eta = hp + sim.b_phys
        assert np.abs(eta[wet]).max() <= 1e-13
        # momentum round-off stays far below the reference's 1e-12 * H * sqrt(g H)
        assert np.abs(sim.hu_phys).max() <= 1e-11 and np.abs(sim.hv_phys).max() <= 1e-11
        orc.step(200)
        compare_state(sim, orc, rtol=RTOL)


@pytest.mark.parametrize("edges", [
    dict(bc_west="tidal", tidal_amplitude=0.5, tidal_period=600.0),
    dict(bc_west="open", bc_east="open", bc_south="open", bc_north="open"),
    dict(bc_west="inflow", inflow_velocity=0.3, bc_east="open"),
    dict(bc_west="discharge", discharge_flux=0.8, bc_east="clamped", clamped_elevation=0.1),
    dict(bc_west="chapman", bc_north="chapman"),
    dict(bc_west="sponge", bc_east="sponge", sponge_width=6, sponge_strength=0.01,
         sponge_h_ref=10.0),
    dict(bc_west="nested", bc_south="open"),
])
def test_boundary_types(edges):
    nx, ny, dx = 96, 64, 10.0
    b = np.asfortranarray(np.tile(np.linspace(-12.0, -8.0, nx)[:, None], (1, ny)))
    h = hump_depth(b, dx, dx, amp=0.4, width=60.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02, **edges)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.advance(120.0)
        orc.advance(120.0)
        assert sim.step_count == orc.step_count
        compare_state(sim, orc, rtol=RTOL)


def test_multi_constituent_tide_setter():
    nx, ny, dx = 80, 48, 20.0
    b = np.asfortranarray(np.tile(np.linspace(-20.0, 2.0, nx)[:, None], (1, ny)))
    h = np.asfortranarray(np.maximum(0.0 - b, 0.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02,
               bc_west="tidal")
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    amp, ph, om = [0.8, 0.2], [0.3, -1.1], [2 * math.pi / 300.0, 2 * math.pi / 170.0]
    with sim:
        sim.set_tidal_constituents(amp, ph, om)
        orc.set_tidal_constituents(amp, ph, om)
        sim.advance(200.0)
        orc.advance(200.0)
        compare_state(sim, orc, rtol=RTOL)


def test_forcing_wind_pressure_rain_coriolis():
    nx, ny, dx = 64, 48, 50.0
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.03,
               coriolis_f=1.0e-4, init_condition="still_water", eta_initial=0.0)
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=11, base=-5.0, amp=(-2.0, 6.0),
                     width=(100.0, 400.0))
    sim, orc = pair(cfg, bathymetry=b)
    rng = np.random.default_rng(5)
    wx = rng.uniform(0.0, 0.3, (nx, ny))
    wy = rng.uniform(-0.1, 0.1, (nx, ny))
    p = rng.uniform(-50.0, 50.0, (nx, ny))  # anomaly: the ghosts stay at 0
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
        compare_state(sim, orc, rtol=RTOL)
        mo, ms = sim.mass_budget()
        assert abs(ms - orc.s.mass_src) <= 1e-10 * abs(orc.s.mass_src)


def test_closed_basin_mass_and_budget():
    """Walls only: mass conserved to round-off, boundary outflux ~ 0."""
    nx, ny, dx = 128, 96, 10.0
    b = gaussian_bed(nx, ny, dx, dx, 12, seed=2, width=(30.0, 200.0))
    h = hump_depth(b, dx, dx, amp=0.5, width=100.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        m0 = sim.h_phys.sum()
        sim.step(300)
        m1 = sim.h_phys.sum()
        assert abs(m1 - m0) <= 1e-12 * m0
        mo, _ = sim.mass_budget()
        orc.step(300)
        assert abs(mo - orc.s.mass_out) <= 1e-9 * max(1.0, abs(orc.s.mass_out))


def test_cfl_interval_and_dt_fixed():
    nx, ny, dx = 64, 64, 10.0
    for extra in (dict(cfl_interval=5), dict(dt_fixed=0.4)):
        cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=30.0, cfl=0.45, **extra)
        sim, orc = pair(cfg)
        with sim:
            sim.advance(25.0)
            orc.advance(25.0)
            assert sim.step_count == orc.step_count
            assert sim.dt == orc.dt
            compare_state(sim, orc, rtol=0.0)


def test_step_clamps_to_t_end_like_reference():
    cfg = dict(nx=8, ny=8, dx=1.0, dy=1.0, t_end=0.2)
    sim, orc = pair(cfg)
    with sim:
        sim.step(2000)
        orc.step(2000)
        assert sim.time == pytest.approx(0.2)
        assert sim.time == orc.time
        compare_state(sim, orc, rtol=0.0)
        with pytest.raises(RuntimeError, match="t_end"):
            sim.step(1)


# ---------------------------------------------------------------------------
# generic Shu-Osher schemes (euler, rk3, rk43): rki_solver.F90:861-926
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("scheme", ["euler", "rk3", "rk43"])
@pytest.mark.parametrize("hllc", [False, True])
def test_generic_schemes_wet_dry_friction(scheme, hllc):
    """Islands, hump, Manning n: every stage, the SSP mixes, dt (x2 for rk43)."""
    nx, ny, dx = 120, 96, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 20, seed=17, width=(20.0, 100.0))
    h = hump_depth(b, dx, dx, width=60.0)
    assert (h == 0.0).sum() > 20
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025,
               use_hllc=hllc, time_scheme=scheme)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(40)
        orc.step(40)
        assert sim.step_count == orc.step_count == 40
        assert sim.time == orc.time
        assert sim.dt == orc.dt
        compare_state(sim, orc, rtol=0.0)
        compare_state(sim, orc, rtol=0.0, fields=("h0", "hu0", "hv0"))


@pytest.mark.parametrize("scheme", ["euler", "rk3", "rk43"])
@pytest.mark.parametrize("edges", [
    dict(bc_west="tidal", tidal_amplitude=0.5, tidal_period=300.0, bc_east="chapman"),
    dict(bc_west="sponge", bc_east="sponge", sponge_width=6, sponge_strength=0.01,
         sponge_h_ref=10.0, bc_south="open", bc_north="inflow", inflow_velocity=0.2),
])
def test_generic_schemes_boundaries(scheme, edges):
    """Stage times t + c_k dt reach the tide; sponge and Chapman per stage."""
    nx, ny, dx = 96, 64, 10.0
    b = np.asfortranarray(np.tile(np.linspace(-12.0, -8.0, nx)[:, None], (1, ny)))
    h = hump_depth(b, dx, dx, amp=0.4, width=60.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02,
               time_scheme=scheme, **edges)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.advance(90.0)
        orc.advance(90.0)
        assert sim.step_count == orc.step_count
        assert sim.time == orc.time
        compare_state(sim, orc, rtol=0.0)


@pytest.mark.parametrize("scheme", ["euler", "rk3", "rk43"])
def test_generic_schemes_forcing_coriolis(scheme):
    """Wind, pressure, rain and the Coriolis rotation by f * beta_k dt."""
    nx, ny, dx = 48, 40, 50.0
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.03,
               coriolis_f=1.0e-4, init_condition="still_water", eta_initial=0.0,
               time_scheme=scheme)
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=12, base=-5.0, amp=(-2.0, 6.0),
                     width=(100.0, 400.0))
    sim, orc = pair(cfg, bathymetry=b)
    rng = np.random.default_rng(8)
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
        sim.step(30)
        orc.step(30)
        compare_state(sim, orc, rtol=0.0)


def test_generic_scheme_graph_chunks_and_fixed_dt():
    """Many steps per graph launch, other tiles and a fixed dt give the same bits."""
    nx, ny, dx = 80, 72, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 12, seed=21, width=(20.0, 80.0))
    h = hump_depth(b, dx, dx, width=50.0)
    for tile, extra in ((0, dict(cfl_interval=3)), (4, dict(dt_fixed=0.05))):
        cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, time_scheme="rk3", **extra)
        sim, orc = pair(cfg, bathymetry=b, initial_h=h)
        with sim:
            sim.set_tile(tile)  # 4: a marching tile, whose generic stages run on 32x16 tiles
            sim.step(150)
            orc.step(150)
            assert sim.dt == orc.dt
            compare_state(sim, orc, rtol=0.0)


def test_generic_schemes_refuse_fp32_and_batches():
    from rakali_b200 import Rakali
    from rakali_b200.ensemble import Ensemble
    cfg = dict(nx=32, ny=32, dx=1.0, dy=1.0, t_end=10.0, time_scheme="rk3")
    with Rakali(**cfg) as sim:
        with pytest.raises(RuntimeError, match="SSP-RK2"):
            sim.set_precision(32)
        assert sim.precision == 64
        with pytest.raises(RuntimeError, match="SSP-RK2"):
            Ensemble([sim])
        sim.step(3)  # still usable


@pytest.mark.parametrize("nghost", [2, 3, 4, 5])
@pytest.mark.parametrize("physics", ["plain", "forcing_coriolis_sponge"])
def test_tma_tiles_against_the_oracle(nghost, physics):
    """The TMA-staged tile kernel (the default) on every ghost parity: its boxes
    start one column left of the tile when nghost is odd.  77 x 50 leaves
    ragged tiles on both axes; the full-physics case runs the kernel built
    with forcing, Coriolis and sponge terms."""
    nx, ny, dx = 77, 50, 20.0
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, nghost=nghost, t_end=1e6, cfl=0.45, manning_n=0.03,
               use_hllc=True)
    if physics != "plain":
        cfg.update(coriolis_f=1.0e-4, bc_west="sponge", sponge_width=5, sponge_strength=0.01,
                   sponge_h_ref=8.0)
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=40 + nghost, base=-6.0, amp=(-2.0, 8.0),
                     width=(60.0, 300.0))
    h = hump_depth(b, dx, dx, width=150.0)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        assert sim._lib.rkb_tma_tile_status(sim._handle) == 0
        assert sim._lib.rkb_get_tile(sim._handle) == 10
        if physics != "plain":
            rng = np.random.default_rng(nghost)
            wx = rng.uniform(0.0, 0.3, (nx, ny))
            wy = rng.uniform(-0.1, 0.1, (nx, ny))
            pr = rng.uniform(-50.0, 50.0, (nx, ny))
            rain = np.full((nx, ny), 1.0e-5)
            sim.set_wind(wx, wy)
            sim.set_atm_pressure(pr)
            sim.set_precipitation(rain)
            g = orc.ng
            for name, arr in (("wind_x", wx), ("wind_y", wy), ("atm", pr), ("precip", rain)):
                orc.arrays[name][g:-g, g:-g] = arr
            orc.s.forcing_active = 1
        sim.step(40)
        orc.step(40)
        assert sim.dt == orc.dt
        compare_state(sim, orc, rtol=0.0)


def test_tiles_agree():
    nx, ny, dx = 150, 70, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 10, seed=9, width=(20.0, 80.0))
    h = hump_depth(b, dx, dx, width=40.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, use_hllc=True)
    ref = None
    for tile in range(11):
        sim, _ = pair(cfg, bathymetry=b, initial_h=h)
        with sim:
            sim.set_tile(tile)
            if tile == 10:  # the TMA-staged kernel, not its fallback
                assert sim._lib.rkb_tma_tile_status(sim._handle) == 0
            sim.step(25)
            cur = sim.h.copy(), sim.hu.copy(), sim.hv.copy()
        if ref is None:
            ref = cur
        else:
            for a, r in zip(cur, ref):
                assert np.array_equal(a, r)


# ---------------------------------------------------------------------------
# kernel-level entry points (device arrays through torch)
# ---------------------------------------------------------------------------

def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).cuda()


def _host(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.mark.parametrize("hllc", [False, True])
def test_kernel_flux_matches_oracle(hllc):
    from oracle import oracle as orc
    from rakali_b200 import _lib
    lib = _lib.load()
    nx, ny, ng = 70, 45, 2
    rng = np.random.default_rng(1)
    b = gaussian_bed(nx + 2 * ng, ny + 2 * ng, 1.0, 1.0, 5, seed=4, base=-1.0, amp=(-0.5, 1.5),
                     width=(3.0, 10.0))
    h = np.asfortranarray(np.maximum(0.3 * rng.random(b.shape) - b, 0.0))
    h[h < 2e-3] *= rng.random((h < 2e-3).sum())  # thin films near the fronts
    hu = np.asfortranarray(rng.normal(0, 0.3, b.shape) * h)
    hv = np.asfortranarray(rng.normal(0, 0.3, b.shape) * h)
    exp = orc.compute_flux(h, hu, hv, b, ng, 1.0, 1.0, hllc=hllc)
    dh, dhu, dhv, db = (_dev(a) for a in (h, hu, hv, b))
    outs = [_dev(np.zeros_like(h)) for _ in range(5)]
    rc = lib.rkb_compute_flux(int(hllc), dh.data_ptr(), dhu.data_ptr(), dhv.data_ptr(),
                              db.data_ptr(), *(o.data_ptr() for o in outs), h.shape[0],
                              h.shape[1], ng, h.shape[0], 1.0, 1.0)
    assert rc == 0
    s = (slice(ng, -ng), slice(ng, -ng))
    for got, want in zip(outs[:3], exp[:3]):
        assert np.array_equal(_host(got)[s], want[s])
    # mass fluxes: right/top faces of the interior plus the first left/bottom face
    assert np.array_equal(_host(outs[3])[ng - 1:-ng, ng:-ng], exp[3][ng - 1:-ng, ng:-ng])
    assert np.array_equal(_host(outs[4])[ng:-ng, ng - 1:-ng], exp[4][ng:-ng, ng - 1:-ng])


def test_kernel_flux_known_answers():
    """test_flux.F90:66-148 (dam break) and :185-229 (lake at rest) on the GPU."""
    from rakali_b200 import _lib
    lib = _lib.load()

    def run(h, hu, hv, b, ng=2):
        ins = [_dev(a) for a in (h, hu, hv, b)]
        outs = [_dev(np.zeros_like(h)) for _ in range(5)]
        rc = lib.rkb_compute_flux(0, *(t.data_ptr() for t in ins), *(o.data_ptr() for o in outs),
                                  h.shape[0], h.shape[1], ng, h.shape[0], 1.0, 1.0)
        assert rc == 0
        return [_host(o) for o in outs]

    nx, ny = 16, 8
    h = np.full((nx, ny), 1.0, order="F")
    h[: nx // 2, :] = 2.0
    z = np.zeros((nx, ny), order="F")
    fh = run(h, z, z, z)[0]
    im = nx // 2 - 1
    for j in range(2, ny - 2):
        assert abs(fh[im, j] + math.sqrt(G / 2)) < 1e-12
        assert abs(fh[im, j] + fh[im + 1, j]) < 1e-13
    i = np.arange(1, 15)[:, None]
    j = np.arange(1, 15)[None, :]
    b = np.asfortranarray(0.5 * np.exp(-0.5 * ((i - 7) ** 2 + (j - 7) ** 2).astype(float)))
    hh = np.asfortranarray(np.maximum(0.0, 2.0 - b))
    out = run(hh, np.zeros_like(b), np.zeros_like(b), b)
    assert max(np.abs(o[2:-2, 2:-2]).max() for o in out[:3]) < 1e-10


def test_kernel_timestep_matches_oracle():
    from oracle import oracle as orc
    from rakali_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(2)
    shape = (38, 27)
    h = np.asfortranarray(rng.random(shape) * 2.0)
    h[h < 0.2] = 0.0
    hu = np.asfortranarray(rng.normal(0, 1, shape))
    hv = np.asfortranarray(rng.normal(0, 1, shape))
    dt_ref, _ = orc.compute_timestep(h, hu, hv, 3, 2.0, 3.0, 0.45)
    ins = [_dev(a) for a in (h, hu, hv)]
    import ctypes
    out = ctypes.c_double()
    rc = lib.rkb_compute_timestep(*(t.data_ptr() for t in ins), shape[0], shape[1], 3, shape[0],
                                  2.0, 3.0, 0.45, ctypes.byref(out))
    assert rc == 0
    assert out.value == dt_ref


# ---------------------------------------------------------------------------
# restart files (rki_save_restart / rki_load_restart)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("precision", [64, 32])
def test_restart_round_trip_continues_bit_identically(tmp_path, precision):
    """save_restart after 30 steps, from_restart into a fresh handle: state and
    clock restored exactly; 30 more steps on both give the same bits."""
    from scipy.io import netcdf_file

    from rakali_b200 import Rakali
    nx, ny, dx = 96, 80, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 12, seed=23, width=(20.0, 90.0))
    h = hump_depth(b, dx, dx, width=50.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim = Rakali(defer_init=True, precision=precision, **cfg)
    sim.set_bathymetry(b)
    sim.set_initial_h(h)
    sim.finalize()
    path = tmp_path / "restart.nc"
    with sim:
        sim.step(30)
        sim.save_restart(path)
        t30 = sim.time
        ref = [getattr(sim, f + "_phys").copy() for f in ("h", "hu", "hv", "b")]
        with netcdf_file(str(path), "r", mmap=False) as f:
            assert np.array_equal(np.asarray(f.variables["h"][:]).T, ref[0])
            assert float(f.variables["time"].getValue()) == t30
        with Rakali.from_restart(path, precision=precision, **cfg) as sim2:
            assert sim2.time == t30
            for fld, r in zip(("h", "hu", "hv", "b"), ref):
                assert np.array_equal(getattr(sim2, fld + "_phys"), r)
            sim.step(30)
            sim2.step(30)
            assert sim2.time == sim.time
            for fld in ("h", "hu", "hv"):
                assert np.array_equal(getattr(sim2, fld + "_phys"), getattr(sim, fld + "_phys"))


def test_checkpoint_matches_oracle_and_run_continues(tmp_path):
    """save_checkpoint after 17 steps: every field with its ghosts (RK2 saves
    included) equals the oracle's bit for bit, the scalar attributes are the
    handle's, and the run then continues bit-identically with the oracle."""
    from scipy.io import netcdf_file
    nx, ny, dx = 72, 56, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 10, seed=29, width=(20.0, 90.0))
    h = hump_depth(b, dx, dx, width=50.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025,
               coriolis_f=1.0e-4)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    path = tmp_path / "step_17.nc"
    with sim:
        sim.step(17)
        orc.step(17)
        sim.save_checkpoint(path)
        ng = orc.ng
        with netcdf_file(str(path), "r", mmap=False) as f:
            assert f.dimensions["x_total"] == nx + 2 * ng
            assert f.dimensions["y_total"] == ny + 2 * ng
            for name in ("h", "hu", "hv", "b", "h0", "hu0", "hv0"):
                v = np.asarray(f.variables[name][:])
                assert f.variables[name].dimensions == ("x_total", "y_total")
                assert np.array_equal(v, orc.arrays[name]), name
            assert f.variables["b"].positive == b"up"
            at = f._attributes
            assert float(at["time"]) == sim.time
            assert int(at["step_count"]) == sim.step_count == 17
            assert float(at["dt"]) == sim.dt
            assert (int(at["nx_phys"]), int(at["ny_phys"]), int(at["nghost"])) == (nx, ny, ng)
            assert (int(at["nx_total"]), int(at["ny_total"])) == (nx + 2 * ng, ny + 2 * ng)
            assert float(at["dx"]) == dx and float(at["dy"]) == dx
            assert float(at["manning_n"]) == 0.025 and float(at["coriolis_f"]) == 1.0e-4
            assert float(at["clamped_elevation"]) == sim.clamped_elevation
        sim.step(9)
        orc.step(9)
        compare_state(sim, orc, rtol=0.0, fields=("h", "hu", "hv", "b", "h0", "hu0", "hv0"))


def test_checkpoint_fp32_form_leaves_the_run_unchanged(tmp_path):
    """FP32 surface form: the checkpoint holds the fields the handle's views
    return, and a run that writes one continues bit-identically to one that
    does not."""
    from scipy.io import netcdf_file

    from rakali_b200 import Rakali
    nx, ny, dx = 64, 48, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 10, seed=41, width=(20.0, 90.0))
    h = hump_depth(b, dx, dx, width=50.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)

    def make():
        s = Rakali(defer_init=True, precision=32, **cfg)
        s.set_bathymetry(b)
        s.set_initial_h(h)
        s.finalize()
        return s

    path = tmp_path / "ck32.nc"
    with make() as a, make() as c:
        a.step(17)
        a.save_checkpoint(path)
        a.step(9)
        c.step(26)
        for f in ("h", "hu", "hv"):
            assert np.array_equal(getattr(a, f), getattr(c, f)), f
        assert a.time == c.time
        with make() as d:
            d.step(17)
            with netcdf_file(str(path), "r", mmap=False) as nc:
                for f in ("h", "hu", "hv", "b", "h0", "hu0", "hv0"):
                    assert np.array_equal(np.asarray(nc.variables[f][:]), getattr(d, f)), f


def test_sync_host_leaves_bed_and_rk2_saves_readable():
    """rki_sync_host refreshes h, hu, hv only; reading the bed (whose ghosts
    the wall fill mirrors every step) or the RK2 saves afterwards still gives
    their current values, as in the oracle, and stepping continues exactly."""
    nx, ny, dx = 48, 40, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=31, width=(20.0, 60.0))
    h = hump_depth(b, dx, dx, width=40.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(6)
        orc.step(6)
        sim.sync_host()
        compare_state(sim, orc, rtol=0.0, fields=("b", "h0", "hu0", "hv0", "h", "hu", "hv"))
        sim.step(4)
        orc.step(4)
        compare_state(sim, orc, rtol=0.0, fields=("h", "hu", "hv", "b", "h0", "hu0", "hv0"))


def test_front_end_layer_accessors_sync_and_xarray():
    """Front-end methods outside the 2D step: the multilayer accessors and
    setters raise RuntimeError as the reference's do when multilayer mode is
    off; sync_from_device hands the host the state and stepping continues
    exactly; to_xarray raises ImportError without xarray, else returns the
    interior snapshot."""
    nx, ny, dx = 40, 32, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=37, width=(20.0, 60.0))
    h = hump_depth(b, dx, dx, width=40.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.025)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        assert sim.nz == 0
        for name in ("h_layer", "salinity", "temperature"):
            with pytest.raises(RuntimeError):
                getattr(sim, name)
        for name in ("set_salinity", "set_temperature"):
            with pytest.raises(RuntimeError, match="multilayer"):
                getattr(sim, name)(np.zeros((nx, ny, 1)))
        sim.step(5)
        orc.step(5)
        sim.sync_from_device()
        compare_state(sim, orc, rtol=0.0, fields=("h", "hu", "hv", "b", "h0", "hu0", "hv0"))
        sim.step(5)
        orc.step(5)
        compare_state(sim, orc, rtol=0.0)
        try:
            import xarray  # noqa: F401
        except ImportError:
            with pytest.raises(ImportError, match="xarray"):
                sim.to_xarray()
        else:
            ds = sim.to_xarray()
            assert np.array_equal(ds["h"].values[0], orc.interior("h"))
            assert float(ds.attrs["time"]) == sim.time


def test_restart_refuses_grid_mismatch_and_finalised_handle(tmp_path):
    from rakali_b200 import Rakali
    path = tmp_path / "r.nc"
    with Rakali(nx=16, ny=12, dx=1.0, dy=1.0, t_end=10.0) as sim:
        sim.step(2)
        sim.save_restart(path)
        raw = str(path).encode()
        assert sim._lib.rki_load_restart(sim._handle, raw, len(raw)) == -2  # finalised
    with pytest.raises(RuntimeError, match="mismatch"):
        Rakali.from_restart(path, nx=17, ny=12, dx=1.0, dy=1.0, t_end=10.0)


def test_bathymetry_file_equals_set_bathymetry(tmp_path):
    """A namelist bathymetry_file (NetCDF classic) loads the same bed as
    set_bathymetry: same ghosts, same initial condition, same steps."""
    from scipy.io import netcdf_file

    from rakali_b200 import Rakali
    nx, ny, dx = 64, 48, 10.0
    b = gaussian_bed(nx, ny, dx, dx, 8, seed=5, width=(30.0, 120.0))
    path = tmp_path / "bed.nc"
    with netcdf_file(str(path), "w", version=2) as f:
        f.createDimension("x", nx)
        f.createDimension("y", ny)
        f.createVariable("elevation", "d", ("y", "x"))[:] = b.T
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02,
               init_condition="still_water", eta_initial=0.2)
    with Rakali(bathymetry_file=str(path), **cfg) as s1, Rakali(defer_init=True, **cfg) as s2:
        s2.set_bathymetry(b)
        s2.finalize()
        assert np.array_equal(s1.b, s2.b) and np.array_equal(s1.h, s2.h)
        s1.step(20)
        s2.step(20)
        assert np.array_equal(s1.h, s2.h) and np.array_equal(s1.hu, s2.hu)


# ---------------------------------------------------------------------------
# gauges (src/io/structured/rki_gauges.F90), recorded on the device
# ---------------------------------------------------------------------------

def _gauge_weights(x, y, dx, dy, nx, ny, ng):
    """compute_local_gauges + compute_interp_weights (rki_gauges.F90:208-336), 0-based."""
    out = []
    for k, (gx, gy) in enumerate(zip(x, y)):
        ig, jg = math.floor(gx / dx) + 1, math.floor(gy / dy) + 1
        if not (1 <= ig <= nx and 1 <= jg <= ny):
            continue
        ia, ja = ig + ng, jg + ng
        xc, yc = (ig - 0.5) * dx, (jg - 0.5) * dy
        if gx < xc:
            i0, wx = (ia - 1, (gx - (xc - dx)) / dx) if ig > 1 else (ia, 0.0)
        else:
            i0, wx = (ia, (gx - xc) / dx) if ig < nx else (ia, 0.0)
        if gy < yc:
            j0, wy = (ja - 1, (gy - (yc - dy)) / dy) if jg > 1 else (ja, 0.0)
        else:
            j0, wy = (ja, (gy - yc) / dy) if jg < ny else (ja, 0.0)
        out.append((k, i0 - 1, j0 - 1, max(0.0, min(1.0, wx)), max(0.0, min(1.0, wy))))
    return out


def _blend(a, i0, j0, wx, wy):
    return ((1.0 - wx) * (1.0 - wy) * a[i0, j0] + wx * (1.0 - wy) * a[i0 + 1, j0]
            + (1.0 - wx) * wy * a[i0, j0 + 1] + wx * wy * a[i0 + 1, j0 + 1])


def test_gauges_match_the_reference_formula_on_the_oracle():
    """Every-step records: bit-identical to gauges_write's formula applied to
    the oracle's state after each step; edge stations clamp; outside dropped."""
    nx, ny, dx = 80, 60, 10.0
    b = gaussian_bed(nx, ny, dx, dx, 10, seed=31, width=(30.0, 120.0))
    h = hump_depth(b, dx, dx, amp=0.4, width=60.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02, use_hllc=True)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    xs = [3.0, 401.7, 795.0, 250.0, 555.5, 900.0, 10.0]
    ys = [2.0, 300.2, 598.0, 5.0, 444.4, 30.0, -1.0]
    w = _gauge_weights(xs, ys, dx, dx, nx, ny, orc.ng)
    with sim:
        kept = sim.set_gauges(xs, ys, names=[f"g{k}" for k in range(len(xs))])
        assert kept == len(w) == 5
        sim.step(12)
        rec = sim.gauge_records()
        assert rec["time"].size == 12 and not rec["overflow"]
        for s in range(12):
            orc.step(1)
            assert rec["time"][s] == orc.time
            A = orc.arrays
            for m, (k, i0, j0, wx, wy) in enumerate(w):
                hh = _blend(A["h"], i0, j0, wx, wy)
                bb = _blend(A["b"], i0, j0, wx, wy)
                hs = max(hh, 1.0e-6)
                assert rec["eta"][s, m] == hh + bb
                assert rec["u"][s, m] == _blend(A["hu"], i0, j0, wx, wy) / hs
                assert rec["v"][s, m] == _blend(A["hv"], i0, j0, wx, wy) / hs
        assert rec["names"] == [f"g{k}" for k, *_ in w]


@pytest.mark.parametrize("precision", [64, 32])
def test_gauge_interval_capacity_and_file(tmp_path, precision):
    """interval > 0 follows the driver's next-time rule; a full buffer sets
    overflow; the file round-trips through scipy."""
    from scipy.io import netcdf_file

    from rakali_b200 import Rakali
    nx, ny, dx = 48, 40, 10.0
    b = gaussian_bed(nx, ny, dx, dx, 6, seed=2, width=(30.0, 100.0))
    h = hump_depth(b, dx, dx, amp=0.4, width=50.0)
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02)
    with Rakali(defer_init=True, precision=precision, **cfg) as sim:
        sim.set_bathymetry(b)
        sim.set_initial_h(h)
        sim.finalize()
        sim.set_gauges([100.0, 250.0], [120.0, 200.0], names=["a", "b"], interval=3.0)
        sim.step(40)
        rec = sim.gauge_records()
    # replay the cadence on the recorded clock: record when t >= next, next += 3
    with Rakali(defer_init=True, precision=precision, **cfg) as ref:
        ref.set_bathymetry(b)
        ref.set_initial_h(h)
        ref.finalize()
        nxt, expect = 3.0, []
        for _ in range(40):
            ref.step(1)
            if ref.time >= nxt:
                expect.append(ref.time)
                nxt += 3.0
    assert np.array_equal(rec["time"], np.array(expect))
    with Rakali(defer_init=True, precision=precision, **cfg) as sim:
        sim.set_bathymetry(b)
        sim.set_initial_h(h)
        sim.finalize()
        sim.set_gauges([100.0], [120.0], capacity=5)
        sim.step(8)
        rec = sim.gauge_records()
        assert rec["time"].size == 5 and rec["overflow"]
        path = tmp_path / "gauges.nc"
        sim.write_gauges(path)
        with netcdf_file(str(path), "r", mmap=False) as f:
            assert np.array_equal(f.variables["eta"][:, 0], rec["eta"][:, 0])
            assert np.array_equal(f.variables["time"][:], rec["time"])


# ---------------------------------------------------------------------------
# narrow and tiny grids (interiors thinner than the ghost width)
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("nx,ny,nghost", [(1, 7, 2), (7, 1, 2), (2, 2, 2), (3, 5, 3), (2, 9, 3)])
def test_narrow_grids_bit_exact_and_fp32_runs(nx, ny, nghost):
    """Grids narrower than max(nghost, 2) fill opposite edges one after the
    other (the reference's W, E, S, N order reads the other side's ghosts);
    FP64 stays bit-identical to the oracle, the FP32 form stays close to it."""
    from rakali_b200 import Rakali
    dx = 10.0
    b = np.asfortranarray(-4.0 + 0.5 * np.add.outer(np.arange(nx), np.arange(ny)) / max(nx, ny))
    h = np.asfortranarray(np.maximum(0.3 * np.exp(-np.add.outer(np.arange(nx) - nx / 2.0,
                                                                 np.arange(ny) - ny / 2.0) ** 2)
                                     - b, 0.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, nghost=nghost, t_end=1e6, cfl=0.45, manning_n=0.02)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(20)
        orc.step(20)
        compare_state(sim, orc, rtol=0.0)
        h64 = sim.h_phys.copy()
    with Rakali(defer_init=True, precision=32, **cfg) as s32:
        s32.set_bathymetry(b)
        s32.set_initial_h(h)
        s32.finalize()
        s32.step(20)
        assert np.all(np.isfinite(s32.h_phys))
        assert np.abs((s32.h_phys + s32.b_phys) - (h64 + b)).max() <= 1e-4


@pytest.mark.parametrize("nx,ny", [(3, 70000), (70000, 3)])
def test_long_grids_beyond_65535_rows(nx, ny):
    """Grids longer than a CUDA grid's y extent (65535) in either direction:
    FP64 bit-identical to the oracle, the FP32 form (whose layout conversions
    walk the rows) close to it."""
    from rakali_b200 import Rakali
    dx = 10.0
    x = np.arange(nx)[:, None] * np.ones((1, ny))
    y = np.ones((nx, 1)) * np.arange(ny)[None, :]
    b = np.asfortranarray(-5.0 + 1.0e-4 * (x + y))
    h = np.asfortranarray(np.maximum(0.2 * np.exp(-((x + y - 35000.0) / 40.0) ** 2) - b, 0.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02)
    sim, orc = pair(cfg, bathymetry=b, initial_h=h)
    with sim:
        sim.step(5)
        orc.step(5)
        compare_state(sim, orc, rtol=0.0)
        e64 = sim.h_phys + sim.b_phys
    with Rakali(defer_init=True, precision=32, **cfg) as s32:
        s32.set_bathymetry(b)
        s32.set_initial_h(h)
        s32.finalize()
        s32.step(5)
        assert np.abs((s32.h_phys + s32.b_phys) - e64).max() <= 1e-4


@pytest.mark.parametrize("precision", [64, 32])
def test_all_dry_domain(precision):
    """No water anywhere: the CFL step falls back to cfl min(dx, dy) / sqrt(g DRY)
    (rki_kernel_timestep.F90:68-72) and nothing moves; FP64 equals the oracle."""
    from rakali_b200 import Rakali
    nx, ny, dx = 40, 30, 5.0
    b = gaussian_bed(nx, ny, dx, dx, 5, seed=4, base=1.0, amp=(0.0, 2.0), width=(20.0, 60.0))
    cfg = dict(nx=nx, ny=ny, dx=dx, dy=dx, t_end=1e6, cfl=0.45, manning_n=0.02,
               init_condition="still_water", eta_initial=0.0)
    if precision == 64:
        sim, orc = pair(cfg, bathymetry=b)
        with sim:
            sim.step(5)
            orc.step(5)
            assert sim.dt == orc.dt == 0.45 * dx / math.sqrt(G * 1.0e-6)
            compare_state(sim, orc, rtol=0.0)
            assert not sim.h_phys.any()
    else:
        with Rakali(defer_init=True, precision=32, **cfg) as sim:
            sim.set_bathymetry(b)
            sim.finalize()
            sim.step(5)
            assert not sim.h_phys.any() and not sim.hu_phys.any() and not sim.hv_phys.any()
