"""Kernel-level entry points on caller-owned device arrays, against the oracle.

The structured kernels of src/core/coastal/kernels/structured/barotropic, one
C entry point each (include/rakali.h): fused_update_stage1/2/_generic
(rki_kernel_fused.F90:22-471), compute_update / compute_rk2_average /
compute_ssp_combine (rki_kernel_update.F90:35-208), apply_friction /
apply_coriolis (rki_kernel_friction.F90:16-152), apply_boundary_conditions
(rki_boundary.F90:40-552) and apply_sponge (rki_kernel_sponge.F90:16-88).
Each is run through the C ABI on device copies of seeded states with wet,
dry and thin-film cells, and compared with the oracle's restatement of the
same kernel: bit-identical, ghosts included where the kernel writes them.
"""
import ctypes

import numpy as np
import pytest

from helpers import gaussian_bed

pytestmark = pytest.mark.gpu

BC = {"wall": 1, "open": 2, "tidal": 3, "nested": 4, "inflow": 5, "discharge": 6,
      "clamped": 7, "sponge": 8, "chapman": 9}


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).cuda()


def _host(t):
    return np.asfortranarray(t.cpu().numpy().T)


@pytest.fixture(scope="module")
def lib():
    from rakali_b200 import _lib
    return _lib.load()


def _state(nx, ny, ng, seed):
    """h, hu, hv, b (with ghosts) over a Gaussian bed: dry islands, thin films,
    strong currents in places (so the clamp, KP07 and the Froude backstop run)."""
    rng = np.random.default_rng(seed)
    b = gaussian_bed(nx + 2 * ng, ny + 2 * ng, 1.0, 1.0, 6, seed=seed + 1, base=-1.0,
                     amp=(-0.5, 1.6), width=(3.0, 9.0))
    h = np.asfortranarray(np.maximum(0.4 * rng.random(b.shape) - b, 0.0))
    thin = h < 3e-3
    h[thin] *= rng.random(thin.sum()) * 0.3
    hu = np.asfortranarray(rng.normal(0, 0.4, b.shape) * np.maximum(h, 1e-7))
    hv = np.asfortranarray(rng.normal(0, 0.4, b.shape) * np.maximum(h, 1e-7))
    fast = rng.random(b.shape) < 0.01
    hu[fast] *= 300.0
    return h, hu, hv, b


def _fluxes(shape, seed, scale=2.0):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.normal(0, scale, shape)) for _ in range(3)]


def _forcing(shape, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(a) for a in (rng.normal(0, 0.3, shape), rng.normal(0, 0.3, shape),
                                           101325.0 + rng.normal(0, 300.0, shape),
                                           rng.random(shape) * 1e-4)]


def _same(got, want, what):
    assert np.array_equal(got, want), (what, float(np.max(np.abs(got - want))))


@pytest.mark.parametrize("stage", [1, 2, 3])
@pytest.mark.parametrize("forcing,coriolis", [(False, 0.0), (True, 1.2e-4)])
def test_fused_update_stages(lib, stage, forcing, coriolis):
    from oracle import oracle as orc
    nx, ny, ng = 61, 37, 2
    h, hu, hv, b = _state(nx, ny, ng, 11 + stage)
    fh, fhu, fhv = _fluxes(h.shape, 5)
    h0 = np.asfortranarray(h + 0.01)
    hu0 = np.asfortranarray(hu * 0.9)
    hv0 = np.asfortranarray(hv * 1.1)
    f4 = _forcing(h.shape, 3) if forcing else [None] * 4
    dt, n, dx, dy = 0.013, 0.03, 1.5, 0.75
    want = [a.copy(order="F") for a in (h, hu, hv, h0, hu0, hv0)]
    kw = dict(manning_n=n, wind_x=f4[0], wind_y=f4[1], atm=f4[2], precip=f4[3],
              coriolis_f=coriolis, forcing_active=forcing, dx=dx, dy=dy)
    if stage == 3:
        orc.fused_stage_generic(*want[:3], fh, fhu, fhv, ng, dt, **kw)
    else:
        orc.fused_stage(stage, *want, fh, fhu, fhv, ng, dt, **kw)
    d = [_dev(a) for a in (h, hu, hv, h0, hu0, hv0, fh, fhu, fhv)]
    fd = [_dev(a) if a is not None else None for a in f4]
    fp = [t.data_ptr() if t is not None else None for t in fd]
    tail = (h.shape[0], h.shape[1], ng, h.shape[0], dx, dy, dt, n, *fp, coriolis, int(forcing))
    if stage == 1:
        rc = lib.rkb_fused_update_stage1(*(t.data_ptr() for t in d), *tail)
    elif stage == 2:
        rc = lib.rkb_fused_update_stage2(*(t.data_ptr() for t in d), *tail)
    else:
        rc = lib.rkb_fused_update_stage_generic(*(t.data_ptr() for t in d[:3] + d[6:]), *tail)
    assert rc == 0
    for k, name in enumerate(("h", "hu", "hv", "h0", "hu0", "hv0")):
        _same(_host(d[k]), want[k], name)


@pytest.mark.parametrize("kind", ["update", "rk2", "ssp"])
def test_update_average_combine(lib, kind):
    from oracle import oracle as orc
    nx, ny, ng = 45, 52, 3
    h, hu, hv, _ = _state(nx, ny, ng, 21)
    h0 = np.asfortranarray(np.abs(h - 0.02))
    hu0 = np.asfortranarray(-hu)
    hv0 = np.asfortranarray(hv * 0.5)
    fh, fhu, fhv = _fluxes(h.shape, 8, scale=5.0)
    want = [a.copy(order="F") for a in (h, hu, hv)]
    d = [_dev(a) for a in (h, hu, hv)]
    G = (h.shape[0], h.shape[1], ng, h.shape[0])
    if kind == "update":
        orc.compute_update(*want, fh, fhu, fhv, ng, 0.05)
        f = [_dev(a) for a in (fh, fhu, fhv)]
        rc = lib.rkb_compute_update(*(t.data_ptr() for t in d + f), *G, 0.05)
    else:
        o = [_dev(a) for a in (h0, hu0, hv0)]
        if kind == "rk2":
            orc.rk2_average(*want, h0, hu0, hv0, ng)
            rc = lib.rkb_compute_rk2_average(*(t.data_ptr() for t in d + o), *G)
        else:
            a_n = 1.0 / 3.0
            orc.ssp_combine(*want, h0, hu0, hv0, a_n, ng)
            rc = lib.rkb_compute_ssp_combine(*(t.data_ptr() for t in d + o), a_n, *G)
    assert rc == 0
    for k, name in enumerate(("h", "hu", "hv")):
        _same(_host(d[k]), want[k], name)


@pytest.mark.parametrize("forcing,include_wind,n", [(False, True, 0.025), (True, True, 0.03),
                                                    (True, False, 0.0)])
def test_friction(lib, forcing, include_wind, n):
    from oracle import oracle as orc
    nx, ny, ng = 50, 33, 2
    h, hu, hv, _ = _state(nx, ny, ng, 31)
    f4 = _forcing(h.shape, 9)
    dt, dx, dy = 0.02, 2.0, 3.0
    want = [a.copy(order="F") for a in (h, hu, hv)]
    orc.apply_friction(*want, ng, dt, n, *f4, forcing_active=forcing, include_wind=include_wind,
                       dx=dx, dy=dy)
    d = [_dev(a) for a in (h, hu, hv)]
    fd = [_dev(a) for a in f4]
    rc = lib.rkb_apply_friction(*(t.data_ptr() for t in d), h.shape[0], h.shape[1], ng,
                                h.shape[0], dx, dy, dt, n, *(t.data_ptr() for t in fd),
                                int(forcing), int(include_wind))
    assert rc == 0
    for k, name in enumerate(("h", "hu", "hv")):
        _same(_host(d[k]), want[k], name)


def test_coriolis(lib):
    from oracle import oracle as orc
    nx, ny, ng = 40, 40, 2
    h, hu, hv, _ = _state(nx, ny, ng, 41)
    want = [a.copy(order="F") for a in (h, hu, hv)]
    orc.apply_coriolis(*want, ng, 37.5, 1.0e-4)
    d = [_dev(a) for a in (h, hu, hv)]
    assert lib.rkb_apply_coriolis(*(t.data_ptr() for t in d), h.shape[0], h.shape[1], ng,
                                  h.shape[0], 37.5, 1.0e-4) == 0
    for k, name in enumerate(("h", "hu", "hv")):
        _same(_host(d[k]), want[k], name)


def _bc_params(edges, **kw):
    from rakali_b200._lib import BcParams
    p = BcParams()
    for k, e in enumerate(edges):
        p.type[k] = BC[e]
    tidal = kw.pop("tidal", ())
    p.n_tidal = len(tidal)
    for k, (a, ph, w) in enumerate(tidal):
        p.tidal_amp[k], p.tidal_phase[k], p.tidal_omega[k] = a, ph, w
    p.tidal_period = kw.pop("tidal_period", 44712.0)
    for key, val in kw.items():
        setattr(p, key, val)
    return p


BC_CASES = [
    (("wall", "wall", "wall", "wall"), {}),
    (("tidal", "open", "wall", "sponge"), dict(tidal_amplitude=0.7, time=1234.5)),
    (("tidal", "wall", "open", "tidal"), dict(tidal=((0.5, 0.3, 1.4e-4), (0.2, 1.1, 7.3e-5)),
                                             time=987.0)),
    (("inflow", "discharge", "clamped", "nested"), dict(inflow_velocity=0.8,
                                                        discharge_flux=1.7,
                                                        clamped_elevation=0.15)),
    (("chapman", "chapman", "chapman", "chapman"), dict(dt=0.07, time=3.0)),
]


@pytest.mark.parametrize("edges,kw", BC_CASES)
@pytest.mark.parametrize("shape", [(48, 31, 2), (40, 26, 3), (1, 9, 2), (5, 2, 3)])
def test_boundary_conditions(lib, edges, kw, shape):
    from oracle import oracle as orc
    nx, ny, ng = shape
    h, hu, hv, b = _state(nx, ny, ng, 51)
    rng = np.random.default_rng(5)
    nxt, nyt = h.shape
    eo = {"west": rng.normal(0.1, 0.05, nyt), "east": rng.normal(0.1, 0.05, nyt),
          "south": rng.normal(0.1, 0.05, nxt), "north": rng.normal(0.1, 0.05, nxt)}
    dx, dy = 1.3, 0.9
    want = [a.copy(order="F") for a in (h, hu, hv, b)]
    okw = dict(kw)
    tidal = okw.pop("tidal", ())
    keep = orc.apply_bc(*want, ng, *edges, dx=dx, dy=dy, tidal=tidal,
                        eta_old={k: v.copy() for k, v in eo.items()}, **okw)
    d = [_dev(a) for a in (h, hu, hv, b)]
    import torch
    eod = [torch.from_numpy(eo[e].copy()).cuda() for e in ("west", "east", "south", "north")]
    p = _bc_params(edges, tidal=tidal, **okw)
    for k in range(4):
        p.eta_old[k] = eod[k].data_ptr()
    rc = lib.rkb_apply_boundary_conditions(*(t.data_ptr() for t in d), nxt, nyt, ng, nxt, dx, dy,
                                           ctypes.byref(p))
    assert rc == 0
    for k, name in enumerate(("h", "hu", "hv", "b")):
        _same(_host(d[k]), want[k], name)
    for k, e in enumerate(("west", "east", "south", "north")):
        if edges[k] == "chapman":
            _same(eod[k].cpu().numpy(), keep[e], "eta_old " + e)


def test_boundary_conditions_refuse_missing_chapman_surface(lib):
    h = np.zeros((12, 10), order="F")
    d = [_dev(h) for _ in range(4)]
    p = _bc_params(("chapman", "wall", "wall", "wall"))
    assert lib.rkb_apply_boundary_conditions(*(t.data_ptr() for t in d), 12, 10, 2, 12, 1.0, 1.0,
                                             ctypes.byref(p)) == -2


@pytest.mark.parametrize("edges", [("sponge", "wall", "sponge", "wall"),
                                   ("sponge", "sponge", "sponge", "sponge"),
                                   ("wall", "sponge", "open", "sponge")])
def test_sponge(lib, edges):
    from oracle import oracle as orc
    nx, ny, ng = 44, 30, 2
    h, hu, hv, _ = _state(nx, ny, ng, 61)
    want = [a.copy(order="F") for a in (h, hu, hv)]
    orc.apply_sponge(*want, ng, 0.4, *edges, sponge_width=7, sponge_strength=0.05,
                     sponge_h_ref=0.3)
    d = [_dev(a) for a in (h, hu, hv)]
    p = _bc_params(edges, sponge_width=7, sponge_strength=0.05, sponge_h_ref=0.3)
    assert lib.rkb_apply_sponge(*(t.data_ptr() for t in d), h.shape[0], h.shape[1], ng,
                                h.shape[0], 0.4, ctypes.byref(p)) == 0
    for k, name in enumerate(("h", "hu", "hv")):
        _same(_host(d[k]), want[k], name)


def test_pieces_reproduce_the_fused_step(lib):
    """compute_flux -> fused_update_stage1 -> boundary fill -> compute_flux ->
    fused_update_stage2, all through the kernel-level entry points, equals one
    SSP-RK2 step of the oracle's solver with the same dt (walls, HLLC,
    friction) - the reference's fused branch (rki_solver.F90:692-815)."""
    from oracle.oracle import OracleSim
    nx, ny, ng = 36, 28, 2
    h, hu, hv, b = _state(nx, ny, ng, 71)
    cfg = dict(nx=nx, ny=ny, dx=1.0, dy=1.0, nghost=ng, t_end=100.0, cfl=0.4, manning_n=0.02,
               use_hllc=True)
    orc = OracleSim.from_config(cfg, bathymetry=b[ng:-ng, ng:-ng].copy(order="F"),
                                initial_h=h[ng:-ng, ng:-ng].copy(order="F"))
    for name, a in (("hu", hu), ("hv", hv)):
        orc.arrays[name][...] = a
    orc.apply_bc()
    state = [orc.arrays[k].copy(order="F") for k in ("h", "hu", "hv", "b")]
    orc.solver_step(0.01, 0.0)  # CFL dt, capped at 0.01 s
    dt = orc.dt
    d = [_dev(a) for a in state]
    z = [_dev(np.zeros_like(h)) for _ in range(8)]  # 3 fluxes, 2 mass fluxes, h0 hu0 hv0
    nxt, nyt = h.shape
    G = (nxt, nyt, ng, nxt)
    p = _bc_params(("wall",) * 4, time=0.0, dt=dt)
    none = [None] * 4

    def flux():
        assert lib.rkb_compute_flux(1, *(t.data_ptr() for t in d), *(t.data_ptr() for t in z[:5]),
                                    *G, 1.0, 1.0) == 0

    flux()
    assert lib.rkb_fused_update_stage1(*(t.data_ptr() for t in d[:3]),
                                       *(t.data_ptr() for t in z[5:8]),
                                       *(t.data_ptr() for t in z[:3]), *G, 1.0, 1.0, dt, 0.02,
                                       *none, 0.0, 0) == 0
    assert lib.rkb_apply_boundary_conditions(*(t.data_ptr() for t in d), *G, 1.0, 1.0,
                                             ctypes.byref(p)) == 0
    flux()
    assert lib.rkb_fused_update_stage2(*(t.data_ptr() for t in d[:3]),
                                       *(t.data_ptr() for t in z[5:8]),
                                       *(t.data_ptr() for t in z[:3]), *G, 1.0, 1.0, dt, 0.02,
                                       *none, 0.0, 0) == 0
    s = (slice(ng, -ng), slice(ng, -ng))
    for k, name in enumerate(("h", "hu", "hv")):
        _same(_host(d[k])[s], orc.arrays[name][s], name)
