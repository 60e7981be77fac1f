"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests, ``__graft_entry__.smoke()`` and the cpu_baseline leg of
``bench.py`` import this module; the product library never does.

``OracleSim`` holds a structured 2D barotropic simulation in numpy arrays
(Fortran order, ghosts included) and drives the C restatement in
``swe_oracle.c``.  ``OracleSim.from_config`` mirrors the reference's
one-shot create path (src/api/rki_api.F90:219-259, ``rki_finalize``):
bathymetry ghost fill, initial condition, boundary setup, Chapman seeding.
Defaults follow src/core/rki_config.F90:36-300.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

BC_CODES = {"wall": 1, "open": 2, "tidal": 3, "nested": 4, "inflow": 5,
            "discharge": 6, "clamped": 7, "sponge": 8, "chapman": 9}
SCHEME_CODES = {"euler": 1, "rk2": 2, "rk3": 3, "rk43": 4}
MAX_TIDAL = 10

# Reference config defaults (src/core/rki_config.F90:36-300) for the keys
# the structured 2D step reads.
DEFAULTS = dict(
    nx=200, ny=1, dx=1.0, dy=1.0, nghost=3,
    t_end=1.0, cfl=0.45, dt_max=1.0e10, dt_fixed=0.0, cfl_interval=1,
    time_scheme="rk2", time_unit="s",
    manning_n=0.0, coriolis_f=0.0, use_hllc=False,
    wind_stress_x=0.0, wind_stress_y=0.0,
    bc_west="wall", bc_east="wall", bc_south="wall", bc_north="wall",
    tidal_amplitude=0.0, tidal_period=44712.0, n_tidal_constituents=0,
    tidal_amp=(), tidal_phase=(), tidal_omega=(),
    inflow_velocity=0.0, discharge_flux=0.0, clamped_elevation=0.0,
    sponge_width=0, sponge_strength=0.0, sponge_h_ref=0.0,
    init_condition="dam_break", eta_initial=0.0, h0=1.0,
    hump_amplitude=0.05, hump_sigma=5.0, hump_x_offset=0.0, hump_y_offset=0.0,
)

TIME_UNITS = {"s": 1.0, "sec": 1.0, "second": 1.0, "seconds": 1.0,
              "min": 60.0, "minute": 60.0, "minutes": 60.0,
              "hr": 3600.0, "hour": 3600.0, "hours": 3600.0, "h": 3600.0,
              "day": 86400.0, "days": 86400.0, "d": 86400.0,
              "year": 365.25 * 86400.0, "years": 365.25 * 86400.0,
              "yr": 365.25 * 86400.0}

_DP = ctypes.POINTER(ctypes.c_double)


class _Bc(ctypes.Structure):
    _fields_ = [
        ("west", ctypes.c_int), ("east", ctypes.c_int),
        ("south", ctypes.c_int), ("north", ctypes.c_int),
        ("n_tidal", ctypes.c_int), ("sponge_width", ctypes.c_int),
        ("tidal_amplitude", ctypes.c_double), ("tidal_period", ctypes.c_double),
        ("time", ctypes.c_double),
        ("tidal_amp", ctypes.c_double * MAX_TIDAL),
        ("tidal_phase", ctypes.c_double * MAX_TIDAL),
        ("tidal_omega", ctypes.c_double * MAX_TIDAL),
        ("inflow_velocity", ctypes.c_double), ("discharge_flux", ctypes.c_double),
        ("clamped_elevation", ctypes.c_double),
        ("sponge_strength", ctypes.c_double), ("sponge_h_ref", ctypes.c_double),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dt", ctypes.c_double),
        ("eta_old_west", _DP), ("eta_old_east", _DP),
        ("eta_old_south", _DP), ("eta_old_north", _DP),
    ]


_FIELDS = ("h", "hu", "hv", "b", "flux_h", "flux_hu", "flux_hv", "mflux_x",
           "mflux_y", "h0", "hu0", "hv0", "wind_x", "wind_y", "atm", "precip")


class _Sim(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("ng", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("cfl", ctypes.c_double), ("dt", ctypes.c_double), ("dt_fixed", ctypes.c_double),
        ("cfl_interval", ctypes.c_int), ("step_count", ctypes.c_int),
        ("use_hllc", ctypes.c_int), ("time_scheme", ctypes.c_int),
        ("manning_n", ctypes.c_double), ("coriolis_f", ctypes.c_double),
        ("forcing_active", ctypes.c_int),
        ("t_current", ctypes.c_double), ("t_end", ctypes.c_double),
        ("mass_out", ctypes.c_double), ("mass_src", ctypes.c_double),
    ] + [(f, _DP) for f in _FIELDS] + [("bc", _Bc)]


_lib = None


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    """Load (building first if needed) the oracle shared library."""
    global _lib
    if _lib is None:
        if not LIB_PATH.is_file():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER(_Sim)
        L.orc_solver_step.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.orc_step_n.argtypes = [P, ctypes.c_int]
        L.orc_advance.argtypes = [P, ctypes.c_double]
        L.orc_total_mass.argtypes = [P]
        L.orc_total_mass.restype = ctypes.c_double
        for name in ("orc_init_dam_break", "orc_init_castro_dam_break",
                     "orc_bc_init_chapman"):
            getattr(L, name).argtypes = [P]
        L.orc_init_gaussian_hump.argtypes = [P] + [ctypes.c_double] * 5
        L.orc_init_still_water.argtypes = [P, ctypes.c_double]
        L.orc_fill_bathymetry_ghosts.argtypes = [_DP, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_compute_timestep.argtypes = [_DP, _DP, _DP, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_double, _DP]
        L.orc_compute_timestep.restype = ctypes.c_double
        L.orc_compute_flux.argtypes = [ctypes.c_int] + [_DP] * 9 + [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        stage_args = [_DP] * 9 + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double] + \
            [_DP] * 4 + [ctypes.c_double, ctypes.c_int]
        L.orc_fused_stage1.argtypes = stage_args
        L.orc_fused_stage2.argtypes = stage_args
        L.orc_fused_stage_generic.argtypes = stage_args[:3] + stage_args[6:]
        I3 = [ctypes.c_int] * 3
        L.orc_compute_update.argtypes = [_DP] * 6 + I3 + [ctypes.c_double]
        L.orc_rk2_average.argtypes = [_DP] * 6 + I3
        L.orc_ssp_combine.argtypes = [_DP] * 6 + [ctypes.c_double] + I3
        L.orc_apply_friction.argtypes = [_DP] * 3 + I3 + [ctypes.c_double] * 4 + [_DP] * 4 + \
            [ctypes.c_int, ctypes.c_int]
        L.orc_apply_coriolis.argtypes = [_DP] * 3 + I3 + [ctypes.c_double] * 2
        L.orc_apply_sponge.argtypes = [_DP] * 3 + I3 + [ctypes.c_double, ctypes.POINTER(_Bc)]
        L.orc_apply_bc.argtypes = [_DP] * 4 + [ctypes.c_int] * 3 + [ctypes.POINTER(_Bc)]
        L.orc_tidal_eta.argtypes = [ctypes.POINTER(_Bc)]
        L.orc_tidal_eta.restype = ctypes.c_double
        L.orc_cr_pow_third.argtypes = [ctypes.c_double]
        L.orc_cr_pow_third.restype = ctypes.c_double
        L.orc_cr_sincos.argtypes = [ctypes.c_double, _DP, _DP]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_set_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def ptr(a):
    """ctypes double* of a contiguous float64 numpy array (or NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous)
    return a.ctypes.data_as(_DP)


def resolve_config(cfg: dict) -> dict:
    """Defaults + user keys, with t_end scaled by time_unit (rki_config.F90:780-810)."""
    out = dict(DEFAULTS)
    for k, v in cfg.items():
        if isinstance(v, np.generic):
            v = v.item()
        out[k] = v
    out["t_end"] = float(out["t_end"]) * TIME_UNITS[str(out["time_unit"])]
    return out


class OracleSim:
    """One oracle simulation; arrays are (nx_total, ny_total) Fortran order."""

    def __init__(self, nx, ny, ng, dx, dy):
        self.nx_phys, self.ny_phys, self.ng = int(nx), int(ny), int(ng)
        self.nxt, self.nyt = self.nx_phys + 2 * self.ng, self.ny_phys + 2 * self.ng
        shape = (self.nxt, self.nyt)
        self.arrays = {f: np.zeros(shape, order="F") for f in _FIELDS}
        self.eta_old = {e: np.zeros(self.nyt if e in ("west", "east") else self.nxt)
                        for e in ("west", "east", "south", "north")}
        s = _Sim()
        s.nx, s.ny, s.ng = self.nxt, self.nyt, self.ng
        s.dx, s.dy = float(dx), float(dy)
        s.cfl, s.dt, s.dt_fixed = 0.45, 0.0, 0.0
        s.cfl_interval, s.step_count = 1, 0
        s.time_scheme = 2
        for f in _FIELDS:
            setattr(s, f, ptr(self.arrays[f]))
        s.bc.west = s.bc.east = s.bc.south = s.bc.north = 1
        s.bc.tidal_period = 44712.0
        s.bc.dx, s.bc.dy = float(dx), float(dy)
        for e, a in self.eta_old.items():
            setattr(s.bc, "eta_old_" + e, ptr(a))
        self.s = s

    def __getattr__(self, name):
        arrays = self.__dict__.get("arrays")
        if arrays is not None and name in arrays:
            return arrays[name]
        raise AttributeError(name)

    # --- setup (rki_finalize order) ------------------------------------
    @classmethod
    def from_config(cls, cfg: dict, bathymetry=None, initial_h=None):
        """Create + finalize like the reference C ABI, from resolved kwargs.

        ``bathymetry`` / ``initial_h`` are optional (nx, ny) interior arrays
        (rki_set_bathymetry / rki_set_initial_h, rki_api.F90:836-890).
        """
        c = resolve_config(cfg)
        o = cls(c["nx"], c["ny"], c["nghost"], c["dx"], c["dy"])
        s = o.s
        s.cfl = float(c["cfl"])
        s.dt_fixed = float(c["dt_fixed"])
        s.cfl_interval = int(c["cfl_interval"])
        s.use_hllc = int(bool(c["use_hllc"]))
        s.time_scheme = SCHEME_CODES[str(c["time_scheme"])]
        s.manning_n = float(c["manning_n"])
        s.coriolis_f = float(c["coriolis_f"])
        s.t_end = float(c["t_end"])
        o.arrays["wind_x"][:] = float(c["wind_stress_x"])
        o.arrays["wind_y"][:] = float(c["wind_stress_y"])
        ng = o.ng
        inner = (slice(ng, ng + o.nx_phys), slice(ng, ng + o.ny_phys))
        if bathymetry is not None:
            o.b[inner] = np.asarray(bathymetry, dtype=np.float64)
        L = lib()
        L.orc_fill_bathymetry_ghosts(ptr(o.b), o.nxt, o.nyt, ng)
        if initial_h is not None:
            o.h[inner] = np.asarray(initial_h, dtype=np.float64)
        else:
            ic = str(c["init_condition"])
            if ic == "still_water":
                L.orc_init_still_water(ctypes.byref(s), float(c["eta_initial"]))
            elif ic == "gaussian_hump":
                L.orc_init_gaussian_hump(ctypes.byref(s), float(c["h0"]),
                                         float(c["hump_amplitude"]), float(c["hump_sigma"]),
                                         float(c["hump_x_offset"]), float(c["hump_y_offset"]))
            elif ic == "castro_dam_break":
                L.orc_init_castro_dam_break(ctypes.byref(s))
            else:
                L.orc_init_dam_break(ctypes.byref(s))
        bc = s.bc
        bc.west, bc.east = BC_CODES[c["bc_west"]], BC_CODES[c["bc_east"]]
        bc.south, bc.north = BC_CODES[c["bc_south"]], BC_CODES[c["bc_north"]]
        bc.tidal_amplitude = float(c["tidal_amplitude"])
        bc.tidal_period = float(c["tidal_period"])
        bc.n_tidal = int(c["n_tidal_constituents"])
        for k, (a, p, w) in enumerate(zip(c["tidal_amp"], c["tidal_phase"], c["tidal_omega"])):
            bc.tidal_amp[k], bc.tidal_phase[k], bc.tidal_omega[k] = a, p, w
        bc.inflow_velocity = float(c["inflow_velocity"])
        bc.discharge_flux = float(c["discharge_flux"])
        bc.clamped_elevation = float(c["clamped_elevation"])
        bc.sponge_width = int(c["sponge_width"])
        bc.sponge_strength = float(c["sponge_strength"])
        bc.sponge_h_ref = float(c["sponge_h_ref"])
        L.orc_bc_init_chapman(ctypes.byref(s))
        return o

    def set_tidal_constituents(self, amp, phase, omega):
        bc = self.s.bc
        for k in range(MAX_TIDAL):
            bc.tidal_amp[k] = bc.tidal_phase[k] = bc.tidal_omega[k] = 0.0
        for k, (a, p, w) in enumerate(zip(amp, phase, omega)):
            bc.tidal_amp[k], bc.tidal_phase[k], bc.tidal_omega[k] = a, p, w
        bc.n_tidal = len(amp)

    # --- stepping -------------------------------------------------------
    def step(self, n=1):
        lib().orc_step_n(ctypes.byref(self.s), int(n))

    def advance(self, target):
        lib().orc_advance(ctypes.byref(self.s), float(target))

    def solver_step(self, dt_max, time):
        lib().orc_solver_step(ctypes.byref(self.s), float(dt_max), float(time))

    def apply_bc(self):
        lib().orc_apply_bc(ptr(self.h), ptr(self.hu), ptr(self.hv), ptr(self.b),
                           self.nxt, self.nyt, self.ng, ctypes.byref(self.s.bc))

    @property
    def time(self):
        return self.s.t_current

    @property
    def dt(self):
        return self.s.dt

    @property
    def step_count(self):
        return self.s.step_count

    def total_mass(self):
        return lib().orc_total_mass(ctypes.byref(self.s))

    def interior(self, name):
        ng = self.ng
        return self.arrays[name][ng:ng + self.nx_phys, ng:ng + self.ny_phys]


# --- kernel-level helpers used by the known-answer tests -----------------

def compute_flux(h, hu, hv, b, ng, dx=1.0, dy=1.0, hllc=False):
    """Flux divergence of every interior cell (rki_kernel_flux.F90:17-102)."""
    h, hu, hv, b = (np.asfortranarray(a, dtype=np.float64) for a in (h, hu, hv, b))
    nx, ny = h.shape
    out = [np.zeros((nx, ny), order="F") for _ in range(5)]
    lib().orc_compute_flux(int(hllc), ptr(h), ptr(hu), ptr(hv), ptr(b), *(ptr(a) for a in out),
                           nx, ny, int(ng), float(dx), float(dy))
    return out


def fused_stage(stage, h, hu, hv, h0, hu0, hv0, fh, fhu, fhv, ng, dt, manning_n=0.0,
                wind_x=None, wind_y=None, atm=None, precip=None, coriolis_f=0.0,
                forcing_active=False, dx=1.0, dy=1.0):
    """Run fused_update_stage1/2 in place on Fortran-order float64 arrays."""
    nx, ny = h.shape
    z = np.zeros((nx, ny), order="F")
    wx = z if wind_x is None else wind_x
    wy = z if wind_y is None else wind_y
    ap = z if atm is None else atm
    pr = z if precip is None else precip
    fn = lib().orc_fused_stage1 if stage == 1 else lib().orc_fused_stage2
    fn(ptr(h), ptr(hu), ptr(hv), ptr(h0), ptr(hu0), ptr(hv0), ptr(fh), ptr(fhu), ptr(fhv),
       nx, ny, int(ng), float(dx), float(dy), float(dt), float(manning_n), ptr(wx), ptr(wy),
       ptr(ap), ptr(pr), float(coriolis_f), int(bool(forcing_active)))


def fused_stage_generic(h, hu, hv, fh, fhu, fhv, ng, dt, manning_n=0.0, wind_x=None,
                        wind_y=None, atm=None, precip=None, coriolis_f=0.0,
                        forcing_active=False, dx=1.0, dy=1.0):
    """fused_update_stage_generic (rki_kernel_fused.F90:22-162) in place."""
    nx, ny = h.shape
    z = np.zeros((nx, ny), order="F")
    f = [z if a is None else a for a in (wind_x, wind_y, atm, precip)]
    lib().orc_fused_stage_generic(ptr(h), ptr(hu), ptr(hv), ptr(fh), ptr(fhu), ptr(fhv), nx, ny,
                                  int(ng), float(dx), float(dy), float(dt), float(manning_n),
                                  *(ptr(a) for a in f), float(coriolis_f),
                                  int(bool(forcing_active)))


def compute_update(h, hu, hv, fh, fhu, fhv, ng, dt):
    """compute_update (rki_kernel_update.F90:35-96) in place."""
    nx, ny = h.shape
    lib().orc_compute_update(*(ptr(a) for a in (h, hu, hv, fh, fhu, fhv)), nx, ny, int(ng),
                             float(dt))


def rk2_average(h, hu, hv, h0, hu0, hv0, ng):
    """compute_rk2_average (rki_kernel_update.F90:98-150) in place."""
    nx, ny = h.shape
    lib().orc_rk2_average(*(ptr(a) for a in (h, hu, hv, h0, hu0, hv0)), nx, ny, int(ng))


def ssp_combine(h, hu, hv, h0, hu0, hv0, a_n, ng):
    """compute_ssp_combine (rki_kernel_update.F90:152-208) in place."""
    nx, ny = h.shape
    lib().orc_ssp_combine(*(ptr(a) for a in (h, hu, hv, h0, hu0, hv0)), float(a_n), nx, ny,
                          int(ng))


def apply_friction(h, hu, hv, ng, dt, manning_n, wind_x=None, wind_y=None, atm=None,
                   precip=None, forcing_active=False, include_wind=True, dx=1.0, dy=1.0):
    """apply_friction (rki_kernel_friction.F90:16-113) in place."""
    nx, ny = h.shape
    z = np.zeros((nx, ny), order="F")
    f = [z if a is None else a for a in (wind_x, wind_y, atm, precip)]
    lib().orc_apply_friction(ptr(h), ptr(hu), ptr(hv), nx, ny, int(ng), float(dx), float(dy),
                             float(dt), float(manning_n), *(ptr(a) for a in f),
                             int(bool(forcing_active)), int(bool(include_wind)))


def apply_coriolis(h, hu, hv, ng, dt, f):
    """apply_coriolis (rki_kernel_friction.F90:115-152) in place."""
    nx, ny = h.shape
    lib().orc_apply_coriolis(ptr(h), ptr(hu), ptr(hv), nx, ny, int(ng), float(dt), float(f))


def apply_sponge(h, hu, hv, ng, dt, west="wall", east="wall", south="wall", north="wall",
                 sponge_width=0, sponge_strength=0.0, sponge_h_ref=0.0):
    """apply_sponge (rki_kernel_sponge.F90:16-88) in place."""
    nx, ny = h.shape
    bc = _Bc()
    bc.west, bc.east = BC_CODES[west], BC_CODES[east]
    bc.south, bc.north = BC_CODES[south], BC_CODES[north]
    bc.sponge_width, bc.sponge_strength, bc.sponge_h_ref = sponge_width, sponge_strength, \
        sponge_h_ref
    lib().orc_apply_sponge(ptr(h), ptr(hu), ptr(hv), nx, ny, int(ng), float(dt),
                           ctypes.byref(bc))


def compute_timestep(h, hu, hv, ng, dx, dy, cfl):
    """(dt, max_speed) from rki_kernel_timestep.F90:16-74."""
    nx, ny = h.shape
    ms = ctypes.c_double(0.0)
    dt = lib().orc_compute_timestep(ptr(h), ptr(hu), ptr(hv), nx, ny, int(ng), float(dx),
                                    float(dy), float(cfl), ctypes.byref(ms))
    return dt, ms.value


def set_threads(n):
    return lib().orc_set_threads(int(n))


if os.environ.get("RAKALI_ORACLE_REBUILD"):
    build()


def apply_bc(h, hu, hv, b, ng, west="wall", east="wall", south="wall", north="wall",
             time=0.0, dt=0.0, dx=1.0, dy=1.0, tidal_amplitude=0.0, tidal_period=44712.0,
             tidal=(), inflow_velocity=0.0, discharge_flux=0.0, clamped_elevation=0.0,
             eta_old=None):
    """apply_boundary_conditions (rki_boundary.F90:40-218) on raw arrays, in place.

    ``tidal`` is a sequence of (amp, phase, omega) constituents; ``eta_old``
    maps edge names to Chapman surfaces (defaults to zeros).
    """
    nx, ny = h.shape
    bc = _Bc()
    bc.west, bc.east = BC_CODES[west], BC_CODES[east]
    bc.south, bc.north = BC_CODES[south], BC_CODES[north]
    bc.time, bc.dt, bc.dx, bc.dy = time, dt, dx, dy
    bc.tidal_amplitude, bc.tidal_period = tidal_amplitude, tidal_period
    bc.n_tidal = len(tidal)
    for k, (a, p, w) in enumerate(tidal):
        bc.tidal_amp[k], bc.tidal_phase[k], bc.tidal_omega[k] = a, p, w
    bc.inflow_velocity, bc.discharge_flux = inflow_velocity, discharge_flux
    bc.clamped_elevation = clamped_elevation
    eo = dict(eta_old or {})
    keep = {}
    for e, n in (("west", ny), ("east", ny), ("south", nx), ("north", nx)):
        arr = np.ascontiguousarray(eo.get(e, np.zeros(n)), dtype=np.float64)
        keep[e] = arr
        setattr(bc, "eta_old_" + e, ptr(arr))
    lib().orc_apply_bc(ptr(h), ptr(hu), ptr(hv), ptr(b), nx, ny, int(ng), ctypes.byref(bc))
    return keep
