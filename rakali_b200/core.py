"""``Rakali``: the structured-grid front end over the B200 ``librakali.so``.

Same calls, argument meaning and error behaviour as the reference wrapper
(python/rakali/_core.py:449-1860): keyword or namelist creation, one-shot or
two-phase (``defer_init``) setup, ``step`` / ``advance`` (with callbacks),
zero-copy Fortran-order field views (``h``, ``h_phys`` ...) that keep the
simulation alive, state and forcing setters, and ``close`` / context-manager
teardown.  Bad input raises a Python exception; the library never stops the
process.

Additions: ``device_fields()`` returns zero-copy torch CUDA views of the
device-resident state, and ``mass_budget()`` the boundary/source volume
accounting of the solver.
"""
from __future__ import annotations

import ctypes
import math
import os
from pathlib import Path

import numpy as np

from . import _lib

TIME_EPS = 1.0e-10  # the stop tolerance of rki_advance (rki_api.F90:401)

# kwarg -> namelist group (python/rakali/_core.py:329-447).  The namelist key is
# the kwarg itself.
_GROUPS = {
    "grid_nml": ("nx", "ny", "dx", "dy", "nghost"),
    "time_nml": ("t_end", "cfl", "dt_max", "dt_fixed", "cfl_interval", "time_scheme"),
    "physics_nml": ("manning_n", "dry_threshold", "wind_stress_x", "wind_stress_y",
                    "coriolis_f", "use_hllc"),
    "output_nml": ("output_to_file", "output_dir", "output_interval", "output_format",
                   "restart_interval", "async_output", "async_buffer_slots", "bathymetry_file",
                   "restart_file", "forcing_file", "forcing_x_origin", "forcing_y_origin",
                   "gauge_file", "gauge_output_interval", "compress_output", "compress_level",
                   "out_h_layer", "out_velocity", "out_salinity", "out_temperature",
                   "out_density", "out_w"),
    "boundary_nml": ("bc_west", "bc_east", "bc_south", "bc_north", "tidal_amplitude",
                     "tidal_period", "n_tidal_constituents", "tidal_amp", "tidal_phase",
                     "tidal_omega", "inflow_velocity", "inflow_salinity", "inflow_temperature",
                     "discharge_flux", "clamped_elevation", "sponge_width", "sponge_strength",
                     "sponge_h_ref", "nesting_file", "nesting_x_origin", "nesting_y_origin"),
    "nonhydrostatic_nml": ("use_nonhydrostatic", "use_multilayer", "nz_layers", "nh_tolerance",
                           "nh_max_iterations", "nh_preconditioner", "nh_solve_interval",
                           "bpg_method", "ml_min_depth", "rho_0", "vmix_nu_max", "vmix_nu_bg",
                           "vmix_ri_alpha", "hdiff_kappa", "smagorinsky_cs", "split_ratio",
                           "split_averaging"),
    "tracer_nml": ("initial_salinity", "S_ref", "beta_S", "S_min", "S_max", "kappa_S_bg",
                   "initial_temperature", "T_ref", "alpha_T", "T_min", "T_max", "kappa_T_bg",
                   "use_ppm_tracer"),
    "initial_condition_nml": ("init_condition", "eta_initial", "h0", "hump_amplitude",
                              "hump_sigma", "hump_x_offset", "hump_y_offset", "init_u_shear"),
    "vcoord_nml": ("vcoord_type", "remap_method", "vcoord_depth_transition",
                   "vcoord_blend_width", "zstar_h_surf_target", "zstar_stretching",
                   "zstar_h_min", "zstar_n_surf"),
    "logging_nml": ("log_level", "status_interval"),
    "metadata_nml": ("reference_time", "institution"),
}
PARAM_GROUP = {k: g for g, keys in _GROUPS.items() for k in keys}

# Read only by the Fortran driver executable, never by the library API: a
# kwarg here would be silently ignored, so it is rejected.
UNSUPPORTED = frozenset(
    ("output_to_file", "output_dir", "output_interval", "output_format", "restart_interval",
     "async_output", "async_buffer_slots", "restart_file", "forcing_file", "forcing_x_origin",
     "forcing_y_origin", "gauge_file", "gauge_output_interval", "compress_output",
     "compress_level", "out_h_layer", "out_velocity", "out_salinity", "out_temperature",
     "out_density", "out_w", "nesting_file", "nesting_x_origin", "nesting_y_origin"))

_BC = ("wall", "open", "tidal", "nested", "inflow", "discharge", "clamped", "sponge", "chapman")
ENUMS = {"bc_west": _BC, "bc_east": _BC, "bc_south": _BC, "bc_north": _BC,
         "time_scheme": ("euler", "rk2", "rk3", "rk43"),
         "remap_method": ("pcm", "plm", "ppm", "ppm_h4", "pqm"),
         "vcoord_type": ("sigma", "zsigma", "zstar", "zstar_lite", "zstar_full",
                         "zstar_sigma")}
POSITIVE = ("nx", "ny", "dx", "dy", "t_end", "cfl", "nz_layers")
INPUT_FILE_KEYS = ("bathymetry_file",)


def _fortran_value(v):
    """One Python value as namelist text."""
    if isinstance(v, np.generic):
        v = v.item()
    if v is None:
        raise ValueError("None is not a valid namelist value")
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, str):
        return '"' + v.replace('"', '""') + '"'
    if isinstance(v, (list, tuple, np.ndarray)):
        return ", ".join(_fortran_value(x) for x in v)
    if isinstance(v, float):
        if not math.isfinite(v):
            raise ValueError(f"non-finite value {v!r} is not allowed")
        return repr(v)
    if isinstance(v, int):
        return str(v)
    raise ValueError(f"unsupported namelist value {v!r}")


def kwargs_to_namelist(kwargs: dict) -> str:
    """Validate keyword arguments and render them as namelist text."""
    by_group: dict[str, list[str]] = {}
    for key, value in kwargs.items():
        if key in UNSUPPORTED:
            raise ValueError(f"'{key}' is read by the Fortran driver executable, not the "
                             "library API, so it would be silently ignored here")
        if key not in PARAM_GROUP:
            raise ValueError(f"Unknown parameter '{key}'. Valid parameters: "
                             f"{sorted(PARAM_GROUP)}")
        if isinstance(value, np.generic):
            value = value.item()
        if key in ENUMS and (not isinstance(value, str) or value.lower() not in ENUMS[key]):
            raise ValueError(f"{key}={value!r} is not valid; choose one of {ENUMS[key]}")
        if key in POSITIVE and not (isinstance(value, (int, float))
                                    and not isinstance(value, bool) and value > 0):
            raise ValueError(f"{key} must be a positive number, got {value!r}")
        by_group.setdefault(PARAM_GROUP[key], []).append(f"  {key} = {_fortran_value(value)}")
    out = ["! namelist written by rakali_b200"]
    for group, lines in by_group.items():
        out.append(f"&{group}")
        out.extend(lines)
        out.append("/")
    return "\n".join(out) + "\n"


def _view(address: int, count: int, owner) -> np.ndarray:
    """numpy float64 view of library memory that keeps `owner` alive."""
    buf = (ctypes.c_double * count).from_address(address)
    buf._rakali_owner = owner  # noqa: SLF001 - the view's base chain holds the sim
    return np.frombuffer(buf, dtype=np.float64)


class _CudaArray:
    """__cuda_array_interface__ exporter for a pitched device field."""

    def __init__(self, ptr, shape, strides, owner):
        self._owner = owner
        self.__cuda_array_interface__ = {
            "shape": shape, "strides": strides, "typestr": "<f8",
            "data": (ptr, False), "version": 3}


class Rakali:
    """Structured 2D shallow-water simulation on one B200 (SSP-RK2, FP64).

    >>> sim = Rakali(nx=200, ny=100, dx=10.0, dy=10.0, t_end=60.0, use_hllc=True)
    >>> sim.advance(60.0)
    >>> sim.h_phys.max()
    """

    def __init__(self, namelist=None, defer_init=False, precision=64, **kwargs):
        self._lib = _lib.load()
        self._handle = ctypes.c_void_p()
        self._alive = False
        if precision not in (32, 64):
            raise ValueError(f"precision must be 32 or 64, got {precision!r}")
        if namelist is not None and kwargs:
            raise ValueError("Pass either a namelist file or keyword arguments, not both")
        if namelist is not None:
            path = Path(namelist)
            if not path.is_file():
                raise FileNotFoundError(f"Namelist file not found: {path}")
            self._check_input_files(self._namelist_inputs(path.read_text()), path.resolve().parent)
            raw = str(path.resolve()).encode()
            fn = self._lib.rki_create if defer_init else self._lib.rki_create_from_namelist
            rc = fn(raw, len(raw), ctypes.byref(self._handle))
        elif kwargs:
            self._check_input_files({k: v for k, v in kwargs.items() if k in INPUT_FILE_KEYS},
                                    Path.cwd())
            text = kwargs_to_namelist(kwargs).encode()
            fn = (self._lib.rki_create_from_string if defer_init
                  else self._lib.rki_create_from_namelist_string)
            rc = fn(text, len(text), ctypes.byref(self._handle))
        else:
            raise ValueError("Pass a namelist file or keyword arguments")
        if rc != 0:
            raise RuntimeError(f"Failed to create simulation (rc={rc}): "
                               f"{_lib.last_error(self._lib)}")
        self._finalised = not defer_init
        self._alive = True
        self._query_grid()
        if precision != 64:
            self.set_precision(precision)

    # --- construction helpers -------------------------------------------
    @staticmethod
    def _namelist_inputs(text: str) -> dict:
        import re
        out = {}
        for m in re.finditer(r'^\s*(bathymetry_file)\s*=\s*["\']([^"\']*)["\']', text,
                             re.IGNORECASE | re.MULTILINE):
            out[m.group(1).lower()] = m.group(2)
        return out

    @staticmethod
    def _check_input_files(entries: dict, base: Path):
        for key, value in entries.items():
            if not value:
                continue
            p = Path(str(value))
            if not p.is_absolute():
                p = Path(base) / p
            if not p.is_file():
                raise FileNotFoundError(f"{key} = {value!r} not found (looked for {p})")

    _kwargs_to_namelist = staticmethod(kwargs_to_namelist)

    def _query_grid(self):
        nx, ny, ng = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        dx, dy = ctypes.c_double(), ctypes.c_double()
        self._lib.rki_get_grid_info(self._handle, ctypes.byref(nx), ctypes.byref(ny),
                                    ctypes.byref(ng), ctypes.byref(dx), ctypes.byref(dy))
        self._nx, self._ny, self._ng = nx.value, ny.value, ng.value
        self._dx, self._dy = dx.value, dy.value

    # --- lifecycle --------------------------------------------------------
    def _destroy_handle(self):
        if getattr(self, "_alive", False):
            self._alive = False
            self._lib.rki_destroy(ctypes.byref(self._handle))

    def close(self):
        """Release the solver handle (idempotent)."""
        self._destroy_handle()

    destroy = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self._destroy_handle()
        return False

    def __del__(self):
        try:
            self._destroy_handle()
        except Exception:
            pass

    def _check_alive(self):
        if not self._alive:
            raise RuntimeError("Simulation has been destroyed")

    def _check_ready(self):
        self._check_alive()
        if not self._finalised:
            raise RuntimeError("Simulation not finalised. Call finalize() after "
                               "set_bathymetry() / set_initial_h().")

    def _rc(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what} failed (rc={rc}): {_lib.last_error(self._lib)}")

    def finalize(self):
        """Complete two-phase setup (bed ghosts, initial condition, BCs, upload)."""
        self._check_alive()
        if self._finalised:
            raise RuntimeError("Simulation already finalised")
        self._rc(self._lib.rki_finalize(self._handle), "Finalize")
        self._finalised = True

    def prepare(self):
        """Alias of :meth:`finalize`."""
        self.finalize()

    # --- fields -----------------------------------------------------------
    def _field(self, name):
        self._check_alive()
        ptr = ctypes.c_void_p()
        nx, ny = ctypes.c_int(), ctypes.c_int()
        rc = getattr(self._lib, f"rki_get_{name}_ptr")(self._handle, ctypes.byref(ptr),
                                                       ctypes.byref(nx), ctypes.byref(ny))
        self._rc(rc, f"rki_get_{name}_ptr")
        arr = _view(ptr.value, nx.value * ny.value, self)
        return arr.reshape((nx.value, ny.value), order="F")

    def _phys(self, a):
        g = self._ng
        return a[g:-g, g:-g]

    h = property(lambda self: self._field("h"), doc="Water depth (with ghosts).")
    hu = property(lambda self: self._field("hu"), doc="x-momentum (with ghosts).")
    hv = property(lambda self: self._field("hv"), doc="y-momentum (with ghosts).")
    b = property(lambda self: self._field("b"), doc="Bed elevation, positive up (with ghosts).")
    h0 = property(lambda self: self._field("h0"), doc="RK2 save of h (start of the last step).")
    hu0 = property(lambda self: self._field("hu0"), doc="RK2 save of hu.")
    hv0 = property(lambda self: self._field("hv0"), doc="RK2 save of hv.")
    def _get_3d_field(self, getter_name):
        """(nx_total, ny_total, nz) view of a layer field; multilayer mode is
        not part of this library, so the getter reports -3 and this raises
        RuntimeError as the reference does when it is inactive
        (python/rakali/_core.py:713-728)."""
        self._check_alive()
        ptr = ctypes.c_void_p()
        nx, ny, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rc = getattr(self._lib, getter_name)(self._handle, ctypes.byref(ptr), ctypes.byref(nx),
                                             ctypes.byref(ny), ctypes.byref(nz))
        if rc != 0:
            raise RuntimeError(f"{getter_name} failed (rc={rc})")
        arr = _view(ptr.value, nx.value * ny.value * nz.value, self)
        return arr.reshape((nx.value, ny.value, nz.value), order="F")

    @property
    def h_layer(self):
        """Layer thickness (multilayer mode only: raises RuntimeError here)."""
        g = self._ng
        return self._get_3d_field("rki_get_h_layer_ptr")[g:-g, g:-g, :]

    def _tracer(self, getter_name):
        q = self._get_3d_field(getter_name)
        lay = self._get_3d_field("rki_get_h_layer_ptr")
        g = self._ng
        q, lay = q[g:-g, g:-g, :], lay[g:-g, g:-g, :]
        with np.errstate(invalid="ignore", divide="ignore"):
            return np.where(lay > 1e-6, q / lay, np.nan)

    @property
    def salinity(self):
        """Layer salinity (multilayer mode only: raises RuntimeError here)."""
        return self._tracer("rki_get_salinity_ptr")

    @property
    def temperature(self):
        """Layer temperature (multilayer mode only: raises RuntimeError here)."""
        return self._tracer("rki_get_temperature_ptr")

    h_phys = property(lambda self: self._phys(self.h), doc="Water depth, interior only.")
    hu_phys = property(lambda self: self._phys(self.hu), doc="x-momentum, interior only.")
    hv_phys = property(lambda self: self._phys(self.hv), doc="y-momentum, interior only.")
    b_phys = property(lambda self: self._phys(self.b), doc="Bed elevation, interior only.")

    @property
    def time(self):
        self._check_alive()
        return self._lib.rki_get_time(self._handle)

    @property
    def dt(self):
        self._check_alive()
        return self._lib.rki_get_dt(self._handle)

    @property
    def step_count(self):
        self._check_alive()
        return self._lib.rki_get_step_count(self._handle)

    @property
    def nz(self):
        self._check_alive()
        return self._lib.rki_get_nz_ml(self._handle)

    nx = property(lambda self: self._nx)
    ny = property(lambda self: self._ny)
    nghost = property(lambda self: self._ng)
    dx = property(lambda self: self._dx)
    dy = property(lambda self: self._dy)

    @property
    def manning_n(self):
        self._check_alive()
        return self._lib.rki_get_manning_n(self._handle)

    @property
    def coriolis_f(self):
        self._check_alive()
        return self._lib.rki_get_coriolis_f(self._handle)

    @property
    def clamped_elevation(self):
        self._check_alive()
        return self._lib.rki_get_clamped_elevation(self._handle)

    # --- stepping ---------------------------------------------------------
    def step(self, n=1):
        """Take n steps (each capped at t_end); raises once t_end is reached."""
        self._check_ready()
        t0 = self.time
        self._rc(self._lib.rki_step(self._handle, int(n)), "Solver step")
        if n > 0 and not self.time > t0:
            raise RuntimeError(f"step() made no progress at t={self.time:g} s: the run has "
                               "reached its t_end. Increase t_end when creating the simulation.")

    def advance(self, target_time, callback=None, callback_interval=None, progress=False):
        """Advance to ``target_time``; with a callback, in chunks with a host sync."""
        self._check_ready()
        target_time = float(target_time)
        bar = None
        if progress:
            try:
                from tqdm.auto import tqdm
                bar = tqdm(total=max(target_time - self.time, 0.0), unit="s",
                           desc=f"advance to t={target_time:.1f}s")
            except ImportError:
                import warnings
                warnings.warn("progress=True requires tqdm", RuntimeWarning, stacklevel=2)
        if callback is None and bar is None:
            self._rc(self._lib.rki_advance(self._handle, target_time), "Advance")
            return
        if callback_interval is None:
            frac = 10.0 if callback is not None else 100.0
            callback_interval = max((target_time - self.time) / frac, TIME_EPS)
        if callback_interval <= 0:
            raise ValueError("callback_interval must be positive")
        try:
            t_now = last = self.time
            while t_now < target_time - TIME_EPS:
                t_next = min(t_now + callback_interval, target_time)
                self._rc(self._lib.rki_advance(self._handle, t_next), "Advance")
                self._lib.rki_sync_host(self._handle)
                if callback is not None:
                    callback(self)
                t_now = self.time
                if bar is not None:
                    bar.update(t_now - last)
                    last = t_now
        finally:
            if bar is not None:
                bar.close()

    def sync_host(self):
        """Refresh the host copies of h, hu, hv (device state stays canonical)."""
        self._check_alive()
        self._lib.rki_sync_host(self._handle)

    def sync_from_device(self):
        """Copy every field home and make the host arrays canonical (the next
        step uploads them again)."""
        self._check_alive()
        self._lib.rki_sync_from_device(self._handle)

    def to_xarray(self, time_dim=True):
        """The current interior state as an ``xarray.Dataset`` (copies): h, b,
        eta, hu, hv and the velocities u, v (NaN where h <= 1e-6) on cell
        centres x, y, with a length-1 ``time`` dimension unless ``time_dim``
        is False; the variables, coordinates and attributes of the reference
        front end's to_xarray (python/rakali/_core.py:1561-1768) without the
        multilayer fields.  Raises ImportError when xarray is not installed.
        """
        try:
            import xarray as xr
        except ImportError as e:
            raise ImportError("to_xarray() requires the xarray package. "
                              "Install with `pip install xarray`.") from e
        self._check_ready()
        self.sync_host()
        nx, ny, dx, dy = self._nx, self._ny, self.dx, self.dy
        coords = {
            "x": ("x", (np.arange(nx) + 0.5) * dx,
                  {"units": "m", "long_name": "distance east of west boundary", "axis": "X"}),
            "y": ("y", (np.arange(ny) + 0.5) * dy,
                  {"units": "m", "long_name": "distance north of south boundary", "axis": "Y"}),
        }
        if time_dim:
            coords["time"] = ("time", np.array([self.time]),
                              {"units": "seconds since simulation start",
                               "long_name": "simulation time", "axis": "T"})
        h, hu, hv, b = (self.h_phys.copy(), self.hu_phys.copy(), self.hv_phys.copy(),
                        self.b_phys.copy())
        with np.errstate(invalid="ignore", divide="ignore"):
            u = np.where(h > 1e-6, hu / h, np.nan)
            v = np.where(h > 1e-6, hv / h, np.nan)

        def wrap(a):
            return (("time", "x", "y"), a[np.newaxis]) if time_dim else (("x", "y"), a)

        data_vars = {
            "h": (*wrap(h), {"units": "m", "long_name": "water depth"}),
            "b": (*wrap(b), {"units": "m", "long_name": "bottom elevation", "positive": "up"}),
            "eta": (*wrap(h + b), {"units": "m", "long_name": "surface elevation (h + b)"}),
            "hu": (*wrap(hu), {"units": "m2 s-1", "long_name": "x-momentum (h*u)"}),
            "hv": (*wrap(hv), {"units": "m2 s-1", "long_name": "y-momentum (h*v)"}),
            "u": (*wrap(u), {"units": "m s-1", "long_name": "x-velocity"}),
            "v": (*wrap(v), {"units": "m s-1", "long_name": "y-velocity"}),
        }
        attrs = {"title": "Rakali simulation snapshot", "source": "rakali_b200 (Rakali.to_xarray)",
                 "Conventions": "CF-1.11", "dx": float(dx), "dy": float(dy), "nx": int(nx),
                 "ny": int(ny), "time": float(self.time), "step_count": int(self.step_count)}
        return xr.Dataset(data_vars=data_vars, coords=coords, attrs=attrs)

    # --- setters ----------------------------------------------------------
    def _shape(self, a, label):
        a = np.asarray(a, dtype=np.float64)
        if a.shape != (self._nx, self._ny):
            raise ValueError(f"{label}: expected shape ({self._nx}, {self._ny}), got {a.shape}")
        return np.asfortranarray(a)

    def _set(self, fn, label, *arrays):
        self._check_alive()
        fs = [self._shape(a, label) for a in arrays]
        ptrs = [f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for f in fs]
        self._rc(getattr(self._lib, fn)(self._handle, *ptrs, self._nx, self._ny), label)

    def set_bathymetry(self, b):
        self._set("rki_set_bathymetry", "set_bathymetry", b)

    def set_initial_h(self, h):
        self._set("rki_set_initial_h", "set_initial_h", h)

    def set_h(self, h):
        self._set("rki_set_h", "set_h", h)

    def set_hu(self, hu):
        self._set("rki_set_hu", "set_hu", hu)

    def set_hv(self, hv):
        self._set("rki_set_hv", "set_hv", hv)

    def _set_tracer(self, fn, label, a):
        self._check_alive()
        nz = self.nz
        if nz <= 0:
            raise RuntimeError(f"{label} requires multilayer mode (nz_layers > 0)")
        a = np.asfortranarray(a, dtype=np.float64)
        if a.shape != (self._nx, self._ny, nz):
            raise ValueError(f"Expected shape {(self._nx, self._ny, nz)}, got {a.shape}")
        rc = getattr(self._lib, fn)(self._handle, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                    self._nx, self._ny, nz)
        if rc != 0:
            raise RuntimeError(f"Failed to {label[4:]} (rc={rc})")

    def set_salinity(self, S):
        """Per-layer salinity (multilayer mode only: raises RuntimeError here,
        as the reference does when nz_layers is 0)."""
        self._set_tracer("rki_set_salinity", "set_salinity", S)

    def set_temperature(self, T):
        """Per-layer temperature (multilayer mode only: raises RuntimeError here)."""
        self._set_tracer("rki_set_temperature", "set_temperature", T)

    def set_wind(self, wx, wy):
        self._set("rki_set_wind", "set_wind", wx, wy)

    def set_atm_pressure(self, p):
        self._set("rki_set_atm_pressure", "set_atm_pressure", p)

    def set_precipitation(self, p):
        self._set("rki_set_precipitation", "set_precipitation", p)

    def set_heat_flux(self, q):
        self._set("rki_set_heat_flux", "set_heat_flux", q)

    def set_evap_minus_precip(self, ep):
        self._set("rki_set_evap_minus_precip", "set_evap_minus_precip", ep)

    def _scalar(self, fn, label, value):
        self._check_alive()
        v = float(value)
        if not math.isfinite(v):
            raise ValueError(f"{label} must be finite, got {value!r}")
        self._rc(getattr(self._lib, fn)(self._handle, v), label)

    def set_inflow_velocity(self, v):
        self._scalar("rki_set_inflow_velocity", "inflow_velocity", v)

    def set_inflow_salinity(self, s):
        self._scalar("rki_set_inflow_salinity", "inflow_salinity", s)

    def set_inflow_temperature(self, t):
        self._scalar("rki_set_inflow_temperature", "inflow_temperature", t)

    def set_discharge_flux(self, q):
        self._scalar("rki_set_discharge_flux", "discharge_flux", q)

    def set_clamped_elevation(self, eta):
        self._scalar("rki_set_clamped_elevation", "clamped_elevation", eta)

    def set_use_hllc(self, enable=True):
        self._check_alive()
        self._rc(self._lib.rki_set_use_hllc(self._handle, int(bool(enable))), "set_use_hllc")

    def set_use_ppm_tracer(self, enable=True):
        self._check_alive()
        self._rc(self._lib.rki_set_use_ppm_tracer(self._handle, int(bool(enable))),
                 "set_use_ppm_tracer")

    def set_tidal_constituents(self, amp, phase, omega):
        self._check_alive()
        a, p, w = (np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
                   for x in (amp, phase, omega))
        if not (a.shape == p.shape == w.shape) or a.ndim != 1:
            raise ValueError("amp, phase and omega must be 1-D arrays of equal length")
        dp = ctypes.POINTER(ctypes.c_double)
        self._rc(self._lib.rki_set_tidal_constituents(
            self._handle, a.ctypes.data_as(dp), p.ctypes.data_as(dp), w.ctypes.data_as(dp),
            int(a.size)), "set_tidal_constituents")

    def save_restart(self, filename):
        """Write h, hu, hv, b and the time to a NetCDF (classic) restart file.

        The variables, dimensions and attributes are those of the reference's
        restart_write (src/io/structured/rki_output.F90:740-853); step count
        and configuration are not saved.
        """
        self._check_ready()
        parent = Path(str(filename)).resolve().parent
        if not parent.is_dir():
            raise FileNotFoundError(f"directory {parent} does not exist")
        raw = str(filename).encode()
        self._rc(self._lib.rki_save_restart(self._handle, raw, len(raw)), "save_restart")

    def save_checkpoint(self, filename):
        """Write a per-step checkpoint: h, hu, hv, b and the RK2 saves h0, hu0,
        hv0 with their ghost cells, plus time, step_count, dt, the grid sizes,
        dx, dy, manning_n, coriolis_f and clamped_elevation as attributes.

        The variables and attributes are those of the reference front end's
        save_checkpoint (python/rakali/_core.py:1433-1499); the file is NetCDF
        classic (64-bit offset) instead of NetCDF-4, readable by any NetCDF
        library.  The simulation keeps running on the device afterwards.
        """
        self._check_ready()
        parent = Path(str(filename)).resolve().parent
        if not parent.is_dir():
            raise FileNotFoundError(f"directory {parent} does not exist")
        raw = str(filename).encode()
        self._rc(self._lib.rkb_save_checkpoint(self._handle, raw, len(raw)), "save_checkpoint")

    # --- gauges (src/io/structured/rki_gauges.F90) --------------------------
    def set_gauges(self, x, y, names=None, interval=0.0, capacity=65536):
        """Record eta, u, v at stations (x, y in metres from the lower-left
        corner) on the device after every step: bilinear stencils as the
        reference's compute_interp_weights, cadence as its driver (every step
        for interval <= 0, else every `interval` seconds).  Stations outside the
        domain are dropped; returns the number kept.  Replaces earlier stations
        and discards their records."""
        self._check_ready()
        x = np.ascontiguousarray(np.atleast_1d(x), dtype=np.float64)
        y = np.ascontiguousarray(np.atleast_1d(y), dtype=np.float64)
        if x.shape != y.shape or x.ndim != 1:
            raise ValueError("x and y must be 1-D arrays of equal length")
        names = [f"gauge_{k + 1}" for k in range(x.size)] if names is None else list(names)
        if len(names) != x.size:
            raise ValueError("one name per station")
        dp = ctypes.POINTER(ctypes.c_double)
        n = self._lib.rkb_set_gauges(self._handle, int(x.size), x.ctypes.data_as(dp),
                                     y.ctypes.data_as(dp), float(interval), int(capacity))
        if n < 0:
            raise RuntimeError(f"set_gauges failed (rc={n}): {_lib.last_error(self._lib)}")
        idx = np.zeros(n, dtype=np.int32)
        bed = np.zeros(n)
        self._lib.rkb_gauge_stations(self._handle, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     bed.ctypes.data_as(dp))
        self._gauges = dict(names=[names[k] for k in idx], x=x[idx], y=y[idx], b=bed,
                            time=[], values=[], overflow=False)
        return int(n)

    def set_gauges_file(self, path, interval=0.0, capacity=65536):
        """Stations from a text file of ``name x y`` lines (``#`` comments and
        blank lines skipped, malformed lines skipped, at most 100 stations;
        read_gauge_file, rki_gauges.F90:129-206)."""
        names, xs, ys = [], [], []
        for line in Path(path).read_text().splitlines():
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            if len(names) == 100:
                break
            parts = line.replace(",", " ").split()
            try:
                x, y = float(parts[1]), float(parts[2])
            except (IndexError, ValueError):
                continue
            names.append(parts[0].strip("'\""))
            xs.append(x)
            ys.append(y)
        return self.set_gauges(xs, ys, names, interval, capacity)

    def gauge_records(self):
        """All records since set_gauges: dict(time (K,), eta, u, v (K, stations),
        names, x, y, b, overflow)."""
        self._check_alive()
        gs = getattr(self, "_gauges", None)
        if gs is None:
            raise RuntimeError("no gauges set")
        n = len(gs["names"])
        dp = ctypes.POINTER(ctypes.c_double)
        while n > 0:
            t = np.zeros(4096)
            v = np.zeros((4096, n, 3))
            ov = ctypes.c_int()
            k = self._lib.rkb_read_gauges(self._handle, 4096, t.ctypes.data_as(dp),
                                          v.ctypes.data_as(dp), ctypes.byref(ov))
            if k < 0:
                raise RuntimeError(f"read_gauges failed (rc={k})")
            gs["overflow"] |= bool(ov.value)
            if k == 0:
                break
            gs["time"].append(t[:k].copy())
            gs["values"].append(v[:k].copy())
        t = np.concatenate(gs["time"]) if gs["time"] else np.zeros(0)
        v = np.concatenate(gs["values"]) if gs["values"] else np.zeros((0, n, 3))
        return dict(time=t, eta=v[:, :, 0], u=v[:, :, 1], v=v[:, :, 2], names=list(gs["names"]),
                    x=gs["x"].copy(), y=gs["y"].copy(), b=gs["b"].copy(), overflow=gs["overflow"])

    def write_gauges(self, filename):
        """Write the records so far as the reference's gauges.nc layout (NetCDF classic)."""
        r = self.gauge_records()
        n = len(r["names"])
        width = 64
        raw = b"".join(nm.encode()[:width].ljust(width, b"\0") for nm in r["names"])
        vals = np.ascontiguousarray(np.stack([r["eta"], r["u"], r["v"]], axis=-1))
        dp = ctypes.POINTER(ctypes.c_double)
        t = np.ascontiguousarray(r["time"])
        rc = self._lib.rkb_write_gauges_netcdf(
            str(filename).encode(), n, raw, width, r["x"].ctypes.data_as(dp),
            r["y"].ctypes.data_as(dp), r["b"].ctypes.data_as(dp), int(t.size),
            t.ctypes.data_as(dp), vals.ctypes.data_as(dp))
        self._rc(rc, "write_gauges")

    @classmethod
    def from_restart(cls, restart_file, namelist=None, **kwargs):
        """Create a simulation whose state (h, hu, hv, b, time) comes from a
        restart file; the namelist or keyword arguments give the configuration,
        whose grid must match the file's (python/rakali/_core.py:1506-1556)."""
        path = Path(str(restart_file))
        if not path.is_file():
            raise FileNotFoundError(f"Restart file not found: {path}")
        raw = str(path.resolve()).encode()
        kwargs.pop("defer_init", None)
        sim = cls(namelist=namelist, defer_init=True, **kwargs)
        try:
            rc = sim._lib.rki_load_restart(sim._handle, raw, len(raw))
            if rc != 0:
                raise RuntimeError(f"rki_load_restart('{path}') failed (rc={rc}): "
                                   f"{_lib.last_error(sim._lib)}")
            sim.finalize()
        except Exception:
            sim.close()
            raise
        return sim

    # --- additions --------------------------------------------------------
    def mass_budget(self):
        """(mass_out, mass_src): boundary outflow and source volume since creation."""
        self._check_ready()
        out = (ctypes.c_double * 3)()
        self._rc(self._lib.rkb_get_mass_budget(self._handle, out), "mass_budget")
        return out[0], out[1]

    def device_fields(self):
        """Zero-copy torch CUDA views (h, hu, hv, b) of the device state, with ghosts.

        Valid until the next step (the state alternates between two buffers).
        """
        import torch
        self._check_ready()
        ptrs = (ctypes.c_void_p * 4)()
        pitch = ctypes.c_int()
        self._rc(self._lib.rkb_get_device_fields(self._handle, ptrs, ctypes.byref(pitch)),
                 "device_fields")
        shape = (self._nx + 2 * self._ng, self._ny + 2 * self._ng)
        strides = (8, 8 * pitch.value)
        return tuple(torch.as_tensor(_CudaArray(p, shape, strides, self), device="cuda")
                     for p in ptrs)

    def set_tile(self, tile: int):
        """Kernel shape of the FP64 stage (0: 32x8, 1: 32x16, 2: 64x4, 3: 16x16 tiles;
        4 / 5: marching strips of 64 / 32 rows; 6 / 7: 32x8 / 32x12 tiles with two extra
        warps; 8: 16x15 tiles; 9: 32x7 tiles with one extra warp; 10: 16x15 tiles
        loaded by TMA copies of their halo boxes)."""
        self._check_alive()
        self._rc(self._lib.rkb_set_tile(self._handle, int(tile)), "set_tile")

    @property
    def precision(self) -> int:
        """64: FP64 depth form (the reference's arithmetic); 32: FP32 surface form."""
        self._check_alive()
        return int(self._lib.rkb_get_precision(self._handle))

    def set_precision(self, bits: int):
        """Switch the step between the FP64 and the FP32 form (state carried over)."""
        self._check_alive()
        if bits not in (32, 64):
            raise ValueError(f"precision must be 32 or 64, got {bits!r}")
        self._rc(self._lib.rkb_set_precision(self._handle, int(bits)), "set_precision")

    def set_sweep(self, cols_per_lane: int = 0, rows: int = 0):
        """FP32 form: columns per lane (2 or 4; 0 = default) and rows per warp (0 = automatic)."""
        self._check_alive()
        self._rc(self._lib.rkb_set_sweep(self._handle, int(cols_per_lane), int(rows)), "set_sweep")


def validate_namelist(text: str):
    """(rc, message) of the library's namelist validation; needs no GPU."""
    lib = _lib.load()
    raw = text.encode()
    buf = ctypes.create_string_buffer(512)
    rc = lib.rkb_validate_namelist(raw, len(raw), buf, len(buf))
    return rc, buf.value.decode()


__all__ = ["Rakali", "kwargs_to_namelist", "validate_namelist"]

if os.environ.get("RAKALI_B200_EAGER_LOAD"):
    _lib.load()
