"""Locate and bind ``librakali.so`` (the B200 build of the structured step).

The search order follows the reference's loader: ``RAKALI_LIB`` first, then
the library built in-tree next to this package (``python -m
rakali_b200.build``).  Signatures are those of ``include/rakali.h``.
"""
from __future__ import annotations

import ctypes
import os
import re
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
HEADER = ROOT / "include" / "rakali.h"
DEFAULT_LIB = PKG / "librakali.so"

_lib = None


def find_library() -> str:
    env = os.environ.get("RAKALI_LIB")
    if env:
        if not os.path.isfile(env):
            raise FileNotFoundError(f"RAKALI_LIB is set to {env!r}, which is not a file")
        return env
    if DEFAULT_LIB.is_file():
        return str(DEFAULT_LIB)
    raise FileNotFoundError(
        f"{DEFAULT_LIB} is missing: build it with `python -m rakali_b200.build` "
        "(needs nvcc) or point RAKALI_LIB at a built librakali.so")


def header_symbols() -> list[str]:
    """Function names declared in include/rakali.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"\b(rk[ib]_\w+)\s*\(", text)


MAX_TIDAL = 10


class BcParams(ctypes.Structure):
    """rkb_bc_params of include/rakali.h (the reference's bc_params_t as the
    boundary and sponge kernels read it)."""
    _fields_ = [
        ("type", ctypes.c_int * 4), ("n_tidal", ctypes.c_int), ("sponge_width", ctypes.c_int),
        ("tidal_amplitude", ctypes.c_double), ("tidal_period", ctypes.c_double),
        ("tidal_amp", ctypes.c_double * MAX_TIDAL), ("tidal_phase", ctypes.c_double * MAX_TIDAL),
        ("tidal_omega", ctypes.c_double * MAX_TIDAL),
        ("inflow_velocity", ctypes.c_double), ("discharge_flux", ctypes.c_double),
        ("clamped_elevation", ctypes.c_double),
        ("sponge_strength", ctypes.c_double), ("sponge_h_ref", ctypes.c_double),
        ("time", ctypes.c_double), ("dt", ctypes.c_double),
        ("eta_old", ctypes.c_void_p * 4),
    ]


def _sig(lib, name, args, res):
    f = getattr(lib, name)
    f.argtypes = args
    f.restype = res


def load(path: str | None = None):
    """Load the library once and attach ctypes signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    lib = ctypes.CDLL(path or find_library())
    H = ctypes.c_void_p
    HP = ctypes.POINTER(ctypes.c_void_p)
    I = ctypes.c_int
    D = ctypes.c_double
    IP = ctypes.POINTER(ctypes.c_int)
    DP = ctypes.POINTER(ctypes.c_double)
    CP = ctypes.c_char_p
    _sig(lib, "rki_working_precision", [], I)
    for n in ("rki_create", "rki_create_from_namelist", "rki_create_from_string",
              "rki_create_from_namelist_string"):
        _sig(lib, n, [CP, I, HP], I)
    _sig(lib, "rki_finalize", [H], I)
    _sig(lib, "rki_destroy", [HP], None)
    _sig(lib, "rki_step", [H, I], I)
    _sig(lib, "rki_advance", [H, D], I)
    _sig(lib, "rki_get_time", [H], D)
    _sig(lib, "rki_get_dt", [H], D)
    _sig(lib, "rki_get_step_count", [H], I)
    _sig(lib, "rki_get_nz_ml", [H], I)
    _sig(lib, "rki_get_grid_info", [H, IP, IP, IP, DP, DP], None)
    for n in ("h", "hu", "hv", "b", "h0", "hu0", "hv0"):
        _sig(lib, f"rki_get_{n}_ptr", [H, HP, IP, IP], I)
    for n in ("h_layer", "hu_layer", "hv_layer", "salinity", "temperature"):
        _sig(lib, f"rki_get_{n}_ptr", [H, HP, IP, IP, IP], I)
    for n in ("bathymetry", "initial_h", "atm_pressure", "precipitation", "heat_flux",
              "evap_minus_precip", "h", "hu", "hv"):
        _sig(lib, f"rki_set_{n}", [H, DP, I, I], I)
    _sig(lib, "rki_set_wind", [H, DP, DP, I, I], I)
    _sig(lib, "rki_set_salinity", [H, DP, I, I, I], I)
    _sig(lib, "rki_set_temperature", [H, DP, I, I, I], I)
    for n in ("inflow_velocity", "inflow_salinity", "inflow_temperature", "discharge_flux",
              "clamped_elevation"):
        _sig(lib, f"rki_set_{n}", [H, D], I)
    for n in ("clamped_elevation", "manning_n", "coriolis_f"):
        _sig(lib, f"rki_get_{n}", [H], D)
    _sig(lib, "rki_set_tidal_constituents", [H, DP, DP, DP, I], I)
    _sig(lib, "rki_sync_host", [H], None)
    _sig(lib, "rki_sync_from_device", [H], None)
    _sig(lib, "rki_save_restart", [H, CP, I], I)
    _sig(lib, "rki_load_restart", [H, CP, I], I)
    _sig(lib, "rkb_save_checkpoint", [H, CP, I], I)
    _sig(lib, "rki_set_use_ppm_tracer", [H, I], I)
    _sig(lib, "rki_set_use_hllc", [H, I], I)
    _sig(lib, "rki_last_error", [], CP)
    _sig(lib, "rkb_validate_namelist", [CP, I, CP, I], I)
    _sig(lib, "rkb_get_mass_budget", [H, DP], I)
    _sig(lib, "rkb_get_device_fields", [H, HP, IP], I)
    _sig(lib, "rkb_set_tile", [H, I], I)
    _sig(lib, "rkb_get_tile", [H], I)
    _sig(lib, "rkb_tma_tile_status", [H], I)
    _sig(lib, "rkb_set_precision", [H, I], I)
    _sig(lib, "rkb_get_precision", [H], I)
    _sig(lib, "rkb_set_sweep", [H, I, I], I)
    _sig(lib, "rkb_set_wait_limit", [H, ctypes.c_longlong], I)
    _sig(lib, "rkb_batch_create", [HP, I, I, HP], I)
    _sig(lib, "rkb_batch_destroy", [HP], None)
    _sig(lib, "rkb_batch_step", [H, I], I)
    _sig(lib, "rkb_batch_advance", [H, D], I)
    _sig(lib, "rkb_batch_time_steps", [H, I, DP], I)
    _sig(lib, "rkb_batch_autotune", [H, I, DP], I)
    _sig(lib, "rkb_batch_profile_steps", [H, I, DP], I)
    _sig(lib, "rkb_batch_set_variant", [H, I, I], I)
    _sig(lib, "rkb_batch_variant", [H, IP, IP], I)
    _sig(lib, "rkb_adjoint_create", [I, I, I, D, D, D, I, I, DP, DP, DP, IP, IP, I, HP], I)
    _sig(lib, "rkb_adjoint_destroy", [HP], None)
    _sig(lib, "rkb_adjoint_set_obs", [H, DP], I)
    _sig(lib, "rkb_adjoint_set_dt", [H, DP], I)
    _sig(lib, "rkb_adjoint_get_dt", [H, DP], I)
    _sig(lib, "rkb_adjoint_forward", [H, DP, DP, D, I, DP, DP], I)
    _sig(lib, "rkb_adjoint_gradient", [H, DP, DP, D, DP, DP, DP], I)
    _sig(lib, "rkb_adjoint_checkpoint_interval", [H], I)
    _sig(lib, "rkb_adjoint_set_state_budget", [H, ctypes.c_longlong], I)
    _sig(lib, "rkb_adjoint_last_ms", [H], D)
    _sig(lib, "rkb_adjoint_batch_create",
         [I, I, I, I, I, D, D, D, I, I, DP, DP, DP, IP, IP, I, HP], I)
    _sig(lib, "rkb_adjoint_members", [H], I)
    _sig(lib, "rkb_adjoint_precision", [H], I)
    _sig(lib, "rkb_adjoint_mass", [H, DP], I)
    _sig(lib, "rkb_adjoint_set_frozen_slopes", [H, I], I)
    _sig(lib, "rkb_test_face_flux", [I, I, DP, DP], None)
    _sig(lib, "rkb_test_face_adj", [I, I, DP, DP, DP], None)
    _sig(lib, "rkb_test_cell", [DP, D, DP], None)
    _sig(lib, "rkb_test_cell_adj", [DP, D, DP, DP], None)
    _sig(lib, "rkb_restart_write", [CP, I, I, DP, DP, DP, DP, D, D, D, I], I)
    _sig(lib, "rkb_restart_read", [CP, I, I, DP, DP, DP, DP, DP], I)
    _sig(lib, "rkb_checkpoint_write", [CP, I, I, ctypes.POINTER(DP), DP, IP], I)
    _sig(lib, "rkb_gauge_stencils", [I, I, I, D, D, DP, DP, I, IP, IP, IP, DP, DP], I)
    _sig(lib, "rkb_bathymetry_read", [CP, I, I, DP], I)
    _sig(lib, "rkb_set_gauges", [H, I, DP, DP, D, I], I)
    _sig(lib, "rkb_gauge_stations", [H, IP, DP], I)
    _sig(lib, "rkb_read_gauges", [H, I, DP, DP, IP], I)
    _sig(lib, "rkb_write_gauges_netcdf", [CP, I, CP, I, DP, DP, DP, I, DP, DP], I)
    _sig(lib, "rkb_time_steps", [H, I, DP], I)
    _sig(lib, "rkb_profile_steps", [H, I, DP], I)
    _sig(lib, "rkb_cr_pow_third", [D], D)
    _sig(lib, "rkb_cr_sincos", [D, DP, DP], None)
    _sig(lib, "rkb_compute_flux", [I, H, H, H, H, H, H, H, H, H, I, I, I, I, D, D], I)
    _sig(lib, "rkb_compute_timestep", [H, H, H, I, I, I, I, D, D, D, DP], I)
    _sig(lib, "rkb_compute_timestep_noalloc", [H, H, H, I, I, I, I, D, D, D, DP], I)
    # kernel-level structured kernels (device pointers as c_void_p)
    G4 = [I, I, I, I]  # nx_total, ny_total, nghost, ld
    stage_tail = [D, D, D, D, H, H, H, H, D, I]  # dx dy dt n  wx wy atm pr  f forcing
    _sig(lib, "rkb_fused_update_stage1", [H] * 9 + G4 + stage_tail, I)
    _sig(lib, "rkb_fused_update_stage2", [H] * 9 + G4 + stage_tail, I)
    _sig(lib, "rkb_fused_update_stage_generic", [H] * 6 + G4 + stage_tail, I)
    _sig(lib, "rkb_compute_update", [H] * 6 + G4 + [D], I)
    _sig(lib, "rkb_compute_rk2_average", [H] * 6 + G4, I)
    _sig(lib, "rkb_compute_ssp_combine", [H] * 6 + [D] + G4, I)
    _sig(lib, "rkb_apply_friction", [H] * 3 + G4 + [D] * 4 + [H] * 4 + [I, I], I)
    _sig(lib, "rkb_apply_coriolis", [H] * 3 + G4 + [D, D], I)
    BP = ctypes.POINTER(BcParams)
    _sig(lib, "rkb_apply_boundary_conditions", [H] * 4 + G4 + [D, D, BP], I)
    _sig(lib, "rkb_apply_sponge", [H] * 3 + G4 + [D, BP], I)
    if lib.rki_working_precision() != 8:
        raise RuntimeError("librakali.so must be the FP64 build")
    lib.wp_dtype = np.float64
    lib.wp_ctype = ctypes.c_double
    if path is None:
        _lib = lib
    return lib


def last_error(lib) -> str:
    msg = lib.rki_last_error()
    return msg.decode() if msg else ""
