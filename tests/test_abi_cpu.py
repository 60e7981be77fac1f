"""C-ABI surface and host-side logic, no GPU needed.

* librakali.so loads and exports every function include/rakali.h declares;
* it exports every symbol the reference's Python wrapper binds at import
  (python/rakali/_core.py:88-283) - and, when the reference package is
  present in this environment, its unmodified loader binds our library;
* namelist parsing/validation behaves like the reference's strict schema
  (src/core/rki_config.F90), returning error codes instead of stopping;
* keyword validation raises ValueError like the reference front end
  (python/tests/test_robustness.py:49-72).
"""
import ctypes
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent

# python/rakali/_core.py:88-283
REFERENCE_BINDS = """rki_working_precision rki_create rki_finalize rki_create_from_namelist
rki_create_from_string rki_create_from_namelist_string rki_destroy rki_step rki_advance
rki_get_time rki_get_dt rki_get_step_count rki_get_nz_ml rki_get_grid_info rki_get_h_ptr
rki_get_hu_ptr rki_get_hv_ptr rki_get_b_ptr rki_get_h0_ptr rki_get_hu0_ptr rki_get_hv0_ptr
rki_get_clamped_elevation rki_get_manning_n rki_get_coriolis_f rki_get_h_layer_ptr
rki_get_hu_layer_ptr rki_get_hv_layer_ptr rki_get_salinity_ptr rki_get_temperature_ptr
rki_set_bathymetry rki_set_initial_h rki_set_wind rki_set_atm_pressure rki_set_precipitation
rki_set_heat_flux rki_set_evap_minus_precip rki_set_h rki_set_hu rki_set_hv rki_set_salinity
rki_set_temperature rki_sync_host rki_sync_from_device rki_save_restart rki_load_restart
rki_set_inflow_velocity rki_set_inflow_salinity rki_set_inflow_temperature
rki_set_discharge_flux rki_set_clamped_elevation rki_set_use_ppm_tracer rki_set_use_hllc
rki_set_tidal_constituents""".split()


@pytest.fixture(scope="module")
def lib():
    from rakali_b200 import _lib
    return _lib.load()


def test_header_symbols_exported(lib):
    from rakali_b200 import _lib
    names = _lib.header_symbols()
    assert len(names) >= 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_reference_wrapper_symbols_exported(lib):
    missing = [n for n in REFERENCE_BINDS if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.rki_working_precision() == 8


@pytest.mark.skipif(not Path("/root/reference/python/rakali/_core.py").is_file(),
                    reason="reference package not present here")
def test_unmodified_reference_loader_binds_library():
    code = ("import sys; sys.path.insert(0, '/root/reference/python');"
            "from rakali import _core; L = _core._load_lib();"
            "print(L._rki_wp_dtype.__name__)")
    env = dict(os.environ, RAKALI_LIB=str(ROOT / "rakali_b200" / "librakali.so"))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip() == "float64"


def test_bad_handles_rejected(lib):
    h = ctypes.c_void_p(0)
    assert lib.rki_step(h, 1) == -100
    assert lib.rki_finalize(h) == -100
    bogus = ctypes.c_void_p(0x1234)
    assert lib.rki_advance(bogus, 1.0) == -100
    assert lib.rki_get_time(bogus) == 0.0
    lib.rki_destroy(ctypes.byref(h))  # null: idempotent no-op
    ptr = ctypes.c_void_p()
    nx, ny = ctypes.c_int(7), ctypes.c_int(7)
    assert lib.rki_get_h_ptr(bogus, ctypes.byref(ptr), ctypes.byref(nx), ctypes.byref(ny)) == -100
    assert ptr.value is None and nx.value == 0 and ny.value == 0


def _validate(text):
    from rakali_b200 import validate_namelist
    return validate_namelist(text)


def test_namelist_schema_and_validation():
    from rakali_b200 import kwargs_to_namelist
    ok = kwargs_to_namelist(dict(nx=200, ny=100, dx=10.0, dy=10.0, t_end=60.0, cfl=0.5,
                                 use_hllc=True, bc_west="tidal", tidal_amp=[0.5, 0.1]))
    assert _validate(ok) == (0, "")
    assert _validate("&grid_nml\n nx = 0\n/\n")[0] == -2
    assert _validate("&grid_nml\n bogus = 1\n/\n")[0] == -2
    assert _validate("&nosuch_nml\n/\n")[0] == -2
    assert _validate("&time_nml\n cfl = 1.5\n/\n")[0] == -2
    assert _validate("&grid_nml nghost = 1 /")[0] == -2  # 5-point stencil needs 2
    assert _validate("&boundary_nml bc_west = 'weird' /")[0] == -2
    assert _validate("&nonhydrostatic_nml use_multilayer = .true. /")[0] == -3
    assert _validate("&grid_nml grid_type = 'unstructured' /")[0] == -3
    assert _validate("&time_nml time_scheme = 'semi_implicit' /")[0] == -3
    # Fortran syntax: comments, d-exponents, repeat counts, element indices,
    # several assignments per record, &end terminators
    txt = ("! comment\n&grid_nml nx=16, ny=8, dx=1.0d0 ! trailing\n dy = 2.5E-1 /\n"
           "&boundary_nml tidal_amp(2) = 0.5, tidal_omega = 3*1.0d-4,\n"
           " bc_west = \"tidal\" &end\n&physics_nml use_hllc = T /\n")
    assert _validate(txt) == (0, "")
    # keys accepted by the reference schema but not used by the 2D step parse
    assert _validate("&vcoord_nml vcoord_type = 'sigma' /\n&si_nml precond = 'none' /")[0] == 0


@pytest.mark.parametrize("bad", [
    dict(bc_west="foo"), dict(nx=0), dict(t_end=-1.0), dict(dx=float("nan")), dict(dx=None),
    dict(time_scheme="semi_implicit"), dict(time_scheme="rk4"), dict(vcoord_type="nope"),
    dict(remap_method="nope"), dict(vcoord_hc=5.0), dict(output_to_file=True),
    dict(forcing_file="f.nc"),
])
def test_bad_kwargs_raise(bad):
    from rakali_b200 import kwargs_to_namelist
    with pytest.raises(ValueError):
        kwargs_to_namelist({**dict(nx=8, ny=8, dx=1.0, dy=1.0, t_end=5.0), **bad})


def test_numpy_scalars_render():
    from rakali_b200 import kwargs_to_namelist
    txt = kwargs_to_namelist(dict(nx=np.int64(8), ny=np.int32(8), dx=np.float64(1.0),
                                  dy=np.float64(1.0), t_end=np.float64(5.0),
                                  use_multilayer=np.bool_(False)))
    assert _validate(txt) == (0, "")


def test_missing_namelist_raises(tmp_path):
    from rakali_b200 import Rakali
    with pytest.raises(FileNotFoundError):
        Rakali(str(tmp_path / "nope.nml"))
    with pytest.raises(FileNotFoundError, match="bathymetry_file"):
        Rakali(nx=8, ny=8, dx=1.0, dy=1.0, t_end=1.0, bathymetry_file=str(tmp_path / "x.nc"))
