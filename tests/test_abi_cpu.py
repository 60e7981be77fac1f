"""C-ABI surface and host-side logic, no GPU needed.

* librakali.so loads and exports every function include/rakali.h declares;
* it exports every symbol the reference's Python wrapper binds at import
  (python/rakali/_core.py:88-283), declared in include/rakali.h with the
  argument and result types of the reference's ctypes signatures (recorded
  in tests/golden/frontend_bindings.json) - and, when RAKALI_REFERENCE_PYTHON
  names the reference's python/ directory, its unmodified loader binds our
  library;
* namelist parsing/validation behaves like the reference's strict schema
  (src/core/rki_config.F90), returning error codes instead of stopping;
* keyword validation raises ValueError like the reference front end
  (python/tests/test_robustness.py:49-72).
"""
import ctypes
import json
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent

# The signatures the reference's own loader binds (python/rakali/_core.py:
# 88-283), recorded by tests/golden/make_frontend_bindings.py.
BINDINGS = json.loads((ROOT / "tests" / "golden" / "frontend_bindings.json").read_text())
REFERENCE_BINDS = sorted(BINDINGS["functions"])

# C spelling of the ctypes types the reference binds with.
_C_OF = {"c_int": "int", "c_double": "double", "c_void_p": "void*", "c_char_p": "char*",
         "POINTER(c_int)": "int*", "POINTER(c_double)": "double*",
         "POINTER(c_void_p)": "void**", "None": "void"}


def _header_prototypes():
    """name -> (result, [argument types]) of every function include/rakali.h
    declares, with const, names and spacing removed."""
    text = (ROOT / "include" / "rakali.h").read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][\w \t\*]*?)\b(r[a-z]+_\w+)\s*\(([^;{]*?)\)\s*;", text):
        def norm(decl, drop_name):
            decl = decl.replace("const", " ").strip()
            stars = decl.count("*")
            words = decl.replace("*", " ").split()
            if drop_name and len(words) > 1:
                words = words[:-1]
            return " ".join(words) + "*" * stars
        args = [a for a in m.group(3).split(",") if a.strip() and a.strip() != "void"]
        protos[m.group(2)] = (norm(m.group(1), False), [norm(a, True) for a in args])
    return protos


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
    assert len(REFERENCE_BINDS) >= 50
    assert not missing, missing
    assert lib.rki_working_precision() == 8
    assert BINDINGS["working_precision_dtype"] == "float64"


def test_header_prototypes_match_reference_bindings():
    """Every function the reference front end binds is declared in
    include/rakali.h with the same number, order and kind of arguments and
    the same result type as the reference's ctypes signature."""
    protos = _header_prototypes()
    bad = []
    for name, sig in BINDINGS["functions"].items():
        if name not in protos:
            bad.append((name, "not declared"))
            continue
        res, args = protos[name]
        want = [_C_OF[t] for t in sig["argtypes"]]
        if args != want or res != _C_OF[sig["restype"]]:
            bad.append((name, res, args, _C_OF[sig["restype"]], want))
    assert not bad, bad


_REF_PY = os.environ.get("RAKALI_REFERENCE_PYTHON")


@pytest.mark.skipif(not (_REF_PY and Path(_REF_PY, "rakali", "_core.py").is_file()),
                    reason="RAKALI_REFERENCE_PYTHON does not name the reference's python/ directory")
def test_unmodified_reference_loader_binds_library():
    code = (f"import sys; sys.path.insert(0, {_REF_PY!r});"
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
    # simulation and batch handles are looked up in registries, never dereferenced
    assert lib.rkb_tma_tile_status(h) == -100
    assert lib.rkb_tma_tile_status(bogus) == -100
    assert lib.rkb_batch_set_variant(h, 10, 0) == -100
    assert lib.rkb_batch_set_variant(bogus, 10, 0) == -100
    assert lib.rkb_adjoint_set_state_budget(h, 0) == -2


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


def test_kernel_entry_points_reject_bad_arguments_before_any_launch(lib):
    """Argument checks of the kernel-level entry points run on the host and
    return -2 before any CUDA call (so they need no GPU): null arrays, a ghost
    width below 2, a leading dimension below nx_total, a bad boundary type,
    a Chapman edge without its surface array."""
    from rakali_b200._lib import BcParams
    fake = ctypes.c_void_p(0x1000)  # never dereferenced: the checks fail first
    n4 = [None] * 4
    assert lib.rkb_compute_update(None, fake, fake, fake, fake, fake, 10, 10, 2, 10, 0.1) == -2
    assert lib.rkb_compute_update(fake, fake, fake, fake, fake, fake, 10, 10, 1, 10, 0.1) == -2
    assert lib.rkb_compute_rk2_average(fake, fake, fake, fake, fake, None, 10, 10, 2, 10) == -2
    assert lib.rkb_compute_ssp_combine(fake, fake, fake, fake, fake, fake, 0.5, 10, 10, 2, 9) == -2
    assert lib.rkb_fused_update_stage1(*([fake] * 9), 10, 10, 2, 10, 1.0, 1.0, 0.1, 0.02,
                                       *n4, 0.0, 1) == -2  # forcing without its arrays
    assert lib.rkb_fused_update_stage2(*([fake] * 5), None, *([fake] * 3), 10, 10, 2, 10, 1.0,
                                       1.0, 0.1, 0.02, *n4, 0.0, 0) == -2
    assert lib.rkb_fused_update_stage_generic(*([fake] * 6), 10, 10, 2, 10, 0.0, 1.0, 0.1, 0.0,
                                              *n4, 0.0, 0) == -2  # dx = 0
    assert lib.rkb_apply_friction(fake, fake, fake, 10, 10, 2, 10, 1.0, 1.0, 0.1, 0.02,
                                  None, None, fake, fake, 1, 1) == -2
    # nothing to do: the reference's early exits return before any launch
    assert lib.rkb_apply_friction(fake, fake, fake, 10, 10, 2, 10, 1.0, 1.0, 0.1, 0.0,
                                  *n4, 0, 1) == 0
    assert lib.rkb_apply_coriolis(fake, fake, fake, 10, 10, 2, 10, 0.1, 0.0) == 0
    p = BcParams()
    for k in range(4):
        p.type[k] = 1
    p.type[2] = 12
    assert lib.rkb_apply_boundary_conditions(fake, fake, fake, fake, 10, 10, 2, 10, 1.0, 1.0,
                                             ctypes.byref(p)) == -2
    p.type[2] = 9  # chapman, no surface array
    assert lib.rkb_apply_boundary_conditions(fake, fake, fake, fake, 10, 10, 2, 10, 1.0, 1.0,
                                             ctypes.byref(p)) == -2
    p.type[2] = 1
    assert lib.rkb_apply_boundary_conditions(fake, fake, fake, fake, 10, 10, 2, 10, 1.0, 1.0,
                                             None) == -2
    assert lib.rkb_apply_sponge(fake, fake, fake, 10, 10, 2, 10, 0.1, ctypes.byref(p)) == 0
