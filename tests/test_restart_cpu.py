"""Restart files (NetCDF classic, 64-bit offset) without a GPU.

rki_save_restart / rki_load_restart write and read the variables of the
reference's restart_write / restart_read (src/io/structured/rki_output.F90:
740-988).  The codec is checked against scipy's independent NetCDF classic
implementation in both directions: files this library writes are read by
scipy with the expected dimensions, variables, units and values, and files
scipy writes are read back by this library; grid mismatches and HDF5
(NetCDF-4) containers are refused.
"""
import ctypes

import numpy as np
import pytest

DP = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def lib():
    from rakali_b200 import _lib
    return _lib.load()


def _fields(nx, ny, seed):
    rng = np.random.default_rng(seed)
    return [np.asfortranarray(rng.standard_normal((nx, ny))) for _ in range(4)]


def _p(a):
    return a.ctypes.data_as(DP)


def test_written_file_reads_in_scipy(lib, tmp_path):
    from scipy.io import netcdf_file
    nx, ny = 7, 5
    h, hu, hv, b = _fields(nx, ny, 1)
    path = tmp_path / "r.nc"
    assert lib.rkb_restart_write(str(path).encode(), nx, ny, _p(h), _p(hu), _p(hv), _p(b), 123.25,
                                 10.0, 5.0, 2) == 0
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions == {"x": nx, "y": ny}
        for name, arr, units in (("h", h, b"m"), ("hu", hu, b"m2 s-1"), ("hv", hv, b"m2 s-1"),
                                 ("b", b, b"m")):
            v = f.variables[name]
            assert v.dimensions == ("y", "x")
            assert v.units == units
            assert np.array_equal(np.asarray(v[:]).T, arr)  # file (y, x) = Fortran (x, y)
        assert float(f.variables["time"].getValue()) == 123.25
        assert f.variables["time"].units == b"seconds since simulation start"
        assert f.Conventions == b"CF-1.11" and f.nghost == b"2"
        assert float(f.dx) == 10.0 and float(f.dy) == 5.0


@pytest.mark.parametrize("version", [1, 2])
def test_scipy_written_file_reads_back(lib, tmp_path, version):
    from scipy.io import netcdf_file
    nx, ny = 6, 9
    h, hu, hv, b = _fields(nx, ny, 2)
    path = tmp_path / "s.nc"
    with netcdf_file(str(path), "w", version=version) as f:
        f.createDimension("x", nx)
        f.createDimension("y", ny)
        f.title = b"written elsewhere"
        for name, arr in (("h", h), ("hu", hu), ("hv", hv), ("b", b)):
            v = f.createVariable(name, "d", ("y", "x"))
            v.units = b"m"
            v[:] = arr.T
        t = f.createVariable("time", "d", ())
        t.data[()] = 3600.5
    out = [np.zeros((nx, ny), order="F") for _ in range(4)]
    tm = ctypes.c_double()
    assert lib.rkb_restart_read(str(path).encode(), nx, ny, *map(_p, out), ctypes.byref(tm)) == 0
    for a, r in zip(out, (h, hu, hv, b)):
        assert np.array_equal(a, r)
    assert tm.value == 3600.5


def test_round_trip_and_refusals(lib, tmp_path):
    from rakali_b200 import _lib
    nx, ny = 5, 4
    h, hu, hv, b = _fields(nx, ny, 3)
    path = tmp_path / "r.nc"
    assert lib.rkb_restart_write(str(path).encode(), nx, ny, _p(h), _p(hu), _p(hv), _p(b), -1.5,
                                 1.0, 1.0, 3) == 0
    out = [np.zeros((nx, ny), order="F") for _ in range(4)]
    tm = ctypes.c_double()
    assert lib.rkb_restart_read(str(path).encode(), nx, ny, *map(_p, out), ctypes.byref(tm)) == 0
    assert all(np.array_equal(a, r) for a, r in zip(out, (h, hu, hv, b))) and tm.value == -1.5
    # grid mismatch
    bad = [np.zeros((nx + 1, ny), order="F") for _ in range(4)]
    assert lib.rkb_restart_read(str(path).encode(), nx + 1, ny, *map(_p, bad),
                                ctypes.byref(tm)) == 1
    assert "mismatch" in _lib.last_error(lib)
    # an HDF5 container (NetCDF-4) and a missing file
    hdf = tmp_path / "n4.nc"
    hdf.write_bytes(b"\x89HDF\r\n\x1a\n" + bytes(64))
    assert lib.rkb_restart_read(str(hdf).encode(), nx, ny, *map(_p, out), ctypes.byref(tm)) == -1
    assert "HDF5" in _lib.last_error(lib)
    assert lib.rkb_restart_read(str(tmp_path / "none.nc").encode(), nx, ny, *map(_p, out),
                                ctypes.byref(tm)) == -1


def _scipy_bed(path, nx, ny, arr, name="b", order="yx", version=2):
    from scipy.io import netcdf_file
    with netcdf_file(str(path), "w", version=version) as f:
        f.createDimension("x", nx)
        f.createDimension("y", ny)
        if order == "yx":  # row-major (y, x): x fastest, the Fortran (x, y) array
            v = f.createVariable(name, "d", ("y", "x"))
            v[:] = arr.T
        else:  # a C-order b[x][y]
            v = f.createVariable(name, "f", ("x", "y"))
            v[:] = arr.astype(np.float32)


@pytest.mark.parametrize("name,order", [("b", "yx"), ("elevation", "xy"), ("depth", "yx")])
def test_bathymetry_file_reads_like_the_reference(lib, tmp_path, name, order):
    """load_bathymetry_into_array (src/io/rki_bathymetry.F90:21-163): b, elevation or
    depth over x, y in either order (a C-order (x, y) variable is read transposed)."""
    nx, ny = 7, 5
    arr = np.asfortranarray(np.random.default_rng(4).standard_normal((nx, ny)))
    path = tmp_path / "bed.nc"
    _scipy_bed(path, nx, ny, arr, name, order)
    out = np.zeros((nx, ny), order="F")
    assert lib.rkb_bathymetry_read(str(path).encode(), nx, ny, _p(out)) == 0
    ref = arr if order == "yx" else arr.astype(np.float32).astype(np.float64)
    assert np.array_equal(out, ref)
    assert lib.rkb_bathymetry_read(str(path).encode(), nx, ny + 1,
                                   _p(np.zeros((nx, ny + 1), order="F"))) == 1


def test_bathymetry_file_without_known_variable(lib, tmp_path):
    from rakali_b200 import _lib
    nx, ny = 4, 3
    path = tmp_path / "bed.nc"
    _scipy_bed(path, nx, ny, np.zeros((nx, ny)), name="topo")
    out = np.zeros((nx, ny), order="F")
    assert lib.rkb_bathymetry_read(str(path).encode(), nx, ny, _p(out)) == -1
    assert "b, elevation, depth" in _lib.last_error(lib)


def test_gauge_file_layout_reads_in_scipy(lib, tmp_path):
    """rkb_write_gauges_netcdf writes create_gauge_netcdf's variables
    (src/io/structured/rki_gauges.F90:338-488)."""
    from scipy.io import netcdf_file
    n, K = 3, 5
    rng = np.random.default_rng(8)
    x, y, b = rng.uniform(0, 100, n), rng.uniform(0, 50, n), rng.uniform(-5, 0, n)
    t = np.arange(K, dtype=np.float64) * 2.5
    vals = np.ascontiguousarray(rng.standard_normal((K, n, 3)))
    names = [b"harbour", b"pier", b"x" * 70]
    raw = b"".join(nm[:64].ljust(64, b"\0") for nm in names)
    path = tmp_path / "gauges.nc"
    assert lib.rkb_write_gauges_netcdf(str(path).encode(), n, raw, 64, _p(x), _p(y), _p(b), K,
                                       _p(t), _p(vals)) == 0
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert f.dimensions == {"station": n, "time": K, "name_strlen": 64}
        assert np.array_equal(f.variables["time"][:], t)
        assert f.variables["time"].units == b"seconds"
        for k, nm in enumerate(names):
            got = bytes(f.variables["station_name"][k]).rstrip(b"\0")
            assert got == nm[:64]
        for name, arr in (("station_x", x), ("station_y", y), ("station_b", b)):
            assert np.array_equal(f.variables[name][:], arr)
        for c, name in enumerate(("eta", "u", "v")):
            assert f.variables[name].dimensions == ("time", "station")
            assert np.array_equal(f.variables[name][:], vals[:, :, c])
        assert f.title == b"Rakali gauge time series"


def test_checkpoint_file_layout_reads_in_scipy(lib, tmp_path):
    """rkb_checkpoint_write (the codec of save_checkpoint) writes the variables
    and attributes of the reference front end's save_checkpoint
    (python/rakali/_core.py:1433-1499): fields with ghosts over (x_total,
    y_total) and the scalars as typed global attributes."""
    from scipy.io import netcdf_file
    nxt, nyt = 13, 9
    rng = np.random.default_rng(12)
    arrs = [np.asfortranarray(rng.standard_normal((nxt, nyt))) for _ in range(7)]
    fields = (DP * 7)(*[_p(a) for a in arrs])
    scal = np.array([123.5, 0.25, 5.0, 7.5, 0.025, 1.0e-4, -0.3])
    cnt = np.array([42, nxt - 4, nyt - 4, 2], dtype=np.int32)
    path = tmp_path / "step_42.nc"
    assert lib.rkb_checkpoint_write(str(path).encode(), nxt, nyt, fields, _p(scal),
                                    cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == 0
    names = ("h", "hu", "hv", "b", "h0", "hu0", "hv0")
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert f.dimensions == {"x_total": nxt, "y_total": nyt}
        for name, a in zip(names, arrs):
            v = f.variables[name]
            assert v.dimensions == ("x_total", "y_total")
            assert np.array_equal(v[:], a), name
        assert f.variables["b"].positive == b"up"
        assert f.variables["hu"].units == b"m2 s-1"
        at = f._attributes
        assert at["title"] == b"Rakali per-step checkpoint (2D barotropic)"
        for key, val in zip(("time", "dt", "dx", "dy", "manning_n", "coriolis_f",
                             "clamped_elevation"), scal):
            assert np.asarray(at[key]).dtype == np.float64 and float(at[key]) == val, key
        for key, val in zip(("step_count", "nx_phys", "ny_phys", "nghost"), cnt):
            assert np.asarray(at[key]).dtype.kind == "i" and int(at[key]) == val, key
        assert (int(at["nx_total"]), int(at["ny_total"])) == (nxt, nyt)
    assert lib.rkb_checkpoint_write(str(path).encode(), 0, nyt, fields, _p(scal),
                                    cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == -2
    # counts that disagree with the extents (nx_total = nx_phys + 2 nghost),
    # a zero ghost width and negative counts are refused
    IP = ctypes.POINTER(ctypes.c_int)
    for bad in ([42, nxt - 2, nyt - 4, 2], [42, nxt - 4, nyt - 4, 3], [42, nxt, nyt, 0],
                [42, -1, nyt - 4, 2]):
        b = np.array(bad, dtype=np.int32)
        assert lib.rkb_checkpoint_write(str(tmp_path / "bad.nc").encode(), nxt, nyt, fields,
                                        _p(scal), b.ctypes.data_as(IP)) == -2, bad
    assert not (tmp_path / "bad.nc").exists()


def test_checkpoint_too_large_for_the_format_is_refused(lib, tmp_path):
    """A field of 4 GiB or more cannot be described by a 64-bit-offset file
    (32-bit variable sizes): the writer refuses it before reading any field,
    and writes no file.  The arrays passed here are one element long; the
    writer must not touch them."""
    n = 23171  # 23171^2 doubles = 4.295e9 bytes > 2^32
    dummy = [np.zeros(1) for _ in range(7)]
    fields = (DP * 7)(*[_p(a) for a in dummy])
    scal = np.zeros(7)
    cnt = np.array([0, n - 4, n - 4, 2], dtype=np.int32)
    path = tmp_path / "huge.nc"
    assert lib.rkb_checkpoint_write(str(path).encode(), n, n, fields, _p(scal),
                                    cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == -1
    assert not path.exists()
    assert b"too large" in lib.rki_last_error()
