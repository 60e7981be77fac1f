// Restart files in the NetCDF classic format (64-bit offset variant), the
// layout of the reference's restart_write / restart_read
// (src/io/structured/rki_output.F90:740-988): dimensions x = nx_phys and
// y = ny_phys, variables h, hu, hv, b (y, x) in FP64 with "units"
// attributes, a scalar "time", and global attributes Conventions, title,
// source, dx, dy, nghost.  The reference writes NetCDF-4 (an HDF5 container)
// through libnetcdf; classic files hold the same variables and every NetCDF
// library (netcdf-fortran's nf90_open included) reads them.  The readers
// accept classic and 64-bit-offset files with fixed-size variables and refuse
// HDF5 containers with a message.
#pragma once

#include <string>

namespace rkb {
namespace nc {

// Interior arrays are (nx, ny) Fortran order (x fastest), which is the
// file's (y, x) row-major order.
bool write_restart(const std::string& path, int nx, int ny, const double* h, const double* hu,
                   const double* hv, const double* b, double time, double dx, double dy, int ng,
                   std::string& err);

// 0: read; 1: the file's grid is not nx x ny; -1: not readable (err says why).
int read_restart(const std::string& path, int nx, int ny, double* h, double* hu, double* hv,
                 double* b, double& time, std::string& err);

// Bathymetry input (src/io/rki_bathymetry.F90:21-163): the first of the
// variables b, elevation, depth, over dimensions x, y in either order, into
// an interior (nx, ny) Fortran-order array.  Return codes as read_restart.
int read_bathymetry(const std::string& path, int nx, int ny, double* b, std::string& err);

// Gauge time series in the layout of create_gauge_netcdf / gauges_write
// (src/io/structured/rki_gauges.F90:338-575): dimensions station, time,
// name_strlen (64); station_name, station_x, station_y, station_b; eta, u, v
// (time, station).  The time dimension has the record count (the reference's
// is unlimited).  names: n fixed-width fields of name_len characters;
// values: [n_records][n][3] (eta, u, v).
bool write_gauges(const std::string& path, int n, const char* names, int name_len,
                  const double* x, const double* y, const double* b, int n_records,
                  const double* times, const double* values, std::string& err);

// Per-step checkpoint in the layout of the reference front end's
// save_checkpoint (python/rakali/_core.py:1433-1499): dimensions x_total,
// y_total; FP64 variables h, hu, hv, b, h0, hu0, hv0 over (x_total, y_total)
// with units / long_name (and positive = up for b); global attributes title,
// source, time, step_count, dt, nx_total, ny_total, nx_phys, ny_phys, nghost,
// dx, dy, manning_n, coriolis_f, clamped_elevation (doubles as NC_DOUBLE,
// counts as NC_INT).  The reference writes NetCDF-4 through xarray; this is
// the same content in a classic (64-bit offset) file.  fields: h, hu, hv, b,
// h0, hu0, hv0, each (nx_total, ny_total) Fortran order with ghosts.
struct CheckpointMeta {
  double time, dt, dx, dy, manning_n, coriolis_f, clamped_elevation;
  int step_count, nx_phys, ny_phys, nghost;
};
bool write_checkpoint(const std::string& path, int nx_total, int ny_total,
                      const double* const fields[7], const CheckpointMeta& m, std::string& err);

}  // namespace nc
}  // namespace rkb
