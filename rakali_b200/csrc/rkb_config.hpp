// Namelist configuration of one structured simulation.
//
// Mirrors the reference's strict namelist schema (src/core/rki_config.F90,
// build_rakali_schema :1234-1253): every group and key the reference accepts
// parses here, unknown groups/keys are errors, and the keys the structured 2D
// step reads are typed and range-checked like validate_config (:886-1183).
// Failures return a message instead of stopping the process.
#pragma once

#include <string>

namespace rkb {

constexpr int kMaxTidalCfg = 10;  // MAX_TIDAL_CONSTITUENTS, rki_config.F90:33

struct Config {
  // &sim_nml, &grid_nml
  std::string sim_type = "coastal";
  std::string grid_type = "structured";
  int nx = 200, ny = 1, nghost = 3;
  double dx = 1.0, dy = 1.0;
  // &time_nml
  double t_end = 1.0, cfl = 0.45, dt_max = 1.0e10, dt_fixed = 0.0;
  int cfl_interval = 1;
  std::string time_scheme = "rk2";
  std::string time_unit = "s";
  // &physics_nml
  double manning_n = 0.0, dry_threshold = 0.001;
  double wind_stress_x = 0.0, wind_stress_y = 0.0, coriolis_f = 0.0;
  bool use_hllc = false, use_linear_bottom_drag = false, wind_surface_layer = false;
  double bottom_drag_r = 0.0;
  // &boundary_nml
  std::string bc_west = "wall", bc_east = "wall", bc_south = "wall", bc_north = "wall";
  double tidal_amplitude = 0.0, tidal_period = 44712.0;
  int n_tidal_constituents = 0;
  double tidal_amp[kMaxTidalCfg] = {}, tidal_phase[kMaxTidalCfg] = {},
         tidal_omega[kMaxTidalCfg] = {};
  double inflow_velocity = 0.0, inflow_salinity = -1.0, inflow_temperature = -999.0;
  double discharge_flux = 0.0, clamped_elevation = 0.0;
  int sponge_width = 0;
  double sponge_strength = 0.0, sponge_h_ref = 0.0;
  std::string nesting_file;
  // &initial_condition_nml
  std::string init_condition = "dam_break";
  double eta_initial = 0.0, h0 = 1.0, hump_amplitude = 0.05, hump_sigma = 5.0;
  double hump_x_offset = 0.0, hump_y_offset = 0.0, init_u_shear = 0.0;
  // &output_nml (only bathymetry_file is read by the library API)
  std::string bathymetry_file;
  // &nonhydrostatic_nml switches that select other solvers
  bool use_nonhydrostatic = false, use_multilayer = false;
  int nz_layers = 2;
  // &tracer_nml (stored for the tracer setters; unused by the 2D step)
  bool use_ppm_tracer = true;
  // &logging_nml
  std::string log_level = "info";
};

// Parse namelist text into `cfg` (defaults first).  Returns true on success;
// on failure `err` names the offending group/key/value.
bool parse_namelist(const std::string& text, Config& cfg, std::string& err);

// validate_config + apply_time_unit_cascade (rki_config.F90:780-889) plus the
// structured-2D scope checks.  Returns 0 when valid, -2 for an invalid value,
// -3 when the configuration asks for a solver mode this library does not run.
int validate(Config& cfg, std::string& err);

int bc_code(const std::string& name);  // rki_boundary_types.F90:106-130
int scheme_code(const std::string& name);  // 1 euler, 2 rk2, 3 rk3, 4 rk43

}  // namespace rkb
