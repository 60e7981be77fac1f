// extern "C" boundary of librakali.so (declared in include/rakali.h).
//
// Handles are opaque pointers to a registry entry; a pointer that is not in
// the registry (null, destroyed, or foreign) is rejected with -100 without
// being dereferenced (the reference checks a magic number instead,
// src/api/rki_handle.F90:116-139).
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <set>
#include <sstream>
#include <string>

#include "../../include/rakali.h"
#include "rkb_batch.hpp"
#include "rkb_netcdf.hpp"
#include "rkb_sim.hpp"

namespace {

constexpr int kBadHandle = -100;

struct Handle {
  unsigned magic;
  rkb::Sim* sim;
};
constexpr unsigned kMagic = 0x72616B53u;  // 'rakS'

std::mutex g_mu;
std::set<Handle*> g_live;
std::set<rkb::Batch*> g_batches;
thread_local std::string g_err;

Handle* resolve(void* p) {
  if (!p) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  auto* h = static_cast<Handle*>(p);
  if (g_live.find(h) == g_live.end()) return nullptr;
  return h;
}

rkb::Sim* sim_of(void* p) {
  Handle* h = resolve(p);
  return h ? h->sim : nullptr;
}

int fail(int rc, const std::string& msg) {
  g_err = msg;
  return rc;
}

int create_impl(const std::string& text, void** out) {
  if (!out) return fail(kBadHandle, "null handle slot");
  *out = nullptr;
  auto* sim = new rkb::Sim();
  std::string err;
  int rc = sim->create(text, err);
  if (rc != 0) {
    delete sim;
    return fail(rc, err);
  }
  auto* h = new Handle{kMagic, sim};
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_live.insert(h);
  }
  *out = h;
  g_err.clear();
  return 0;
}

int field(void* handle, int which, void** ptr, int* nx, int* ny) {
  if (ptr) *ptr = nullptr;
  if (nx) *nx = 0;
  if (ny) *ny = 0;
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  *ptr = s->field_ptr(which);
  *nx = s->g.nxt;
  *ny = s->g.nyt;
  return 0;
}

int layer_field(void* handle, void** ptr, int* nx, int* ny, int* nz) {
  if (ptr) *ptr = nullptr;
  if (nx) *nx = 0;
  if (ny) *ny = 0;
  if (nz) *nz = 0;
  if (!sim_of(handle)) return kBadHandle;
  return fail(-1, "multilayer mode is not active");
}

int set_state(void* handle, int which, const double* data, int nx, int ny) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (!data) return fail(-2, "null data");
  return s->set_interior(which, data, nx, ny);
}

int set_forcing(void* handle, int which, const double* data, int nx, int ny) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (!data) return fail(-2, "null data");
  return s->set_forcing(which, data, nx, ny);
}

std::string read_file(const char* name, int len) {
  std::string path(name, name + (len > 0 ? len : 0));
  std::ifstream f(path);
  if (!f) return std::string();  // missing file keeps the defaults (rki_config.F90:648-657)
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

}  // namespace

extern "C" {

int rki_working_precision(void) { return 8; }

const char* rki_last_error(void) { return g_err.c_str(); }

int rki_create(const char* filename, int len, void** handle) {
  if (!filename || len < 0) return fail(-2, "bad filename");
  return create_impl(read_file(filename, len), handle);
}

int rki_create_from_string(const char* text, int len, void** handle) {
  if (!text || len < 0) return fail(-2, "bad namelist buffer");
  return create_impl(std::string(text, text + len), handle);
}

int rki_finalize(void* handle) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (s->is_finalised) return -2;
  std::string err;
  int rc = s->finalize(err);
  if (rc != 0) return fail(rc, err);
  return 0;
}

int rki_create_from_namelist(const char* filename, int len, void** handle) {
  int rc = rki_create(filename, len, handle);
  if (rc != 0) return rc;
  rc = rki_finalize(*handle);
  if (rc != 0) rki_destroy(handle);
  return rc;
}

int rki_create_from_namelist_string(const char* text, int len, void** handle) {
  int rc = rki_create_from_string(text, len, handle);
  if (rc != 0) return rc;
  rc = rki_finalize(*handle);
  if (rc != 0) rki_destroy(handle);
  return rc;
}

void rki_destroy(void** handle) {
  if (!handle || !*handle) return;
  Handle* h = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto* p = static_cast<Handle*>(*handle);
    auto it = g_live.find(p);
    if (it == g_live.end()) return;
    g_live.erase(it);
    h = p;
  }
  if (h->sim->batch) static_cast<rkb::Batch*>(h->sim->batch)->detach(h->sim);
  delete h->sim;
  h->magic = 0;
  delete h;
  *handle = nullptr;
}

int rki_step(void* handle, int n_steps) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  int rc = s->step(n_steps);
  return rc ? fail(rc, s->error_text().empty() ? "device step failed" : s->error_text()) : 0;
}

int rki_advance(void* handle, double target_time) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  int rc = s->advance(target_time);
  return rc ? fail(rc, s->error_text().empty() ? "device advance failed" : s->error_text()) : 0;
}

double rki_get_time(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return s ? s->time() : 0.0;
}

double rki_get_dt(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return (s && s->is_initialised) ? s->dt() : 0.0;
}

void rki_get_grid_info(void* handle, int* nx, int* ny, int* nghost, double* dx, double* dy) {
  rkb::Sim* s = sim_of(handle);
  const bool ok = s && s->is_initialised;
  if (nx) *nx = ok ? s->cfg.nx : 0;
  if (ny) *ny = ok ? s->cfg.ny : 0;
  if (nghost) *nghost = ok ? s->cfg.nghost : 0;
  if (dx) *dx = ok ? s->cfg.dx : 0.0;
  if (dy) *dy = ok ? s->cfg.dy : 0.0;
}

int rki_get_step_count(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return (s && s->is_initialised) ? s->step_count() : 0;
}

int rki_get_nz_ml(void* handle) {
  (void)handle;
  return 0;
}

int rki_get_h_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 0, p, nx, ny); }
int rki_get_hu_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 1, p, nx, ny); }
int rki_get_hv_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 2, p, nx, ny); }
int rki_get_b_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 3, p, nx, ny); }
int rki_get_h0_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 4, p, nx, ny); }
int rki_get_hu0_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 5, p, nx, ny); }
int rki_get_hv0_ptr(void* h, void** p, int* nx, int* ny) { return field(h, 6, p, nx, ny); }

int rki_get_h_layer_ptr(void* h, void** p, int* nx, int* ny, int* nz) { return layer_field(h, p, nx, ny, nz); }
int rki_get_hu_layer_ptr(void* h, void** p, int* nx, int* ny, int* nz) { return layer_field(h, p, nx, ny, nz); }
int rki_get_hv_layer_ptr(void* h, void** p, int* nx, int* ny, int* nz) { return layer_field(h, p, nx, ny, nz); }
int rki_get_salinity_ptr(void* h, void** p, int* nx, int* ny, int* nz) { return layer_field(h, p, nx, ny, nz); }
int rki_get_temperature_ptr(void* h, void** p, int* nx, int* ny, int* nz) { return layer_field(h, p, nx, ny, nz); }

int rki_set_bathymetry(void* h, const double* b, int nx, int ny) { return set_state(h, 3, b, nx, ny); }
int rki_set_initial_h(void* h, const double* d, int nx, int ny) { return set_state(h, 10, d, nx, ny); }
int rki_set_h(void* h, const double* d, int nx, int ny) { return set_state(h, 0, d, nx, ny); }
int rki_set_hu(void* h, const double* d, int nx, int ny) { return set_state(h, 1, d, nx, ny); }
int rki_set_hv(void* h, const double* d, int nx, int ny) { return set_state(h, 2, d, nx, ny); }

int rki_set_wind(void* h, const double* wx, const double* wy, int nx, int ny) {
  int rc = set_forcing(h, 0, wx, nx, ny);
  if (rc != 0) return rc;
  return set_forcing(h, 1, wy, nx, ny);
}
int rki_set_atm_pressure(void* h, const double* p, int nx, int ny) { return set_forcing(h, 2, p, nx, ny); }
int rki_set_precipitation(void* h, const double* p, int nx, int ny) { return set_forcing(h, 3, p, nx, ny); }
int rki_set_heat_flux(void* h, const double* q, int nx, int ny) { return set_forcing(h, 4, q, nx, ny); }
int rki_set_evap_minus_precip(void* h, const double* e, int nx, int ny) { return set_forcing(h, 5, e, nx, ny); }

int rki_set_salinity(void* h, const double* d, int nx, int ny, int nz) {
  (void)d; (void)nx; (void)ny; (void)nz;
  rkb::Sim* s = sim_of(h);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  return fail(-3, "multilayer mode is not active");
}
int rki_set_temperature(void* h, const double* d, int nx, int ny, int nz) {
  return rki_set_salinity(h, d, nx, ny, nz);
}

#define RKB_BC_SCALAR(fn, stmt)                 \
  int fn(void* handle, double value) {          \
    rkb::Sim* s = sim_of(handle);               \
    if (!s) return kBadHandle;                  \
    if (!s->is_initialised) return -1;          \
    stmt;                                       \
    s->params_dirty = true;                     \
    return 0;                                   \
  }
RKB_BC_SCALAR(rki_set_inflow_velocity, (s->bc.inflow_velocity = value, s->cfg.inflow_velocity = value))
RKB_BC_SCALAR(rki_set_inflow_salinity, s->cfg.inflow_salinity = value)
RKB_BC_SCALAR(rki_set_inflow_temperature, s->cfg.inflow_temperature = value)
RKB_BC_SCALAR(rki_set_discharge_flux, (s->bc.discharge_flux = value, s->cfg.discharge_flux = value))
RKB_BC_SCALAR(rki_set_clamped_elevation, (s->bc.clamped_elevation = value, s->cfg.clamped_elevation = value))
#undef RKB_BC_SCALAR

double rki_get_clamped_elevation(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return (s && s->is_initialised) ? s->cfg.clamped_elevation : 0.0;
}
double rki_get_manning_n(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return (s && s->is_initialised) ? s->phys.manning_n : 0.0;
}
double rki_get_coriolis_f(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return (s && s->is_initialised) ? s->phys.coriolis_f : 0.0;
}

int rki_set_tidal_constituents(void* handle, const double* amp, const double* phase,
                               const double* omega, int n) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (n < 0 || n > rkb::kMaxTidal) return -2;
  if (n > 0 && (!amp || !phase || !omega)) return fail(-2, "null constituent arrays");
  for (int k = 0; k < rkb::kMaxTidal; ++k) {
    s->bc.amp[k] = k < n ? amp[k] : 0.0;
    s->bc.phase[k] = k < n ? phase[k] : 0.0;
    s->bc.omega[k] = k < n ? omega[k] : 0.0;
    s->cfg.tidal_amp[k] = s->bc.amp[k];
    s->cfg.tidal_phase[k] = s->bc.phase[k];
    s->cfg.tidal_omega[k] = s->bc.omega[k];
  }
  s->bc.n_tidal = n;
  s->cfg.n_tidal_constituents = n;
  s->params_dirty = true;
  return 0;
}

void rki_sync_host(void* handle) {
  rkb::Sim* s = sim_of(handle);
  if (s) s->sync_host();
}

void rki_sync_from_device(void* handle) {
  rkb::Sim* s = sim_of(handle);
  if (s) s->sync_from_device();
}

int rki_save_restart(void* handle, const char* filename, int len) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (!s->is_finalised) return -2;
  if (!filename || len <= 0) return fail(-3, "empty restart file name");
  std::string err;
  const int rc = s->save_restart(std::string(filename, (size_t)len), err);
  return rc == 0 ? 0 : fail(-3, err);
}

int rkb_save_checkpoint(void* handle, const char* filename, int len) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (!s->is_finalised) return -2;
  if (!filename || len <= 0) return fail(-3, "empty checkpoint file name");
  std::string err;
  const int rc = s->save_checkpoint(std::string(filename, (size_t)len), err);
  return rc == 0 ? 0 : fail(-3, err);
}

int rki_load_restart(void* handle, const char* filename, int len) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  if (s->is_finalised) return -2;
  if (!filename || len <= 0) return fail(-3, "empty restart file name");
  std::string err;
  const int rc = s->load_restart(std::string(filename, (size_t)len), err);
  return rc == 0 ? 0 : fail(-3, err);
}

int rkb_set_gauges(void* handle, int n, const double* x, const double* y, double interval,
                   int capacity) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised || !s->is_finalised) return -1;
  std::string err;
  const int rc = s->set_gauges(n, x, y, interval, capacity, err);
  return rc >= 0 ? rc : fail(rc, err.empty() ? "gauge setup failed" : err);
}

int rkb_gauge_stations(void* handle, int* station, double* station_b) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  return s->gauge_stations(station, station_b);
}

int rkb_read_gauges(void* handle, int max_records, double* times, double* values, int* overflow) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (max_records < 0) return -2;
  return s->read_gauges(max_records, times, values, overflow);
}

int rkb_write_gauges_netcdf(const char* path, int n, const char* names, int name_len,
                            const double* x, const double* y, const double* b, int n_records,
                            const double* times, const double* values) {
  if (!path || n < 0 || n_records < 0 || (n > 0 && (!x || !y || !b)) ||
      (n_records > 0 && (!times || (n > 0 && !values))))
    return fail(-2, "invalid arguments");
  std::string err;
  if (!rkb::nc::write_gauges(path, n, names, name_len, x, y, b, n_records, times, values, err))
    return fail(-1, err);
  return 0;
}

// Host-only codec entry points (no simulation, no GPU): interior (nx, ny)
// Fortran-order arrays; read returns 0, 1 (grid mismatch) or -1.
int rkb_restart_write(const char* path, int nx, int ny, const double* h, const double* hu,
                      const double* hv, const double* b, double time, double dx, double dy,
                      int nghost) {
  if (!path || !h || !hu || !hv || !b || nx < 1 || ny < 1) return fail(-2, "invalid arguments");
  std::string err;
  if (!rkb::nc::write_restart(path, nx, ny, h, hu, hv, b, time, dx, dy, nghost, err))
    return fail(-1, err);
  return 0;
}

int rkb_checkpoint_write(const char* path, int nx_total, int ny_total,
                         const double* const* fields, const double* scalars, const int* counts) {
  if (!path || !fields || !scalars || !counts || nx_total < 1 || ny_total < 1)
    return fail(-2, "invalid arguments");
  for (int k = 0; k < 7; ++k)
    if (!fields[k]) return fail(-2, "invalid arguments");
  // the counts must describe the arrays: nx_total = nx_phys + 2 nghost, as
  // the reference's grid derives it (rki_grid.F90)
  if (counts[3] < 1 || counts[1] < 1 || counts[2] < 1 ||
      (long long)nx_total != (long long)counts[1] + 2LL * counts[3] ||
      (long long)ny_total != (long long)counts[2] + 2LL * counts[3])
    return fail(-2, "checkpoint counts disagree with the array extents");
  rkb::nc::CheckpointMeta m{};
  m.time = scalars[0];
  m.dt = scalars[1];
  m.dx = scalars[2];
  m.dy = scalars[3];
  m.manning_n = scalars[4];
  m.coriolis_f = scalars[5];
  m.clamped_elevation = scalars[6];
  m.step_count = counts[0];
  m.nx_phys = counts[1];
  m.ny_phys = counts[2];
  m.nghost = counts[3];
  std::string err;
  if (!rkb::nc::write_checkpoint(path, nx_total, ny_total, fields, m, err)) return fail(-1, err);
  return 0;
}

int rkb_gauge_stencils(int nx, int ny, int nghost, double dx, double dy, const double* x,
                       const double* y, int n, int* station, int* ix0, int* iy0, double* wx,
                       double* wy) {
  if (nx < 1 || ny < 1 || nghost < 1 || !(dx > 0.0) || !(dy > 0.0) || n < 0 ||
      (n > 0 && (!x || !y || !station || !ix0 || !iy0 || !wx || !wy)))
    return fail(-2, "invalid arguments");
  rkb::Grid g{};
  g.ng = nghost;
  g.nxt = nx + 2 * nghost;
  g.nyt = ny + 2 * nghost;
  g.pitch = g.nxt;
  g.dx = dx;
  g.dy = dy;
  rkb::GaugeStencils st;
  rkb::gauge_stencils(g, x, y, n, st);
  for (size_t k = 0; k < st.station.size(); ++k) {
    station[k] = st.station[k];
    ix0[k] = st.ix0[k];
    iy0[k] = st.iy0[k];
    wx[k] = st.wx[k];
    wy[k] = st.wy[k];
  }
  return (int)st.station.size();
}

int rkb_bathymetry_read(const char* path, int nx, int ny, double* b) {
  if (!path || !b || nx < 1 || ny < 1) return fail(-2, "invalid arguments");
  std::string err;
  const int rc = rkb::nc::read_bathymetry(path, nx, ny, b, err);
  return rc == 0 ? 0 : fail(rc, err);
}

int rkb_restart_read(const char* path, int nx, int ny, double* h, double* hu, double* hv,
                     double* b, double* time) {
  if (!path || !h || !hu || !hv || !b || !time || nx < 1 || ny < 1)
    return fail(-2, "invalid arguments");
  std::string err;
  const int rc = rkb::nc::read_restart(path, nx, ny, h, hu, hv, b, *time, err);
  return rc == 0 ? 0 : fail(rc, err);
}

int rki_set_use_ppm_tracer(void* handle, int flag) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  s->cfg.use_ppm_tracer = flag != 0;
  return 0;
}

int rki_set_use_hllc(void* handle, int flag) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_initialised) return -1;
  s->phys.use_hllc = flag != 0 ? 1 : 0;
  s->cfg.use_hllc = flag != 0;
  s->params_dirty = true;
  return 0;
}

// ---- additions ------------------------------------------------------------

int rkb_validate_namelist(const char* text, int len, char* err, int err_len) {
  if (!text || len < 0) return -2;
  rkb::Config c;
  std::string e;
  int rc = 0;
  if (!rkb::parse_namelist(std::string(text, text + len), c, e)) rc = -2;
  else rc = rkb::validate(c, e);
  if (err && err_len > 0) {
    std::snprintf(err, (size_t)err_len, "%s", e.c_str());
  }
  return rc;
}

int rkb_get_mass_budget(void* handle, double* out) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  if (!out) return -2;
  s->mass_budget(out);
  return 0;
}

int rkb_get_device_fields(void* handle, void** ptrs, int* pitch) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  if (s->precision() != 64)
    return fail(-3, "device field views are FP64 depth-form arrays; the handle runs the FP32 "
                    "surface form (rkb_set_precision(handle, 64) first)");
  if (s->ensure_device() != 0) return -1;
  rkb::StepArgs a = s->device_args();
  rkb::FieldSet F = s->current_buffer() ? a.U1 : a.U0;
  ptrs[0] = F.h;
  ptrs[1] = F.hu;
  ptrs[2] = F.hv;
  ptrs[3] = a.b;
  *pitch = a.g.pitch;
  return 0;
}

int rkb_set_tile(void* handle, int tile) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (tile < 0 || tile >= rkb::kNumTiles) return -2;
  s->tile = tile;
  s->params_dirty = true;
  return 0;
}

int rkb_time_steps(void* handle, int n, double* ms) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  if (!ms) return -2;
  return s->time_steps(n, ms);
}

int rkb_profile_steps(void* handle, int n, double* out5) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (!s->is_finalised) return -1;
  if (!out5) return -2;
  const int rc = s->profile_steps(n, out5);
  return rc == 0 ? 0 : fail(rc, s->error_text());
}

int rkb_get_tile(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return s ? s->tile : kBadHandle;
}

int rkb_tma_tile_status(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return s ? s->tma_status() : kBadHandle;
}

// ---- batches ----------------------------------------------------------------

static rkb::Batch* batch_of(void* p) {
  if (!p) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  auto* b = static_cast<rkb::Batch*>(p);
  return g_batches.count(b) ? b : nullptr;
}

int rkb_batch_create(void** handles, int n, int precision, void** batch) {
  if (!batch) return fail(kBadHandle, "null batch slot");
  *batch = nullptr;
  if (!handles || n <= 0) return fail(-2, "a batch needs at least one simulation");
  std::vector<rkb::Sim*> sims;
  for (int i = 0; i < n; ++i) {
    rkb::Sim* s = sim_of(handles[i]);
    if (!s) return fail(kBadHandle, "invalid simulation handle in the batch");
    sims.push_back(s);
  }
  auto* b = new rkb::Batch();
  std::string err;
  const int rc = b->create(sims, precision, err);
  if (rc != 0) {
    delete b;
    return fail(rc, err);
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_batches.insert(b);
  }
  *batch = b;
  g_err.clear();
  return 0;
}

void rkb_batch_destroy(void** batch) {
  if (!batch || !*batch) return;
  rkb::Batch* b = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto* p = static_cast<rkb::Batch*>(*batch);
    if (!g_batches.count(p)) return;
    g_batches.erase(p);
    b = p;
  }
  delete b;
  *batch = nullptr;
}

int rkb_batch_step(void* batch, int n_steps) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  const int rc = b->step(n_steps);
  return rc ? fail(rc, b->error().empty() ? "batch step failed" : b->error()) : 0;
}

int rkb_batch_advance(void* batch, double target_time) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  const int rc = b->advance(target_time);
  return rc ? fail(rc, b->error().empty() ? "batch advance failed" : b->error()) : 0;
}

int rkb_batch_time_steps(void* batch, int n, double* ms) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  if (!ms) return -2;
  const int rc = b->time_steps(n, ms);
  return rc ? fail(rc, b->error().empty() ? "batch timing failed" : b->error()) : 0;
}

int rkb_batch_profile_steps(void* batch, int n, double* out5) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  if (!out5) return -2;
  const int rc = b->profile_steps(n, out5);
  return rc ? fail(rc, b->error().empty() ? "batch profiling failed" : b->error()) : 0;
}

int rkb_batch_autotune(void* batch, int trial_steps, double* best_ms_per_step) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  const int rc = b->autotune(trial_steps, best_ms_per_step);
  return rc ? fail(rc, b->error().empty() ? "batch autotune failed" : b->error()) : 0;
}

int rkb_batch_variant(void* batch, int* a, int* b_) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  b->variant(a, b_);
  return 0;
}

int rkb_batch_set_variant(void* batch, int a, int b_) {
  rkb::Batch* b = batch_of(batch);
  if (!b) return kBadHandle;
  const int rc = b->set_variant(a, b_);
  return rc == 0 ? 0 : fail(rc, b->error().empty() ? "batch variant refused" : b->error());
}

int rkb_set_precision(void* handle, int bits) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (bits != 32 && bits != 64) return fail(-2, "precision must be 32 or 64");
  const int rc = s->set_precision(bits);
  return rc == 0 ? 0 : fail(rc, s->error_text());
}

int rkb_get_precision(void* handle) {
  rkb::Sim* s = sim_of(handle);
  return s ? s->precision() : kBadHandle;
}

int rkb_set_sweep(void* handle, int cols_per_lane, int rows) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  if (cols_per_lane != 0 && cols_per_lane != 2 && cols_per_lane != 4)
    return fail(-2, "cols_per_lane must be 0 (default), 2 or 4");
  if (rows < 0) return fail(-2, "rows must be >= 0 (0 selects the automatic value)");
  s->sweep_cpl = cols_per_lane == 0 ? 2 : cols_per_lane;
  s->sweep_rows = rows;
  s->params_dirty = true;
  return 0;
}

int rkb_set_wait_limit(void* handle, long long cycles) {
  rkb::Sim* s = sim_of(handle);
  if (!s) return kBadHandle;
  s->wait_cycles = cycles > 0 ? cycles : rkb::kWaitCyclesDefault;
  s->drop_step_graphs();  // the step graphs hold the sweep's arguments by value
  s->params_dirty = true;
  return 0;
}

}  // extern "C"

namespace rkb {
// Message for rki_last_error() from entry points defined in other files.
void set_last_error(const std::string& msg) { g_err = msg; }
}  // namespace rkb
