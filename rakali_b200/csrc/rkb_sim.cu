// Host driver of one structured simulation (see rkb_sim.hpp).
#include "rkb_sim.hpp"
#include "rkb_cell.cuh"

#include "rkb_netcdf.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>

namespace rkb {

namespace {

size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

std::string trim_copy(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return {};
  return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
}

// Shu-Osher coefficients of the time schemes (rki_timestepper.F90:60-100):
// stage k steps beta_k dt from X_k at time t + c_k dt, then mixes alpha_k U^n
// + (1 - alpha_k) X_k+1 when alpha_k != 0.  ssp_coeff scales the CFL step.
void fill_scheme(Physics& p, int code) {
  for (int k = 0; k < 4; ++k) p.alpha[k] = p.beta[k] = p.c[k] = 0.0;
  p.scheme = code;
  p.ssp_coeff = 1.0;
  switch (code) {
    case 1:
      p.n_stages = 1;
      p.beta[0] = 1.0;
      break;
    case 3:
      p.n_stages = 3;
      p.alpha[1] = 0.75;
      p.alpha[2] = 1.0 / 3.0;
      p.beta[0] = p.beta[1] = p.beta[2] = 1.0;
      p.c[1] = 1.0;
      p.c[2] = 0.5;
      break;
    case 4:
      p.n_stages = 4;
      p.ssp_coeff = 2.0;
      p.alpha[2] = 2.0 / 3.0;
      p.beta[0] = p.beta[1] = p.beta[2] = p.beta[3] = 0.5;
      p.c[1] = 0.5;
      p.c[2] = 1.0;
      p.c[3] = 0.5;
      break;
    default:
      p.scheme = 2;
      p.n_stages = 2;
      p.alpha[1] = 0.5;
      p.beta[0] = p.beta[1] = 1.0;
      p.c[1] = 1.0;
      break;
  }
}

#define RKB_TRY(expr)                      \
  do {                                     \
    cudaError_t e_ = (expr);               \
    if (e_ != cudaSuccess) return -1;      \
  } while (0)

}  // namespace

Sim::~Sim() {
  drop_graphs();
  if (gauge_mem_) cudaFree(gauge_mem_);
  gauge_mem_ = nullptr;
  free_device();
  for (auto& p : hf_) {
    if (p) cudaFreeHost(p);
    p = nullptr;
  }
  if (hctl_) cudaFreeHost(hctl_);
  if (stream_) cudaStreamDestroy(stream_);
}

namespace {
constexpr size_t kStageBytes = size_t(16) << 20;  // per staging buffer

// Two pinned staging buffers shared by every simulation of the process (one
// upload at a time holds them), allocated by the first finalize on a device
// so no timed upload pays for the pinned allocation.  Their events are
// recorded on whichever stream used them last.
struct Staging {
  std::mutex mu;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool used[2] = {false, false};
  int ensure() {
    for (int k = 0; k < 2; ++k) {
      if (!buf[k] && cudaMallocHost(&buf[k], kStageBytes) != cudaSuccess) {
        buf[k] = nullptr;
        return -1;
      }
      if (!ev[k] && cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess) {
        ev[k] = nullptr;
        return -1;
      }
    }
    return 0;
  }
};
Staging& staging() {
  static Staging* st = new Staging();  // lives until exit (pinned memory freed by the driver)
  return *st;
}

// rows [r0, r1) of an (nx)-wide row-major block copied with up to `nt`
// threads (each a contiguous band of rows)
void copy_rows(double* dst, const double* src, size_t nx, int r0, int r1) {
  const int rows = r1 - r0;
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max(1u, std::min(hw ? hw : 1u, 8u));
  const size_t bytes = (size_t)rows * nx * sizeof(double);
  if (nt == 1 || bytes < (size_t(1) << 20)) {
    std::memcpy(dst, src + (size_t)r0 * nx, bytes);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (int t = 0; t < nt; ++t) {
    const int a = r0 + rows * t / nt, b = r0 + rows * (t + 1) / nt;
    if (a < b)
      th.emplace_back([=] {
        std::memcpy(dst + (size_t)(a - r0) * nx, src + (size_t)a * nx,
                    (size_t)(b - a) * nx * sizeof(double));
      });
  }
  for (auto& t : th) t.join();
}
}  // namespace

int Sim::upload_rows(double* dst, const double* src, int nx, int ny) {
  const size_t row_bytes = (size_t)nx * sizeof(double);
  const int chunk = (int)std::max<size_t>(1, kStageBytes / row_bytes);
  if ((size_t)chunk * row_bytes > kStageBytes) {  // one row exceeds a buffer
    RKB_TRY(cudaMemcpy2DAsync(dst, (size_t)g.pitch * sizeof(double), src, row_bytes, row_bytes,
                              ny, cudaMemcpyHostToDevice, stream_));
    return 0;
  }
  Staging& st = staging();
  std::lock_guard<std::mutex> lk(st.mu);
  if (st.ensure() != 0) return -1;
  int k = 0;
  for (int r0 = 0; r0 < ny; r0 += chunk, k ^= 1) {
    const int r1 = std::min(ny, r0 + chunk);
    if (st.used[k]) RKB_TRY(cudaEventSynchronize(st.ev[k]));  // its previous DMA is done
    copy_rows(static_cast<double*>(st.buf[k]), src, (size_t)nx, r0, r1);
    RKB_TRY(cudaMemcpy2DAsync(dst + (size_t)r0 * g.pitch, (size_t)g.pitch * sizeof(double),
                              st.buf[k], row_bytes, row_bytes, r1 - r0, cudaMemcpyHostToDevice,
                              stream_));
    RKB_TRY(cudaEventRecord(st.ev[k], stream_));
    st.used[k] = true;
  }
  // the buffers are free again once this stream's copies are done
  RKB_TRY(cudaEventSynchronize(st.ev[k ^ 1]));
  return 0;
}

int Sim::create(const std::string& text, std::string& err) {
  Config c;
  if (!parse_namelist(text, c, err)) return -2;
  int rc = validate(c, err);
  if (rc != 0) return rc;
  cfg = c;
  g.ng = cfg.nghost;
  g.nxt = cfg.nx + 2 * cfg.nghost;
  g.nyt = cfg.ny + 2 * cfg.nghost;
  g.pitch = (int)round_up((size_t)g.nxt, 32);
  g.dx = cfg.dx;
  g.dy = cfg.dy;
  ncell_ = (size_t)g.nxt * (size_t)g.nyt;

  if (cudaGetDevice(&device_) != cudaSuccess) {
    err = "no CUDA device available";
    return -1;
  }
  for (auto& p : hf_) {
    if (cudaMallocHost((void**)&p, ncell_ * sizeof(double)) != cudaSuccess) {
      err = "pinned host allocation failed";
      return -1;
    }
    std::memset(p, 0, ncell_ * sizeof(double));
  }
  if (cudaMallocHost((void**)&hctl_, sizeof(StepCtl)) != cudaSuccess) {
    err = "pinned host allocation failed";
    return -1;
  }
  std::memset(hctl_, 0, sizeof(StepCtl));

  // Physics and time control (state_init_from_config, rki_state.F90:134-301)
  phys = Physics{};
  phys.cfl = cfg.cfl;
  phys.dt_fixed = cfg.dt_fixed;
  phys.t_end = cfg.t_end;
  phys.cfl_interval = cfg.cfl_interval;
  phys.manning_n = cfg.manning_n;
  phys.coriolis_f = cfg.coriolis_f;
  phys.use_hllc = cfg.use_hllc ? 1 : 0;
  phys.forcing_active = 0;
  fill_scheme(phys, scheme_code(cfg.time_scheme));
  params_dirty = true;
  t_current_ = 0.0;
  dt_ = 0.0;
  step_count_ = 0;
  is_initialised = true;
  is_finalised = false;
  return 0;
}

// init_from_config (src/core/rki_init.F90:196-216) on the host arrays.
void Sim::init_condition() {
  const int nxt = g.nxt, nyt = g.nyt, ng = g.ng;
  double* h = hf_[0];
  double* hu = hf_[1];
  double* hv = hf_[2];
  double* b = hf_[3];
  auto at = [&](int i, int j) { return (size_t)i + (size_t)j * (size_t)nxt; };
  bool has_b = false;
  for (size_t k = 0; k < ncell_ && !has_b; ++k) has_b = b[k] != 0.0;
  const std::string& ic = cfg.init_condition;
  if (ic == "still_water") {
    for (size_t k = 0; k < ncell_; ++k) {
      h[k] = std::max(cfg.eta_initial - b[k], 0.0);
      hu[k] = 0.0;
      hv[k] = 0.0;
    }
  } else if (ic == "gaussian_hump") {
    const double xc = (double)cfg.nx * g.dx * 0.5 + cfg.hump_x_offset;
    const double yc = (double)cfg.ny * g.dy * 0.5 + cfg.hump_y_offset;
    const double s2 = 2.0 * (cfg.hump_sigma * cfg.hump_sigma);
    for (int j = 0; j < nyt; ++j)
      for (int i = 0; i < nxt; ++i) {
        const double x = ((double)(i + 1 - ng) - 0.5) * g.dx;
        const double y = ((double)(j + 1 - ng) - 0.5) * g.dy;
        const double r2 = (x - xc) * (x - xc) + (y - yc) * (y - yc);
        const size_t q = at(i, j);
        if (!has_b) b[q] = 0.0;
        h[q] = cfg.h0 + cfg.hump_amplitude * std::exp(-r2 / s2);
        hu[q] = 0.0;
        hv[q] = 0.0;
      }
  } else if (ic == "castro_dam_break") {
    const double x0 = -0.5 * (double)cfg.nx * g.dx;
    const double y0 = -0.5 * (double)cfg.ny * g.dy;
    for (int j = 0; j < nyt; ++j)
      for (int i = 0; i < nxt; ++i) {
        const double x = x0 + ((double)(i + 1 - ng) - 0.5) * g.dx;
        const double y = y0 + ((double)(j + 1 - ng) - 0.5) * g.dy;
        const size_t q = at(i, j);
        b[q] = -(1.0 - 0.4 * std::exp(-x * x - y * y));
        h[q] = (x * x + y * y <= 0.36) ? 3.0 - b[q] : 1.0 - b[q];
        hu[q] = 0.0;
        hv[q] = 0.0;
      }
  } else {  // dam_break
    const int mid_x = ng + cfg.nx / 2;
    for (int j = 0; j < nyt; ++j)
      for (int i = 0; i < nxt; ++i) {
        const size_t q = at(i, j);
        if (!has_b) b[q] = 0.0;
        hu[q] = 0.0;
        hv[q] = 0.0;
        h[q] = (i + 1 <= mid_x) ? 2.0 : 1.0;
      }
  }
}

int Sim::finalize(std::string& err) {
  const int nxt = g.nxt, nyt = g.nyt, ng = g.ng;
  double* b = hf_[3];
  auto at = [&](int i, int j) { return (size_t)i + (size_t)j * (size_t)nxt; };
  // bathymetry_file unless the caller set the bed (rki_api.F90:238-240)
  const std::string bfile = trim_copy(cfg.bathymetry_file);
  if (!user_set_bathymetry && !bfile.empty()) {
    std::vector<double> bi((size_t)cfg.nx * cfg.ny);
    if (nc::read_bathymetry(bfile, cfg.nx, cfg.ny, bi.data(), err) != 0) return -3;
    for (int j = 0; j < cfg.ny; ++j)
      std::memcpy(b + at(ng, ng + j), bi.data() + (size_t)j * cfg.nx, (size_t)cfg.nx * sizeof(double));
  }
  // fill_bathymetry_ghosts_array (src/io/rki_bathymetry.F90:165-196)
  for (int j = 0; j < nyt; ++j)
    for (int i = 0; i < ng; ++i) {
      b[at(i, j)] = b[at(ng, j)];
      b[at(ng + cfg.nx + i, j)] = b[at(ng + cfg.nx - 1, j)];
    }
  for (int j = 0; j < ng; ++j)
    for (int i = 0; i < nxt; ++i) {
      b[at(i, j)] = b[at(i, ng)];
      b[at(i, ng + cfg.ny + j)] = b[at(i, ng + cfg.ny - 1)];
    }
  if (!user_set_h) init_condition();

  // bc_init_from_config (rki_boundary_types.F90:132-154)
  bc = BcParams{};
  bc.type[0] = bc_code(cfg.bc_west);
  bc.type[1] = bc_code(cfg.bc_east);
  bc.type[2] = bc_code(cfg.bc_south);
  bc.type[3] = bc_code(cfg.bc_north);
  bc.tidal_amplitude = cfg.tidal_amplitude;
  bc.tidal_period = cfg.tidal_period;
  bc.n_tidal = cfg.n_tidal_constituents;
  for (int k = 0; k < kMaxTidal; ++k) {
    bc.amp[k] = cfg.tidal_amp[k];
    bc.phase[k] = cfg.tidal_phase[k];
    bc.omega[k] = cfg.tidal_omega[k];
  }
  bc.inflow_velocity = cfg.inflow_velocity;
  bc.discharge_flux = cfg.discharge_flux;
  bc.clamped_elevation = cfg.clamped_elevation;
  bc.sponge_width = cfg.sponge_width;
  bc.sponge_strength = cfg.sponge_strength;
  bc.sponge_h_ref = cfg.sponge_h_ref;
  // bc_init_chapman (rki_boundary_types.F90:156-202)
  eta_old_[0].assign(nyt, 0.0);
  eta_old_[1].assign(nyt, 0.0);
  eta_old_[2].assign(nxt, 0.0);
  eta_old_[3].assign(nxt, 0.0);
  const double* h = hf_[0];
  if (bc.type[0] == kChapman || bc.type[1] == kChapman)
    for (int j = 0; j < nyt; ++j) {
      eta_old_[0][j] = h[at(ng, j)] + b[at(ng, j)];
      eta_old_[1][j] = h[at(nxt - ng - 1, j)] + b[at(nxt - ng - 1, j)];
    }
  if (bc.type[2] == kChapman || bc.type[3] == kChapman)
    for (int i = 0; i < nxt; ++i) {
      eta_old_[2][i] = h[at(i, ng)] + b[at(i, ng)];
      eta_old_[3][i] = h[at(i, nyt - ng - 1)] + b[at(i, nyt - ng - 1)];
    }
  params_dirty = true;

  int rc = alloc_device(err);
  if (rc != 0) return rc;
  {  // the setters' staging buffers, once per process
    Staging& st = staging();
    std::lock_guard<std::mutex> lk(st.mu);
    if (st.ensure() != 0) {
      err = "pinned staging allocation failed";
      return -1;
    }
  }
  for (int w = 0; w < 4; ++w)
    RKB_TRY(cudaMemcpyAsync(args_.eta_old[w], eta_old_[w].data(),
                            eta_old_[w].size() * sizeof(double), cudaMemcpyHostToDevice,
                            stream_));
  rc = upload_state();
  if (rc != 0) return rc;
  RKB_TRY(cudaStreamSynchronize(stream_));
  on_device_ = true;
  mark_host_stale();
  is_finalised = true;
  return 0;
}

int Sim::alloc_device(std::string& err) {
  if (dmem_) return 0;
  if (cudaSetDevice(device_) != cudaSuccess) { err = "cudaSetDevice failed"; return -1; }
  if (!stream_ && cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) {
    err = "stream creation failed";
    return -1;
  }
  const size_t field = round_up((size_t)g.pitch * (size_t)g.nyt, 64);  // doubles
  size_t npart = 0;
  for (int t = 0; t < kNumTiles; ++t) npart = std::max(npart, partials_doubles(g, t));
  npart = round_up(npart, 64);
  const size_t neta = round_up(2 * (size_t)g.nyt + 2 * (size_t)g.nxt, 64);
  const size_t ctl_bytes = round_up(sizeof(StepCtl), 256) + round_up(sizeof(Physics), 256) +
                           round_up(sizeof(BcParams), 256);
  const size_t bytes = (10 * field + npart + neta) * sizeof(double) + ctl_bytes;
  if (cudaMalloc(&dmem_, bytes) != cudaSuccess) {
    dmem_ = nullptr;
    err = "device allocation failed";
    return -1;
  }
  if (cudaMemsetAsync(dmem_, 0, bytes, stream_) != cudaSuccess) return -1;
  double* p = (double*)dmem_;
  auto take = [&](size_t n) {
    double* q = p;
    p += n;
    return q;
  };
  args_.g = g;
  args_.U0 = {take(field), take(field), take(field)};
  args_.U1 = {take(field), take(field), take(field)};
  args_.S = {take(field), take(field), take(field)};
  args_.b = take(field);
  args_.partials = take(npart);
  double* eo = take(neta);
  args_.eta_old[0] = eo;
  args_.eta_old[1] = eo + g.nyt;
  args_.eta_old[2] = eo + 2 * g.nyt;
  args_.eta_old[3] = eo + 2 * g.nyt + g.nxt;
  char* cp = (char*)p;
  args_.ctl = (StepCtl*)cp;
  cp += round_up(sizeof(StepCtl), 256);
  args_.phys = (const Physics*)cp;
  cp += round_up(sizeof(Physics), 256);
  args_.bc = (const BcParams*)cp;
  args_.fo = Forcing{nullptr, nullptr, nullptr, nullptr};
  args_.tile = tile;
  args_.hllc = phys.use_hllc;
  args_.scheme = phys.scheme;
  args_.n_stages = phys.n_stages;
  args_.wait_cycles = wait_cycles;
  tma_status_ = encode_tile_maps(args_, &maps_);
  args_.maps = tma_status_ == 0 ? &maps_ : nullptr;
  cur_ = 0;
  // the clock starts at the restart time when a restart file was loaded
  hctl_->t = t_current_;
  if (cudaMemcpyAsync(&args_.ctl->t, &hctl_->t, sizeof(double), cudaMemcpyHostToDevice,
                      stream_) != cudaSuccess ||
      cudaStreamSynchronize(stream_) != cudaSuccess)
    return -1;
  return 0;
}

void Sim::drop_graphs() {
  for (auto& ge : graphs_) {
    if (ge.exec) cudaGraphExecDestroy(ge.exec);
    if (ge.graph) cudaGraphDestroy(ge.graph);
  }
  graphs_.clear();
}

// gauges_init (src/io/structured/rki_gauges.F90:80-123) without the file
// parsing: stations outside the domain are dropped; station_b is the
// bilinear bed at each station (create_gauge_netcdf, :455-467).  The gauge
// clock starts at the current time (rki_driver.F90:346-352).
int Sim::set_gauges(int n, const double* x, const double* y, double interval, int capacity,
                    std::string& err) {
  if (n < 0 || capacity < 1 || (n > 0 && (!x || !y))) {
    err = "invalid gauge arguments";
    return -2;
  }
  if (cudaSetDevice(device_) != cudaSuccess) return -1;
  if (on_device_ && cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
  drop_graphs();
  ++gauge_gen_;
  if (gauge_mem_) cudaFree(gauge_mem_);
  gauge_mem_ = nullptr;
  gauge_dev_ = nullptr;
  gauge_host_ = GaugeDev{};
  gauge_station_.clear();
  gauge_b_.clear();
  GaugeStencils st;
  gauge_stencils(g, x, y, n, st);
  const int nl = (int)st.station.size();
  if (nl == 0) return 0;
  const size_t head = 256, ints = 2 * (size_t)nl * sizeof(int), dbl = 2 * (size_t)nl * 8;
  const size_t recs = (size_t)capacity * (1 + 3 * (size_t)nl) * 8;
  const size_t bytes = head + ((ints + 255) / 256) * 256 + dbl + recs;
  if (cudaMalloc(&gauge_mem_, bytes) != cudaSuccess) {
    gauge_mem_ = nullptr;
    err = "device allocation of the gauge buffer failed";
    return -1;
  }
  char* p = (char*)gauge_mem_;
  gauge_dev_ = (GaugeDev*)p;
  int* ix0 = (int*)(p + head);
  int* iy0 = ix0 + nl;
  double* wx = (double*)(p + head + ((ints + 255) / 256) * 256);
  double* wy = wx + nl;
  double* rec_t = wy + nl;
  double* rec = rec_t + capacity;
  GaugeDev h{};
  h.n = nl;
  h.cap = capacity;
  h.interval = interval;
  h.next = interval > 0.0 ? t_current_ + interval : t_current_;
  h.ix0 = ix0;
  h.iy0 = iy0;
  h.wx = wx;
  h.wy = wy;
  h.rec_t = rec_t;
  h.rec = rec;
  RKB_TRY(cudaMemcpy(ix0, st.ix0.data(), nl * sizeof(int), cudaMemcpyHostToDevice));
  RKB_TRY(cudaMemcpy(iy0, st.iy0.data(), nl * sizeof(int), cudaMemcpyHostToDevice));
  RKB_TRY(cudaMemcpy(wx, st.wx.data(), nl * sizeof(double), cudaMemcpyHostToDevice));
  RKB_TRY(cudaMemcpy(wy, st.wy.data(), nl * sizeof(double), cudaMemcpyHostToDevice));
  RKB_TRY(cudaMemcpy(gauge_dev_, &h, sizeof(GaugeDev), cudaMemcpyHostToDevice));
  gauge_host_ = h;
  gauge_station_ = st.station;
  // the bed at each station from the host bed (ghosts filled at finalize)
  const double* b = hf_[3];
  auto at = [&](int i, int j) { return (size_t)i + (size_t)j * (size_t)g.nxt; };
  for (int k = 0; k < nl; ++k) {
    const int i0 = st.ix0[k], j0 = st.iy0[k];
    const double a = st.wx[k], c = st.wy[k];
    gauge_b_.push_back((1.0 - a) * (1.0 - c) * b[at(i0, j0)] + a * (1.0 - c) * b[at(i0 + 1, j0)] +
                       (1.0 - a) * c * b[at(i0, j0 + 1)] + a * c * b[at(i0 + 1, j0 + 1)]);
  }
  return nl;
}

cudaError_t Sim::record_gauges(cudaStream_t s) {
  const int n = gauge_host_.n;
  if (n <= 0) return cudaSuccess;
  if (precision_ == 32)
    return launch_gauge_record32(args32_.g, args_.ctl, gauge_dev_, n, args32_.U0, args32_.U1,
                                 args32_.b, s);
  return launch_gauge_record(g, args_.ctl, gauge_dev_, n, args_.U0, args_.U1, args_.b, s);
}

int Sim::gauge_stations(int* station, double* station_b) const {
  for (size_t k = 0; k < gauge_station_.size(); ++k) {
    if (station) station[k] = gauge_station_[k];
    if (station_b) station_b[k] = gauge_b_[k];
  }
  return (int)gauge_station_.size();
}

int Sim::read_gauges(int max_records, double* times, double* values, int* overflow) {
  if (overflow) *overflow = 0;
  if (!gauge_dev_) return 0;
  if (cudaSetDevice(device_) != cudaSuccess) return -1;
  if (on_device_ && cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
  GaugeDev h{};
  RKB_TRY(cudaMemcpy(&h, gauge_dev_, sizeof(GaugeDev), cudaMemcpyDeviceToHost));
  const int k = h.count < max_records ? h.count : max_records;
  if (k > 0) {
    if (times) RKB_TRY(cudaMemcpy(times, h.rec_t, (size_t)k * 8, cudaMemcpyDeviceToHost));
    if (values)
      RKB_TRY(cudaMemcpy(values, h.rec, (size_t)k * h.n * 3 * 8, cudaMemcpyDeviceToHost));
  }
  if (overflow) *overflow = h.overflow;
  // the records read are consumed; later ones move to the front
  const int rest = h.count - k;
  if (rest > 0) {
    RKB_TRY(cudaMemcpy(h.rec_t, h.rec_t + k, (size_t)rest * 8, cudaMemcpyDeviceToDevice));
    RKB_TRY(cudaMemcpy(h.rec, h.rec + (size_t)k * h.n * 3, (size_t)rest * h.n * 3 * 8,
                       cudaMemcpyDeviceToDevice));
  }
  const int counters[2] = {rest, 0};
  RKB_TRY(cudaMemcpy(&gauge_dev_->count, counters, sizeof(counters), cudaMemcpyHostToDevice));
  return k;
}

// Per-step checkpoint (python/rakali/_core.py:1433-1499): every field with
// ghosts, RK2 saves included, after a full pull that leaves the device state
// canonical.
int Sim::save_checkpoint(const std::string& path, std::string& err) {
  if (on_device_) {
    cudaSetDevice(device_);
    if (pull_missing(7) != 0) {
      err = "copying the state to the host failed";
      return -1;
    }
  }
  nc::CheckpointMeta m{};
  m.time = t_current_;
  m.dt = dt_;
  m.dx = cfg.dx;
  m.dy = cfg.dy;
  m.manning_n = phys.manning_n;
  m.coriolis_f = phys.coriolis_f;
  m.clamped_elevation = cfg.clamped_elevation;
  m.step_count = step_count_;
  m.nx_phys = cfg.nx;
  m.ny_phys = cfg.ny;
  m.nghost = g.ng;
  const double* f[7] = {hf_[0], hf_[1], hf_[2], hf_[3], hf_[4], hf_[5], hf_[6]};
  return nc::write_checkpoint(path, g.nxt, g.nyt, f, m, err) ? 0 : -1;
}

// restart_write (src/io/structured/rki_output.F90:740-853): interior h, hu,
// hv, b and the clock, after refresh_host.
int Sim::save_restart(const std::string& path, std::string& err) {
  if (on_device_ && !host_is_current_) sync_host();
  const int nx = cfg.nx, ny = cfg.ny;
  std::vector<double> f[4];
  for (int k = 0; k < 4; ++k) {
    f[k].resize((size_t)nx * ny);
    for (int j = 0; j < ny; ++j)
      std::memcpy(f[k].data() + (size_t)j * nx, hf_[k] + (size_t)g.ng + (size_t)(g.ng + j) * g.nxt,
                  (size_t)nx * sizeof(double));
  }
  return nc::write_restart(path, nx, ny, f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                           t_current_, g.dx, g.dy, g.ng, err)
             ? 0
             : -3;
}

// restart_read (rki_output.F90:855-988) before finalize: the interior state
// and bed come from the file (the initial condition is then not applied) and
// the clock starts at the file's time.  1: grid mismatch.
int Sim::load_restart(const std::string& path, std::string& err) {
  const int nx = cfg.nx, ny = cfg.ny;
  std::vector<double> f[4];
  for (auto& v : f) v.resize((size_t)nx * ny);
  double t = 0.0;
  const int rc = nc::read_restart(path, nx, ny, f[0].data(), f[1].data(), f[2].data(), f[3].data(),
                                  t, err);
  if (rc != 0) return rc;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < ny; ++j)
      std::memcpy(hf_[k] + (size_t)g.ng + (size_t)(g.ng + j) * g.nxt, f[k].data() + (size_t)j * nx,
                  (size_t)nx * sizeof(double));
  user_set_h = true;
  user_set_bathymetry = true;
  t_current_ = t;
  return 0;
}

void Sim::free_device() {
  if (dmem_) cudaFree(dmem_);
  dmem_ = nullptr;
  if (dmem32_) cudaFree(dmem32_);
  dmem32_ = nullptr;
  for (double* f : {const_cast<double*>(args_.fo.wind_x), const_cast<double*>(args_.fo.wind_y),
                    const_cast<double*>(args_.fo.atm), const_cast<double*>(args_.fo.precip)})
    if (f) cudaFree(f);
  args_.fo = Forcing{nullptr, nullptr, nullptr, nullptr};
}

// Host arrays -> device (solver_enter_data): h, hu, hv into the current
// buffer, the bed, and the forcing fields when active.
int Sim::upload_state() {
  const size_t wbytes = (size_t)g.nxt * sizeof(double);
  const size_t dpitch = (size_t)g.pitch * sizeof(double);
  FieldSet F = cur_ ? args_.U1 : args_.U0;
  double* dst[4] = {F.h, F.hu, F.hv, args_.b};
  for (int k = 0; k < 4; ++k)
    RKB_TRY(cudaMemcpy2DAsync(dst[k], dpitch, hf_[k], wbytes, wbytes, g.nyt,
                              cudaMemcpyHostToDevice, stream_));
  // The other state buffer and the stage scratch start as copies too: ghost
  // cells that no boundary rule rewrites (nested edges) then keep their
  // values in every buffer, as the reference's single array does.
  const size_t fbytes = (size_t)g.pitch * (size_t)g.nyt * sizeof(double);
  FieldSet O = cur_ ? args_.U0 : args_.U1;
  double* copies[2][3] = {{O.h, O.hu, O.hv}, {args_.S.h, args_.S.hu, args_.S.hv}};
  for (auto& c : copies)
    for (int k = 0; k < 3; ++k)
      RKB_TRY(cudaMemcpyAsync(c[k], dst[k], fbytes, cudaMemcpyDeviceToDevice, stream_));
  if (stepped_) {
    // the other buffer's interior is the RK2 save U^n (the h0 views)
    const size_t off_d = (size_t)g.ng + (size_t)g.ng * (size_t)g.pitch;
    const size_t off_h = (size_t)g.ng + (size_t)g.ng * (size_t)g.nxt;
    for (int k = 0; k < 3; ++k)
      RKB_TRY(cudaMemcpy2DAsync(copies[0][k] + off_d, dpitch, hf_[4 + k] + off_h, wbytes,
                                (size_t)g.nx_phys() * sizeof(double), g.ny_phys(),
                                cudaMemcpyHostToDevice, stream_));
  }
  if (phys.forcing_active && upload_forcing() != 0) return -1;
  if (precision_ == 32 && to_surface(false) != 0) return -1;
  hctl_->ms_valid = 0;
  RKB_TRY(cudaMemcpyAsync(&args_.ctl->ms_valid, &hctl_->ms_valid, sizeof(int),
                          cudaMemcpyHostToDevice, stream_));
  params_dirty = true;
  return 0;
}

// Forcing fields -> device (solver_update_forcing, rki_solver.F90:421-434) and
// the precipitation sum the mass budget adds each stage.
int Sim::upload_forcing() {
  const size_t wbytes = (size_t)g.nxt * sizeof(double);
  const size_t dpitch = (size_t)g.pitch * sizeof(double);
  if (!args_.fo.wind_x) {
    double* f[4];
    for (int k = 0; k < 4; ++k)
      RKB_TRY(cudaMalloc((void**)&f[k], (size_t)g.pitch * g.nyt * sizeof(double)));
    args_.fo = Forcing{f[0], f[1], f[2], f[3]};
    drop_graphs();  // graphs hold the old (null) forcing pointers
  }
  const double* dstf[4] = {args_.fo.wind_x, args_.fo.wind_y, args_.fo.atm, args_.fo.precip};
  for (int k = 0; k < 4; ++k)
    RKB_TRY(cudaMemcpy2DAsync(const_cast<double*>(dstf[k]), dpitch, forcing_[k].data(), wbytes,
                              wbytes, g.nyt, cudaMemcpyHostToDevice, stream_));
  double acc = 0.0;
  for (int j = g.ng; j < g.nyt - g.ng; ++j)
    for (int i = g.ng; i < g.nxt - g.ng; ++i) acc = acc + forcing_[3][(size_t)i + (size_t)j * g.nxt];
  hctl_->precip_sum = acc;
  RKB_TRY(cudaMemcpyAsync(&args_.ctl->precip_sum, &hctl_->precip_sum, sizeof(double),
                          cudaMemcpyHostToDevice, stream_));
  return cudaStreamSynchronize(stream_) == cudaSuccess ? 0 : -1;
}

int Sim::upload_params() {
  if (!params_dirty) return 0;
  // The stream is synchronised after every run, so the pinned staging copies
  // are free to reuse.
  static_assert(sizeof(Physics) + sizeof(BcParams) < 4096, "param staging");
  RKB_TRY(cudaMemcpyAsync(const_cast<Physics*>(args_.phys), &phys, sizeof(Physics),
                          cudaMemcpyHostToDevice, stream_));
  RKB_TRY(cudaMemcpyAsync(const_cast<BcParams*>(args_.bc), &bc, sizeof(BcParams),
                          cudaMemcpyHostToDevice, stream_));
  RKB_TRY(cudaStreamSynchronize(stream_));
  args_.hllc = phys.use_hllc;
  args_.tile = tile;
  args_.scheme = phys.scheme;
  args_.n_stages = phys.n_stages;
  args_.plain = plain_physics(phys, bc) ? 1 : 0;
  args_.wait_cycles = wait_cycles > 0 ? wait_cycles : kWaitCyclesDefault;
  RKB_TRY(configure_kernels(args_.tile, args_.hllc));
  params_dirty = false;
  return 0;
}

int Sim::ensure_device() {
  if (cudaSetDevice(device_) != cudaSuccess) return -1;
  if (!on_device_) {
    if (upload_state() != 0) return -1;
    on_device_ = true;
  } else if (handed_[0] || handed_[1] || handed_[2] || handed_[3]) {
    // Fields whose host arrays went out through a pointer since the last run
    // may have been written there: they move back, and only they (the
    // reference's ensure_device uploads every array, rki_api.F90:116-123).
    if (precision_ == 32 && handed_[3]) {
      // a new bed changes every surface eta = h + b: the depths come home
      // under the old bed, then the whole state goes up again
      if (pull_missing(7) != 0) return -1;
      if (upload_state() != 0) return -1;
    } else {
      for (int f = 0; f < 4; ++f)
        if (handed_[f] && push_field(f) != 0) return -1;
    }
  }
  for (bool& h : handed_) h = false;
  mark_host_stale();
  return 0;
}

// Device -> host of h, hu, hv (solver_update_host); with `full`, also the
// bed and the RK2 save arrays (solver_exit_data).
static int pull(const StepArgs& a, int cur, bool stepped, bool full, double* const* hf,
                const Grid& g, cudaStream_t s) {
  const size_t wbytes = (size_t)g.nxt * sizeof(double);
  const size_t spitch = (size_t)g.pitch * sizeof(double);
  FieldSet F = cur ? a.U1 : a.U0;
  const double* src[4] = {F.h, F.hu, F.hv, a.b};
  const int n = full ? 4 : 3;
  for (int k = 0; k < n; ++k)
    if (cudaMemcpy2DAsync(hf[k], wbytes, src[k], spitch, wbytes, g.nyt, cudaMemcpyDeviceToHost, s) !=
        cudaSuccess)
      return -1;
  if (full && stepped && a.scheme != 2) {
    // generic schemes: the save arrays are whole copies of U^n, ghosts
    // included (solver_save_state), which is the other buffer
    FieldSet O = cur ? a.U0 : a.U1;
    const double* so[3] = {O.h, O.hu, O.hv};
    for (int k = 0; k < 3; ++k)
      if (cudaMemcpy2DAsync(hf[4 + k], wbytes, so[k], spitch, wbytes, g.nyt,
                            cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return -1;
  } else if (full && stepped) {
    // RK2 save arrays: interior of U^n from the other buffer; the reference
    // never writes their ghosts in the fused RK2 path (left at zero here).
    FieldSet O = cur ? a.U0 : a.U1;
    const double* so[3] = {O.h, O.hu, O.hv};
    const size_t off_d = (size_t)g.ng + (size_t)g.ng * (size_t)g.pitch;
    const size_t off_h = (size_t)g.ng + (size_t)g.ng * (size_t)g.nxt;
    for (int k = 0; k < 3; ++k)
      if (cudaMemcpy2DAsync(hf[4 + k] + off_h, wbytes, so[k] + off_d, spitch,
                            (size_t)g.nx_phys() * sizeof(double), g.ny_phys(),
                            cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return -1;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}

int Sim::pull_state(bool full) {
  if (precision_ == 32 && to_depth(full) != 0) return -1;
  if (pull(args_, cur_, stepped_, full, hf_, g, stream_) != 0) return -1;
  for (int f = 0; f < (full ? 7 : 3); ++f) fcur_[f] = true;
  return 0;
}

// One field of pull(): 0..2 the current state, 3 the bed, 4..6 the RK2 saves
// (written by the first step; before it the host arrays hold their values).
int Sim::pull_field(int f) {
  if (f >= 4 && !stepped_) {
    fcur_[f] = true;
    return 0;
  }
  if (precision_ == 32 && to_depth(f >= 4) != 0) return -1;
  const size_t wbytes = (size_t)g.nxt * sizeof(double);
  const size_t spitch = (size_t)g.pitch * sizeof(double);
  const FieldSet F = cur_ ? args_.U1 : args_.U0;
  const FieldSet O = cur_ ? args_.U0 : args_.U1;
  const double* src[7] = {F.h, F.hu, F.hv, args_.b, O.h, O.hu, O.hv};
  if (f < 4 || args_.scheme != 2) {
    RKB_TRY(cudaMemcpy2DAsync(hf_[f], wbytes, src[f], spitch, wbytes, g.nyt,
                              cudaMemcpyDeviceToHost, stream_));
  } else {
    const size_t off_d = (size_t)g.ng + (size_t)g.ng * (size_t)g.pitch;
    const size_t off_h = (size_t)g.ng + (size_t)g.ng * (size_t)g.nxt;
    RKB_TRY(cudaMemcpy2DAsync(hf_[f] + off_h, wbytes, src[f] + off_d, spitch,
                              (size_t)g.nx_phys() * sizeof(double), g.ny_phys(),
                              cudaMemcpyDeviceToHost, stream_));
  }
  RKB_TRY(cudaStreamSynchronize(stream_));
  fcur_[f] = true;
  return 0;
}

int Sim::pull_missing(int upto) {
  for (int f = 0; f < upto; ++f)
    if (!field_current(f) && pull_field(f) != 0) return -1;
  return 0;
}

// Host array f (0..2 a state field of the current buffer, 3 the bed) to the
// device, ghosts included; the CFL maxima are recomputed before the next step.
int Sim::push_field(int f) {
  const size_t wbytes = (size_t)g.nxt * sizeof(double);
  const size_t dpitch = (size_t)g.pitch * sizeof(double);
  const FieldSet F = cur_ ? args_.U1 : args_.U0;
  double* dst[4] = {F.h, F.hu, F.hv, args_.b};
  RKB_TRY(cudaMemcpy2DAsync(dst[f], dpitch, hf_[f], wbytes, wbytes, g.nyt,
                            cudaMemcpyHostToDevice, stream_));
  if (f <= 2) {
    if (precision_ == 32 && to_surface(true, f) != 0) return -1;
    hctl_->ms_valid = 0;
    RKB_TRY(cudaMemcpyAsync(&args_.ctl->ms_valid, &hctl_->ms_valid, sizeof(int),
                            cudaMemcpyHostToDevice, stream_));
  }
  RKB_TRY(cudaStreamSynchronize(stream_));
  return 0;
}

// The host arrays become canonical (a pointer to them is handed out, or they
// are about to be written): pull what is not current, then the next run
// uploads them.
void Sim::ensure_host() {
  if (on_device_) {
    cudaSetDevice(device_);
    // fields already current (some perhaps written through a view since)
    // are kept; the others come home
    pull_missing(7);
    on_device_ = false;
    mark_host_current();
    for (bool& h : handed_) h = false;
  }
}

void Sim::sync_host() {
  if (is_initialised && on_device_) {
    cudaSetDevice(device_);
    pull_missing(3);  // h, hu, hv only: the bed and RK2 saves stay on the device
    host_state_current_ = true;
  }
}

void Sim::sync_from_device() {
  if (is_initialised && on_device_) {
    cudaSetDevice(device_);
    pull_state(true);
    on_device_ = false;
    mark_host_current();
    for (bool& h : handed_) h = false;
  }
}

// rki_get_*_ptr (rki_api.F90:502-700): the reference brings every array home
// and unmaps the device copy (ensure_host); here only the field asked for
// comes home, and the next run uploads it again in case the caller wrote
// through the pointer.  Before finalize and after ensure_host the host
// arrays are canonical already.
double* Sim::field_ptr(int which) {
  if (on_device_) {
    cudaSetDevice(device_);
    if (!field_current(which)) pull_field(which);
    handed_[which] = true;
  }
  return hf_[which];
}

int Sim::set_interior(int which, const double* data, int nx, int ny) {
  if (nx != cfg.nx || ny != cfg.ny) return -2;
  const bool state_field = which <= 2;
  const bool pre_final = (which == 3) || (which == 10);  // bathymetry, initial h
  if (pre_final) {
    if (on_device_) ensure_host();
  }
  const int f = which == 10 ? 0 : which;
  // A state field set while the device holds the state goes straight from
  // the caller's array to the device, and the host array is marked stale
  // (the next pointer to it brings the new values home) - unless a pointer
  // to it is out, in which case the host array is the caller's view and
  // takes the values too.
  const bool direct = state_field && on_device_ && !handed_[f];
  double* dst = hf_[f];
  if (!direct)
    for (int j = 0; j < ny; ++j)
      std::memcpy(dst + (size_t)g.ng + (size_t)(g.ng + j) * g.nxt, data + (size_t)j * nx,
                  (size_t)nx * sizeof(double));
  if (which == 3) {
    user_set_bathymetry = true;
    if (is_finalised) {
      double* b = dst;
      auto at = [&](int i, int j) { return (size_t)i + (size_t)j * (size_t)g.nxt; };
      for (int j = 0; j < g.nyt; ++j)
        for (int i = 0; i < g.ng; ++i) {
          b[at(i, j)] = b[at(g.ng, j)];
          b[at(g.ng + cfg.nx + i, j)] = b[at(g.ng + cfg.nx - 1, j)];
        }
      for (int j = 0; j < g.ng; ++j)
        for (int i = 0; i < g.nxt; ++i) {
          b[at(i, j)] = b[at(i, g.ng)];
          b[at(i, g.ng + cfg.ny + j)] = b[at(i, g.ng + cfg.ny - 1)];
        }
    }
  }
  if (which == 10 || which == 0) user_set_h = true;
  if (state_field && on_device_) {
    // The reference refreshes the host state, writes the interior and pushes
    // h, hu and hv (rki_api.F90:126-143); the device already holds the other
    // two fields and this one's ghosts, so only this field's interior moves.
    cudaSetDevice(device_);
    const size_t wbytes = (size_t)g.nxt * sizeof(double);
    const size_t dpitch = (size_t)g.pitch * sizeof(double);
    // FP32: the depth staging buffers take the current state first, so the
    // conversion of this field back carries the device's ghosts
    if (precision_ == 32 && to_depth(false) != 0) return -1;
    FieldSet F = cur_ ? args_.U1 : args_.U0;
    double* dstd[3] = {F.h, F.hu, F.hv};
    const size_t off_d = (size_t)g.ng + (size_t)g.ng * (size_t)g.pitch;
    const size_t off_h = (size_t)g.ng + (size_t)g.ng * (size_t)g.nxt;
    if (direct) {
      if (upload_rows(dstd[f] + off_d, data, nx, ny) != 0) return -1;
    } else if (cudaMemcpy2DAsync(dstd[f] + off_d, dpitch, hf_[f] + off_h, wbytes,
                                 (size_t)nx * sizeof(double), ny, cudaMemcpyHostToDevice,
                                 stream_) != cudaSuccess) {
      return -1;
    }
    if (precision_ == 32 && to_surface(true, f) != 0) return -1;
    hctl_->ms_valid = 0;
    if (cudaMemcpyAsync(&args_.ctl->ms_valid, &hctl_->ms_valid, sizeof(int),
                        cudaMemcpyHostToDevice, stream_) != cudaSuccess)
      return -1;
    if (cudaStreamSynchronize(stream_) != cudaSuccess) return -1;
    // FP64 through the host array: a host array that was current stays
    // current (same interior on both sides).  Direct, or FP32 (the device
    // holds the field rounded to the surface form): the host copy is stale.
    for (int k = 0; k < 7; ++k) fcur_[k] = field_current(k);
    host_is_current_ = host_state_current_ = false;
    if (direct || precision_ == 32) fcur_[f] = false;
  }
  return 0;
}

int Sim::set_forcing(int which, const double* data, int nx, int ny) {
  if (nx != cfg.nx || ny != cfg.ny) return -2;
  if (forcing_[0].empty()) {
    // state%forcing arrays: uniform config wind stress, zero elsewhere
    forcing_[0].assign(ncell_, cfg.wind_stress_x);
    forcing_[1].assign(ncell_, cfg.wind_stress_y);
    for (int k = 2; k < 6; ++k) forcing_[k].assign(ncell_, 0.0);
  }
  double* dst = forcing_[which].data();
  for (int j = 0; j < ny; ++j)
    std::memcpy(dst + (size_t)g.ng + (size_t)(g.ng + j) * g.nxt, data + (size_t)j * nx,
                (size_t)nx * sizeof(double));
  if (which <= 3) {
    phys.forcing_active = 1;
    params_dirty = true;
  }
  if (on_device_ && which <= 3) return upload_forcing();
  return 0;
}

void Sim::pull_ctl() {
  cudaMemcpyAsync(hctl_, args_.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream_);
  cudaStreamSynchronize(stream_);
  t_current_ = hctl_->t;
  dt_ = hctl_->dt_prev;
  step_count_ = hctl_->step_count;
  cur_ = hctl_->cur;
}

cudaGraphExec_t Sim::graph_for(int steps) {
  const int rows = precision_ == 32 ? args32_.rows * 8 + args32_.cpl : 0;
  const int plain = precision_ == 32 ? args32_.plain : args_.plain;
  for (auto& ge : graphs_)
    if (ge.steps == steps && ge.hllc == args_.hllc && ge.tile == args_.tile &&
        ge.prec == precision_ && ge.rows == rows && ge.plain == plain)
      return ge.exec;
  GraphEntry ge{steps, args_.hllc, args_.tile, precision_, rows, plain, nullptr, nullptr};
  if (cudaStreamSynchronize(stream_) != cudaSuccess) return nullptr;
  if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return nullptr;
  const int ngauge = gauge_host_.n;
  for (int k = 0; k < steps; ++k) {
    if (precision_ == 32) {
      launch_step32(args32_, stream_);
      if (ngauge > 0)
        launch_gauge_record32(args32_.g, args_.ctl, gauge_dev_, ngauge, args32_.U0, args32_.U1,
                              args32_.b, stream_);
    } else {
      launch_step(args_, stream_);
      if (ngauge > 0)
        launch_gauge_record(g, args_.ctl, gauge_dev_, ngauge, args_.U0, args_.U1, args_.b,
                            stream_);
    }
  }
  if (cudaStreamEndCapture(stream_, &ge.graph) != cudaSuccess) return nullptr;
  if (cudaGraphInstantiate(&ge.exec, ge.graph, 0) != cudaSuccess) return nullptr;
  graphs_.push_back(ge);
  return ge.exec;
}

int Sim::prepare_run(int mode, double target, int nsteps) {
  if (ensure_device() != 0) return -1;
  if (upload_params() != 0) return -1;
  // the kernels read the control block; set the run mode
  hctl_->mode = mode;
  hctl_->target = target;
  hctl_->remaining = nsteps;
  RKB_TRY(cudaMemcpyAsync(&args_.ctl->target, &hctl_->target, sizeof(double),
                          cudaMemcpyHostToDevice, stream_));
  RKB_TRY(cudaMemcpyAsync(&args_.ctl->mode, &hctl_->mode, sizeof(int), cudaMemcpyHostToDevice,
                          stream_));
  RKB_TRY(cudaMemcpyAsync(&args_.ctl->remaining, &hctl_->remaining, sizeof(int),
                          cudaMemcpyHostToDevice, stream_));
  // CFL maxima of the current state if no step epilogue has produced them
  RKB_TRY(cudaMemcpyAsync(&hctl_->ms_valid, &args_.ctl->ms_valid, sizeof(int),
                          cudaMemcpyDeviceToHost, stream_));
  RKB_TRY(cudaStreamSynchronize(stream_));
  if (precision_ == 32) {
    sync_args32();
    if (!hctl_->ms_valid) RKB_TRY(launch_max_speed32(args32_, stream_));
  } else if (!hctl_->ms_valid) {
    RKB_TRY(launch_max_speed(args_, stream_));
  }
  return 0;
}

int Sim::run(int mode, double target, int nsteps) {
  if (prepare_run(mode, target, nsteps) != 0) return -1;

  if (mode == 1) {
    int left = nsteps;
    while (left > 0) {
      int k = 1;
      while (k * 2 <= left && k * 2 <= steps_per_graph_cap) k *= 2;
      cudaGraphExec_t ge = graph_for(k);
      if (!ge) return -1;
      RKB_TRY(cudaGraphLaunch(ge, stream_));
      left -= k;
    }
    pull_ctl();
  } else {
    pull_ctl();
    while (t_current_ < target - 1.0e-10) {
      int k = 1;
      if (dt_ > 0.0) {
        const double est = std::ceil((target - t_current_) / dt_ * 1.02) + 1.0;
        while (k < est && k < steps_per_graph_cap) k *= 2;
      }
      cudaGraphExec_t ge = graph_for(k);
      if (!ge) return -1;
      RKB_TRY(cudaGraphLaunch(ge, stream_));
      const double t_before = t_current_;
      const int steps_before = step_count_;
      pull_ctl();
      if (check_device_error() != 0) return -1;
      if (!(t_current_ > t_before) && step_count_ == steps_before) return -1;  // no progress
    }
  }
  if (check_device_error() != 0) return -1;
  if (cudaGetLastError() != cudaSuccess) return -1;
  stepped_ = true;
  mark_host_stale();
  return 0;
}

int Sim::time_steps(int n, double* ms) {
  if (n <= 0) return -2;
  if (prepare_run(1, 0.0, n) != 0) return -1;
  // capture the graphs first so instantiation stays outside the timed region
  for (int k = 1; k <= steps_per_graph_cap; k *= 2)
    if (k <= n && !graph_for(k)) return -1;
  cudaEvent_t e0, e1;
  RKB_TRY(cudaEventCreate(&e0));
  RKB_TRY(cudaEventCreate(&e1));
  RKB_TRY(cudaEventRecord(e0, stream_));
  int left = n;
  while (left > 0) {
    int k = 1;
    while (k * 2 <= left && k * 2 <= steps_per_graph_cap) k *= 2;
    RKB_TRY(cudaGraphLaunch(graph_for(k), stream_));
    left -= k;
  }
  RKB_TRY(cudaEventRecord(e1, stream_));
  RKB_TRY(cudaEventSynchronize(e1));
  float f = 0.0f;
  RKB_TRY(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  pull_ctl();
  if (check_device_error() != 0) return -1;
  stepped_ = true;
  mark_host_stale();
  return 0;
}

int Sim::profile_steps(int n, double out[5]) {
  if (n <= 0) return -2;
  if (phys.scheme != 2) {
    err_text_ = "stage timing covers the two fused SSP-RK2 stages only";
    return -2;
  }
  if (prepare_run(1, 0.0, n) != 0) return -1;
  cudaEvent_t ev[5];
  for (auto& e : ev) RKB_TRY(cudaEventCreate(&e));
  double acc[4] = {0, 0, 0, 0};
  for (int s = 0; s < n; ++s) {
    const bool f32 = precision_ == 32;
    RKB_TRY(cudaEventRecord(ev[0], stream_));
    RKB_TRY(f32 ? launch_bc32(args32_, 1, stream_) : launch_bc(args_, 1, stream_));
    RKB_TRY(cudaEventRecord(ev[1], stream_));
    RKB_TRY(f32 ? launch_stage32_only(args32_, 1, stream_) : launch_stage_only(args_, 1, stream_));
    RKB_TRY(cudaEventRecord(ev[2], stream_));
    RKB_TRY(f32 ? launch_bc32(args32_, 2, stream_) : launch_bc(args_, 2, stream_));
    RKB_TRY(cudaEventRecord(ev[3], stream_));
    RKB_TRY(f32 ? launch_stage32_only(args32_, 2, stream_) : launch_stage_only(args_, 2, stream_));
    RKB_TRY(cudaEventRecord(ev[4], stream_));
    RKB_TRY(cudaEventSynchronize(ev[4]));
    for (int k = 0; k < 4; ++k) {
      float f = 0.0f;
      RKB_TRY(cudaEventElapsedTime(&f, ev[k], ev[k + 1]));
      acc[k] += f;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < 4; ++k) out[k] = acc[k] / n;
  out[4] = (double)(precision_ == 32 ? launches_per_step32(args32_) : launches_per_step(args_));
  pull_ctl();
  if (check_device_error() != 0) return -1;
  stepped_ = true;
  mark_host_stale();
  return 0;
}

// ---------------------------------------------------------------------------
// FP32 surface form
// ---------------------------------------------------------------------------

int Sim::set_precision(int p) {
  if (p != 32 && p != 64) return -2;
  if (p == precision_) return 0;
  if (p == 32 && phys.scheme != 2) {
    err_text_ = "the FP32 surface form runs the SSP-RK2 scheme only";
    return -2;
  }
  if (is_finalised && on_device_) ensure_host();  // state home in the old form
  precision_ = p;
  params_dirty = true;
  return 0;
}

// Surface-form buffers: U0, U1, S (eta, hu, hv in FP32), the bed in FP64 and
// the per-warp partials, in one allocation.  Rows start 128-byte aligned at
// the first interior column; the pitch covers the last strip's right halo.
int Sim::alloc_device32() {
  if (dmem32_) return 0;
  if (!stream_) return -1;
  Grid g32 = g;
  const int off = (32 - g.ng % 32) % 32;
  const size_t need = (size_t)off + sweep_row_extent(g);
  g32.pitch = (int)round_up(std::max(need, (size_t)off + (size_t)g.nxt), 32);
  const size_t field = round_up((size_t)g32.pitch * (size_t)g.nyt, 64);  // elements
  const size_t npart = round_up(partials_doubles32(g, 4), 64);
  const size_t bytes = 9 * field * sizeof(float) + field * sizeof(double) + npart * sizeof(double);
  if (cudaMalloc(&dmem32_, bytes) != cudaSuccess) {
    dmem32_ = nullptr;
    err_text_ = "device allocation of the FP32 surface form failed";
    return -1;
  }
  if (cudaMemsetAsync(dmem32_, 0, bytes, stream_) != cudaSuccess) return -1;
  float* fp = (float*)dmem32_;
  auto f32 = [&](int k) { return fp + (size_t)k * field + off; };
  args32_ = StepArgs32{};
  args32_.g = g32;
  args32_.U0 = {f32(0), f32(1), f32(2)};
  args32_.U1 = {f32(3), f32(4), f32(5)};
  args32_.S = {f32(6), f32(7), f32(8)};
  double* dp = (double*)(fp + 9 * field);
  args32_.b = dp + off;
  args32_.partials = dp + field;
  if (configure_kernels32() != cudaSuccess) return -1;
  auto_rows_[0] = auto_rows32(g, 2);
  auto_rows_[1] = auto_rows32(g, 4);
  sync_args32();
  return 0;
}

// Shared pointers and launch shape of the surface form (forcing fields may be
// allocated late; the sweep rows may be overridden).
void Sim::sync_args32() {
  args32_.ctl = args_.ctl;
  args32_.phys = args_.phys;
  args32_.bc = args_.bc;
  args32_.fo = args_.fo;
  args32_.fpitch = g.pitch;
  for (int w = 0; w < 4; ++w) args32_.eta_old[w] = args_.eta_old[w];
  args32_.hllc = phys.use_hllc;
  args32_.plain = !phys.forcing_active && !(std::fabs(phys.coriolis_f) > 1.0e-20) &&
                  !(bc.sponge_width > 0 && bc.sponge_strength > 0.0);
  args32_.cpl = sweep_cpl == 4 ? 4 : 2;
  int rows = sweep_rows > 0 ? sweep_rows : auto_rows_[args32_.cpl == 4 ? 1 : 0];
  if (rows < 4) rows = 4;
  args32_.rows = rows;
  args32_.wait_cycles = wait_cycles > 0 ? wait_cycles : kWaitCyclesDefault;
  sweep_shape(g, rows, args32_.cpl, args32_.nstrips, args32_.nrowblk);
}

// FP64 staging buffers -> surface form: all three buffers (after an upload)
// or the current one (after a setter).
int Sim::to_surface(bool cur_only, int field) {
  if (alloc_device32() != 0) return -1;
  const FieldSet src[3] = {args_.U0, args_.U1, args_.S};
  const FieldSet32 dst[3] = {args32_.U0, args32_.U1, args32_.S};
  for (int k = 0; k < 3; ++k) {
    if (cur_only && k != cur_) continue;
    FieldSet s = src[k];
    if (field >= 0) {  // one state field of the current buffer; the bed is unchanged
      if (field != 0) s.h = nullptr;
      if (field != 1) s.hu = nullptr;
      if (field != 2) s.hv = nullptr;
    }
    double* bed = field < 0 && k == (cur_only ? cur_ : 0) ? args32_.b : nullptr;
    RKB_TRY(launch_to_surface(g, args32_.g, s, args_.b, dst[k], bed, stream_));
  }
  return 0;
}

// Surface form -> FP64 depth buffers ahead of a host read: the current state
// and the bed, plus the RK2 save buffer when `full`.
int Sim::to_depth(bool full) {
  if (!dmem32_) return 0;
  const FieldSet src64[2] = {args_.U0, args_.U1};
  const FieldSet32 src32[2] = {args32_.U0, args32_.U1};
  RKB_TRY(launch_to_depth(args32_.g, g, src32[cur_], args32_.b, src64[cur_], args_.b, stream_));
  if (full && stepped_)
    RKB_TRY(launch_to_depth(args32_.g, g, src32[cur_ ^ 1], args32_.b, src64[cur_ ^ 1], nullptr,
                            stream_));
  return 0;
}

int Sim::check_device_error() {
  if (!hctl_->error) return 0;
  const int code = hctl_->error;
  err_text_ = code == kErrPhysics
                  ? "the step kernel was built for other physics than the device held; the step "
                    "was abandoned"
              : code == kErrNonFinite
                  ? "a non-finite value (NaN or infinity) appeared in the state at step " +
                        std::to_string(step_count_) + " (t = " + std::to_string(t_current_) +
                        "); the run stopped after that step"
                  : "a bounded device-side wait for a bulk copy expired (a bulk or TMA copy into "
                    "shared memory); the step was abandoned";
  hctl_->error = 0;
  cudaMemcpyAsync(&args_.ctl->error, &hctl_->error, sizeof(int), cudaMemcpyHostToDevice, stream_);
  cudaStreamSynchronize(stream_);
  return -1;
}

// ---------------------------------------------------------------------------
// Batch membership
// ---------------------------------------------------------------------------

int Sim::batch_prepare(int mode, double target, int nsteps) {
  if (prepare_run(mode, target, nsteps) != 0) return -1;
  return cudaStreamSynchronize(stream_) == cudaSuccess ? 0 : -1;
}

int Sim::batch_finish() {
  pull_ctl();
  if (check_device_error() != 0) return -1;
  stepped_ = true;
  mark_host_stale();
  return 0;
}

// The state goes home (fields, RK2 save, bed, clock); trial steps may then run
// on the device; restore() re-uploads exactly that state and clock.  The FP32
// surface form round-trips through the FP64 host arrays bit for bit.
int Sim::snapshot() {
  if (ensure_device() != 0) return -1;
  ensure_host();
  pull_ctl();
  snap_ctl_ = *hctl_;
  for (int w = 0; w < 4; ++w)  // Chapman surfaces change with every boundary fill
    RKB_TRY(cudaMemcpyAsync(eta_old_[w].data(), args_.eta_old[w],
                            eta_old_[w].size() * sizeof(double), cudaMemcpyDeviceToHost,
                            stream_));
  if (gauge_dev_)  // trial steps must leave no gauge records behind
    RKB_TRY(cudaMemcpyAsync(&snap_gauge_, gauge_dev_, sizeof(GaugeDev), cudaMemcpyDeviceToHost,
                            stream_));
  RKB_TRY(cudaStreamSynchronize(stream_));
  snap_cur_ = cur_;
  snap_t_ = t_current_;
  snap_dt_ = dt_;
  snap_steps_ = step_count_;
  snap_stepped_ = stepped_;
  return 0;
}

int Sim::restore() {
  if (cudaSetDevice(device_) != cudaSuccess) return -1;
  *hctl_ = snap_ctl_;
  hctl_->done_blocks = 0u;
  hctl_->ms_done_blocks = 0u;
  hctl_->msx_next = 0ull;
  hctl_->msy_next = 0ull;
  hctl_->error = 0;
  RKB_TRY(cudaMemcpyAsync(args_.ctl, hctl_, sizeof(StepCtl), cudaMemcpyHostToDevice, stream_));
  for (int w = 0; w < 4; ++w)
    RKB_TRY(cudaMemcpyAsync(args_.eta_old[w], eta_old_[w].data(),
                            eta_old_[w].size() * sizeof(double), cudaMemcpyHostToDevice,
                            stream_));
  if (gauge_dev_)
    RKB_TRY(cudaMemcpyAsync(gauge_dev_, &snap_gauge_, sizeof(GaugeDev), cudaMemcpyHostToDevice,
                            stream_));
  RKB_TRY(cudaStreamSynchronize(stream_));
  cur_ = snap_cur_;
  t_current_ = snap_t_;
  dt_ = snap_dt_;
  step_count_ = snap_steps_;
  stepped_ = snap_stepped_;
  on_device_ = false;  // the next run uploads the host arrays, which hold the snapshot
  mark_host_current();
  for (bool& h : handed_) h = false;
  return 0;
}

int Sim::step(int n) {
  if (n <= 0) return 0;
  return run(1, 0.0, n);
}

int Sim::advance(double target) {
  if (!(t_current_ < target - 1.0e-10)) return 0;
  return run(0, target, 0);
}

void Sim::mass_budget(double out[3]) {
  if (dmem_) {
    cudaMemcpyAsync(hctl_, args_.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream_);
    cudaStreamSynchronize(stream_);
  }
  out[0] = hctl_->mass_out;
  out[1] = hctl_->mass_src;
  out[2] = 0.0;
}

}  // namespace rkb
