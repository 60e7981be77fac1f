// One structured simulation: host mirror, device state and the step driver.
//
// The host side mirrors the reference handle's state machine
// (src/api/rki_api.F90:48-150, on_device / host_is_current) so the zero-copy
// field views behave the same: reading a field pointer brings the device
// state home, and the next step uploads whatever the caller left in it.
#pragma once

#include <string>
#include <vector>

#include "rkb_config.hpp"
#include "rkb_gauges.hpp"
#include "rkb_kernels.h"

namespace rkb {

class Sim {
 public:
  Sim() = default;
  ~Sim();
  Sim(const Sim&) = delete;
  Sim& operator=(const Sim&) = delete;

  // rki_create / rki_create_from_string: parse, validate, allocate host state.
  int create(const std::string& namelist_text, std::string& err);
  // rki_finalize: ghost-fill the bed, initial condition, BCs, device upload.
  int finalize(std::string& err);

  int step(int n);                 // rki_step
  // n steps bracketed by CUDA events on the simulation's stream; *ms = elapsed.
  int time_steps(int n, double* ms);
  // n steps launched one kernel at a time with events between launches;
  // out[k] = mean ms of launch k of a step (bc1, stage1, bc2, stage2 in order,
  // the boundary launches summed), out[4] = launches per step.
  int profile_steps(int n, double out[5]);
  int save_restart(const std::string& path, std::string& err);  // NetCDF classic
  int save_checkpoint(const std::string& path, std::string& err);  // NetCDF classic
  // Gauge stations recorded on the device after every step (rkb_gauges.cu):
  // returns the number of stations inside the domain, or < 0.
  int set_gauges(int n, const double* x, const double* y, double interval, int capacity,
                 std::string& err);
  int gauge_stations(int* station, double* station_b) const;  // the stations inside
  // Drain the recorded series: count returned, times [count], values
  // [count][n][3] (eta, u, v), *overflow = records dropped since the last read.
  int read_gauges(int max_records, double* times, double* values, int* overflow);
  // For batches: the recorder kernel of this simulation (nothing without
  // stations), and a number that changes whenever the stations change.
  cudaError_t record_gauges(cudaStream_t s);
  int gauge_generation() const { return gauge_gen_; }
  int load_restart(const std::string& path, std::string& err);  // before finalize; 1 = grid mismatch
  int advance(double target_time);  // rki_advance

  // Field access (F-order host arrays with ghosts).  `which`: 0 h, 1 hu,
  // 2 hv, 3 b, 4 h0, 5 hu0, 6 hv0.
  double* field_ptr(int which);
  int set_interior(int which, const double* data, int nx, int ny);  // setters
  int set_forcing(int which, const double* data, int nx, int ny);   // 0 wx, 1 wy, 2 atm, 3 precip
  void sync_host();          // rki_sync_host
  void sync_from_device();   // rki_sync_from_device

  // bookkeeping the API reads
  double time() const { return t_current_; }
  double dt() const { return dt_; }
  int step_count() const { return step_count_; }
  void mass_budget(double out[3]);

  Config cfg;
  Grid g{};
  bool is_initialised = false, is_finalised = false;
  bool user_set_bathymetry = false, user_set_h = false;
  BcParams bc{};
  Physics phys{};
  bool params_dirty = true;
  int tile = kTile16x15t;  // fastest measured FP64 variant on B200 (4096^2 workload)
  int steps_per_graph_cap = 256;
  int sweep_rows = 0;     // FP32 sweep: rows per warp (0: one wave of resident warps)
  int sweep_cpl = 2;      // FP32 sweep: columns per lane (2 or 4)
  // FP32 sweep: limit of its waits for bulk copies, in clock cycles (the
  // default unless a test shortens it to make a wait give up)
  long long wait_cycles = kWaitCyclesDefault;
  void drop_step_graphs() { drop_graphs(); }

  // Arithmetic form of the step: 64 = FP64 depth form (the reference's
  // arithmetic), 32 = FP32 surface form (rkb_step_f32.cu).  Switching brings
  // the state home in the old form and uploads it in the new one.
  int precision() const { return precision_; }
  int set_precision(int p);
  const std::string& error_text() const { return err_text_; }

  // ---- membership of a batch (rkb_batch.cu) ----
  // Set up a run of the device clock (mode 0: advance to `target`, mode 1:
  // `nsteps` steps) without launching steps: state and parameters resident,
  // CFL maxima current, kernel arguments in sync.
  int batch_prepare(int mode, double target, int nsteps);
  // After a batch ran steps on this simulation: read the device clock back.
  int batch_finish();
  // Trial runs (autotuning) on the live state: bring it home, then put it back.
  int snapshot();
  int restore();
  StepArgs32 device_args32() const { return args32_; }
  void* batch = nullptr;  // the batch this simulation belongs to (at most one)

  // Device pointers for the torch / kernel-level paths.
  StepArgs device_args() const { return args_; }
  int tma_status() const { return tma_status_; }
  const TileMaps& tile_maps() const { return maps_; }
  int current_buffer() const { return cur_; }
  cudaStream_t stream() const { return stream_; }
  int ensure_device();
  void ensure_host();

 private:
  int alloc_device(std::string& err);
  void free_device();
  int upload_state();
  int upload_params();
  int alloc_device32();
  int to_surface(bool cur_only, int field = -1);  // field 0..2: that state field only
  int to_depth(bool full);
  int pull_state(bool full);
  void sync_args32();
  int check_device_error();
  int upload_forcing();
  int run(int mode, double target, int nsteps);
  int prepare_run(int mode, double target, int nsteps);
  cudaGraphExec_t graph_for(int steps);
  void pull_ctl();
  void init_condition();

  size_t ncell_ = 0;
  double* hf_[7] = {};  // pinned host fields
  std::vector<double> forcing_[6];  // wind_x, wind_y, atm, precip, heat_flux, e-p (contiguous)
  std::vector<double> eta_old_[4];
  bool forcing_dev_ = false;

  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  void* dmem_ = nullptr;
  StepArgs args_{};
  TileMaps maps_{};  // TMA maps of the state buffers (args_.maps points here when encoded)
  int tma_status_ = -1;  // encode_tile_maps' result (-1: no device buffers yet)
  StepCtl* hctl_ = nullptr;  // pinned
  // host_is_current_: every host array (state, bed, RK2 saves) equals the
  // device's; host_state_current_: h, hu, hv do (after rki_sync_host).
  bool on_device_ = false, host_is_current_ = false, stepped_ = false;
  bool host_state_current_ = false;
  // Per-field bookkeeping while the device holds the state (fields 0 h, 1 hu,
  // 2 hv, 3 b, 4-6 the RK2 saves): fcur_[f], host array f equals the
  // device's value; handed_[f], a pointer to host array f went out since the
  // last device run, so the caller may have written through it and the next
  // run uploads it (the RK2 saves are rewritten by every step and are not).
  bool fcur_[7] = {};
  bool handed_[7] = {};
  void mark_host_stale() {
    host_is_current_ = host_state_current_ = false;
    for (bool& f : fcur_) f = false;
  }
  void mark_host_current() {
    host_is_current_ = host_state_current_ = true;
    for (bool& f : fcur_) f = true;
  }
  bool field_current(int f) const {
    return host_is_current_ || fcur_[f] || (f <= 2 && host_state_current_);
  }
  // Caller's (nx, ny) interior rows -> device rows starting at `dst` (pitch
  // in elements), through two pinned staging buffers: host threads copy one
  // chunk of rows while the previous chunk's DMA runs.
  int upload_rows(double* dst, const double* src, int nx, int ny);
  int pull_field(int f);      // device -> host array f (FP32: through the depth form)
  int pull_missing(int upto);  // every field f < upto whose host array is not current
  int push_field(int f);      // host array f -> device (f <= 3)
  int cur_ = 0;
  double t_current_ = 0.0, dt_ = 0.0;
  int step_count_ = 0;
  int precision_ = 64;
  std::string err_text_;

  // FP32 surface form: one more allocation, same control/parameter blocks
  void* dmem32_ = nullptr;
  StepArgs32 args32_{};
  int auto_rows_[2] = {0, 0};  // automatic rows for 2 and 4 columns per lane
  StepCtl snap_ctl_{};
  int snap_cur_ = 0, snap_steps_ = 0;
  double snap_t_ = 0.0, snap_dt_ = 0.0;
  bool snap_stepped_ = false;

  // gauges
  void drop_graphs();
  void* gauge_mem_ = nullptr;
  GaugeDev* gauge_dev_ = nullptr;
  GaugeDev gauge_host_{};
  std::vector<int> gauge_station_;
  std::vector<double> gauge_b_;
  int gauge_gen_ = 0;
  GaugeDev snap_gauge_{};  // recorder state at the last snapshot

  struct GraphEntry {
    int steps, hllc, tile, prec, rows, plain;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs_;
};

}  // namespace rkb
