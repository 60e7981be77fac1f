/*
 * librakali.so (B200 build): C ABI of the structured 2D shallow-water step.
 *
 * Part 1 is the drop-in boundary: every symbol the reference's Python
 * wrapper binds at import (python/rakali/_core.py:88-283), with the
 * reference's signatures and return codes (src/api/rki_api.F90:157-1507).
 * The unmodified `rakali` package loads this library through RAKALI_LIB.
 *
 * Return codes (src/api/rki_api.F90:22-27):
 *     0  success
 *    -1  not initialised / not finalised / device failure
 *    -2  grid mismatch / already finalised / invalid namelist value
 *    -3  mode not active (multilayer, restart, unsupported solver mode)
 *  -100  invalid handle (null, destroyed or foreign pointer)
 * Invalid configurations return an error code (the reference stops the
 * process); rki_last_error() gives the message.
 *
 * Field pointers are host memory owned by the library, Fortran order
 * (nx_total, ny_total) with ghost cells, valid until rki_destroy.
 *
 * Part 2 adds entry points with no counterpart in the reference: kernel-level
 * calls on caller-owned device arrays (mirroring the structured kernels of
 * src/core/coastal/kernels/structured/barotropic), device-resident views for
 * zero-copy torch interop, and diagnostics.
 */
#ifndef RAKALI_B200_H
#define RAKALI_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: reference C ABI ------------------------------------------ */

/* rki_api.F90:157-167 */
int rki_working_precision(void);

/* rki_api.F90:169-217; a missing file keeps the defaults, as the reference. */
int rki_create(const char *filename, int len, void **handle);
/* rki_api.F90:219-259 */
int rki_finalize(void *handle);
/* rki_api.F90:261-272 */
int rki_create_from_namelist(const char *filename, int len, void **handle);
/* rki_api.F90:274-313 */
int rki_create_from_string(const char *text, int len, void **handle);
/* rki_api.F90:315-326 */
int rki_create_from_namelist_string(const char *text, int len, void **handle);
/* rki_api.F90:328-356 (nulls *handle; idempotent) */
void rki_destroy(void **handle);

/* rki_api.F90:358-383: n steps, each capped at t_end - t */
int rki_step(void *handle, int n_steps);
/* rki_api.F90:385-410: steps while t < target - 1e-10, last one capped */
int rki_advance(void *handle, double target_time);

/* rki_api.F90:412-498 */
double rki_get_time(void *handle);
double rki_get_dt(void *handle);
void rki_get_grid_info(void *handle, int *nx, int *ny, int *nghost, double *dx, double *dy);
int rki_get_step_count(void *handle);
int rki_get_nz_ml(void *handle);

/* rki_api.F90:502-698: zero-copy host views, (nx_total, ny_total) F-order */
int rki_get_h_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_hu_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_hv_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_b_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_h0_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_hu0_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);
int rki_get_hv0_ptr(void *handle, void **ptr, int *nx_total, int *ny_total);

/* rki_api.F90:702-834: multilayer fields (return -1: multilayer not active) */
int rki_get_h_layer_ptr(void *handle, void **ptr, int *nx_total, int *ny_total, int *nz);
int rki_get_hu_layer_ptr(void *handle, void **ptr, int *nx_total, int *ny_total, int *nz);
int rki_get_hv_layer_ptr(void *handle, void **ptr, int *nx_total, int *ny_total, int *nz);
int rki_get_salinity_ptr(void *handle, void **ptr, int *nx_total, int *ny_total, int *nz);
int rki_get_temperature_ptr(void *handle, void **ptr, int *nx_total, int *ny_total, int *nz);

/* rki_api.F90:836-890 (pre-finalize fields, interior (nx, ny) F-order) */
int rki_set_bathymetry(void *handle, const double *b, int nx, int ny);
int rki_set_initial_h(void *handle, const double *h, int nx, int ny);

/* rki_api.F90:896-1036 (forcing; wind/pressure/precipitation activate it) */
int rki_set_wind(void *handle, const double *wx, const double *wy, int nx, int ny);
int rki_set_atm_pressure(void *handle, const double *p, int nx, int ny);
int rki_set_precipitation(void *handle, const double *p, int nx, int ny);
int rki_set_heat_flux(void *handle, const double *q, int nx, int ny);
int rki_set_evap_minus_precip(void *handle, const double *ep, int nx, int ny);

/* rki_api.F90:1040-1123 (mid-run state injection) */
int rki_set_h(void *handle, const double *h, int nx, int ny);
int rki_set_hu(void *handle, const double *hu, int nx, int ny);
int rki_set_hv(void *handle, const double *hv, int nx, int ny);
/* rki_api.F90:1125-1199 (multilayer tracers: -3 when not multilayer) */
int rki_set_salinity(void *handle, const double *s, int nx, int ny, int nz);
int rki_set_temperature(void *handle, const double *t, int nx, int ny, int nz);

/* rki_api.F90:1205-1303 (boundary scalars) */
int rki_set_inflow_velocity(void *handle, double v);
int rki_set_inflow_salinity(void *handle, double s);
int rki_set_inflow_temperature(void *handle, double t);
int rki_set_discharge_flux(void *handle, double q);
int rki_set_clamped_elevation(void *handle, double eta);
double rki_get_clamped_elevation(void *handle);
double rki_get_manning_n(void *handle);
double rki_get_coriolis_f(void *handle);
/* rki_api.F90:1335-1366 */
int rki_set_tidal_constituents(void *handle, const double *amp, const double *phase,
                               const double *omega, int n);

/* rki_api.F90:1372-1403 */
void rki_sync_host(void *handle);
void rki_sync_from_device(void *handle);

/* rki_api.F90:1409-1471: restart files.  save (finalised handle) writes
 * interior h, hu, hv, b and the time as NetCDF classic (64-bit offset);
 * load (before finalize) restores them and the clock; -3 on a grid
 * mismatch or an unreadable file (NetCDF-4/HDF5 containers included). */
int rki_save_restart(void *handle, const char *filename, int len);
int rki_load_restart(void *handle, const char *filename, int len);

/* Replaces the reference front end's Rakali.save_checkpoint
 * (python/rakali/_core.py:1433-1499, written there through xarray): a per-step
 * checkpoint of a finalised handle with every field including ghosts (h, hu,
 * hv, b and the RK2 saves h0, hu0, hv0 over dimensions x_total, y_total) and
 * the clock, grid and physics scalars as global attributes, in a NetCDF
 * classic (64-bit offset) file.  The device state stays canonical.  -1 not
 * initialised, -2 not finalised, -3 on an empty name or a failed write. */
int rkb_save_checkpoint(void *handle, const char *filename, int len);

/* rki_api.F90:1473-1507 */
int rki_set_use_ppm_tracer(void *handle, int flag);
int rki_set_use_hllc(void *handle, int flag);

/* ---- Part 2: additions (no counterpart in the reference) ---------------- */

/* Message of the last failed call on this thread ("" if none). */
const char *rki_last_error(void);

/* Parse + validate a namelist without a GPU: 0, -2 or -3 as rki_create. */
int rkb_validate_namelist(const char *text, int len, char *err, int err_len);

/* Boundary volume budget: out[0] = mass_out, out[1] = mass_src
 * (rki_solver.F90:507-657).  Returns 0 or an error code. */
int rkb_get_mass_budget(void *handle, double *out);

/* Device views of the current state for zero-copy torch interop: ptrs[0..3]
 * = h, hu, hv, b (device, pitched), *pitch in elements.  Valid until the
 * next step (the state ping-pongs between two buffers). */
int rkb_get_device_fields(void *handle, void **ptrs, int *pitch);

/* Kernel shape of the FP64 stage (0: 32x8, 1: 32x16, 2: 64x4, 3: 16x16
 * tiles; 4 / 5: marching strips of 64 / 32 rows; 6 / 7: 32x8 / 32x12 tiles
 * with two extra warps; 8: 16x15 tiles; 9: 32x7 tiles with one extra warp;
 * 10: 16x15 tiles loaded by TMA copies of their halo boxes (the 16x15
 * kernel where its maps cannot be encoded, see rkb_tma_tile_status)).  Results do not depend on the shape.  -2 for any other
 * value. */
int rkb_set_tile(void *handle, int tile);
int rkb_get_tile(void *handle);
/* Whether tile 10 runs TMA-staged on this simulation: 0 yes; -1 not yet
 * finalised; otherwise why not (1 misaligned rows, 2 misaligned buffer, 3 no
 * tensor-map encoder, 100 + a runtime error or 200 + an entry-point query
 * result while finding it, 1000 + the encoder's CUresult).  No counterpart
 * in the reference. */
int rkb_tma_tile_status(void *handle);

/* Arithmetic form of the step: 64 = FP64 depth form (the reference's
 * arithmetic, the default), 32 = FP32 surface form (eta = h + b, hu, hv in
 * FP32; bed differences, wet/dry tests and mass sums in FP64).  May be called
 * before or after rki_finalize; the host views and setters keep their FP64
 * arrays in both forms.  -2 for any other value. */
int rkb_set_precision(void *handle, int bits);
int rkb_get_precision(void *handle);
/* FP32 form: columns per lane of the sweep kernel (0 = default 2, or 2, 4)
 * and rows each warp sweeps (0 = one wave of resident warps).  Results do
 * not depend on either. */
int rkb_set_sweep(void *handle, int cols_per_lane, int rows);
/* Limit, in GPU clock cycles, of the device-side waits for asynchronous
 * copies: the FP32 sweep's bulk row copies and the TMA tile copies of the
 * FP64 TMA-staged tile kernel (tile 10) (<= 0: the default, about one second;
 * a limit shorter than one clock read gives up at once).  A wait that runs out makes the step fail
 * with -1 and a message in rki_last_error(); the copies in flight are still
 * waited for (with the default limit) before the kernel returns.  No
 * counterpart in the reference: it exists so that the error path can be
 * exercised. */
int rkb_set_wait_limit(void *handle, long long cycles);

/* Batches of independent simulations (ensembles of uneven sizes): every
 * member is advanced by one launch per phase covering all members, chunks of
 * steps captured in CUDA graphs; each member keeps its own dt, clock,
 * boundary parameters and host views.  Members must be finalised, share the
 * Riemann solver and be at least max(nghost, 2) cells wide; a simulation
 * belongs to one batch at most.  `precision` (64 or 32) is applied to every
 * member.  Destroying a member makes later calls on the batch return -1. */
int rkb_batch_create(void **handles, int n, int precision, void **batch);
void rkb_batch_destroy(void **batch);
int rkb_batch_step(void *batch, int n_steps);
int rkb_batch_advance(void *batch, double target_time);
/* n steps of every member between CUDA events on the batch's stream. */
int rkb_batch_time_steps(void *batch, int n, double *ms);
/* n steps of every member launched phase by phase with CUDA events between
 * the launches: out5[0..3] = mean ms per step of the stage-1 boundary fills,
 * stage 1, the stage-2 fills and stage 2; out5[4] = mean ms per step of the
 * whole sequence.  Set beside rkb_batch_time_steps (the same steps replayed
 * from CUDA graphs) it shows what the launches themselves cost. */
int rkb_batch_profile_steps(void *batch, int n, double *out5);
/* Times each candidate kernel shape (FP64: the shared-memory tiles; FP32: 2 or 4
 * columns per lane x rows per warp sweep) for trial_steps steps on the live
 * state, restores the state exactly, keeps the fastest shape. */
int rkb_batch_autotune(void *batch, int trial_steps, double *best_ms_per_step);
/* Kernel shape in use: FP64 (tile, 0); FP32 (columns per lane, rows). */
int rkb_batch_variant(void *batch, int *a, int *b);
/* Sets the kernel shape without trials: FP64 (a shared-memory tile: 0-3,
 * 6-10; tile 10, TMA-staged, needs every member's tensor maps and otherwise
 * runs the 16x15 kernel), 0); FP32 (2 or 4 columns per lane, rows per warp
 * sweep >= 0, 0 = one wave of resident warps).  -2 for any other shape. */
int rkb_batch_set_variant(void *batch, int a, int b);

/* Gauge-misfit adjoint of the FP64 step (walls, HLL or HLLC, Manning
 * friction with a per-cell n field).  J = sum over steps 1..n_steps and the
 * gauges of (h + b - obs)^2 on a fixed dt sequence; gradients by
 * hand-written reverse kernels with sqrt(n_steps) checkpointing (or every
 * state kept in device memory, rkb_adjoint_set_state_budget).  Interior
 * arrays are (nx, ny) Fortran order on the host; gauges are interior
 * (i, j), 0-based, distinct; obs is (n_steps, n_gauges) row-major. */
int rkb_adjoint_create(int nx, int ny, int nghost, double dx, double dy, double cfl, int use_hllc,
                       int n_steps, const double *h0, const double *hu0, const double *hv0,
                       const int *gauge_i, const int *gauge_j, int n_gauges, void **adj);
void rkb_adjoint_destroy(void **adj);
int rkb_adjoint_set_obs(void *adj, const double *obs);
int rkb_adjoint_set_dt(void *adj, const double *dts);
int rkb_adjoint_get_dt(void *adj, double *dts);
/* Forward run: record_dt != 0 takes CFL steps and stores them (else the
 * stored sequence is replayed).  n_field may be NULL (uniform n_scalar).
 * eta_gauges (optional) receives (n_steps, n_gauges) surfaces. */
int rkb_adjoint_forward(void *adj, const double *b, const double *n_field, double n_scalar,
                        int record_dt, double *J, double *eta_gauges);
/* J and dJ/db, dJ/dn (interior (nx, ny) arrays) on the stored dt sequence. */
int rkb_adjoint_gradient(void *adj, const double *b, const double *n_field, double n_scalar,
                         double *J, double *grad_b, double *grad_n);
/* 1 once a gradient run kept every state, else the sqrt(n_steps) interval. */
int rkb_adjoint_checkpoint_interval(void *adj);
/* Device bytes a gradient run may allocate to keep every state U^0..U^N
 * (3 (N + 1) fields) instead of recomputing them from sqrt(N) checkpoints:
 * 0 (the default) never, < 0 half the free device memory at that run.  The
 * gradients are the same bits either way.  No counterpart in the reference. */
int rkb_adjoint_set_state_budget(void *adj, long long bytes);
/* Device milliseconds of the last forward / gradient call (CUDA events). */
double rkb_adjoint_last_ms(void *adj);
/* A batch of n_members equally sized problems advanced together (every
 * kernel launch covers all members), in FP64 (precision 64) or FP32 (32;
 * misfit and mass sums stay FP64).  Per-member arrays are stacked member by
 * member: h0/hu0/hv0/b/n_field/grad_* are (n_members, nx*ny) with each
 * member Fortran-ordered, gauge_i/j are (n_members, n_gauges), obs and
 * eta_gauges are (n_steps, n_members, n_gauges), dts (n_members, n_steps),
 * J (n_members).  hu0, hv0 may be NULL (zero).  rkb_adjoint_create is this
 * call with precision 64 and one member; the functions above take either. */
int rkb_adjoint_batch_create(int precision, int n_members, int nx, int ny, int nghost, double dx,
                             double dy, double cfl, int use_hllc, int n_steps, const double *h0,
                             const double *hu0, const double *hv0, const int *gauge_i,
                             const int *gauge_j, int n_gauges, void **adj);
int rkb_adjoint_members(void *adj);
int rkb_adjoint_precision(void *adj);
/* FP64 interior mass sum(h) per member before (out[m]) and after
 * (out[n_members + m]) the last forward run. */
int rkb_adjoint_mass(void *adj, double *out);
/* on != 0: later gradients hold the limited slopes of each state fixed (their
 * adjoints are dropped): not the exact derivative, but one that stays bounded
 * over long windows, where the exact derivative of the minmod limiter grows. */
int rkb_adjoint_set_frozen_slopes(void *adj, int on);
/* Host builds of the face flux / cell update and their adjoints (for
 * finite-difference checks without a GPU). */
void rkb_test_face_flux(int dir, int hllc, const double *in8, double *out6);
void rkb_test_face_adj(int dir, int hllc, const double *in8, const double *gout6, double *gin8);
void rkb_test_cell(const double *in4, double dt, double *out3);
void rkb_test_cell_adj(const double *in4, double dt, const double *gout3, double *gin4);

/* NetCDF classic (64-bit offset) restart codec without a simulation: the
 * variables of rki_save_restart (h, hu, hv, b as (y, x) FP64 with units,
 * scalar time; dimensions x, y; global Conventions, title, source, dx, dy,
 * nghost).  Arrays are interior (nx, ny) Fortran order.  read returns 0,
 * 1 when the file's grid is not nx x ny, -1 when unreadable (NetCDF-4/HDF5
 * containers included), -2 on bad arguments. */
int rkb_restart_write(const char *path, int nx, int ny, const double *h, const double *hu,
                      const double *hv, const double *b, double time, double dx, double dy,
                      int nghost);
int rkb_restart_read(const char *path, int nx, int ny, double *h, double *hu, double *hv,
                     double *b, double *time);
/* The per-step checkpoint codec of rkb_save_checkpoint without a simulation:
 * fields = h, hu, hv, b, h0, hu0, hv0, each (nx_total, ny_total) Fortran order
 * with ghosts; scalars = time, dt, dx, dy, manning_n, coriolis_f,
 * clamped_elevation; counts = step_count, nx_phys, ny_phys, nghost.  0 written,
 * -1 write failed, -2 bad arguments. */
int rkb_checkpoint_write(const char *path, int nx_total, int ny_total,
                         const double *const *fields, const double *scalars, const int *counts);

/* Gauge stencils without a simulation (compute_local_gauges /
 * compute_interp_weights, src/io/structured/rki_gauges.F90:208-336): of the n
 * stations (x, y in metres from the lower-left corner) those inside the
 * nx x ny interior, in order: their index, the 0-based array indices (ghosts
 * included) of the lower-left stencil cell and the clamped bilinear weights.
 * Returns how many stations are inside (arrays hold n entries), -2 on bad
 * arguments. */
int rkb_gauge_stencils(int nx, int ny, int nghost, double dx, double dy, const double *x,
                       const double *y, int n, int *station, int *ix0, int *iy0, double *wx,
                       double *wy);

/* bathymetry_file input (src/io/rki_bathymetry.F90:21-163): variable b,
 * elevation or depth over dimensions x, y (either order) of a NetCDF classic
 * file into an interior (nx, ny) Fortran-order array; return codes as
 * rkb_restart_read.  rki_finalize reads the namelist's bathymetry_file this
 * way unless rki_set_bathymetry was called. */
int rkb_bathymetry_read(const char *path, int nx, int ny, double *b);

/* Gauge stations (src/io/structured/rki_gauges.F90) recorded on the device
 * after every step, without host synchronisation: x, y in metres from the
 * domain's lower-left corner; stations outside the domain are dropped;
 * bilinear stencils and weights as compute_interp_weights (:245-336);
 * interval = gauge_output_interval (s, <= 0: every step) with the driver's
 * cadence (rki_driver.F90:469-473); capacity = records held on the device.
 * Needs a finalised handle; returns the number of stations kept.  n = 0
 * removes the stations. */
int rkb_set_gauges(void *handle, int n, const double *x, const double *y, double interval,
                   int capacity);
/* For the kept stations: station[k] = index in the list given, station_b[k] =
 * bilinear bed (either may be NULL); returns their number. */
int rkb_gauge_stations(void *handle, int *station, double *station_b);
/* Move up to max_records records to the host: times [count], values
 * [count][stations][3] = eta, u, v (gauges_write, :490-575); returns count;
 * *overflow = 1 if records were dropped because the buffer was full. */
int rkb_read_gauges(void *handle, int max_records, double *times, double *values, int *overflow);
/* Write a gauge file in the layout of create_gauge_netcdf (:338-488) as
 * NetCDF classic: names are n fixed-width fields of name_len characters. */
int rkb_write_gauges_netcdf(const char *path, int n, const char *names, int name_len,
                            const double *x, const double *y, const double *b, int n_records,
                            const double *times, const double *values);

/* Run n steps bracketed by CUDA events on the simulation's own stream;
 * *ms = device time of the n steps (state already resident). */
int rkb_time_steps(void *handle, int n, double *ms);
/* Run n steps one launch at a time; out5[0..3] = mean ms per step of the
 * stage-1 boundary fill, stage 1, stage-2 boundary fill, stage 2 (with the
 * close of the step); out5[4] = kernel launches per step. */
int rkb_profile_steps(void *handle, int n, double *out5);

/* Correctly rounded h**fl(1/3) and sin/cos, the host builds of the device
 * functions the step uses for the friction, tidal and Coriolis terms. */
double rkb_cr_pow_third(double h);
void rkb_cr_sincos(double x, double *sn, double *cs);

/*
 * Kernel-level entry points on caller-owned DEVICE arrays, Fortran order
 * with leading dimension `ld` (>= nx_total).  All run on the current
 * device's legacy default stream and synchronise before returning.
 */
/* compute_flux_hll / compute_flux_hllc (rki_kernel_flux.F90:17-102):
 * flux divergence and per-face HLL mass fluxes of every interior cell. */
int rkb_compute_flux(int use_hllc, const double *h, const double *hu, const double *hv,
                     const double *b, double *flux_h, double *flux_hu, double *flux_hv,
                     double *mass_flux_x, double *mass_flux_y, int nx_total, int ny_total,
                     int nghost, int ld, double dx, double dy);

/* compute_timestep (rki_kernel_timestep.F90:16-74): *dt_out on the host. */
int rkb_compute_timestep(const double *h, const double *hu, const double *hv, int nx_total,
                         int ny_total, int nghost, int ld, double dx, double dy, double cfl,
                         double *dt_out);

/* The remaining structured kernels of src/core/coastal, one entry point each,
 * on caller-owned device arrays in the same layout.  Each updates the
 * interior cells nghost .. n_total - nghost - 1 in place, with the
 * reference's arithmetic (bit-identical results); ghosts are left as they
 * are.  Optional forcing arrays (wind_x, wind_y, atm, precip) may be NULL
 * only when forcing_active is 0.  Returns 0, -2 for bad arguments, -1 for a
 * CUDA error. */

/* fused_update_stage1 (rki_kernel_fused.F90:164-303): (h0, hu0, hv0) <- U,
 * U <- U + dt F, clamp / KP07 / Froude backstop, Manning friction, wind,
 * pressure gradient, Coriolis rotation, precipitation. */
int rkb_fused_update_stage1(double *h, double *hu, double *hv, double *h0, double *hu0,
                            double *hv0, const double *flux_h, const double *flux_hu,
                            const double *flux_hv, int nx_total, int ny_total, int nghost, int ld,
                            double dx, double dy, double dt, double manning_n,
                            const double *wind_x, const double *wind_y, const double *atm,
                            const double *precip, double coriolis_f, int forcing_active);
/* fused_update_stage2 (rki_kernel_fused.F90:305-471): the stage-1 update
 * without the save, then U <- (U0 + U) / 2 and a second clamp. */
int rkb_fused_update_stage2(double *h, double *hu, double *hv, const double *h0,
                            const double *hu0, const double *hv0, const double *flux_h,
                            const double *flux_hu, const double *flux_hv, int nx_total,
                            int ny_total, int nghost, int ld, double dx, double dy, double dt,
                            double manning_n, const double *wind_x, const double *wind_y,
                            const double *atm, const double *precip, double coriolis_f,
                            int forcing_active);
/* fused_update_stage_generic (rki_kernel_fused.F90:22-162): one Euler stage
 * of the selectable schemes (dt = beta_k dt_step), no save, no average. */
int rkb_fused_update_stage_generic(double *h, double *hu, double *hv, const double *flux_h,
                                   const double *flux_hu, const double *flux_hv, int nx_total,
                                   int ny_total, int nghost, int ld, double dx, double dy,
                                   double dt, double manning_n, const double *wind_x,
                                   const double *wind_y, const double *atm,
                                   const double *precip, double coriolis_f, int forcing_active);
/* compute_update (rki_kernel_update.F90:35-96): U <- U + dt F, then clamp. */
int rkb_compute_update(double *h, double *hu, double *hv, const double *flux_h,
                       const double *flux_hu, const double *flux_hv, int nx_total, int ny_total,
                       int nghost, int ld, double dt);
/* compute_rk2_average (rki_kernel_update.F90:98-150): U <- (U0 + U) / 2,
 * then clamp. */
int rkb_compute_rk2_average(double *h, double *hu, double *hv, const double *h0,
                            const double *hu0, const double *hv0, int nx_total, int ny_total,
                            int nghost, int ld);
/* compute_ssp_combine (rki_kernel_update.F90:152-208):
 * U <- a_n U0 + (1 - a_n) U, then clamp. */
int rkb_compute_ssp_combine(double *h, double *hu, double *hv, const double *h0,
                            const double *hu0, const double *hv0, double a_n, int nx_total,
                            int ny_total, int nghost, int ld);
/* apply_friction (rki_kernel_friction.F90:16-113): semi-implicit Manning
 * friction, then (forcing_active) wind stress (include_wind), pressure
 * gradient and precipitation; the reference's optional forcing_active and
 * include_wind default to 1 there and are explicit here. */
int rkb_apply_friction(double *h, double *hu, double *hv, int nx_total, int ny_total, int nghost,
                       int ld, double dx, double dy, double dt, double manning_n,
                       const double *wind_x, const double *wind_y, const double *atm,
                       const double *precip, int forcing_active, int include_wind);
/* apply_coriolis (rki_kernel_friction.F90:115-152): exact rotation of
 * (hu, hv) by f dt in wet cells. */
int rkb_apply_coriolis(const double *h, double *hu, double *hv, int nx_total, int ny_total,
                       int nghost, int ld, double dt, double f);

/* bc_params_t (src/core/structured/rki_boundary_types.F90:38-100) as the
 * boundary and sponge kernels read it.  type[]: west, east, south, north,
 * 1 wall, 2 open, 3 tidal, 4 nested, 5 inflow, 6 discharge, 7 clamped,
 * 8 sponge, 9 chapman (rki_boundary_types.F90:19-36).  eta_old[]: the
 * Chapman surfaces of the four edges, device arrays of ny_total (W, E) or
 * nx_total (S, N) doubles, read and refreshed by the fill (NULL where the
 * edge is not Chapman). */
#define RKB_MAX_TIDAL 10
typedef struct {
  int type[4];
  int n_tidal;
  int sponge_width;
  double tidal_amplitude, tidal_period;
  double tidal_amp[RKB_MAX_TIDAL], tidal_phase[RKB_MAX_TIDAL], tidal_omega[RKB_MAX_TIDAL];
  double inflow_velocity, discharge_flux, clamped_elevation;
  double sponge_strength, sponge_h_ref;
  double time;  /* bc%time: the boundary clock of this fill */
  double dt;    /* bc%dt: the step the Chapman condition uses */
  double *eta_old[4];
} rkb_bc_params;

/* apply_boundary_conditions (rki_boundary.F90:40-218): ghost layers of the
 * W, E, S, N edges in that order; wall and sponge edges also mirror the bed
 * b into their ghosts. */
int rkb_apply_boundary_conditions(double *h, double *hu, double *hv, double *b, int nx_total,
                                  int ny_total, int nghost, int ld, double dx, double dy,
                                  const rkb_bc_params *bc);
/* apply_sponge (rki_kernel_sponge.F90:16-88): relaxation towards
 * (sponge_h_ref, 0, 0) within sponge_width cells of sponge edges. */
int rkb_apply_sponge(double *h, double *hu, double *hv, int nx_total, int ny_total, int nghost,
                     int ld, double dt, const rkb_bc_params *bc);

/* No counterpart in the reference.  The same dt as rkb_compute_timestep for
 * callers that cannot allocate device memory when they need it: a host
 * application whose memory pool already owns the GPU, or a driver loop that
 * must not block (cudaMalloc/cudaFree synchronise the device).  It allocates
 * nothing: its scratch is a fixed array inside the library (2 doubles per
 * interior row plus one, for at most 32768 interior rows; about 512 KB on
 * every GPU that loads the library, held until exit).  More rows return -2
 * with the reason in rki_last_error().  Each call looks up the array's
 * device address with the caller's device current, so a device reset or a
 * new context is followed; the first call on a device may load the
 * library's GPU code, so make it before any stream capture.  There is one
 * array per GPU and every call uses it: calls that overlap on the GPU (other
 * host threads, other streams) race, so serialise them.  The result is read
 * back before returning. */
int rkb_compute_timestep_noalloc(const double *h, const double *hu, const double *hv,
                                 int nx_total, int ny_total, int nghost, int ld, double dx,
                                 double dy, double cfl, double *dt_out);

#ifdef __cplusplus
}
#endif
#endif
