/*
 * CPU oracle for the structured 2D shallow-water SSP-RK2 step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the Fortran
 * reference kernels, used by tests/, by __graft_entry__.smoke() and by the
 * cpu_baseline leg of bench.py as the checker.  The product library never
 * links or calls it.
 *
 * Every array is Fortran order (column-major), shape (nx_total, ny_total),
 * ghost cells included: element (i, j) with 0-based i, j lives at
 * a[i + j*nx_total].  The reference's 1-based interior range
 * nghost+1 .. n_total-nghost becomes 0-based nghost .. n_total-nghost-1.
 *
 * Arithmetic follows the reference expression by expression (left-to-right
 * evaluation, no contraction: build with -ffp-contract=off).
 */
#ifndef SWE_ORACLE_H
#define SWE_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary-condition tags (src/core/structured/rki_boundary_types.F90:19-36). */
enum {
  ORC_BC_WALL = 1, ORC_BC_OPEN = 2, ORC_BC_TIDAL = 3, ORC_BC_NESTED = 4,
  ORC_BC_INFLOW = 5, ORC_BC_DISCHARGE = 6, ORC_BC_CLAMPED = 7,
  ORC_BC_SPONGE = 8, ORC_BC_CHAPMAN = 9
};

#define ORC_MAX_TIDAL 10

/* Boundary parameters (rki_boundary_types.F90:38-100, bc_params_t). */
typedef struct {
  int west, east, south, north;
  int n_tidal;
  int sponge_width;
  double tidal_amplitude, tidal_period, time;
  double tidal_amp[ORC_MAX_TIDAL], tidal_phase[ORC_MAX_TIDAL], tidal_omega[ORC_MAX_TIDAL];
  double inflow_velocity, discharge_flux, clamped_elevation;
  double sponge_strength, sponge_h_ref;
  double dx, dy, dt;
  /* Chapman persistent surfaces; length ny_total (W/E) and nx_total (S/N). */
  double *eta_old_west, *eta_old_east, *eta_old_south, *eta_old_north;
} orc_bc;

/* One simulation (state_t + the handle's clock, reduced to the 2D path).
 * All arrays are caller-owned, nx_total*ny_total doubles. */
typedef struct {
  int nx, ny, ng;              /* nx_total, ny_total, nghost */
  double dx, dy;
  double cfl, dt, dt_fixed;
  int cfl_interval, step_count;
  int use_hllc;
  int time_scheme;             /* 1 euler, 2 rk2, 3 rk3, 4 rk43 */
  double manning_n, coriolis_f;
  int forcing_active;
  double t_current, t_end;
  double mass_out, mass_src;
  double *h, *hu, *hv, *b;
  double *flux_h, *flux_hu, *flux_hv, *mflux_x, *mflux_y;
  double *h0, *hu0, *hv0;
  double *wind_x, *wind_y, *atm, *precip;
  orc_bc bc;
} orc_sim;

/* OpenMP thread count for timing runs; returns the count in effect. */
int orc_set_threads(int n);

/* Correctly rounded h**(1/3) (as h**fl(1/3)), sin, cos (crmath.c): the
 * platform-independent values of the reference's libm calls. */
double orc_cr_pow_third(double h);
double orc_cr_sin(double x);
double orc_cr_cos(double x);
void orc_cr_sincos(double x, double *sn, double *cs);

/* rki_kernel_flux.F90:17-102 (compute_flux_hll / compute_flux_hllc). */
void orc_compute_flux(int use_hllc, const double *h, const double *hu, const double *hv,
                      const double *b, double *flux_h, double *flux_hu, double *flux_hv,
                      double *mflux_x, double *mflux_y, int nx, int ny, int ng,
                      double dx, double dy);

/* rki_kernel_fused.F90:164-303 / :305-471 / :22-162. */
void orc_fused_stage1(double *h, double *hu, double *hv, double *h0, double *hu0, double *hv0,
                      const double *fh, const double *fhu, const double *fhv,
                      int nx, int ny, int ng, double dx, double dy, double dt, double manning_n,
                      const double *wind_x, const double *wind_y, const double *atm,
                      const double *precip, double coriolis_f, int forcing_active);
void orc_fused_stage2(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                      const double *hv0, const double *fh, const double *fhu, const double *fhv,
                      int nx, int ny, int ng, double dx, double dy, double dt, double manning_n,
                      const double *wind_x, const double *wind_y, const double *atm,
                      const double *precip, double coriolis_f, int forcing_active);
void orc_fused_stage_generic(double *h, double *hu, double *hv,
                             const double *fh, const double *fhu, const double *fhv,
                             int nx, int ny, int ng, double dx, double dy, double dt,
                             double manning_n, const double *wind_x, const double *wind_y,
                             const double *atm, const double *precip, double coriolis_f,
                             int forcing_active);

/* rki_kernel_update.F90:35-208. */
void orc_compute_update(double *h, double *hu, double *hv, const double *fh, const double *fhu,
                        const double *fhv, int nx, int ny, int ng, double dt);
void orc_rk2_average(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                     const double *hv0, int nx, int ny, int ng);
void orc_ssp_combine(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                     const double *hv0, double a_n, int nx, int ny, int ng);

/* rki_kernel_friction.F90:16-152 (unfused friction/forcing, Coriolis). */
void orc_apply_friction(double *h, double *hu, double *hv, int nx, int ny, int ng, double dx,
                        double dy, double dt, double manning_n, const double *wind_x,
                        const double *wind_y, const double *atm, const double *precip,
                        int forcing_active, int include_wind);
void orc_apply_coriolis(const double *h, double *hu, double *hv, int nx, int ny, int ng,
                        double dt, double f);

/* rki_kernel_timestep.F90:16-74: returns dt; *max_speed_out gets the reduction. */
double orc_compute_timestep(const double *h, const double *hu, const double *hv, int nx, int ny,
                            int ng, double dx, double dy, double cfl, double *max_speed_out);

/* rki_boundary.F90:40-552 (edges W, E, S, N in order). */
void orc_apply_bc(double *h, double *hu, double *hv, double *b, int nx, int ny, int ng,
                  orc_bc *bc);
/* Tidal surface for the current bc->time (rki_boundary.F90:92-101). */
double orc_tidal_eta(const orc_bc *bc);

/* rki_kernel_sponge.F90:16-88. */
void orc_apply_sponge(double *h, double *hu, double *hv, int nx, int ny, int ng, double dt,
                      const orc_bc *bc);

/* src/io/rki_bathymetry.F90:165-196. */
void orc_fill_bathymetry_ghosts(double *b, int nx, int ny, int ng);

/* src/core/rki_init.F90:29-194. */
void orc_init_dam_break(orc_sim *s);
void orc_init_gaussian_hump(orc_sim *s, double h0, double amp, double sigma, double xoff,
                            double yoff);
void orc_init_castro_dam_break(orc_sim *s);
void orc_init_still_water(orc_sim *s, double eta0);
/* rki_boundary_types.F90:156-202 (seed Chapman surfaces). */
void orc_bc_init_chapman(orc_sim *s);

/* src/core/rki_init.F90:287-316. */
double orc_total_mass(const orc_sim *s);

/* rki_solver.F90:659-926: one step, dt capped by dt_max (pass a huge value
 * for "no cap"), BC clock set to `time`. */
void orc_solver_step(orc_sim *s, double dt_max, double time);
/* src/api/rki_api.F90:358-410. */
void orc_step_n(orc_sim *s, int n);
void orc_advance(orc_sim *s, double target_time);

#ifdef __cplusplus
}
#endif
#endif
