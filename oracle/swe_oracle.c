/*
 * CPU oracle: plain-C restatement of the reference's structured 2D
 * barotropic step.  TEST INFRASTRUCTURE ONLY (see swe_oracle.h).
 *
 * Each function names the Fortran routine (file:line, paths relative to the
 * reference project root) it restates.  Loops keep the reference's structure
 * (cell-centred, every interior face evaluated twice, one pass per kernel)
 * so the oracle stays an independent check of the fused GPU kernels.
 */
#include "swe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Thread count for the OpenMP loops (cpu_baseline timing); results do not
 * depend on it because every parallel loop writes disjoint cells. */
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

/* src/core/rki_constants.F90:38-157 */
static const double G = 9.80665;
static const double RHO = 1035.0;
static const double DRY = 1.0e-6;
static const double THIN = 1.0e-3;
static const double FR_BACK = 50.0;
/* DESING_EPS = 1.5e-4; its 4th power folded at compile time (correctly rounded). */
static const double EPS4 = 5.062499999999998e-16;
static const double SQRT2 = 1.4142135623730951;
static const double TWO_PI_C = 6.283185307179586;

#define AT(a, i, j) (a)[(size_t)(i) + (size_t)(j) * (size_t)nx]

/* ---------------------------------------------------------------------- */
/* Flux kernel: rki_kernel_flux.F90                                       */
/* ---------------------------------------------------------------------- */

/* minmod, rki_kernel_flux.F90:380-393 */
static double minmod(double a, double b) {
  if (a * b <= 0.0) return 0.0;
  if (fabs(a) < fabs(b)) return a;
  return b;
}

/* extract_velocity, rki_kernel_flux.F90:395-408 */
static void velocity(double hv_, double qx, double qy, double *u, double *v) {
  if (hv_ > DRY) {
    *u = qx / hv_;
    *v = qy / hv_;
  } else {
    *u = 0.0;
    *v = 0.0;
  }
}

/* Wave-speed bounds shared by HLL/HLLC (rki_kernel_flux.F90:438-467).
 * `un_*` is the face-normal velocity of each side. */
static void wave_speeds(double hl, double hr, double unl, double unr, double *sl, double *sr) {
  double al = sqrt(G * fmax(hl, 0.0));
  double ar = sqrt(G * fmax(hr, 0.0));
  /* fmax(x, 0) equals Fortran max(x, 0.0) for every non-NaN x. */
  if (hr <= DRY) {
    *sl = unl - al;
    *sr = unl + 2.0 * al;
  } else if (hl <= DRY) {
    *sl = unr - 2.0 * ar;
    *sr = unr + ar;
  } else {
    double a = unl - al, b = unr - ar;
    double c = unl + al, d = unr + ar;
    *sl = (a < b) ? a : b;
    *sr = (c > d) ? c : d;
  }
}

/*
 * HLL / HLLC across one face.  dir=0: x-face (normal momentum is the 2nd
 * component), dir=1: y-face (normal momentum is the 3rd component).
 * hll_flux_x :410-495, hll_flux_y :497-582, hllc_flux_x :584-684,
 * hllc_flux_y :686-783.
 */
static void riemann(int dir, int hllc, double hl, double qxl, double qyl, double hr, double qxr,
                    double qyr, double *fh, double *fqx, double *fqy) {
  double ul, vl, ur, vr;
  velocity(hl, qxl, qyl, &ul, &vl);
  velocity(hr, qxr, qyr, &ur, &vr);
  double sl, sr;
  if (dir == 0)
    wave_speeds(hl, hr, ul, ur, &sl, &sr);
  else
    wave_speeds(hl, hr, vl, vr, &sl, &sr);

  double l_h, l_x, l_y, r_h, r_x, r_y;
  if (dir == 0) {
    l_h = qxl;
    l_x = qxl * ul + 0.5 * G * hl * hl;
    l_y = qxl * vl;
    r_h = qxr;
    r_x = qxr * ur + 0.5 * G * hr * hr;
    r_y = qxr * vr;
  } else {
    l_h = qyl;
    l_x = qxl * vl;
    l_y = qyl * vl + 0.5 * G * hl * hl;
    r_h = qyr;
    r_x = qxr * vr;
    r_y = qyr * vr + 0.5 * G * hr * hr;
  }

  if (sl >= 0.0) {
    *fh = l_h; *fqx = l_x; *fqy = l_y;
    return;
  }
  if (sr <= 0.0) {
    *fh = r_h; *fqx = r_x; *fqy = r_y;
    return;
  }
  double inv = 1.0 / (sr - sl);
  *fh = (sr * l_h - sl * r_h + sl * sr * (hr - hl)) * inv;
  if (dir == 0) {
    *fqx = (sr * l_x - sl * r_x + sl * sr * (qxr - qxl)) * inv;
    if (!hllc) {
      *fqy = (sr * l_y - sl * r_y + sl * sr * (qyr - qyl)) * inv;
    } else {
      double den = hr * (ur - sr) - hl * (ul - sl);
      double ss;
      if (fabs(den) > DRY)
        ss = (sl * hr * (ur - sr) - sr * hl * (ul - sl)) / den;
      else
        ss = 0.5 * (ul + ur);
      *fqy = (ss >= 0.0) ? (*fh) * vl : (*fh) * vr;
    }
  } else {
    *fqy = (sr * l_y - sl * r_y + sl * sr * (qyr - qyl)) * inv;
    if (!hllc) {
      *fqx = (sr * l_x - sl * r_x + sl * sr * (qxr - qxl)) * inv;
    } else {
      double den = hr * (vr - sr) - hl * (vl - sl);
      double ss;
      if (fabs(den) > DRY)
        ss = (sl * hr * (vr - sr) - sr * hl * (vl - sl)) / den;
      else
        ss = 0.5 * (vl + vr);
      *fqx = (ss >= 0.0) ? (*fh) * ul : (*fh) * ur;
    }
  }
}

/*
 * One face from two reconstructed side states (left side L, right side R)
 * with the Audusse hydrostatic reconstruction, rki_kernel_flux.F90:186-224
 * (repeated four times in flux_cell).  Returns the flux and the side depths
 * used by the well-balanced correction.
 */
static void face(int dir, int hllc, double etaL, double qxL, double qyL, double bL, double etaR,
                 double qxR, double qyR, double bR, double *fh, double *fqx, double *fqy,
                 double *hpreL, double *hhydL, double *hpreR, double *hhydR) {
  double hL = fmax(0.0, etaL - bL);
  double hR = fmax(0.0, etaR - bR);
  double bmax = fmax(bL, bR);
  double hyl = fmax(0.0, hL + bL - bmax);
  double hyr = fmax(0.0, hR + bR - bmax);
  double ul, vl, ur, vr;
  velocity(hL, qxL, qyL, &ul, &vl);
  velocity(hR, qxR, qyR, &ur, &vr);
  riemann(dir, hllc, hyl, hyl * ul, hyl * vl, hyr, hyr * ur, hyr * vr, fh, fqx, fqy);
  *hpreL = hL;
  *hhydL = hyl;
  *hpreR = hR;
  *hhydR = hyr;
}

/*
 * flux_cell, rki_kernel_flux.F90:104-378: net flux divergence of cell
 * (i, j) plus its four HLL mass fluxes.
 */
static void flux_cell(int hllc, const double *h, const double *hu, const double *hv,
                      const double *b, int nx, int i, int j, double dx, double dy, double *o_fh,
                      double *o_fhu, double *o_fhv, double *mxl, double *mxr, double *myb,
                      double *myt) {
  const double half_g = 0.5 * G;
  double e_c = AT(h, i, j) + AT(b, i, j);
  double e_im1 = AT(h, i - 1, j) + AT(b, i - 1, j);
  double e_ip1 = AT(h, i + 1, j) + AT(b, i + 1, j);
  double e_im2 = AT(h, i - 2, j) + AT(b, i - 2, j);
  double e_ip2 = AT(h, i + 2, j) + AT(b, i + 2, j);
  double e_jm1 = AT(h, i, j - 1) + AT(b, i, j - 1);
  double e_jp1 = AT(h, i, j + 1) + AT(b, i, j + 1);
  double e_jm2 = AT(h, i, j - 2) + AT(b, i, j - 2);
  double e_jp2 = AT(h, i, j + 2) + AT(b, i, j + 2);

  double se_x, su_x, sv_x, se_y, su_y, sv_y;
  if (AT(h, i, j) < THIN || AT(h, i - 1, j) < DRY || AT(h, i + 1, j) < DRY) {
    se_x = su_x = sv_x = 0.0;
  } else {
    se_x = minmod(e_c - e_im1, e_ip1 - e_c);
    su_x = minmod(AT(hu, i, j) - AT(hu, i - 1, j), AT(hu, i + 1, j) - AT(hu, i, j));
    sv_x = minmod(AT(hv, i, j) - AT(hv, i - 1, j), AT(hv, i + 1, j) - AT(hv, i, j));
  }
  if (AT(h, i, j) < THIN || AT(h, i, j - 1) < DRY || AT(h, i, j + 1) < DRY) {
    se_y = su_y = sv_y = 0.0;
  } else {
    se_y = minmod(e_c - e_jm1, e_jp1 - e_c);
    su_y = minmod(AT(hu, i, j) - AT(hu, i, j - 1), AT(hu, i, j + 1) - AT(hu, i, j));
    sv_y = minmod(AT(hv, i, j) - AT(hv, i, j - 1), AT(hv, i, j + 1) - AT(hv, i, j));
  }

  double sn_e, sn_u, sn_v;
  double fxl_h, fxl_u, fxl_v, fxr_h, fxr_u, fxr_v;
  double fyb_h, fyb_u, fyb_v, fyt_h, fyt_u, fyt_v;
  double dummy1, dummy2;
  double hyd_left, pre_left, hyd_right, pre_right;
  double hyd_bot, pre_bot, hyd_top, pre_top;

  /* left face (i-1/2): neighbour i-1 reconstructs with its own slope */
  if (AT(h, i - 1, j) < THIN || AT(h, i - 2, j) < DRY || AT(h, i, j) < DRY) {
    sn_e = sn_u = sn_v = 0.0;
  } else {
    sn_e = minmod(e_im1 - e_im2, e_c - e_im1);
    sn_u = minmod(AT(hu, i - 1, j) - AT(hu, i - 2, j), AT(hu, i, j) - AT(hu, i - 1, j));
    sn_v = minmod(AT(hv, i - 1, j) - AT(hv, i - 2, j), AT(hv, i, j) - AT(hv, i - 1, j));
  }
  face(0, hllc, e_im1 + 0.5 * sn_e, AT(hu, i - 1, j) + 0.5 * sn_u, AT(hv, i - 1, j) + 0.5 * sn_v,
       AT(b, i - 1, j), e_c - 0.5 * se_x, AT(hu, i, j) - 0.5 * su_x, AT(hv, i, j) - 0.5 * sv_x,
       AT(b, i, j), &fxl_h, &fxl_u, &fxl_v, &dummy1, &dummy2, &pre_left, &hyd_left);

  /* right face (i+1/2) */
  if (AT(h, i + 1, j) < THIN || AT(h, i, j) < DRY || AT(h, i + 2, j) < DRY) {
    sn_e = sn_u = sn_v = 0.0;
  } else {
    sn_e = minmod(e_ip1 - e_c, e_ip2 - e_ip1);
    sn_u = minmod(AT(hu, i + 1, j) - AT(hu, i, j), AT(hu, i + 2, j) - AT(hu, i + 1, j));
    sn_v = minmod(AT(hv, i + 1, j) - AT(hv, i, j), AT(hv, i + 2, j) - AT(hv, i + 1, j));
  }
  face(0, hllc, e_c + 0.5 * se_x, AT(hu, i, j) + 0.5 * su_x, AT(hv, i, j) + 0.5 * sv_x,
       AT(b, i, j), e_ip1 - 0.5 * sn_e, AT(hu, i + 1, j) - 0.5 * sn_u,
       AT(hv, i + 1, j) - 0.5 * sn_v, AT(b, i + 1, j), &fxr_h, &fxr_u, &fxr_v, &pre_right,
       &hyd_right, &dummy1, &dummy2);

  /* bottom face (j-1/2) */
  if (AT(h, i, j - 1) < THIN || AT(h, i, j - 2) < DRY || AT(h, i, j) < DRY) {
    sn_e = sn_u = sn_v = 0.0;
  } else {
    sn_e = minmod(e_jm1 - e_jm2, e_c - e_jm1);
    sn_u = minmod(AT(hu, i, j - 1) - AT(hu, i, j - 2), AT(hu, i, j) - AT(hu, i, j - 1));
    sn_v = minmod(AT(hv, i, j - 1) - AT(hv, i, j - 2), AT(hv, i, j) - AT(hv, i, j - 1));
  }
  face(1, hllc, e_jm1 + 0.5 * sn_e, AT(hu, i, j - 1) + 0.5 * sn_u, AT(hv, i, j - 1) + 0.5 * sn_v,
       AT(b, i, j - 1), e_c - 0.5 * se_y, AT(hu, i, j) - 0.5 * su_y, AT(hv, i, j) - 0.5 * sv_y,
       AT(b, i, j), &fyb_h, &fyb_u, &fyb_v, &dummy1, &dummy2, &pre_bot, &hyd_bot);

  /* top face (j+1/2) */
  if (AT(h, i, j + 1) < THIN || AT(h, i, j) < DRY || AT(h, i, j + 2) < DRY) {
    sn_e = sn_u = sn_v = 0.0;
  } else {
    sn_e = minmod(e_jp1 - e_c, e_jp2 - e_jp1);
    sn_u = minmod(AT(hu, i, j + 1) - AT(hu, i, j), AT(hu, i, j + 2) - AT(hu, i, j + 1));
    sn_v = minmod(AT(hv, i, j + 1) - AT(hv, i, j), AT(hv, i, j + 2) - AT(hv, i, j + 1));
  }
  face(1, hllc, e_c + 0.5 * se_y, AT(hu, i, j) + 0.5 * su_y, AT(hv, i, j) + 0.5 * sv_y,
       AT(b, i, j), e_jp1 - 0.5 * sn_e, AT(hu, i, j + 1) - 0.5 * sn_u,
       AT(hv, i, j + 1) - 0.5 * sn_v, AT(b, i, j + 1), &fyt_h, &fyt_u, &fyt_v, &pre_top,
       &hyd_top, &dummy1, &dummy2);

  /* Divergence with the well-balanced correction, :358-369. */
  *o_fh = -((fxr_h - fxl_h) / dx) - (fyt_h - fyb_h) / dy;
  *o_fhu = -((fxr_u - fxl_u) / dx) - (fyt_u - fyb_u) / dy -
           half_g *
               (hyd_left * hyd_left - pre_left * pre_left - hyd_right * hyd_right +
                pre_right * pre_right) /
               dx;
  *o_fhv = -((fxr_v - fxl_v) / dx) - (fyt_v - fyb_v) / dy -
           half_g *
               (hyd_bot * hyd_bot - pre_bot * pre_bot - hyd_top * hyd_top + pre_top * pre_top) /
               dy;
  *mxl = fxl_h;
  *mxr = fxr_h;
  *myb = fyb_h;
  *myt = fyt_h;
}

void orc_compute_flux(int use_hllc, const double *h, const double *hu, const double *hv,
                      const double *b, double *flux_h, double *flux_hu, double *flux_hv,
                      double *mflux_x, double *mflux_y, int nx, int ny, int ng, double dx,
                      double dy) {
#pragma omp parallel for schedule(static)
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double fh, fhu, fhv, mxl, mxr, myb, myt;
      flux_cell(use_hllc, h, hu, hv, b, nx, i, j, dx, dy, &fh, &fhu, &fhv, &mxl, &mxr, &myb,
                &myt);
      AT(flux_h, i, j) = fh;
      AT(flux_hu, i, j) = fhu;
      AT(flux_hv, i, j) = fhv;
      if (mflux_x) {
        AT(mflux_x, i, j) = mxr;
        if (i == ng) AT(mflux_x, i - 1, j) = mxl;
      }
      if (mflux_y) {
        AT(mflux_y, i, j) = myt;
        if (j == ng) AT(mflux_y, i, j - 1) = myb;
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* Update kernels: rki_kernel_fused.F90, rki_kernel_update.F90            */
/* ---------------------------------------------------------------------- */

/* Clamp + KP07 desingularisation + Froude backstop, repeated verbatim in
 * rki_kernel_fused.F90:93-119 and :441-463 and rki_kernel_update.F90:64-95. */
static void protect(double *ph, double *pu, double *pv) {
  double h = *ph, u = *pu, v = *pv;
  if (h < 0.0) {
    h = 0.0;
    u = 0.0;
    v = 0.0;
  } else if (h < DRY) {
    u = 0.0;
    v = 0.0;
  } else {
    double h2 = h * h;
    double h4 = h2 * h2;
    if (h4 < EPS4) {
      double uu = SQRT2 * h * u / sqrt(h4 + EPS4);
      double vv = SQRT2 * h * v / sqrt(h4 + EPS4);
      u = h * uu;
      v = h * vv;
    }
    double sp2 = (u * u + v * v) / (h * h);
    double fr2 = FR_BACK * FR_BACK * G * h;
    if (sp2 > fr2) {
      double sc = sqrt(fr2 / sp2);
      u = u * sc;
      v = v * sc;
    }
  }
  *ph = h;
  *pu = u;
  *pv = v;
}

/* Friction + forcing + Coriolis + precipitation for one cell,
 * rki_kernel_fused.F90:121-154. */
static void sources(double *ph, double *pu, double *pv, int nx, int i, int j, double dx,
                    double dy, double dt, double manning_n, double n_sq, int has_fric,
                    int has_cor, double cosf, double sinf, const double *wind_x,
                    const double *wind_y, const double *atm, const double *precip,
                    int forcing_active) {
  double h = *ph, u = *pu, v = *pv;
  (void)manning_n;
  if (h > DRY) {
    if (has_fric) {
      double uu = u / h;
      double vv = v / h;
      double speed = sqrt(uu * uu + vv * vv);
      double cf = G * n_sq / orc_cr_pow_third(h);
      double den = 1.0 + dt * cf * speed / h;
      u = u / den;
      v = v / den;
    }
    if (forcing_active) {
      u = u + dt * AT(wind_x, i, j) / RHO;
      v = v + dt * AT(wind_y, i, j) / RHO;
      double dpdx = (AT(atm, i + 1, j) - AT(atm, i - 1, j)) / (2.0 * dx);
      double dpdy = (AT(atm, i, j + 1) - AT(atm, i, j - 1)) / (2.0 * dy);
      u = u - dt * h * dpdx / RHO;
      v = v - dt * h * dpdy / RHO;
    }
    if (has_cor) {
      double uo = u, vo = v;
      u = uo * cosf + vo * sinf;
      v = -(uo * sinf) + vo * cosf;
    }
  }
  if (forcing_active) h = h + dt * AT(precip, i, j);
  *ph = h;
  *pu = u;
  *pv = v;
}

typedef struct {
  double n_sq, cosf, sinf;
  int has_fric, has_cor;
} src_consts;

static src_consts make_src(double manning_n, double coriolis_f, double dt) {
  src_consts c;
  c.n_sq = manning_n * manning_n;
  c.has_fric = manning_n > 0.0;
  c.has_cor = fabs(coriolis_f) > 1.0e-20;
  c.cosf = c.has_cor ? orc_cr_cos(coriolis_f * dt) : 0.0;
  c.sinf = c.has_cor ? orc_cr_sin(coriolis_f * dt) : 0.0;
  return c;
}

void orc_fused_stage1(double *h, double *hu, double *hv, double *h0, double *hu0, double *hv0,
                      const double *fh, const double *fhu, const double *fhv, int nx, int ny,
                      int ng, double dx, double dy, double dt, double manning_n,
                      const double *wind_x, const double *wind_y, const double *atm,
                      const double *precip, double coriolis_f, int forcing_active) {
  src_consts c = make_src(manning_n, coriolis_f, dt);
#pragma omp parallel for schedule(static)
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = AT(h, i, j), u = AT(hu, i, j), v = AT(hv, i, j);
      AT(h0, i, j) = a;
      AT(hu0, i, j) = u;
      AT(hv0, i, j) = v;
      a = a + dt * AT(fh, i, j);
      u = u + dt * AT(fhu, i, j);
      v = v + dt * AT(fhv, i, j);
      protect(&a, &u, &v);
      sources(&a, &u, &v, nx, i, j, dx, dy, dt, manning_n, c.n_sq, c.has_fric, c.has_cor,
              c.cosf, c.sinf, wind_x, wind_y, atm, precip, forcing_active);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

void orc_fused_stage2(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                      const double *hv0, const double *fh, const double *fhu, const double *fhv,
                      int nx, int ny, int ng, double dx, double dy, double dt, double manning_n,
                      const double *wind_x, const double *wind_y, const double *atm,
                      const double *precip, double coriolis_f, int forcing_active) {
  src_consts c = make_src(manning_n, coriolis_f, dt);
#pragma omp parallel for schedule(static)
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = AT(h, i, j), u = AT(hu, i, j), v = AT(hv, i, j);
      a = a + dt * AT(fh, i, j);
      u = u + dt * AT(fhu, i, j);
      v = v + dt * AT(fhv, i, j);
      protect(&a, &u, &v);
      sources(&a, &u, &v, nx, i, j, dx, dy, dt, manning_n, c.n_sq, c.has_fric, c.has_cor,
              c.cosf, c.sinf, wind_x, wind_y, atm, precip, forcing_active);
      a = 0.5 * (AT(h0, i, j) + a);
      u = 0.5 * (AT(hu0, i, j) + u);
      v = 0.5 * (AT(hv0, i, j) + v);
      protect(&a, &u, &v);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

void orc_fused_stage_generic(double *h, double *hu, double *hv, const double *fh,
                             const double *fhu, const double *fhv, int nx, int ny, int ng,
                             double dx, double dy, double dt, double manning_n,
                             const double *wind_x, const double *wind_y, const double *atm,
                             const double *precip, double coriolis_f, int forcing_active) {
  src_consts c = make_src(manning_n, coriolis_f, dt);
#pragma omp parallel for schedule(static)
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = AT(h, i, j), u = AT(hu, i, j), v = AT(hv, i, j);
      a = a + dt * AT(fh, i, j);
      u = u + dt * AT(fhu, i, j);
      v = v + dt * AT(fhv, i, j);
      protect(&a, &u, &v);
      sources(&a, &u, &v, nx, i, j, dx, dy, dt, manning_n, c.n_sq, c.has_fric, c.has_cor,
              c.cosf, c.sinf, wind_x, wind_y, atm, precip, forcing_active);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

void orc_compute_update(double *h, double *hu, double *hv, const double *fh, const double *fhu,
                        const double *fhv, int nx, int ny, int ng, double dt) {
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = AT(h, i, j) + dt * AT(fh, i, j);
      double u = AT(hu, i, j) + dt * AT(fhu, i, j);
      double v = AT(hv, i, j) + dt * AT(fhv, i, j);
      protect(&a, &u, &v);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

void orc_rk2_average(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                     const double *hv0, int nx, int ny, int ng) {
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = 0.5 * (AT(h0, i, j) + AT(h, i, j));
      double u = 0.5 * (AT(hu0, i, j) + AT(hu, i, j));
      double v = 0.5 * (AT(hv0, i, j) + AT(hv, i, j));
      protect(&a, &u, &v);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

/* rki_kernel_update.F90:152-208 */
void orc_ssp_combine(double *h, double *hu, double *hv, const double *h0, const double *hu0,
                     const double *hv0, double a_n, int nx, int ny, int ng) {
  double a_prev = 1.0 - a_n;
#pragma omp parallel for schedule(static)
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double a = a_n * AT(h0, i, j) + a_prev * AT(h, i, j);
      double u = a_n * AT(hu0, i, j) + a_prev * AT(hu, i, j);
      double v = a_n * AT(hv0, i, j) + a_prev * AT(hv, i, j);
      protect(&a, &u, &v);
      AT(h, i, j) = a;
      AT(hu, i, j) = u;
      AT(hv, i, j) = v;
    }
  }
}

/* rki_kernel_friction.F90:16-113 (forcing_active and include_wind are the
 * reference's optional arguments, default .true.) */
void orc_apply_friction(double *h, double *hu, double *hv, int nx, int ny, int ng, double dx,
                        double dy, double dt, double manning_n, const double *wind_x,
                        const double *wind_y, const double *atm, const double *precip,
                        int forcing_active, int include_wind) {
  int has_fric = manning_n > 0.0;
  if (!has_fric && !forcing_active) return;
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double hval = AT(h, i, j);
      if (hval > DRY) {
        double u = AT(hu, i, j) / hval;
        double v = AT(hv, i, j) / hval;
        double speed = sqrt(u * u + v * v);
        if (has_fric) {
          double cf = G * manning_n * manning_n / orc_cr_pow_third(hval);
          double den = 1.0 + dt * cf * speed / hval;
          AT(hu, i, j) = AT(hu, i, j) / den;
          AT(hv, i, j) = AT(hv, i, j) / den;
        }
        if (forcing_active) {
          if (include_wind) { /* :89-94, skipped when wind goes to the surface layer */
            AT(hu, i, j) = AT(hu, i, j) + dt * AT(wind_x, i, j) / RHO;
            AT(hv, i, j) = AT(hv, i, j) + dt * AT(wind_y, i, j) / RHO;
          }
          double dpdx = (AT(atm, i + 1, j) - AT(atm, i - 1, j)) / (2.0 * dx);
          double dpdy = (AT(atm, i, j + 1) - AT(atm, i, j - 1)) / (2.0 * dy);
          AT(hu, i, j) = AT(hu, i, j) - dt * hval * dpdx / RHO;
          AT(hv, i, j) = AT(hv, i, j) - dt * hval * dpdy / RHO;
        }
      }
      if (forcing_active) AT(h, i, j) = AT(h, i, j) + dt * AT(precip, i, j);
    }
  }
}

/* rki_kernel_friction.F90:115-150 */
void orc_apply_coriolis(const double *h, double *hu, double *hv, int nx, int ny, int ng,
                        double dt, double f) {
  if (fabs(f) < 1.0e-20) return;
  double cosf_ = orc_cr_cos(f * dt), sinf_ = orc_cr_sin(f * dt);
  for (int j = ng; j < ny - ng; ++j)
    for (int i = ng; i < nx - ng; ++i)
      if (AT(h, i, j) > DRY) {
        double uo = AT(hu, i, j), vo = AT(hv, i, j);
        AT(hu, i, j) = uo * cosf_ + vo * sinf_;
        AT(hv, i, j) = -(uo * sinf_) + vo * cosf_;
      }
}

/* ---------------------------------------------------------------------- */
/* CFL timestep: rki_kernel_timestep.F90:16-74                            */
/* ---------------------------------------------------------------------- */

double orc_compute_timestep(const double *h, const double *hu, const double *hv, int nx, int ny,
                            int ng, double dx, double dy, double cfl, double *max_speed_out) {
  double ms = 0.0;
  for (int j = ng; j < ny - ng; ++j) {
    for (int i = ng; i < nx - ng; ++i) {
      double hh = AT(h, i, j);
      if (hh > DRY) {
        double c = sqrt(G * hh);
        double h2 = hh * hh;
        double den = sqrt(h2 * h2 + EPS4);
        double ua = fabs(AT(hu, i, j)) * SQRT2 * hh / den;
        double va = fabs(AT(hv, i, j)) * SQRT2 * hh / den;
        double sx = (ua + c) / dx;
        double sy = (va + c) / dy;
        if (sx > ms) ms = sx;
        if (sy > ms) ms = sy;
      }
    }
  }
  if (max_speed_out) *max_speed_out = ms;
  if (ms > 0.0) return cfl / ms;
  return cfl * fmin(dx, dy) / sqrt(G * DRY);
}

/* ---------------------------------------------------------------------- */
/* Boundary conditions: rki_boundary.F90:40-552                           */
/* ---------------------------------------------------------------------- */

/* Edge geometry (rki_boundary.F90:75-84) in 0-based indices: first ghost
 * cell (ig0, jg0), outward step per layer (din, djn), step along the edge
 * (dit, djt), tangential extent, sign of the outward normal, and whether
 * the normal momentum is hu. */
typedef struct {
  int ig0, jg0, din, djn, dit, djt, n_tan;
  double sgn;
  int normal_u;
} edge;

static edge make_edge(int which, int nx, int ny, int ng) {
  edge e;
  switch (which) {
    case 0: /* west */
      e.ig0 = ng - 1; e.jg0 = 0; e.din = -1; e.djn = 0; e.dit = 0; e.djt = 1;
      e.n_tan = ny; e.sgn = -1.0; e.normal_u = 1;
      break;
    case 1: /* east */
      e.ig0 = nx - ng; e.jg0 = 0; e.din = 1; e.djn = 0; e.dit = 0; e.djt = 1;
      e.n_tan = ny; e.sgn = 1.0; e.normal_u = 1;
      break;
    case 2: /* south */
      e.ig0 = 0; e.jg0 = ng - 1; e.din = 0; e.djn = -1; e.dit = 1; e.djt = 0;
      e.n_tan = nx; e.sgn = -1.0; e.normal_u = 0;
      break;
    default: /* north */
      e.ig0 = 0; e.jg0 = ny - ng; e.din = 0; e.djn = 1; e.dit = 1; e.djt = 0;
      e.n_tan = nx; e.sgn = 1.0; e.normal_u = 0;
      break;
  }
  return e;
}

/* bc_wall_edge :220-291 */
static void wall_edge(double *h, double *hu, double *hv, double *b, int nx, int ng, edge e) {
  for (int t = 0; t < e.n_tan; ++t) {
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int im = ig - (2 * k - 1) * e.din;
      int jm = jg - (2 * k - 1) * e.djn;
      AT(b, ig, jg) = AT(b, im, jm);
      AT(h, ig, jg) = fmax(0.0, AT(h, im, jm) + AT(b, im, jm) - AT(b, ig, jg));
      if (e.normal_u) {
        AT(hu, ig, jg) = -AT(hu, im, jm);
        AT(hv, ig, jg) = AT(hv, im, jm);
      } else {
        AT(hv, ig, jg) = -AT(hv, im, jm);
        AT(hu, ig, jg) = AT(hu, im, jm);
      }
    }
  }
}

/* bc_flather_edge :293-345 */
static void flather_edge(double *h, double *hu, double *hv, const double *b, int nx, int ng,
                         edge e, double eta_ext, int prescribe_h) {
  for (int t = 0; t < e.n_tan; ++t) {
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int ii = e.ig0 + t * e.dit - e.din;
      int ji = e.jg0 + t * e.djt - e.djn;
      double hi = AT(h, ii, ji);
      double ei = hi + AT(b, ii, ji);
      double hmax = fmax(hi, 1.0e-6);
      double c = sqrt(G * hmax);
      double hg = prescribe_h ? fmax(0.0, eta_ext - AT(b, ig, jg)) : hi;
      AT(h, ig, jg) = hg;
      if (e.normal_u) {
        AT(hu, ig, jg) = hg * (AT(hu, ii, ji) / hmax + e.sgn * c * (ei - eta_ext) / hmax);
        AT(hv, ig, jg) = AT(hv, ii, ji);
      } else {
        AT(hv, ig, jg) = hg * (AT(hv, ii, ji) / hmax + e.sgn * c * (ei - eta_ext) / hmax);
        AT(hu, ig, jg) = AT(hu, ii, ji);
      }
    }
  }
}

/* bc_inflow_edge :347-390 */
static void inflow_edge(double *h, double *hu, double *hv, int nx, int ng, edge e, double vel) {
  double in_sgn = -e.sgn;
  for (int t = 0; t < e.n_tan; ++t) {
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int ii = e.ig0 + t * e.dit - e.din;
      int ji = e.jg0 + t * e.djt - e.djn;
      double hi = AT(h, ii, ji);
      AT(h, ig, jg) = hi;
      if (e.normal_u) {
        AT(hu, ig, jg) = in_sgn * hi * vel;
        AT(hv, ig, jg) = AT(hv, ii, ji);
      } else {
        AT(hv, ig, jg) = in_sgn * hi * vel;
        AT(hu, ig, jg) = AT(hu, ii, ji);
      }
    }
  }
}

/* bc_disch_edge :392-434 */
static void discharge_edge(double *h, double *hu, double *hv, int nx, int ng, edge e,
                           double flux) {
  double in_sgn = -e.sgn;
  for (int t = 0; t < e.n_tan; ++t) {
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int ii = e.ig0 + t * e.dit - e.din;
      int ji = e.jg0 + t * e.djt - e.djn;
      AT(h, ig, jg) = AT(h, ii, ji);
      if (e.normal_u) {
        AT(hu, ig, jg) = in_sgn * flux;
        AT(hv, ig, jg) = AT(hv, ii, ji);
      } else {
        AT(hv, ig, jg) = in_sgn * flux;
        AT(hu, ig, jg) = AT(hu, ii, ji);
      }
    }
  }
}

/* bc_clamped_edge :436-469 */
static void clamped_edge(double *h, double *hu, double *hv, const double *b, int nx, int ng,
                         edge e, double eta) {
  for (int t = 0; t < e.n_tan; ++t) {
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int ii = e.ig0 + t * e.dit - e.din;
      int ji = e.jg0 + t * e.djt - e.djn;
      AT(h, ig, jg) = fmax(0.0, eta - AT(b, ig, jg));
      AT(hu, ig, jg) = AT(hu, ii, ji);
      AT(hv, ig, jg) = AT(hv, ii, ji);
    }
  }
}

/* bc_chapman_edge :471-552.  The reference runs the (t, k) pairs as one
 * do concurrent; the k == 1 refresh of eta_old(t) is read by the other
 * layers of the same t.  Here every k of a given t reads the pre-refresh
 * value (the refresh is applied after the t's layers are filled), which is
 * the only race-free reading of that loop. */
static void chapman_edge(double *h, double *hu, double *hv, const double *b, int nx, int ny,
                         int ng, edge e, double *eta_old, double dt, double dx, double dy) {
  double dd = e.normal_u ? dx : dy;
  for (int t = 0; t < e.n_tan; ++t) {
    double eta_old_val = eta_old[t];
    double refresh = eta_old_val;
    for (int k = 1; k <= ng; ++k) {
      int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      int ii = e.ig0 + t * e.dit - e.din;
      int ji = e.jg0 + t * e.djt - e.djn;
      int i2 = ii - e.din;
      int j2 = ji - e.djn;
      double hi = AT(h, ii, ji);
      double ei = hi + AT(b, ii, ji);
      double hmax = fmax(hi, 1.0e-6);
      double c = sqrt(G * hmax);
      double eg;
      if (dt > 0.0) {
        double detadt = (ei - eta_old_val) / dt;
        double detadx;
        if (i2 >= 0 && i2 < nx && j2 >= 0 && j2 < ny)
          detadx = (AT(h, i2, j2) + AT(b, i2, j2) - ei) / dd;
        else
          detadx = 0.0;
        double cp = (fabs(detadx) > 1.0e-10) ? -detadt / detadx : 0.0;
        cp = fmax(0.0, fmin(cp, c));
        eg = eta_old_val - cp * dt / dd * (eta_old_val - ei);
      } else {
        eg = ei;
      }
      if (k == 1) refresh = ei;
      double hg = fmax(0.0, eg - AT(b, ig, jg));
      AT(h, ig, jg) = hg;
      if (e.normal_u) {
        AT(hu, ig, jg) = hg * (AT(hu, ii, ji) / hmax + e.sgn * c * (ei - eg) / hmax);
        AT(hv, ig, jg) = AT(hv, ii, ji);
      } else {
        AT(hv, ig, jg) = hg * (AT(hv, ii, ji) / hmax + e.sgn * c * (ei - eg) / hmax);
        AT(hu, ig, jg) = AT(hu, ii, ji);
      }
    }
    eta_old[t] = refresh;
  }
}

double orc_tidal_eta(const orc_bc *bc) {
  double eta = 0.0;
  if (bc->n_tidal > 0) {
    for (int n = 0; n < bc->n_tidal; ++n)
      eta = eta + bc->tidal_amp[n] * orc_cr_cos(bc->tidal_omega[n] * bc->time - bc->tidal_phase[n]);
  } else if (bc->tidal_period > 0.0) {
    eta = bc->tidal_amplitude * orc_cr_sin(TWO_PI_C * bc->time / bc->tidal_period);
  }
  return eta;
}

void orc_apply_bc(double *h, double *hu, double *hv, double *b, int nx, int ny, int ng,
                  orc_bc *bc) {
  double tide = orc_tidal_eta(bc);
  int types[4] = {bc->west, bc->east, bc->south, bc->north};
  double *eta_old[4] = {bc->eta_old_west, bc->eta_old_east, bc->eta_old_south,
                        bc->eta_old_north};
  for (int w = 0; w < 4; ++w) {
    edge e = make_edge(w, nx, ny, ng);
    switch (types[w]) {
      case ORC_BC_WALL:
      case ORC_BC_SPONGE:
        wall_edge(h, hu, hv, b, nx, ng, e);
        break;
      case ORC_BC_OPEN:
        flather_edge(h, hu, hv, b, nx, ng, e, 0.0, 0);
        break;
      case ORC_BC_TIDAL:
        flather_edge(h, hu, hv, b, nx, ng, e, tide, 1);
        break;
      case ORC_BC_INFLOW:
        inflow_edge(h, hu, hv, nx, ng, e, bc->inflow_velocity);
        break;
      case ORC_BC_DISCHARGE:
        discharge_edge(h, hu, hv, nx, ng, e, bc->discharge_flux);
        break;
      case ORC_BC_CLAMPED:
        clamped_edge(h, hu, hv, b, nx, ng, e, bc->clamped_elevation);
        break;
      case ORC_BC_CHAPMAN:
        chapman_edge(h, hu, hv, b, nx, ny, ng, e, eta_old[w], bc->dt, bc->dx, bc->dy);
        break;
      default: /* nested: filled elsewhere */
        break;
    }
  }
}

/* rki_kernel_sponge.F90:16-88 */
void orc_apply_sponge(double *h, double *hu, double *hv, int nx, int ny, int ng, double dt,
                      const orc_bc *bc) {
  int sw = bc->sponge_width;
  if (sw <= 0) return;
  double strength = bc->sponge_strength, href = bc->sponge_h_ref;
  if (strength <= 0.0) return;
  int i0 = ng, i1 = nx - ng - 1, j0 = ng, j1 = ny - ng - 1;
  for (int j = j0; j <= j1; ++j) {
    for (int i = i0; i <= i1; ++i) {
      int dmin = sw + 1;
      if (bc->west == ORC_BC_SPONGE && i - i0 < sw && i - i0 < dmin) dmin = i - i0;
      if (bc->east == ORC_BC_SPONGE && i1 - i < sw && i1 - i < dmin) dmin = i1 - i;
      if (bc->south == ORC_BC_SPONGE && j - j0 < sw && j - j0 < dmin) dmin = j - j0;
      if (bc->north == ORC_BC_SPONGE && j1 - j < sw && j1 - j < dmin) dmin = j1 - j;
      if (dmin < sw) {
        double ratio = (double)(sw - dmin) / (double)sw;
        double alpha = strength * ratio * ratio;
        AT(h, i, j) = AT(h, i, j) - dt * alpha * (AT(h, i, j) - href);
        AT(hu, i, j) = AT(hu, i, j) - dt * alpha * AT(hu, i, j);
        AT(hv, i, j) = AT(hv, i, j) - dt * alpha * AT(hv, i, j);
      }
    }
  }
}

/* src/io/rki_bathymetry.F90:165-196 (constant extrapolation) */
void orc_fill_bathymetry_ghosts(double *b, int nx, int ny, int ng) {
  int nxp = nx - 2 * ng, nyp = ny - 2 * ng;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < ng; ++i) {
      AT(b, i, j) = AT(b, ng, j);
      AT(b, ng + nxp + i, j) = AT(b, ng + nxp - 1, j);
    }
  for (int j = 0; j < ng; ++j)
    for (int i = 0; i < nx; ++i) {
      AT(b, i, j) = AT(b, i, ng);
      AT(b, i, ng + nyp + j) = AT(b, i, ng + nyp - 1);
    }
}

/* ---------------------------------------------------------------------- */
/* Initial conditions: src/core/rki_init.F90                              */
/* ---------------------------------------------------------------------- */

static int any_nonzero(const double *b, size_t n) {
  for (size_t k = 0; k < n; ++k)
    if (b[k] != 0.0) return 1;
  return 0;
}

void orc_init_dam_break(orc_sim *s) {
  int nx = s->nx, ny = s->ny;
  int mid_x = s->ng + (nx - 2 * s->ng) / 2; /* 1-based column of the dam */
  int has_b = any_nonzero(s->b, (size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      if (!has_b) AT(s->b, i, j) = 0.0;
      AT(s->hu, i, j) = 0.0;
      AT(s->hv, i, j) = 0.0;
      AT(s->h, i, j) = (i + 1 <= mid_x) ? 2.0 : 1.0;
    }
}

void orc_init_gaussian_hump(orc_sim *s, double h0, double amp, double sigma, double xoff,
                            double yoff) {
  int nx = s->nx, ny = s->ny, ng = s->ng;
  double xc = (double)(nx - 2 * ng) * s->dx * 0.5 + xoff;
  double yc = (double)(ny - 2 * ng) * s->dy * 0.5 + yoff;
  int has_b = any_nonzero(s->b, (size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double x = ((double)(i + 1 - ng) - 0.5) * s->dx;
      double y = ((double)(j + 1 - ng) - 0.5) * s->dy;
      double r2 = (x - xc) * (x - xc) + (y - yc) * (y - yc);
      if (!has_b) AT(s->b, i, j) = 0.0;
      AT(s->h, i, j) = h0 + amp * exp(-r2 / (2.0 * (sigma * sigma)));
      AT(s->hu, i, j) = 0.0;
      AT(s->hv, i, j) = 0.0;
    }
}

void orc_init_castro_dam_break(orc_sim *s) {
  int nx = s->nx, ny = s->ny, ng = s->ng;
  double x0 = -0.5 * (double)(nx - 2 * ng) * s->dx;
  double y0 = -0.5 * (double)(ny - 2 * ng) * s->dy;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double x = x0 + ((double)(i + 1 - ng) - 0.5) * s->dx;
      double y = y0 + ((double)(j + 1 - ng) - 0.5) * s->dy;
      double depth = 1.0 - 0.4 * exp(-x * x - y * y);
      AT(s->b, i, j) = -depth;
      double r2 = x * x + y * y;
      AT(s->h, i, j) = (r2 <= 0.36) ? 3.0 - AT(s->b, i, j) : 1.0 - AT(s->b, i, j);
      AT(s->hu, i, j) = 0.0;
      AT(s->hv, i, j) = 0.0;
    }
}

void orc_init_still_water(orc_sim *s, double eta0) {
  int nx = s->nx, ny = s->ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      AT(s->h, i, j) = fmax(eta0 - AT(s->b, i, j), 0.0);
      AT(s->hu, i, j) = 0.0;
      AT(s->hv, i, j) = 0.0;
    }
}

void orc_bc_init_chapman(orc_sim *s) {
  int nx = s->nx, ny = s->ny, ng = s->ng;
  orc_bc *bc = &s->bc;
  if (bc->west == ORC_BC_CHAPMAN || bc->east == ORC_BC_CHAPMAN)
    for (int j = 0; j < ny; ++j) {
      bc->eta_old_west[j] = AT(s->h, ng, j) + AT(s->b, ng, j);
      bc->eta_old_east[j] = AT(s->h, nx - ng - 1, j) + AT(s->b, nx - ng - 1, j);
    }
  if (bc->south == ORC_BC_CHAPMAN || bc->north == ORC_BC_CHAPMAN)
    for (int i = 0; i < nx; ++i) {
      bc->eta_old_south[i] = AT(s->h, i, ng) + AT(s->b, i, ng);
      bc->eta_old_north[i] = AT(s->h, i, ny - ng - 1) + AT(s->b, i, ny - ng - 1);
    }
}

double orc_total_mass(const orc_sim *s) {
  int nx = s->nx, ny = s->ny, ng = s->ng;
  double area = s->dx * s->dy, acc = 0.0;
  for (int j = ng; j < ny - ng; ++j)
    for (int i = ng; i < nx - ng; ++i) {
      double hh = AT(s->h, i, j);
      if (hh > 0.0 && hh < 1.0e6) acc = acc + hh * area;
    }
  return acc;
}

/* ---------------------------------------------------------------------- */
/* Solver: rki_solver.F90:507-926                                          */
/* ---------------------------------------------------------------------- */

static double interior_sum(const double *a, int nx, int ny, int ng) {
  double acc = 0.0;
  for (int j = ng; j < ny - ng; ++j)
    for (int i = ng; i < nx - ng; ++i) acc = acc + AT(a, i, j);
  return acc;
}

/* accumulate_boundary_mass_out :507-537 */
static void mass_out(orc_sim *s, double w) {
  double acc = interior_sum(s->flux_h, s->nx, s->ny, s->ng);
  s->mass_out = s->mass_out - w * s->dt * acc * (s->dx * s->dy);
}

/* accumulate_mass_src :539-606 (2D path: precipitation only) */
static void mass_src(orc_sim *s, double w) {
  if (!s->forcing_active) return;
  double acc = interior_sum(s->precip, s->nx, s->ny, s->ng);
  s->mass_src = s->mass_src + w * s->dt * acc * (s->dx * s->dy);
}

/* accumulate_sponge_mass_src :608-657 */
static void sponge_stage(orc_sim *s, double w, double dt) {
  if (s->bc.sponge_width <= 0) {
    orc_apply_sponge(s->h, s->hu, s->hv, s->nx, s->ny, s->ng, dt, &s->bc);
    return;
  }
  double before = interior_sum(s->h, s->nx, s->ny, s->ng);
  orc_apply_sponge(s->h, s->hu, s->hv, s->nx, s->ny, s->ng, dt, &s->bc);
  double after = interior_sum(s->h, s->nx, s->ny, s->ng);
  s->mass_src = s->mass_src + w * (after - before) * (s->dx * s->dy);
}

static void bc(orc_sim *s) { orc_apply_bc(s->h, s->hu, s->hv, s->b, s->nx, s->ny, s->ng, &s->bc); }

static void flux(orc_sim *s) {
  orc_compute_flux(s->use_hllc, s->h, s->hu, s->hv, s->b, s->flux_h, s->flux_hu, s->flux_hv,
                   s->mflux_x, s->mflux_y, s->nx, s->ny, s->ng, s->dx, s->dy);
}

/* Shu-Osher tables, src/core/rki_timestepper.F90:60-100 */
static void scheme_table(int scheme, int *n, double *ssp, double *alpha, double *beta,
                         double *c) {
  for (int k = 0; k < 4; ++k) alpha[k] = beta[k] = c[k] = 0.0;
  switch (scheme) {
    case 1:
      *n = 1; *ssp = 1.0; beta[0] = 1.0;
      break;
    case 3:
      *n = 3; *ssp = 1.0;
      alpha[1] = 0.75; alpha[2] = 1.0 / 3.0;
      beta[0] = beta[1] = beta[2] = 1.0;
      c[1] = 1.0; c[2] = 0.5;
      break;
    case 4:
      *n = 4; *ssp = 2.0;
      alpha[2] = 2.0 / 3.0;
      beta[0] = beta[1] = beta[2] = beta[3] = 0.5;
      c[1] = 0.5; c[2] = 1.0; c[3] = 0.5;
      break;
    default:
      *n = 2; *ssp = 1.0;
      alpha[1] = 0.5;
      beta[0] = beta[1] = 1.0;
      c[1] = 1.0;
      break;
  }
}

/* solver_advance_2d_generic :861-926 */
static void advance_generic(orc_sim *s, int nst, const double *alpha, const double *beta,
                            const double *c) {
  size_t n = (size_t)s->nx * s->ny;
  /* solver_save_state copies the whole arrays. */
  memcpy(s->h0, s->h, n * sizeof(double));
  memcpy(s->hu0, s->hu, n * sizeof(double));
  memcpy(s->hv0, s->hv, n * sizeof(double));
  double t_base = s->bc.time;
  for (int st = 0; st < nst; ++st) {
    double dts = beta[st] * s->dt;
    s->bc.time = t_base + c[st] * s->dt;
    bc(s);
    flux(s);
    orc_fused_stage_generic(s->h, s->hu, s->hv, s->flux_h, s->flux_hu, s->flux_hv, s->nx, s->ny,
                            s->ng, s->dx, s->dy, dts, s->manning_n, s->wind_x, s->wind_y,
                            s->atm, s->precip, s->coriolis_f, s->forcing_active);
    if (alpha[st] != 0.0)
      orc_ssp_combine(s->h, s->hu, s->hv, s->h0, s->hu0, s->hv0, alpha[st], s->nx, s->ny, s->ng);
    orc_apply_sponge(s->h, s->hu, s->hv, s->nx, s->ny, s->ng, dts, &s->bc);
  }
  s->bc.time = t_base + s->dt;
}

void orc_solver_step(orc_sim *s, double dt_max, double time) {
  int nst;
  double ssp, alpha[4], beta[4], c[4];
  scheme_table(s->time_scheme, &nst, &ssp, alpha, beta, c);

  s->bc.time = time;
  s->bc.dx = s->dx;
  s->bc.dy = s->dy;

  bc(s);
  if (s->dt_fixed > 0.0) {
    s->dt = s->dt_fixed;
    s->dt = fmin(s->dt, dt_max);
  } else if (s->step_count % s->cfl_interval == 0 || s->dt <= 0.0) {
    s->dt = orc_compute_timestep(s->h, s->hu, s->hv, s->nx, s->ny, s->ng, s->dx, s->dy, s->cfl,
                                 NULL);
    s->dt = s->dt * ssp;
    s->dt = fmin(s->dt, dt_max);
  }
  s->step_count = s->step_count + 1;
  s->bc.dt = s->dt;

  if (s->time_scheme != 2) {
    advance_generic(s, nst, alpha, beta, c);
    return;
  }

  /* fused RK2 stage 1 */
  bc(s);
  flux(s);
  mass_out(s, 0.5);
  orc_fused_stage1(s->h, s->hu, s->hv, s->h0, s->hu0, s->hv0, s->flux_h, s->flux_hu, s->flux_hv,
                   s->nx, s->ny, s->ng, s->dx, s->dy, s->dt, s->manning_n, s->wind_x, s->wind_y,
                   s->atm, s->precip, s->coriolis_f, s->forcing_active);
  mass_src(s, 0.5);
  sponge_stage(s, 0.5, s->dt);

  /* fused RK2 stage 2 */
  s->bc.time = s->bc.time + s->dt;
  bc(s);
  flux(s);
  mass_out(s, 0.5);
  orc_fused_stage2(s->h, s->hu, s->hv, s->h0, s->hu0, s->hv0, s->flux_h, s->flux_hu, s->flux_hv,
                   s->nx, s->ny, s->ng, s->dx, s->dy, s->dt, s->manning_n, s->wind_x, s->wind_y,
                   s->atm, s->precip, s->coriolis_f, s->forcing_active);
  mass_src(s, 0.5);
  sponge_stage(s, 0.5, s->dt);
}

void orc_step_n(orc_sim *s, int n) {
  for (int k = 0; k < n; ++k) {
    orc_solver_step(s, s->t_end - s->t_current, s->t_current);
    s->t_current = s->t_current + s->dt;
  }
}

void orc_advance(orc_sim *s, double target_time) {
  while (s->t_current < target_time - 1.0e-10) {
    orc_solver_step(s, target_time - s->t_current, s->t_current);
    s->t_current = s->t_current + s->dt;
  }
}
