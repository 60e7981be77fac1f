// Reverse-mode derivatives of the structured step's pointwise pieces (FP64).
//
// Each *_adj function recomputes the forward values it needs from the same
// inputs as the forward function (rkb_face.cuh, rkb_common.cuh) and
// propagates adjoints back to those inputs, branch by branch: the branches the
// forward took (wet/dry tests, wave-speed min/max, HLL sub/supercritical
// cases, the HLLC contact sign, clamps) are held fixed, as the derivative of a
// piecewise-smooth function inside one piece.  All functions are host+device
// so they can be checked against finite differences on the CPU.
#pragma once

#include "rkb_common.cuh"
#include "rkb_crmath.cuh"
#include "rkb_face.cuh"

namespace rkb {

// Derivative of velocity(): u = q/h when h > DRY_THRESHOLD, else 0.
RKB_HD void velocity_adj(double h, double qx, double qy, double gu, double gv, double& gh,
                         double& gqx, double& gqy) {
  if (h > kDry) {
    const double u = qx / h, v = qy / h;
    gqx += gu / h;
    gqy += gv / h;
    gh += -(gu * u + gv * v) / h;
  }
}

// Adjoint of riemann<DIR, HLLC>(hl, qxl, qyl, hr, qxr, qyr) given the output
// adjoints (gfh, gfqx, gfqy); accumulates into g[6] = (hl, qxl, qyl, hr, qxr, qyr).
template <int DIR, bool HLLC>
RKB_HD void riemann_adj(double hl, double qxl, double qyl, double hr, double qxr, double qyr,
                        double gfh, double gfqx, double gfqy, double g[6]) {
  double ul, vl, ur, vr;
  velocity(hl, qxl, qyl, ul, vl);
  velocity(hr, qxr, qyr, ur, vr);
  const double al = sqrt(kG * pos(hl));
  const double ar = sqrt(kG * pos(hr));
  const double nl = DIR == 0 ? ul : vl;
  const double nr = DIR == 0 ? ur : vr;
  int branch;
  double sl, sr;
  bool sl_first = true, sr_first = true;  // which argument of min / max was taken
  if (hr <= kDry) {
    branch = 0;
    sl = nl - al;
    sr = nl + 2.0 * al;
  } else if (hl <= kDry) {
    branch = 1;
    sl = nr - 2.0 * ar;
    sr = nr + ar;
  } else {
    branch = 2;
    const double a1 = nl - al, a2 = nr - ar, b1 = nl + al, b2 = nr + ar;
    sl_first = a1 < a2;  // dmin(a, b) = a < b ? a : b
    sl = sl_first ? a1 : a2;
    sr_first = b1 > b2;  // dmax(a, b) = a > b ? a : b
    sr = sr_first ? b1 : b2;
  }
  // side fluxes L, R (h, x, y components) and states U
  double L[3], R[3];
  if (DIR == 0) {
    L[0] = qxl; L[1] = qxl * ul + kHalfG * hl * hl; L[2] = qxl * vl;
    R[0] = qxr; R[1] = qxr * ur + kHalfG * hr * hr; R[2] = qxr * vr;
  } else {
    L[0] = qyl; L[1] = qxl * vl; L[2] = qyl * vl + kHalfG * hl * hl;
    R[0] = qyr; R[1] = qxr * vr; R[2] = qyr * vr + kHalfG * hr * hr;
  }
  const double UL[3] = {hl, qxl, qyl}, UR[3] = {hr, qxr, qyr};
  double gF[3] = {gfh, gfqx, gfqy};
  double gL[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, gUL[3] = {0, 0, 0}, gUR[3] = {0, 0, 0};
  double gsl = 0.0, gsr = 0.0;
  double gul = 0.0, gvl = 0.0, gur = 0.0, gvr = 0.0;
  if (sl >= 0.0) {
    for (int k = 0; k < 3; ++k) gL[k] += gF[k];
  } else if (sr <= 0.0) {
    for (int k = 0; k < 3; ++k) gR[k] += gF[k];
  } else {
    const double inv = 1.0 / (sr - sl);
    const double slsr = sl * sr;
    const int t = DIR == 0 ? 2 : 1;  // tangential component
    if (HLLC) {
      // tangential flux = fh * (upwind tangential velocity) (rki_kernel_flux.F90:584-783)
      const double un_l = DIR == 0 ? ul : vl, un_r = DIR == 0 ? ur : vr;
      const double ut_l = DIR == 0 ? vl : ul, ut_r = DIR == 0 ? vr : ur;
      const double hrr = hr, hll = hl;
      const double den = hrr * (un_r - sr) - hll * (un_l - sl);
      double ss;
      if (fabs(den) > kDry)
        ss = (sl * hrr * (un_r - sr) - sr * hll * (un_l - sl)) / den;
      else
        ss = 0.5 * (un_l + un_r);
      const double fh = (sr * L[0] - sl * R[0] + slsr * (UR[0] - UL[0])) * inv;
      const double gt = gF[t];
      gF[0] += gt * (ss >= 0.0 ? ut_l : ut_r);
      if (ss >= 0.0) {
        if (DIR == 0) gvl += gt * fh; else gul += gt * fh;
      } else {
        if (DIR == 0) gvr += gt * fh; else gur += gt * fh;
      }
      gF[t] = 0.0;
    }
    for (int k = 0; k < 3; ++k) {
      if (HLLC && k == t) continue;
      const double d = UR[k] - UL[k];
      const double F = (sr * L[k] - sl * R[k] + slsr * d) * inv;
      gL[k] += gF[k] * sr * inv;
      gR[k] += -gF[k] * sl * inv;
      gUR[k] += gF[k] * slsr * inv;
      gUL[k] += -gF[k] * slsr * inv;
      gsr += gF[k] * ((L[k] + sl * d) * inv - F * inv);
      gsl += gF[k] * ((-R[k] + sr * d) * inv + F * inv);
    }
  }
  // wave speeds
  double gnl = 0.0, gnr = 0.0, gal = 0.0, gar = 0.0;
  if (branch == 0) {
    gnl += gsl + gsr;
    gal += -gsl + 2.0 * gsr;
  } else if (branch == 1) {
    gnr += gsl + gsr;
    gar += -2.0 * gsl + gsr;
  } else {
    if (sl_first) { gnl += gsl; gal -= gsl; } else { gnr += gsl; gar -= gsl; }
    if (sr_first) { gnl += gsr; gal += gsr; } else { gnr += gsr; gar += gsr; }
  }
  if (DIR == 0) { gul += gnl; gur += gnr; } else { gvl += gnl; gvr += gnr; }
  double ghl = 0.0, ghr = 0.0;
  if (al > 0.0) ghl += gal * kG / (2.0 * al);
  if (ar > 0.0) ghr += gar * kG / (2.0 * ar);
  // side fluxes -> (q, u, v, h)
  double gqxl = 0.0, gqyl = 0.0, gqxr = 0.0, gqyr = 0.0;
  if (DIR == 0) {
    gqxl += gL[0] + gL[1] * ul + gL[2] * vl;
    gul += gL[1] * qxl;
    gvl += gL[2] * qxl;
    ghl += gL[1] * 2.0 * kHalfG * hl;
    gqxr += gR[0] + gR[1] * ur + gR[2] * vr;
    gur += gR[1] * qxr;
    gvr += gR[2] * qxr;
    ghr += gR[1] * 2.0 * kHalfG * hr;
  } else {
    gqyl += gL[0] + gL[2] * vl;
    gqxl += gL[1] * vl;
    gvl += gL[1] * qxl + gL[2] * qyl;
    ghl += gL[2] * 2.0 * kHalfG * hl;
    gqyr += gR[0] + gR[2] * vr;
    gqxr += gR[1] * vr;
    gvr += gR[1] * qxr + gR[2] * qyr;
    ghr += gR[2] * 2.0 * kHalfG * hr;
  }
  ghl += gUL[0]; gqxl += gUL[1]; gqyl += gUL[2];
  ghr += gUR[0]; gqxr += gUR[1]; gqyr += gUR[2];
  velocity_adj(hl, qxl, qyl, gul, gvl, ghl, gqxl, gqyl);
  velocity_adj(hr, qxr, qyr, gur, gvr, ghr, gqxr, gqyr);
  g[0] += ghl; g[1] += gqxl; g[2] += gqyl;
  g[3] += ghr; g[4] += gqxr; g[5] += gqyr;
}

// Adjoint of face_flux<DIR, HLLC>(eL, qxL, qyL, bL, eR, qxR, qyR, bR) given
// gout = adjoints of (fh, fqx, fqy, wbR, hL2, pL2); accumulates into
// gin[8] = (eL, qxL, qyL, bL, eR, qxR, qyR, bR).
template <int DIR, bool HLLC>
RKB_HD void face_adj(double eL, double qxL, double qyL, double bL, double eR, double qxR,
                     double qyR, double bR, const double gout[6], double gin[8]) {
  const double hL = pos(eL - bL);
  const double hR = pos(eR - bR);
  const bool bl_max = bL > bR;  // dmax(bL, bR) = bL > bR ? bL : bR
  const double bmax = bl_max ? bL : bR;
  const double xl = hL + bL - bmax, xr = hR + bR - bmax;
  const double hyl = pos(xl);
  const double hyr = pos(xr);
  double ul, vl, ur, vr;
  velocity(hL, qxL, qyL, ul, vl);
  velocity(hR, qxR, qyR, ur, vr);
  double gr[6] = {0, 0, 0, 0, 0, 0};
  riemann_adj<DIR, HLLC>(hyl, hyl * ul, hyl * vl, hyr, hyr * ur, hyr * vr, gout[0], gout[1],
                         gout[2], gr);
  double ghyl = gr[0], ghyr = gr[3];
  double gul = 0.0, gvl = 0.0, gur = 0.0, gvr = 0.0;
  ghyl += gr[1] * ul + gr[2] * vl;
  gul += gr[1] * hyl;
  gvl += gr[2] * hyl;
  ghyr += gr[4] * ur + gr[5] * vr;
  gur += gr[4] * hyr;
  gvr += gr[5] * hyr;
  double ghL = 0.0, ghR = 0.0;
  ghyr += 2.0 * hyr * gout[3];
  ghR += -2.0 * hR * gout[3];
  ghyl += 2.0 * hyl * gout[4];
  ghL += 2.0 * hL * gout[5];
  double gqxL = 0.0, gqyL = 0.0, gqxR = 0.0, gqyR = 0.0;
  velocity_adj(hL, qxL, qyL, gul, gvl, ghL, gqxL, gqyL);
  velocity_adj(hR, qxR, qyR, gur, gvr, ghR, gqxR, gqyR);
  double gbL = 0.0, gbR = 0.0, gbmax = 0.0;
  if (xl > 0.0) { ghL += ghyl; gbL += ghyl; gbmax -= ghyl; }
  if (xr > 0.0) { ghR += ghyr; gbR += ghyr; gbmax -= ghyr; }
  if (bl_max) gbL += gbmax; else gbR += gbmax;
  double geL = 0.0, geR = 0.0;
  if (eL - bL > 0.0) { geL += ghL; gbL -= ghL; }
  if (eR - bR > 0.0) { geR += ghR; gbR -= ghR; }
  gin[0] += geL; gin[1] += gqxL; gin[2] += gqyL; gin[3] += gbL;
  gin[4] += geR; gin[5] += gqxR; gin[6] += gqyR; gin[7] += gbR;
}

// Adjoint of protect(h, u, v) at input (h, u, v): (gh, gu, gv) are the output
// adjoints on entry and the input adjoints on return.
RKB_HD void protect_adj(double h, double u, double v, double& gh, double& gu, double& gv) {
  if (h < 0.0) {
    gh = 0.0; gu = 0.0; gv = 0.0;
    return;
  }
  if (h < kDry) {
    gu = 0.0; gv = 0.0;
    return;
  }
  // forward with intermediates
  const double h2 = h * h;
  const double h4 = h2 * h2;
  const bool kp = h4 < kEps4;
  double u1 = u, v1 = v, r = 0.0;
  if (kp) {
    r = sqrt(h4 + kEps4);
    u1 = h * (kSqrt2 * h * u / r);
    v1 = h * (kSqrt2 * h * v / r);
  }
  const double sp2 = (u1 * u1 + v1 * v1) / (h * h);
  const double fr2 = kFroude * kFroude * kG * h;
  double ghh = gh, gu1 = gu, gv1 = gv;
  if (sp2 > fr2) {
    // u2 = u1 sqrt(fr2 / sp2) = u1 sqrt(F^2 g h^3 / (u1^2 + v1^2))
    const double sc = sqrt(fr2 / sp2);
    const double q2 = u1 * u1 + v1 * v1;
    // d sc / d u1 = -sc u1 / q2, d sc / d h = 1.5 sc / h
    const double gsc = gu * u1 + gv * v1;
    gu1 = gu * sc - gsc * sc * u1 / q2;
    gv1 = gv * sc - gsc * sc * v1 / q2;
    ghh += gsc * 1.5 * sc / h;
  }
  double gu0 = gu1, gv0 = gv1;
  if (kp) {
    // u1 = sqrt2 h^2 u / r, r = sqrt(h^4 + eps4): d/du = sqrt2 h^2 / r,
    // d/dh = sqrt2 u (2 h / r - h^2 * 2 h^3 / r^3)
    const double f = kSqrt2 * h2 / r;
    const double df = kSqrt2 * (2.0 * h / r - h2 * 2.0 * h * h2 / (r * r * r));
    gu0 = gu1 * f;
    gv0 = gv1 * f;
    ghh += (gu1 * u + gv1 * v) * df;
  }
  gh = ghh;
  gu = gu0;
  gv = gv0;
}

// Manning friction of sources() with a per-cell n (rki_kernel_fused.F90:121-130).
RKB_HD void friction(double h, double& u, double& v, double n, double dt) {
  if (h > kDry && n > 0.0) {
    const double n_sq = n * n;
    const double uu = u / h;
    const double vv = v / h;
    const double speed = sqrt(uu * uu + vv * vv);
    const double cf = kG * n_sq / cr_pow_third(h);
    const double den = 1.0 + dt * cf * speed / h;
    u = u / den;
    v = v / den;
  }
}

// Adjoint of friction at input (h, u, v, n): (gu, gv) output adjoints in,
// input adjoints out; gh, gn accumulated.
RKB_HD void friction_adj(double h, double u, double v, double n, double dt, double& gh,
                         double& gu, double& gv, double& gn) {
  if (!(h > kDry && n > 0.0)) return;
  const double uu = u / h, vv = v / h;
  const double sp = sqrt(uu * uu + vv * vv);
  const double c3 = cr_pow_third(h);
  const double cf = kG * n * n / c3;
  const double den = 1.0 + dt * cf * sp / h;
  const double gden = -(gu * u + gv * v) / (den * den);
  double gu0 = gu / den, gv0 = gv / den;
  const double gcf = gden * dt * sp / h;
  const double gsp = gden * dt * cf / h;
  gh += gden * (-dt * cf * sp / (h * h));
  gn += gcf * 2.0 * kG * n / c3;
  const double gc3 = -gcf * cf / c3;
  gh += gc3 * c3 / (3.0 * h);
  if (sp > 0.0) {
    const double guu = gsp * uu / sp, gvv = gsp * vv / sp;
    gu0 += guu / h;
    gv0 += gvv / h;
    gh += -(guu * uu + gvv * vv) / h;
  }
  gu = gu0;
  gv = gv0;
}

// minmod branch: 0 = zero, 1 = first argument, 2 = second (rki_kernel_flux.F90:380-393)
RKB_HD int minmod_choice(double a, double b) {
  if (a * b <= 0.0) return 0;
  return fabs(a) < fabs(b) ? 1 : 2;
}

}  // namespace rkb
