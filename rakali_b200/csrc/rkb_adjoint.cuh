// Reverse-mode derivatives of the structured step's pointwise pieces.
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

// h^(1/3): correctly rounded in FP64 (the production step's friction term),
// the CUDA / libm cube root in FP32.
RKB_HD double pow_third(double h) { return cr_pow_third(h); }
RKB_HD float pow_third(float h) { return cbrtf(h); }

// Derivative of velocity(): u = q/h when h > DRY_THRESHOLD, else 0.  The
// five quotients by h share one reciprocal: they only scale adjoints (no
// branch depends on them), so a last-bit difference from the divisions is
// immaterial, and the reverse sweep is dominated by division sequences.
template <typename T>
RKB_HD void velocity_adj(T h, T qx, T qy, T gu, T gv, T& gh,
                         T& gqx, T& gqy) {
  if (h > T(kDry)) {
    const T rh = T(1) / h;
    const T u = qx * rh, v = qy * rh;
    gqx += gu * rh;
    gqy += gv * rh;
    gh += -(gu * u + gv * v) * rh;
  }
}

// Adjoint of riemann<DIR, HLLC>(hl, qxl, qyl, hr, qxr, qyr) given the output
// adjoints (gfh, gfqx, gfqy); accumulates into g[6] = (hl, qxl, qyl, hr, qxr, qyr).
template <int DIR, bool HLLC, typename T>
RKB_HD void riemann_adj(T hl, T qxl, T qyl, T hr, T qxr, T qyr,
                        T gfh, T gfqx, T gfqy, T g[6]) {
  T ul, vl, ur, vr;
  velocity(hl, qxl, qyl, ul, vl);
  velocity(hr, qxr, qyr, ur, vr);
  const T al = sqrt(T(kG) * pos(hl));
  const T ar = sqrt(T(kG) * pos(hr));
  const T nl = DIR == 0 ? ul : vl;
  const T nr = DIR == 0 ? ur : vr;
  int branch;
  T sl, sr;
  bool sl_first = true, sr_first = true;  // which argument of min / max was taken
  if (hr <= T(kDry)) {
    branch = 0;
    sl = nl - al;
    sr = nl + T(2) * al;
  } else if (hl <= T(kDry)) {
    branch = 1;
    sl = nr - T(2) * ar;
    sr = nr + ar;
  } else {
    branch = 2;
    const T a1 = nl - al, a2 = nr - ar, b1 = nl + al, b2 = nr + ar;
    sl_first = a1 < a2;  // dmin(a, b) = a < b ? a : b
    sl = sl_first ? a1 : a2;
    sr_first = b1 > b2;  // dmax(a, b) = a > b ? a : b
    sr = sr_first ? b1 : b2;
  }
  // side fluxes L, R (h, x, y components) and states U
  T L[3], R[3];
  if (DIR == 0) {
    L[0] = qxl; L[1] = qxl * ul + T(kHalfG) * hl * hl; L[2] = qxl * vl;
    R[0] = qxr; R[1] = qxr * ur + T(kHalfG) * hr * hr; R[2] = qxr * vr;
  } else {
    L[0] = qyl; L[1] = qxl * vl; L[2] = qyl * vl + T(kHalfG) * hl * hl;
    R[0] = qyr; R[1] = qxr * vr; R[2] = qyr * vr + T(kHalfG) * hr * hr;
  }
  const T UL[3] = {hl, qxl, qyl}, UR[3] = {hr, qxr, qyr};
  T gF[3] = {gfh, gfqx, gfqy};
  T gL[3] = {0, 0, 0}, gR[3] = {0, 0, 0}, gUL[3] = {0, 0, 0}, gUR[3] = {0, 0, 0};
  T gsl = T(0), gsr = T(0);
  T gul = T(0), gvl = T(0), gur = T(0), gvr = T(0);
  if (sl >= T(0)) {
    for (int k = 0; k < 3; ++k) gL[k] += gF[k];
  } else if (sr <= T(0)) {
    for (int k = 0; k < 3; ++k) gR[k] += gF[k];
  } else {
    const T inv = T(1) / (sr - sl);
    const T slsr = sl * sr;
    const int t = DIR == 0 ? 2 : 1;  // tangential component
    if (HLLC) {
      // tangential flux = fh * (upwind tangential velocity) (rki_kernel_flux.F90:584-783)
      const T un_l = DIR == 0 ? ul : vl, un_r = DIR == 0 ? ur : vr;
      const T ut_l = DIR == 0 ? vl : ul, ut_r = DIR == 0 ? vr : ur;
      const T hrr = hr, hll = hl;
      const T den = hrr * (un_r - sr) - hll * (un_l - sl);
      T ss;
      if (fabs(den) > T(kDry))
        ss = (sl * hrr * (un_r - sr) - sr * hll * (un_l - sl)) / den;
      else
        ss = T(0.5) * (un_l + un_r);
      const T fh = (sr * L[0] - sl * R[0] + slsr * (UR[0] - UL[0])) * inv;
      const T gt = gF[t];
      gF[0] += gt * (ss >= T(0) ? ut_l : ut_r);
      if (ss >= T(0)) {
        if (DIR == 0) gvl += gt * fh; else gul += gt * fh;
      } else {
        if (DIR == 0) gvr += gt * fh; else gur += gt * fh;
      }
      gF[t] = T(0);
    }
    for (int k = 0; k < 3; ++k) {
      if (HLLC && k == t) continue;
      const T d = UR[k] - UL[k];
      const T F = (sr * L[k] - sl * R[k] + slsr * d) * inv;
      gL[k] += gF[k] * sr * inv;
      gR[k] += -gF[k] * sl * inv;
      gUR[k] += gF[k] * slsr * inv;
      gUL[k] += -gF[k] * slsr * inv;
      gsr += gF[k] * ((L[k] + sl * d) * inv - F * inv);
      gsl += gF[k] * ((-R[k] + sr * d) * inv + F * inv);
    }
  }
  // wave speeds
  T gnl = T(0), gnr = T(0), gal = T(0), gar = T(0);
  if (branch == 0) {
    gnl += gsl + gsr;
    gal += -gsl + T(2) * gsr;
  } else if (branch == 1) {
    gnr += gsl + gsr;
    gar += -T(2) * gsl + gsr;
  } else {
    if (sl_first) { gnl += gsl; gal -= gsl; } else { gnr += gsl; gar -= gsl; }
    if (sr_first) { gnl += gsr; gal += gsr; } else { gnr += gsr; gar += gsr; }
  }
  if (DIR == 0) { gul += gnl; gur += gnr; } else { gvl += gnl; gvr += gnr; }
  T ghl = T(0), ghr = T(0);
  if (al > T(0)) ghl += gal * T(kG) / (T(2) * al);
  if (ar > T(0)) ghr += gar * T(kG) / (T(2) * ar);
  // side fluxes -> (q, u, v, h)
  T gqxl = T(0), gqyl = T(0), gqxr = T(0), gqyr = T(0);
  if (DIR == 0) {
    gqxl += gL[0] + gL[1] * ul + gL[2] * vl;
    gul += gL[1] * qxl;
    gvl += gL[2] * qxl;
    ghl += gL[1] * T(2) * T(kHalfG) * hl;
    gqxr += gR[0] + gR[1] * ur + gR[2] * vr;
    gur += gR[1] * qxr;
    gvr += gR[2] * qxr;
    ghr += gR[1] * T(2) * T(kHalfG) * hr;
  } else {
    gqyl += gL[0] + gL[2] * vl;
    gqxl += gL[1] * vl;
    gvl += gL[1] * qxl + gL[2] * qyl;
    ghl += gL[2] * T(2) * T(kHalfG) * hl;
    gqyr += gR[0] + gR[2] * vr;
    gqxr += gR[1] * vr;
    gvr += gR[1] * qxr + gR[2] * qyr;
    ghr += gR[2] * T(2) * T(kHalfG) * hr;
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
template <int DIR, bool HLLC, typename T>
RKB_HD void face_adj(T eL, T qxL, T qyL, T bL, T eR, T qxR,
                     T qyR, T bR, const T gout[6], T gin[8]) {
  const T hL = pos(eL - bL);
  const T hR = pos(eR - bR);
  const bool bl_max = bL > bR;  // dmax(bL, bR) = bL > bR ? bL : bR
  const T bmax = bl_max ? bL : bR;
  const T xl = hL + bL - bmax, xr = hR + bR - bmax;
  const T hyl = pos(xl);
  const T hyr = pos(xr);
  T ul, vl, ur, vr;
  velocity(hL, qxL, qyL, ul, vl);
  velocity(hR, qxR, qyR, ur, vr);
  T gr[6] = {0, 0, 0, 0, 0, 0};
  riemann_adj<DIR, HLLC>(hyl, hyl * ul, hyl * vl, hyr, hyr * ur, hyr * vr, gout[0], gout[1],
                         gout[2], gr);
  T ghyl = gr[0], ghyr = gr[3];
  T gul = T(0), gvl = T(0), gur = T(0), gvr = T(0);
  ghyl += gr[1] * ul + gr[2] * vl;
  gul += gr[1] * hyl;
  gvl += gr[2] * hyl;
  ghyr += gr[4] * ur + gr[5] * vr;
  gur += gr[4] * hyr;
  gvr += gr[5] * hyr;
  T ghL = T(0), ghR = T(0);
  ghyr += T(2) * hyr * gout[3];
  ghR += -T(2) * hR * gout[3];
  ghyl += T(2) * hyl * gout[4];
  ghL += T(2) * hL * gout[5];
  T gqxL = T(0), gqyL = T(0), gqxR = T(0), gqyR = T(0);
  velocity_adj(hL, qxL, qyL, gul, gvl, ghL, gqxL, gqyL);
  velocity_adj(hR, qxR, qyR, gur, gvr, ghR, gqxR, gqyR);
  T gbL = T(0), gbR = T(0), gbmax = T(0);
  if (xl > T(0)) { ghL += ghyl; gbL += ghyl; gbmax -= ghyl; }
  if (xr > T(0)) { ghR += ghyr; gbR += ghyr; gbmax -= ghyr; }
  if (bl_max) gbL += gbmax; else gbR += gbmax;
  T geL = T(0), geR = T(0);
  if (eL - bL > T(0)) { geL += ghL; gbL -= ghL; }
  if (eR - bR > T(0)) { geR += ghR; gbR -= ghR; }
  gin[0] += geL; gin[1] += gqxL; gin[2] += gqyL; gin[3] += gbL;
  gin[4] += geR; gin[5] += gqxR; gin[6] += gqyR; gin[7] += gbR;
}

// Adjoint of protect(h, u, v) at input (h, u, v): (gh, gu, gv) are the output
// adjoints on entry and the input adjoints on return.
template <typename T>
RKB_HD void protect_adj(T h, T u, T v, T& gh, T& gu, T& gv) {
  if (h < T(0)) {
    gh = T(0); gu = T(0); gv = T(0);
    return;
  }
  if (h < T(kDry)) {
    gu = T(0); gv = T(0);
    return;
  }
  // forward with intermediates
  const T h2 = h * h;
  const T h4 = h2 * h2;
  const bool kp = h4 < T(kEps4);
  T u1 = u, v1 = v, r = T(0);
  if (kp) {
    r = sqrt(h4 + T(kEps4));
    u1 = h * (T(kSqrt2) * h * u / r);
    v1 = h * (T(kSqrt2) * h * v / r);
  }
  const T sp2 = (u1 * u1 + v1 * v1) / (h * h);
  const T fr2 = T(kFroude) * T(kFroude) * T(kG) * h;
  T ghh = gh, gu1 = gu, gv1 = gv;
  if (sp2 > fr2) {
    // u2 = u1 sqrt(fr2 / sp2) = u1 sqrt(F^2 g h^3 / (u1^2 + v1^2))
    const T sc = sqrt(fr2 / sp2);
    const T q2 = u1 * u1 + v1 * v1;
    // d sc / d u1 = -sc u1 / q2, d sc / d h = 1.5 sc / h
    const T gsc = gu * u1 + gv * v1;
    gu1 = gu * sc - gsc * sc * u1 / q2;
    gv1 = gv * sc - gsc * sc * v1 / q2;
    ghh += gsc * T(1.5) * sc / h;
  }
  T gu0 = gu1, gv0 = gv1;
  if (kp) {
    // u1 = sqrt2 h^2 u / r, r = sqrt(h^4 + eps4): d/du = sqrt2 h^2 / r,
    // d/dh = sqrt2 u (2 h / r - h^2 * 2 h^3 / r^3)
    const T f = T(kSqrt2) * h2 / r;
    const T df = T(kSqrt2) * (T(2) * h / r - h2 * T(2) * h * h2 / (r * r * r));
    gu0 = gu1 * f;
    gv0 = gv1 * f;
    ghh += (gu1 * u + gv1 * v) * df;
  }
  gh = ghh;
  gu = gu0;
  gv = gv0;
}

// Manning friction of sources() with a per-cell n (rki_kernel_fused.F90:121-130).
template <typename T>
RKB_HD void friction(T h, T& u, T& v, T n, T dt) {
  if (h > T(kDry) && n > T(0)) {
    const T n_sq = n * n;
    const T uu = u / h;
    const T vv = v / h;
    const T speed = sqrt(uu * uu + vv * vv);
    const T cf = T(kG) * n_sq / pow_third(h);
    const T den = T(1) + dt * cf * speed / h;
    u = u / den;
    v = v / den;
  }
}

// Adjoint of friction at input (h, u, v, n): (gu, gv) output adjoints in,
// input adjoints out; gh, gn accumulated.
// The quotients share one reciprocal per denominator (h, h^(1/3), den, sp),
// and h^(1/3) is the math library's cube root rather than the correctly
// rounded one of the forward step: here they only scale adjoints, and no
// branch depends on them.
template <typename T>
RKB_HD void friction_adj(T h, T u, T v, T n, T dt, T& gh,
                         T& gu, T& gv, T& gn) {
  if (!(h > T(kDry) && n > T(0))) return;
  const T rh = T(1) / h;
  const T uu = u * rh, vv = v * rh;
  const T sp = sqrt(uu * uu + vv * vv);
  const T c3 = cbrt(h);
  const T rc3 = T(1) / c3;
  const T cf = T(kG) * n * n * rc3;
  const T den = T(1) + dt * cf * sp * rh;
  const T rden = T(1) / den;
  const T gden = -(gu * u + gv * v) * rden * rden;
  T gu0 = gu * rden, gv0 = gv * rden;
  const T gcf = gden * dt * sp * rh;
  const T gsp = gden * dt * cf * rh;
  gh += gden * (-dt * cf * sp * rh * rh);
  gn += gcf * T(2) * T(kG) * n * rc3;
  const T gc3 = -gcf * cf * rc3;
  gh += gc3 * c3 * rh * T(1.0 / 3.0);
  if (sp > T(0)) {
    const T rsp = T(1) / sp;
    const T guu = gsp * uu * rsp, gvv = gsp * vv * rsp;
    gu0 += guu * rh;
    gv0 += gvv * rh;
    gh += -(guu * uu + gvv * vv) * rh;
  }
  gu = gu0;
  gv = gv0;
}

// minmod branch: 0 = zero, 1 = first argument, 2 = second (rki_kernel_flux.F90:380-393)
template <typename T>
RKB_HD int minmod_choice(T a, T b) {
  if (a * b <= T(0)) return 0;
  return fabs(a) < fabs(b) ? 1 : 2;
}

}  // namespace rkb
