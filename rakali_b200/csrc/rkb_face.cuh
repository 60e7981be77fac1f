// Face-level numerics of the structured barotropic flux (FP64).
//
// One call evaluates one cell face: Audusse hydrostatic reconstruction of the
// two side states, then the HLL or HLLC Riemann flux.  The reference
// (rki_kernel_flux.F90:104-378, flux_cell) evaluates every interior face
// twice, once from each neighbour, and the two evaluations are bit-identical;
// the B200 kernels evaluate each face once and share it through shared memory.
#pragma once

#include "rkb_common.cuh"

namespace rkb {

// Outputs of one face.  wbR is the right-side well-balanced term
// h_hyd^2 - h_pre^2 (the neighbour to the right adds it first); hL2 and pL2
// are the left side's h_hyd^2 and h_pre^2, subtracted and added in that order
// by the neighbour to the left (rki_kernel_flux.F90:361-369).
struct FaceOut {
  double fh, fqx, fqy;
  double wbR, hL2, pL2;
};

__host__ __device__ __forceinline__ void velocity(double h, double qx, double qy, double& u, double& v) {
  if (h > kDry) {
    u = qx / h;
    v = qy / h;
  } else {
    u = 0.0;
    v = 0.0;
  }
}

// HLL / HLLC in direction DIR (0: x, normal momentum qx; 1: y, normal qy).
// hll_flux_x/y rki_kernel_flux.F90:410-582, hllc_flux_x/y :584-783.
template <int DIR, bool HLLC>
__host__ __device__ __forceinline__ void riemann(double hl, double qxl, double qyl, double hr, double qxr,
                                        double qyr, double& fh, double& fqx, double& fqy) {
  double ul, vl, ur, vr;
  velocity(hl, qxl, qyl, ul, vl);
  velocity(hr, qxr, qyr, ur, vr);
  const double al = sqrt(kG * pos(hl));
  const double ar = sqrt(kG * pos(hr));
  const double nl = DIR == 0 ? ul : vl;
  const double nr = DIR == 0 ? ur : vr;
  double sl, sr;
  if (hr <= kDry) {
    sl = nl - al;
    sr = nl + 2.0 * al;
  } else if (hl <= kDry) {
    sl = nr - 2.0 * ar;
    sr = nr + ar;
  } else {
    sl = dmin(nl - al, nr - ar);
    sr = dmax(nl + al, nr + ar);
  }
  double lh, lx, ly, rh, rx, ry;
  if (DIR == 0) {
    lh = qxl;
    lx = qxl * ul + kHalfG * hl * hl;
    ly = qxl * vl;
    rh = qxr;
    rx = qxr * ur + kHalfG * hr * hr;
    ry = qxr * vr;
  } else {
    lh = qyl;
    lx = qxl * vl;
    ly = qyl * vl + kHalfG * hl * hl;
    rh = qyr;
    rx = qxr * vr;
    ry = qyr * vr + kHalfG * hr * hr;
  }
  if (sl >= 0.0) {
    fh = lh; fqx = lx; fqy = ly;
    return;
  }
  if (sr <= 0.0) {
    fh = rh; fqx = rx; fqy = ry;
    return;
  }
  const double inv = 1.0 / (sr - sl);
  const double slsr = sl * sr;
  fh = (sr * lh - sl * rh + slsr * (hr - hl)) * inv;
  if (DIR == 0) {
    fqx = (sr * lx - sl * rx + slsr * (qxr - qxl)) * inv;
    if (!HLLC) {
      fqy = (sr * ly - sl * ry + slsr * (qyr - qyl)) * inv;
    } else {
      const double den = hr * (ur - sr) - hl * (ul - sl);
      double ss;
      if (fabs(den) > kDry)
        ss = (sl * hr * (ur - sr) - sr * hl * (ul - sl)) / den;
      else
        ss = 0.5 * (ul + ur);
      fqy = ss >= 0.0 ? fh * vl : fh * vr;
    }
  } else {
    fqy = (sr * ly - sl * ry + slsr * (qyr - qyl)) * inv;
    if (!HLLC) {
      fqx = (sr * lx - sl * rx + slsr * (qxr - qxl)) * inv;
    } else {
      const double den = hr * (vr - sr) - hl * (vl - sl);
      double ss;
      if (fabs(den) > kDry)
        ss = (sl * hr * (vr - sr) - sr * hl * (vl - sl)) / den;
      else
        ss = 0.5 * (vl + vr);
      fqx = ss >= 0.0 ? fh * ul : fh * ur;
    }
  }
}

// One face from the reconstructed side values (eta, hu, hv) and the beds.
// The Audusse step follows rki_kernel_flux.F90:186-224.
template <int DIR, bool HLLC>
__host__ __device__ __forceinline__ void face_flux(double eL, double qxL, double qyL, double bL, double eR,
                                          double qxR, double qyR, double bR, FaceOut& o) {
  const double hL = pos(eL - bL);
  const double hR = pos(eR - bR);
  const double bmax = dmax(bL, bR);
  const double hyl = pos(hL + bL - bmax);
  const double hyr = pos(hR + bR - bmax);
  double ul, vl, ur, vr;
  velocity(hL, qxL, qyL, ul, vl);
  velocity(hR, qxR, qyR, ur, vr);
  riemann<DIR, HLLC>(hyl, hyl * ul, hyl * vl, hyr, hyr * ur, hyr * vr, o.fh, o.fqx, o.fqy);
  o.wbR = hyr * hyr - hR * hR;
  o.hL2 = hyl * hyl;
  o.pL2 = hL * hL;
}

// Limited slope of one cell along one direction (rki_kernel_flux.F90:159-181):
// zero near wet/dry fronts, else minmod of the one-sided differences.
__host__ __device__ __forceinline__ void cell_slope(double hm, double hc, double hp, double em, double ec,
                                           double ep, double um, double uc, double up, double vm,
                                           double vc, double vp, double& se, double& su,
                                           double& sv) {
  if (hc < kThin || hm < kDry || hp < kDry) {
    se = 0.0; su = 0.0; sv = 0.0;
  } else {
    se = minmod(ec - em, ep - ec);
    su = minmod(uc - um, up - uc);
    sv = minmod(vc - vm, vp - vc);
  }
}

}  // namespace rkb
