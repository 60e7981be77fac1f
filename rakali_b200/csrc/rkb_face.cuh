// Face-level numerics of the structured barotropic flux.
//
// Templates on the real type T (double in the production step and the FP64
// adjoint, float in the FP32 adjoint); constants enter as T(c).
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
template <typename T>
struct FaceOutT {
  T fh, fqx, fqy;
  T wbR, hL2, pL2;
};
using FaceOut = FaceOutT<double>;

template <typename T>
__host__ __device__ __forceinline__ void velocity(T h, T qx, T qy, T& u, T& v) {
  if (h > T(kDry)) {
    u = qx / h;
    v = qy / h;
  } else {
    u = T(0);
    v = T(0);
  }
}

// HLL / HLLC in direction DIR (0: x, normal momentum qx; 1: y, normal qy).
// hll_flux_x/y rki_kernel_flux.F90:410-582, hllc_flux_x/y :584-783.
template <int DIR, bool HLLC, typename T>
__host__ __device__ __forceinline__ void riemann(T hl, T qxl, T qyl, T hr, T qxr, T qyr, T& fh,
                                                 T& fqx, T& fqy) {
  T ul, vl, ur, vr;
  velocity(hl, qxl, qyl, ul, vl);
  velocity(hr, qxr, qyr, ur, vr);
  const T al = sqrt(T(kG) * pos(hl));
  const T ar = sqrt(T(kG) * pos(hr));
  const T nl = DIR == 0 ? ul : vl;
  const T nr = DIR == 0 ? ur : vr;
  T sl, sr;
  if (hr <= T(kDry)) {
    sl = nl - al;
    sr = nl + T(2) * al;
  } else if (hl <= T(kDry)) {
    sl = nr - T(2) * ar;
    sr = nr + ar;
  } else {
    sl = dmin(nl - al, nr - ar);
    sr = dmax(nl + al, nr + ar);
  }
  T lh, lx, ly, rh, rx, ry;
  if (DIR == 0) {
    lh = qxl;
    lx = qxl * ul + T(kHalfG) * hl * hl;
    ly = qxl * vl;
    rh = qxr;
    rx = qxr * ur + T(kHalfG) * hr * hr;
    ry = qxr * vr;
  } else {
    lh = qyl;
    lx = qxl * vl;
    ly = qyl * vl + T(kHalfG) * hl * hl;
    rh = qyr;
    rx = qxr * vr;
    ry = qyr * vr + T(kHalfG) * hr * hr;
  }
  if (sl >= T(0)) {
    fh = lh; fqx = lx; fqy = ly;
    return;
  }
  if (sr <= T(0)) {
    fh = rh; fqx = rx; fqy = ry;
    return;
  }
  const T inv = T(1) / (sr - sl);
  const T slsr = sl * sr;
  fh = (sr * lh - sl * rh + slsr * (hr - hl)) * inv;
  if (DIR == 0) {
    fqx = (sr * lx - sl * rx + slsr * (qxr - qxl)) * inv;
    if (!HLLC) {
      fqy = (sr * ly - sl * ry + slsr * (qyr - qyl)) * inv;
    } else {
      const T den = hr * (ur - sr) - hl * (ul - sl);
      T ss;
      if (fabs(den) > T(kDry))
        ss = (sl * hr * (ur - sr) - sr * hl * (ul - sl)) / den;
      else
        ss = T(0.5) * (ul + ur);
      fqy = ss >= T(0) ? fh * vl : fh * vr;
    }
  } else {
    fqy = (sr * ly - sl * ry + slsr * (qyr - qyl)) * inv;
    if (!HLLC) {
      fqx = (sr * lx - sl * rx + slsr * (qxr - qxl)) * inv;
    } else {
      const T den = hr * (vr - sr) - hl * (vl - sl);
      T ss;
      if (fabs(den) > T(kDry))
        ss = (sl * hr * (vr - sr) - sr * hl * (vl - sl)) / den;
      else
        ss = T(0.5) * (vl + vr);
      fqx = ss >= T(0) ? fh * ul : fh * ur;
    }
  }
}

// One face from the reconstructed side values (eta, hu, hv) and the beds.
// The Audusse step follows rki_kernel_flux.F90:186-224.
template <int DIR, bool HLLC, typename T>
__host__ __device__ __forceinline__ void face_flux(T eL, T qxL, T qyL, T bL, T eR, T qxR, T qyR,
                                                   T bR, FaceOutT<T>& o) {
  const T hL = pos(eL - bL);
  const T hR = pos(eR - bR);
  const T bmax = dmax(bL, bR);
  const T hyl = pos(hL + bL - bmax);
  const T hyr = pos(hR + bR - bmax);
  T ul, vl, ur, vr;
  velocity(hL, qxL, qyL, ul, vl);
  velocity(hR, qxR, qyR, ur, vr);
  riemann<DIR, HLLC>(hyl, hyl * ul, hyl * vl, hyr, hyr * ur, hyr * vr, o.fh, o.fqx, o.fqy);
  o.wbR = hyr * hyr - hR * hR;
  o.hL2 = hyl * hyl;
  o.pL2 = hL * hL;
}

// Limited slope of one cell along one direction (rki_kernel_flux.F90:159-181):
// zero near wet/dry fronts, else minmod of the one-sided differences.
template <typename T>
__host__ __device__ __forceinline__ void cell_slope(T hm, T hc, T hp, T em, T ec, T ep, T um, T uc,
                                                    T up, T vm, T vc, T vp, T& se, T& su, T& sv) {
  if (hc < T(kThin) || hm < T(kDry) || hp < T(kDry)) {
    se = T(0); su = T(0); sv = T(0);
  } else {
    se = minmod(ec - em, ep - ec);
    su = minmod(uc - um, up - uc);
    sv = minmod(vc - vm, vp - vc);
  }
}

}  // namespace rkb
