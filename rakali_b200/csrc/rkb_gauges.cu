// Gauge (station) time series recorded on the device (src/io/structured/
// rki_gauges.F90).  Stations get the reference's bilinear stencil and weights
// on the host (compute_local_gauges / compute_interp_weights, :208-336); after
// every step a one-block kernel, captured in the step graphs, decides from
// the device clock whether this step is a gauge time (rki_driver.F90:469-473,
// :777-799: every step when the interval is <= 0, else when t >= the next
// gauge time, which then advances by one interval) and appends eta, u, v of
// every station to a device buffer (gauges_write, rki_gauges.F90:490-575).
// No host synchronisation per step; the host drains the buffer on demand.
//
// Compiled with --fmad=false: the interpolation is evaluated in the
// reference's expression order, so with the FP64 form the records equal the
// same formula applied to the oracle's state bit for bit.
#include <cmath>

#include "rkb_gauges.hpp"

namespace rkb {

namespace {

// Bilinear value of a field at stencil (i0, j0) with weights (wx, wy),
// (1-wx)(1-wy) a00 + wx(1-wy) a10 + (1-wx)wy a01 + wx wy a11.
__device__ __forceinline__ double blend(double a00, double a10, double a01, double a11, double wx,
                                        double wy) {
  return (1.0 - wx) * (1.0 - wy) * a00 + wx * (1.0 - wy) * a10 + (1.0 - wx) * wy * a01 +
         wx * wy * a11;
}

// Thread 0 decides whether this step is a gauge time and claims a record.
__device__ __forceinline__ int claim_record(const StepCtl* ctl, GaugeDev* gd) {
  __shared__ int slot;
  if (threadIdx.x == 0) {
    slot = -1;
    if (ctl->active) {
      const double t = ctl->t;
      if (gd->interval <= 0.0 || t >= gd->next) {
        if (gd->count < gd->cap) {
          slot = gd->count;
          gd->count = slot + 1;
          gd->rec_t[slot] = t;
        } else {
          gd->overflow = 1;
        }
        if (gd->interval > 0.0) gd->next = gd->next + gd->interval;
      }
    }
  }
  __syncthreads();
  return slot;
}

__device__ __forceinline__ void store(GaugeDev* gd, int s, int k, double h, double hu, double hv,
                                      double b) {
  const double h_safe = h > 1.0e-6 ? h : 1.0e-6;  // MIN_DEPTH, rki_gauges.F90:507
  double* r = gd->rec + ((size_t)s * gd->n + k) * 3;
  r[0] = h + b;
  r[1] = hu / h_safe;
  r[2] = hv / h_safe;
}

__global__ void k_gauge_record(Grid g, const StepCtl* ctl, GaugeDev* gd, FieldSet U0, FieldSet U1,
                               const double* __restrict__ bed) {
  const int s = claim_record(ctl, gd);
  if (s < 0) return;
  const FieldSet F = ctl->cur ? U1 : U0;  // the state after the step
  for (int k = threadIdx.x; k < gd->n; k += blockDim.x) {
    const int i0 = gd->ix0[k], j0 = gd->iy0[k];
    const double wx = gd->wx[k], wy = gd->wy[k];
    const size_t q00 = g.at(i0, j0), q10 = g.at(i0 + 1, j0), q01 = g.at(i0, j0 + 1),
                 q11 = g.at(i0 + 1, j0 + 1);
    const double h = blend(F.h[q00], F.h[q10], F.h[q01], F.h[q11], wx, wy);
    const double hu = blend(F.hu[q00], F.hu[q10], F.hu[q01], F.hu[q11], wx, wy);
    const double hv = blend(F.hv[q00], F.hv[q10], F.hv[q01], F.hv[q11], wx, wy);
    const double b = blend(bed[q00], bed[q10], bed[q01], bed[q11], wx, wy);
    store(gd, s, k, h, hu, hv, b);
  }
}

// FP32 surface form: depth max(0, eta - b) in FP64 at each corner.
__global__ void k_gauge_record32(Grid g, const StepCtl* ctl, GaugeDev* gd, FieldSet32 U0,
                                 FieldSet32 U1, const double* __restrict__ bed) {
  const int s = claim_record(ctl, gd);
  if (s < 0) return;
  const FieldSet32 F = ctl->cur ? U1 : U0;
  for (int k = threadIdx.x; k < gd->n; k += blockDim.x) {
    const int i0 = gd->ix0[k], j0 = gd->iy0[k];
    const double wx = gd->wx[k], wy = gd->wy[k];
    const size_t q[4] = {g.at(i0, j0), g.at(i0 + 1, j0), g.at(i0, j0 + 1), g.at(i0 + 1, j0 + 1)};
    double hh[4], uu[4], vv[4], bb[4];
    for (int c = 0; c < 4; ++c) {
      bb[c] = bed[q[c]];
      const double d = (double)F.eta[q[c]] - bb[c];
      hh[c] = d > 0.0 ? d : 0.0;
      uu[c] = (double)F.hu[q[c]];
      vv[c] = (double)F.hv[q[c]];
    }
    store(gd, s, k, blend(hh[0], hh[1], hh[2], hh[3], wx, wy),
          blend(uu[0], uu[1], uu[2], uu[3], wx, wy), blend(vv[0], vv[1], vv[2], vv[3], wx, wy),
          blend(bb[0], bb[1], bb[2], bb[3], wx, wy));
  }
}

}  // namespace

void gauge_stencils(const Grid& g, const double* x, const double* y, int n, GaugeStencils& out) {
  const int nx = g.nx_phys(), ny = g.ny_phys(), ng = g.ng;
  const double dx = g.dx, dy = g.dy;
  out = GaugeStencils{};
  for (int k = 0; k < n; ++k) {
    // compute_local_gauges (:208-243): the 1-based physical cell of the
    // station.  floor(q) + 1 lies in [1, n] exactly when q = x / dx lies in
    // [0, n), so testing q first gives the reference's inside-domain answer
    // for every finite coordinate and drops NaN, infinite and huge ones
    // before any conversion to int.
    const double qx = x[k] / dx, qy = y[k] / dy;
    if (!(qx >= 0.0 && qx < (double)nx && qy >= 0.0 && qy < (double)ny)) continue;
    const int ig = (int)std::floor(qx) + 1;
    const int jg = (int)std::floor(qy) + 1;
    // compute_interp_weights (:245-336), 1-based array indices ia, ja
    const int ia = ig + ng, ja = jg + ng;
    const double xc = ((double)ig - 0.5) * dx, yc = ((double)jg - 0.5) * dy;
    int ix0, iy0;
    double wx, wy;
    if (x[k] < xc) {
      if (ig > 1) { ix0 = ia - 1; wx = (x[k] - (xc - dx)) / dx; }
      else { ix0 = ia; wx = 0.0; }
    } else {
      if (ig < nx) { ix0 = ia; wx = (x[k] - xc) / dx; }
      else { ix0 = ia; wx = 0.0; }
    }
    if (y[k] < yc) {
      if (jg > 1) { iy0 = ja - 1; wy = (y[k] - (yc - dy)) / dy; }
      else { iy0 = ja; wy = 0.0; }
    } else {
      if (jg < ny) { iy0 = ja; wy = (y[k] - yc) / dy; }
      else { iy0 = ja; wy = 0.0; }
    }
    wx = std::fmax(0.0, std::fmin(1.0, wx));
    wy = std::fmax(0.0, std::fmin(1.0, wy));
    out.station.push_back(k);
    out.ix0.push_back(ix0 - 1);  // 0-based
    out.iy0.push_back(iy0 - 1);
    out.wx.push_back(wx);
    out.wy.push_back(wy);
  }
}

cudaError_t launch_gauge_record(const Grid& g, const StepCtl* ctl, GaugeDev* gd, int n,
                                const FieldSet& U0, const FieldSet& U1, const double* b,
                                cudaStream_t s) {
  const int tpb = n > 128 ? 256 : 128;
  k_gauge_record<<<1, tpb, 0, s>>>(g, ctl, gd, U0, U1, b);
  return cudaGetLastError();
}

cudaError_t launch_gauge_record32(const Grid& g, const StepCtl* ctl, GaugeDev* gd, int n,
                                  const FieldSet32& U0, const FieldSet32& U1, const double* b,
                                  cudaStream_t s) {
  const int tpb = n > 128 ? 256 : 128;
  k_gauge_record32<<<1, tpb, 0, s>>>(g, ctl, gd, U0, U1, b);
  return cudaGetLastError();
}

}  // namespace rkb
