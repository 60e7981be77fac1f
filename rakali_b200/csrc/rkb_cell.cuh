// Pointwise cell terms of the FP64 stage update, shared by the fused stage
// kernels and the kernel-level entry points (both compiled with
// --fmad=false): Manning friction, wind, pressure gradient, Coriolis and
// precipitation (rki_kernel_fused.F90:121-154), and the sponge relaxation
// (rki_kernel_sponge.F90:16-88).
#pragma once

#include "rkb_crmath.cuh"
#include "rkb_kernels.h"
#include "rkb_stepctl.cuh"

namespace rkb {

// Pointwise sources after the Euler update: Manning friction, wind,
// pressure gradient, Coriolis, precipitation (rki_kernel_fused.F90:121-154).
__device__ __forceinline__ void sources(double& h, double& u, double& v, const Physics* p, double dt,
                                        double n_sq, double cosf, double sinf, bool has_cor,
                                        const Grid& g, int i, int j, const Forcing& fo) {
  if (h > kDry) {
    if (p->manning_n > 0.0) {
      const double uu = u / h;
      const double vv = v / h;
      const double speed = sqrt(uu * uu + vv * vv);
      const double cf = kG * n_sq / cr_pow_third(h);
      const double den = 1.0 + dt * cf * speed / h;
      u = u / den;
      v = v / den;
    }
    if (p->forcing_active) {
      const size_t q = g.at(i, j);
      u = u + dt * fo.wind_x[q] / kRho;
      v = v + dt * fo.wind_y[q] / kRho;
      const double dpdx = (fo.atm[g.at(i + 1, j)] - fo.atm[g.at(i - 1, j)]) / (2.0 * g.dx);
      const double dpdy = (fo.atm[g.at(i, j + 1)] - fo.atm[g.at(i, j - 1)]) / (2.0 * g.dy);
      u = u - dt * h * dpdx / kRho;
      v = v - dt * h * dpdy / kRho;
    }
    if (has_cor) {
      const double uo = u, vo = v;
      u = uo * cosf + vo * sinf;
      v = -(uo * sinf) + vo * cosf;
    }
  }
  if (p->forcing_active) h = h + dt * fo.precip[g.at(i, j)];
}

// Sponge relaxation of interior cell (i, j) (rki_kernel_sponge.F90:16-88).
__device__ __forceinline__ void sponge(double& h, double& u, double& v, const BcParams* bc,
                                       const Grid& g, int i, int j, double dt) {
  const double alpha = sponge_alpha(bc, g, i, j);
  if (alpha > 0.0) {
    h = h - dt * alpha * (h - bc->sponge_h_ref);
    u = u - dt * alpha * u;
    v = v - dt * alpha * v;
  }
}

}  // namespace rkb
