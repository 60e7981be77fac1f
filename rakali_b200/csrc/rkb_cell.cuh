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

// Semi-implicit Manning friction of a wet cell (rki_kernel_fused.F90:121-131).
__device__ __forceinline__ void manning(double h, double& u, double& v, double dt, double n_sq) {
  const double uu = u / h;
  const double vv = v / h;
  const double speed = sqrt(uu * uu + vv * vv);
  const double cf = kG * n_sq / cr_pow_third(h);
  const double den = 1.0 + dt * cf * speed / h;
  u = u / den;
  v = v / den;
}

// Pointwise sources after the Euler update: Manning friction, wind,
// pressure gradient, Coriolis, precipitation (rki_kernel_fused.F90:121-154).
__device__ __forceinline__ void sources(double& h, double& u, double& v, const Physics* p, double dt,
                                        double n_sq, double cosf, double sinf, bool has_cor,
                                        const Grid& g, int i, int j, const Forcing& fo) {
  if (h > kDry) {
    if (p->manning_n > 0.0) manning(h, u, v, dt, n_sq);
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

// The sources of a stage without forcing, Coriolis or sponge terms: Manning
// friction alone (the same expressions as sources()).
__device__ __forceinline__ void sources_plain(double& h, double& u, double& v, double manning_n,
                                              double dt, double n_sq) {
  if (h > kDry && manning_n > 0.0) manning(h, u, v, dt, n_sq);
}

// True when a stage has no forcing, Coriolis or sponge terms: the stage
// kernels then run their plain-physics build.
__host__ __device__ __forceinline__ bool plain_physics(const Physics& p, const BcParams& bc) {
  return p.forcing_active == 0 && !(fabs(p.coriolis_f) > 1.0e-20) &&
         !(bc.sponge_width > 0 && bc.sponge_strength > 0.0);
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
