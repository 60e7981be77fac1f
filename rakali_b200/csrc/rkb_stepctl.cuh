// Step control, boundary-edge geometry and block reductions shared by the
// FP64 and FP32 step kernels.  Each translation unit compiles these with its
// own floating-point flags; everything here is FP64 arithmetic on scalars.
#pragma once

#include "rkb_common.cuh"
#include "rkb_crmath.cuh"

namespace rkb {

// Decide whether this step runs and its dt (rki_api.F90:385-410 loop test,
// rki_solver.F90:731-748).  Reads only fields that stay fixed during a step,
// so every thread of the first launch computes the same answer.
__device__ __forceinline__ bool step_begin(const StepCtl* c, const Physics* p, const Grid& g,
                                           double& dt) {
  double dt_max;
  bool active;
  if (c->mode == 0) {
    active = c->t < c->target - 1.0e-10;
    dt_max = c->target - c->t;
  } else {
    active = c->remaining > 0;
    dt_max = p->t_end - c->t;
  }
  dt = c->dt_prev;
  if (c->error != 0) active = false;  // a step reported an error: the rest of the chunk idles
  if (!active) return false;
  if (p->dt_fixed > 0.0) {
    dt = dmin(p->dt_fixed, dt_max);
  } else if (c->step_count % p->cfl_interval == 0 || c->dt_prev <= 0.0) {
    dt = cfl_dt(c->msx, c->msy, g, p->cfl) * p->ssp_coeff;
    dt = dmin(dt, dt_max);
  }
  return true;
}

// Sponge relaxation rate of interior cell (i, j) (rki_kernel_sponge.F90:16-88):
// strength * ((width - d) / width)^2 with d the distance to the nearest sponge
// edge, 0 outside every sponge layer.
__device__ __forceinline__ double sponge_alpha(const BcParams* bc, const Grid& g, int i, int j) {
  const int sw = bc->sponge_width;
  if (sw <= 0 || bc->sponge_strength <= 0.0) return 0.0;
  const int i0 = g.ng, i1 = g.nxt - g.ng - 1, j0 = g.ng, j1 = g.nyt - g.ng - 1;
  int dmn = sw + 1;
  if (bc->type[0] == kSponge && i - i0 < sw && i - i0 < dmn) dmn = i - i0;
  if (bc->type[1] == kSponge && i1 - i < sw && i1 - i < dmn) dmn = i1 - i;
  if (bc->type[2] == kSponge && j - j0 < sw && j - j0 < dmn) dmn = j - j0;
  if (bc->type[3] == kSponge && j1 - j < sw && j1 - j < dmn) dmn = j1 - j;
  if (dmn >= sw) return 0.0;
  const double ratio = (double)(sw - dmn) / (double)sw;
  return bc->sponge_strength * ratio * ratio;
}

// Boundary edge geometry (rki_boundary.F90:40-218)

struct Edge {
  int ig0, jg0, din, djn, dit, djt, n_tan;
  double sgn;
  bool normal_u;
};

// Edge geometry of rki_boundary.F90:75-84 in 0-based indices.
__device__ __forceinline__ Edge make_edge(int w, const Grid& g) {
  Edge e;
  switch (w) {
    case 0: e = {g.ng - 1, 0, -1, 0, 0, 1, g.nyt, -1.0, true}; break;
    case 1: e = {g.nxt - g.ng, 0, 1, 0, 0, 1, g.nyt, 1.0, true}; break;
    case 2: e = {0, g.ng - 1, 0, -1, 1, 0, g.nxt, -1.0, false}; break;
    default: e = {0, g.nyt - g.ng, 0, 1, 1, 0, g.nxt, 1.0, false}; break;
  }
  return e;
}

__device__ __forceinline__ double tidal_eta(const BcParams* bc, double time) {
  double eta = 0.0;
  if (bc->n_tidal > 0) {
    for (int n = 0; n < bc->n_tidal; ++n)
      eta = eta + bc->amp[n] * cr_cos(bc->omega[n] * time - bc->phase[n]);
  } else if (bc->tidal_period > 0.0) {
    eta = bc->tidal_amplitude * cr_sin(kTwoPi * time / bc->tidal_period);
  }
  return eta;
}

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Close a step (one block: k_close after the last FP64 stage, or the last
// block of a marching or FP32 sweep kernel): fixed-order sums of the
// partials, the mass budget in the reference's order
// (rki_solver.F90:507-657), the CFL maxima of the new state and the clock.
// `budget` false: the generic Shu-Osher schemes, which do not accumulate the
// boundary mass budget (rki_solver.F90:861-926).
static __device__ void finalize_step(const Grid& g, StepCtl* ctl, const Physics* phys,
                              double* partials, unsigned int nparts, double dt, int cur,
                              bool budget = true) {
  const int tid = threadIdx.x;
  const int nthr = (int)blockDim.x;  // a multiple of 32
  const double area = g.dx * g.dy;
  // Fixed-order sums of the partials over every thread of this block: thread
  // t adds partials t, t + nthr, ... in order (L2 loads: earlier kernels or
  // blocks wrote them), each warp combines its lanes by butterfly, and thread
  // 0 adds the warp results in warp order.
  __shared__ double red[4][32];
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (budget) {
    // eight rows of loads in flight per thread; the additions keep their order
#pragma unroll 8
    for (unsigned int k = tid; k < nparts; k += nthr)
      for (int s = 0; s < 4; ++s) acc[s] = acc[s] + __ldcg(partials + (size_t)s * nparts + k);
  }
  for (int s = 0; s < 4; ++s) {
    const double w = warp_sum(acc[s]);
    if ((tid & 31) == 0) red[s][tid >> 5] = w;
  }
  __syncthreads();
  double sums[4] = {0.0, 0.0, 0.0, 0.0};
  if (tid == 0)
    for (int w = 0; w < nthr / 32; ++w)
      for (int s = 0; s < 4; ++s) sums[s] = sums[s] + red[s][w];
  if (tid == 0 && budget) {
    double mo = ctl->mass_out;
    mo = mo - 0.5 * dt * sums[0] * area;
    mo = mo - 0.5 * dt * sums[2] * area;
    ctl->mass_out = mo;
    double ms = ctl->mass_src;
    if (phys->forcing_active) ms = ms + 0.5 * dt * ctl->precip_sum * area;
    ms = ms + 0.5 * sums[1] * area;
    if (phys->forcing_active) ms = ms + 0.5 * dt * ctl->precip_sum * area;
    ms = ms + 0.5 * sums[3] * area;
    ctl->mass_src = ms;
  }
  if (tid == 0) {
    volatile StepCtl* vc = ctl;
    ctl->msx = __longlong_as_double((long long)vc->msx_next);
    ctl->msy = __longlong_as_double((long long)vc->msy_next);
    ctl->msx_next = 0ull;
    ctl->msy_next = 0ull;
    ctl->ms_valid = 1;
    ctl->t = ctl->t + dt;
    ctl->dt_prev = dt;
    ctl->step_count = ctl->step_count + 1;
    ctl->remaining = ctl->remaining - 1;
    ctl->steps_run = ctl->steps_run + 1;
    ctl->cur = cur ^ 1;
    ctl->done_blocks = 0u;
  }
}

}  // namespace rkb
