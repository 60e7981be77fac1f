// Ghost-cell fill of one boundary edge (rki_boundary.F90:40-552), shared by
// the step's boundary launches and the kernel-level
// apply_boundary_conditions entry point.  Compiled with --fmad=false in both
// translation units, so both fill the same bits.
#pragma once

#include "rkb_kernels.h"
#include "rkb_stepctl.cuh"

namespace rkb {

// Fill the ghost layers of position t along edge w (0 W, 1 E, 2 S, 3 N) of
// F from its first interior cells, at boundary time `time` with the fill's dt
// `dtb` (Chapman).  Every ghost value also goes to (h2, hu2, hv2) when h2 is
// not null.  Wall and sponge edges mirror the bed into their ghosts, as the
// reference does (b is modified).  eo: the Chapman surface of this edge (one
// value per tangential position), read and then refreshed; chapman_fresh
// makes the fill use the current interior surface instead of the stored one
// (the extra fill the reference runs before computing dt).
__device__ __forceinline__ void fill_edge(const Grid& g, const BcParams* bc, double* __restrict__ b,
                                          const FieldSet& F, double* h2, double* hu2,
                                          double* hv2, int w, int t, double time, double dtb,
                                          double* eo, bool chapman_fresh) {
  const int type = bc->type[w];
  if (type == kNested) return;
  const Edge e = make_edge(w, g);
  if (t >= e.n_tan) return;
  double* h = F.h;
  double* hu = F.hu;
  double* hv = F.hv;

  // ghost (k) and first interior cell along the inward normal
  const int ii = e.ig0 + t * e.dit - e.din;
  const int ji = e.jg0 + t * e.djt - e.djn;

  auto put = [&](int ig, int jg, double vh, double vu, double vv) {
    const size_t q = g.at(ig, jg);
    h[q] = vh; hu[q] = vu; hv[q] = vv;
    if (h2) { h2[q] = vh; hu2[q] = vu; hv2[q] = vv; }
  };

  if (type == kWall || type == kSponge) {
    // bc_wall_edge :220-291 (bed and surface mirrored, normal momentum negated)
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const int im = ig - (2 * k - 1) * e.din;
      const int jm = jg - (2 * k - 1) * e.djn;
      const size_t m = g.at(im, jm);
      const double bm = b[m];
      b[g.at(ig, jg)] = bm;
      const double vh = pos(h[m] + bm - bm);
      double vu, vv;
      if (e.normal_u) { vu = -hu[m]; vv = hv[m]; } else { vv = -hv[m]; vu = hu[m]; }
      put(ig, jg, vh, vu, vv);
    }
    return;
  }

  const size_t qi = g.at(ii, ji);
  const double hi = h[qi];
  const double qu = hu[qi];
  const double qv = hv[qi];
  if (type == kOpen || type == kTidal) {
    // bc_flather_edge :293-345
    const bool prescribe = type == kTidal;
    const double eta_ext = prescribe ? tidal_eta(bc, time) : 0.0;
    const double ei = hi + b[qi];
    const double hmax = dmax(hi, 1.0e-6);
    const double c = sqrt(kG * hmax);
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const double hg = prescribe ? pos(eta_ext - b[g.at(ig, jg)]) : hi;
      if (e.normal_u)
        put(ig, jg, hg, hg * (qu / hmax + e.sgn * c * (ei - eta_ext) / hmax), qv);
      else
        put(ig, jg, hg, qu, hg * (qv / hmax + e.sgn * c * (ei - eta_ext) / hmax));
    }
  } else if (type == kInflow) {
    // bc_inflow_edge :347-390
    const double in_sgn = -e.sgn;
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      if (e.normal_u)
        put(ig, jg, hi, in_sgn * hi * bc->inflow_velocity, qv);
      else
        put(ig, jg, hi, qu, in_sgn * hi * bc->inflow_velocity);
    }
  } else if (type == kDischarge) {
    // bc_disch_edge :392-434
    const double in_sgn = -e.sgn;
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      if (e.normal_u)
        put(ig, jg, hi, in_sgn * bc->discharge_flux, qv);
      else
        put(ig, jg, hi, qu, in_sgn * bc->discharge_flux);
    }
  } else if (type == kClamped) {
    // bc_clamped_edge :436-469
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      put(ig, jg, pos(bc->clamped_elevation - b[g.at(ig, jg)]), qu, qv);
    }
  } else if (type == kChapman) {
    // bc_chapman_edge :471-552; every layer reads the surface stored before
    // this call, then position t's surface is refreshed once.
    const double dd = e.normal_u ? g.dx : g.dy;
    // The reference fills the ghosts once more before computing dt
    // (rki_solver.F90:719); for Chapman that extra call refreshes the stored
    // surface to the current interior one, which the first stage then sees.
    const double ei0 = hi + b[qi];
    const double eov = chapman_fresh ? ei0 : eo[t];
    const double ei = hi + b[qi];
    const double hmax = dmax(hi, 1.0e-6);
    const double c = sqrt(kG * hmax);
    const int i2 = ii - e.din;
    const int j2 = ji - e.djn;
    double eg;
    if (dtb > 0.0) {
      const double detadt = (ei - eov) / dtb;
      double detadx = 0.0;
      if (i2 >= 0 && i2 < g.nxt && j2 >= 0 && j2 < g.nyt) {
        const size_t q2 = g.at(i2, j2);
        detadx = (h[q2] + b[q2] - ei) / dd;
      }
      double cp = fabs(detadx) > 1.0e-10 ? -detadt / detadx : 0.0;
      cp = pos(dmin(cp, c));
      eg = eov - cp * dtb / dd * (eov - ei);
    } else {
      eg = ei;
    }
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const double hg = pos(eg - b[g.at(ig, jg)]);
      if (e.normal_u)
        put(ig, jg, hg, hg * (qu / hmax + e.sgn * c * (ei - eg) / hmax), qv);
      else
        put(ig, jg, hg, qu, hg * (qv / hmax + e.sgn * c * (ei - eg) / hmax));
    }
    eo[t] = ei;
  }
}

}  // namespace rkb
