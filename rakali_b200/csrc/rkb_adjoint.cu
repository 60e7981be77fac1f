// FP64 instance of the gauge-misfit adjoint (rkb_adjoint_impl.cuh), compiled
// with --fmad=false so its forward is bit-identical to the production step,
// and the C ABI of both precisions (the FP32 instance is rkb_adjoint32.cu).
#include "rkb_adjoint_impl.cuh"

namespace rkb {

AdjointBase* make_adjoint64(int nm, int nx, int ny, int ng, double dx, double dy, double cfl,
                            int hllc, int nsteps, const double* h0, const double* hu0,
                            const double* hv0, const int* gi, const int* gj, int ngauge,
                            std::string& err, int& rc) {
  return adj::make_adjoint<double>(nm, nx, ny, ng, dx, dy, cfl, hllc, nsteps, h0, hu0, hv0, gi, gj,
                                   ngauge, err, rc);
}

void set_last_error(const std::string& msg);

}  // namespace rkb

// ---------------------------------------------------------------------------
// C ABI (declared in include/rakali.h)
// ---------------------------------------------------------------------------

namespace {
rkb::AdjointBase* as_adj(void* a) { return static_cast<rkb::AdjointBase*>(a); }
}  // namespace

extern "C" {

int rkb_adjoint_batch_create(int precision, int n_members, int nx, int ny, int nghost, double dx,
                             double dy, double cfl, int use_hllc, int n_steps, const double* h0,
                             const double* hu0, const double* hv0, const int* gauge_i,
                             const int* gauge_j, int n_gauges, void** adj) {
  if (!adj) return -2;
  *adj = nullptr;
  if (precision != 32 && precision != 64) {
    rkb::set_last_error("precision must be 32 or 64");
    return -2;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    rkb::set_last_error("no CUDA device available");
    return -1;
  }
  std::string err;
  int rc = 0;
  rkb::AdjointBase* a =
      precision == 64
          ? rkb::make_adjoint64(n_members, nx, ny, nghost, dx, dy, cfl, use_hllc, n_steps, h0, hu0,
                                hv0, gauge_i, gauge_j, n_gauges, err, rc)
          : rkb::make_adjoint32(n_members, nx, ny, nghost, dx, dy, cfl, use_hllc, n_steps, h0, hu0,
                                hv0, gauge_i, gauge_j, n_gauges, err, rc);
  if (!a) {
    rkb::set_last_error(err.empty() ? "adjoint setup failed" : err);
    return rc != 0 ? rc : -1;
  }
  *adj = a;
  return 0;
}

int rkb_adjoint_create(int nx, int ny, int nghost, double dx, double dy, double cfl, int use_hllc,
                       int n_steps, const double* h0, const double* hu0, const double* hv0,
                       const int* gauge_i, const int* gauge_j, int n_gauges, void** adj) {
  return rkb_adjoint_batch_create(64, 1, nx, ny, nghost, dx, dy, cfl, use_hllc, n_steps, h0, hu0,
                                  hv0, gauge_i, gauge_j, n_gauges, adj);
}

void rkb_adjoint_destroy(void** adj) {
  if (!adj || !*adj) return;
  delete as_adj(*adj);
  *adj = nullptr;
}

int rkb_adjoint_set_obs(void* adj, const double* obs) {
  if (!adj || !obs) return -2;
  return as_adj(adj)->set_obs(obs);
}

int rkb_adjoint_set_dt(void* adj, const double* dts) {
  if (!adj || !dts) return -2;
  return as_adj(adj)->set_dt(dts);
}

int rkb_adjoint_get_dt(void* adj, double* dts) {
  if (!adj || !dts) return -2;
  as_adj(adj)->get_dt(dts);
  return 0;
}

int rkb_adjoint_forward(void* adj, const double* b, const double* n_field, double n_scalar,
                        int record_dt, double* J, double* eta_gauges) {
  if (!adj || !b || !J) return -2;
  return as_adj(adj)->forward(b, n_field, n_scalar, record_dt != 0, J, eta_gauges);
}

int rkb_adjoint_gradient(void* adj, const double* b, const double* n_field, double n_scalar,
                         double* J, double* grad_b, double* grad_n) {
  if (!adj || !b || !J || !grad_b || !grad_n) return -2;
  return as_adj(adj)->gradient(b, n_field, n_scalar, J, grad_b, grad_n);
}

int rkb_adjoint_checkpoint_interval(void* adj) {
  return adj ? as_adj(adj)->checkpoint_interval() : -2;
}

int rkb_adjoint_set_state_budget(void* adj, long long bytes) {
  if (!adj) return -2;
  as_adj(adj)->set_state_budget(bytes);
  return 0;
}

double rkb_adjoint_last_ms(void* adj) { return adj ? as_adj(adj)->last_ms() : -1.0; }

int rkb_adjoint_members(void* adj) { return adj ? as_adj(adj)->members() : -2; }

int rkb_adjoint_precision(void* adj) { return adj ? as_adj(adj)->precision() : -2; }

int rkb_adjoint_set_frozen_slopes(void* adj, int on) {
  if (!adj) return -2;
  as_adj(adj)->set_frozen_slopes(on != 0);
  return 0;
}

int rkb_adjoint_mass(void* adj, double* out) {
  if (!adj || !out) return -2;
  as_adj(adj)->mass(out);
  return 0;
}

// Host builds of the face and cell derivatives, for finite-difference checks.
void rkb_test_face_flux(int dir, int hllc, const double* in8, double* out6) {
  rkb::FaceOut o;
  if (dir == 0) {
    if (hllc) rkb::face_flux<0, true>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], o);
    else rkb::face_flux<0, false>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], o);
  } else {
    if (hllc) rkb::face_flux<1, true>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], o);
    else rkb::face_flux<1, false>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], o);
  }
  out6[0] = o.fh; out6[1] = o.fqx; out6[2] = o.fqy;
  out6[3] = o.wbR; out6[4] = o.hL2; out6[5] = o.pL2;
}

void rkb_test_face_adj(int dir, int hllc, const double* in8, const double* gout6, double* gin8) {
  for (int k = 0; k < 8; ++k) gin8[k] = 0.0;
  if (dir == 0) {
    if (hllc) rkb::face_adj<0, true>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], gout6, gin8);
    else rkb::face_adj<0, false>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], gout6, gin8);
  } else {
    if (hllc) rkb::face_adj<1, true>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], gout6, gin8);
    else rkb::face_adj<1, false>(in8[0], in8[1], in8[2], in8[3], in8[4], in8[5], in8[6], in8[7], gout6, gin8);
  }
}

// out3 = protect then friction of (h, u, v) with n and dt; the adjoint maps
// gout3 to gin4 = (h, u, v, n).
void rkb_test_cell(const double* in4, double dt, double* out3) {
  double h = in4[0], u = in4[1], v = in4[2];
  rkb::protect(h, u, v);
  rkb::friction(h, u, v, in4[3], dt);
  out3[0] = h; out3[1] = u; out3[2] = v;
}

void rkb_test_cell_adj(const double* in4, double dt, const double* gout3, double* gin4) {
  double h = in4[0], u = in4[1], v = in4[2];
  double h1 = h, u1 = u, v1 = v;
  rkb::protect(h1, u1, v1);
  double gh = gout3[0], gu = gout3[1], gv = gout3[2], gn = 0.0;
  rkb::friction_adj(h1, u1, v1, in4[3], dt, gh, gu, gv, gn);
  rkb::protect_adj(h, u, v, gh, gu, gv);
  gin4[0] = gh; gin4[1] = gu; gin4[2] = gv; gin4[3] = gn;
}

}  // extern "C"
