// FP32 instance of the gauge-misfit adjoint (rkb_adjoint_impl.cuh): the same
// forward and reverse kernels in FP32 arithmetic (fused multiply-adds, fast
// division and square root); misfit sums and domain mass in FP64.
#include "rkb_adjoint_impl.cuh"

namespace rkb {

AdjointBase* make_adjoint32(int nm, int nx, int ny, int ng, double dx, double dy, double cfl,
                            int hllc, int nsteps, const double* h0, const double* hu0,
                            const double* hv0, const int* gi, const int* gj, int ngauge,
                            std::string& err, int& rc) {
  return adj::make_adjoint<float>(nm, nx, ny, ng, dx, dy, cfl, hllc, nsteps, h0, hu0, hv0, gi, gj,
                                  ngauge, err, rc);
}

}  // namespace rkb
