// Kernel-level C entry points on caller-owned device arrays
// (declared in include/rakali.h, Part 2).
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/rakali.h"
#include "rkb_kernels.h"

namespace rkb {
namespace {

// Max over wet interior cells of (|u|+c) along x and y, into two bit-pattern
// accumulators (rki_kernel_timestep.F90:52-66).
__global__ void k_timestep_reduce(Grid g, const double* __restrict__ h,
                                  const double* __restrict__ hu, const double* __restrict__ hv,
                                  unsigned long long* acc) {
  const int nxp = g.nx_phys(), nyp = g.ny_phys();
  const long long n = (long long)nxp * nyp;
  double mx = 0.0, my = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = g.ng + (int)(k % nxp);
    const int j = g.ng + (int)(k / nxp);
    const size_t q = g.at(i, j);
    double sx, sy;
    wave_speed(h[q], hu[q], hv[q], sx, sy);
    if (sx > mx) mx = sx;
    if (sy > my) my = sy;
  }
  for (int o = 16; o > 0; o >>= 1) {
    double a = __shfl_xor_sync(0xffffffffu, mx, o);
    double b = __shfl_xor_sync(0xffffffffu, my, o);
    mx = a > mx ? a : mx;
    my = b > my ? b : my;
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&acc[0], mx);
    atomic_max_pos(&acc[1], my);
  }
}

Grid make_grid(int nxt, int nyt, int ng, int ld, double dx, double dy) {
  Grid g;
  g.nxt = nxt;
  g.nyt = nyt;
  g.ng = ng;
  g.pitch = ld;
  g.dx = dx;
  g.dy = dy;
  return g;
}

bool grid_ok(int nxt, int nyt, int ng, int ld) {
  return ng >= 2 && nxt > 2 * ng && nyt > 2 * ng && ld >= nxt;
}

}  // namespace

// Shared by rkb_compute_timestep and its caller-provided-scratch variants.
cudaError_t timestep_reduce(const Grid& g, const double* h, const double* hu, const double* hv,
                            unsigned long long* acc, cudaStream_t s) {
  const long long n = (long long)g.nx_phys() * g.ny_phys();
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  k_timestep_reduce<<<(unsigned)blocks, 256, 0, s>>>(g, h, hu, hv, acc);
  return cudaGetLastError();
}

}  // namespace rkb

extern "C" {

int rkb_compute_flux(int use_hllc, const double* h, const double* hu, const double* hv,
                     const double* b, double* flux_h, double* flux_hu, double* flux_hv,
                     double* mass_flux_x, double* mass_flux_y, int nx_total, int ny_total,
                     int nghost, int ld, double dx, double dy) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv || !b || !flux_h || !flux_hu || !flux_hv) return -2;
  rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, dx, dy);
  rkb::FieldSet in{const_cast<double*>(h), const_cast<double*>(hu), const_cast<double*>(hv)};
  rkb::FluxOut out{flux_h, flux_hu, flux_hv, mass_flux_x, mass_flux_y};
  cudaError_t e = rkb::launch_flux(g, use_hllc, in, b, out, rkb::kTile32x8, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  return e == cudaSuccess ? 0 : -1;
}

int rkb_compute_timestep(const double* h, const double* hu, const double* hv, int nx_total,
                         int ny_total, int nghost, int ld, double dx, double dy, double cfl,
                         double* dt_out) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv || !dt_out) return -2;
  rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, dx, dy);
  unsigned long long* acc = nullptr;
  if (cudaMalloc((void**)&acc, 2 * sizeof(unsigned long long)) != cudaSuccess) return -1;
  unsigned long long host[2] = {0ull, 0ull};
  cudaError_t e = cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), 0);
  if (e == cudaSuccess) e = rkb::timestep_reduce(g, h, hu, hv, acc, 0);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host, acc, sizeof(host), cudaMemcpyDeviceToHost, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  cudaFree(acc);
  if (e != cudaSuccess) return -1;
  double msx, msy;
  std::memcpy(&msx, &host[0], sizeof(double));
  std::memcpy(&msy, &host[1], sizeof(double));
  *dt_out = rkb::cfl_dt(msx, msy, g, cfl);
  return 0;
}

}  // extern "C"

// Host builds of the correctly rounded transcendental terms the kernels use
// (rkb_crmath.cuh), exposed so the same code can be checked without a GPU.
#include "rkb_crmath.cuh"

extern "C" {

double rkb_cr_pow_third(double h) { return rkb::cr_pow_third(h); }

void rkb_cr_sincos(double x, double* sn, double* cs) { rkb::cr_sincos(x, *sn, *cs); }

}  // extern "C"
