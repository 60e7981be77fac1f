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

// ---------------------------------------------------------------------------
// Allocation-free CFL timestep.
//
// Some callers of this library cannot allocate device memory at the point
// where they need dt: a host application that has reserved the GPU's memory
// for its own pool (the reference's OpenACC runtime maps all model arrays up
// front), or a driver loop that must not block - cudaMalloc and cudaFree
// synchronise the whole device.  rkb_compute_timestep_noalloc therefore does
// its two-pass reduction in a fixed scratch array compiled into the library:
// one slot pair per interior row, plus the result.
//
// Limits: ny_total - 2*nghost <= kNoAllocMaxRows rows.  The array is device
// memory of every GPU that loads the library, held until the process exits.
// Every call shares it and it keeps the last call's contents; the row pass
// writes every slot it later reads, so nothing needs clearing.  Calls that
// overlap on the GPU (other host threads, other streams) race on it.
// ---------------------------------------------------------------------------

#include <string>

namespace rkb {
void set_last_error(const std::string& msg);  // rkb_api.cu
namespace {

constexpr int kNoAllocMaxRows = 32768;
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxRows + 2];

// One warp per interior row: the row's maxima of (|u|+c) along x and y.
__global__ void k_row_speed(Grid g, const double* __restrict__ h, const double* __restrict__ hu,
                            const double* __restrict__ hv, double* scratch) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int nyp = g.ny_phys();
  if (row >= nyp) return;
  const int j = g.ng + row;
  double mx = 0.0, my = 0.0;
  for (int i = g.ng + lane; i < g.nxt - g.ng; i += 32) {
    const size_t q = g.at(i, j);
    double sx, sy;
    wave_speed(h[q], hu[q], hv[q], sx, sy);
    if (sx > mx) mx = sx;
    if (sy > my) my = sy;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, mx, o);
    const double b = __shfl_xor_sync(0xffffffffu, my, o);
    mx = a > mx ? a : mx;
    my = b > my ? b : my;
  }
  if (lane == 0) {
    scratch[row] = mx;
    scratch[kNoAllocMaxRows + row] = my;
  }
}

// One block folds the row maxima and stores dt in the last slot.
__global__ void k_rows_to_dt(Grid g, double cfl, double* scratch) {
  const int nyp = g.ny_phys();
  double mx = 0.0, my = 0.0;
  for (int r = threadIdx.x; r < nyp; r += blockDim.x) {
    const double a = scratch[r], b = scratch[kNoAllocMaxRows + r];
    if (a > mx) mx = a;
    if (b > my) my = b;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double a = __shfl_xor_sync(0xffffffffu, mx, o);
    const double b = __shfl_xor_sync(0xffffffffu, my, o);
    mx = a > mx ? a : mx;
    my = b > my ? b : my;
  }
  __shared__ double wx[32], wy[32];
  if ((threadIdx.x & 31) == 0) {
    wx[threadIdx.x >> 5] = mx;
    wy[threadIdx.x >> 5] = my;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      if (wx[w] > mx) mx = wx[w];
      if (wy[w] > my) my = wy[w];
    }
    scratch[2 * kNoAllocMaxRows] = cfl_dt(mx, my, g, cfl);
  }
}

// Device address of the scratch array in the current device's context (the
// symbol's host-side name is not a device address).  Looked up on every
// call rather than cached: after cudaDeviceReset the runtime loads the module
// again, possibly elsewhere, and a cached address would go stale.  The
// lookup is a host-side table read once the module is loaded.
double* scratch_address() {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
  return static_cast<double*>(p);
}

}  // namespace
}  // namespace rkb

extern "C" {

int rkb_compute_timestep_noalloc(const double* h, const double* hu, const double* hv,
                                 int nx_total, int ny_total, int nghost, int ld, double dx,
                                 double dy, double cfl, double* dt_out) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv || !dt_out) return -2;
  if (ny_total - 2 * nghost > rkb::kNoAllocMaxRows) {
    rkb::set_last_error("rkb_compute_timestep_noalloc: " + std::to_string(ny_total - 2 * nghost) +
                        " interior rows exceed the fixed scratch of " +
                        std::to_string(rkb::kNoAllocMaxRows) + " rows");
    return -2;
  }
  double* scratch = rkb::scratch_address();
  if (!scratch) {
    rkb::set_last_error("rkb_compute_timestep_noalloc: no device address for the scratch array");
    return -1;
  }
  rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, dx, dy);
  const int rows = g.ny_phys();
  const int warps_per_block = 8;
  rkb::k_row_speed<<<(rows + warps_per_block - 1) / warps_per_block, 32 * warps_per_block>>>(
      g, h, hu, hv, scratch);
  rkb::k_rows_to_dt<<<1, 1024>>>(g, cfl, scratch);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpy(dt_out, scratch + 2 * rkb::kNoAllocMaxRows, sizeof(double),
                   cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
