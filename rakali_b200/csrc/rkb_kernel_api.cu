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

// ---------------------------------------------------------------------------
// The remaining structured kernels of src/core/coastal as kernel-level entry
// points: the stage updates, the update / average / SSP combine, friction,
// Coriolis, the boundary fills and the sponge.  Each runs one grid-stride
// kernel over the interior (or over the edges) with the device functions the
// fused step uses, so the results are those of the fused step's pieces.
// ---------------------------------------------------------------------------

#include "rkb_bc.cuh"
#include "rkb_cell.cuh"

namespace rkb {
namespace {

// Interior cell k of a grid-stride loop.
__device__ __forceinline__ bool interior_cell(const Grid& g, long long k, int& i, int& j) {
  const int nxp = g.nx_phys();
  const long long n = (long long)nxp * g.ny_phys();
  if (k >= n) return false;
  i = g.ng + (int)(k % nxp);
  j = g.ng + (int)(k / nxp);
  return true;
}

__device__ __forceinline__ long long stride() { return (long long)gridDim.x * blockDim.x; }
__device__ __forceinline__ long long first() {
  return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}

// MODE 1: fused_update_stage1, 2: fused_update_stage2, 3: the generic stage.
template <int MODE>
__global__ void k_fused_update(Grid g, FieldSet U, FieldSet U0, const double* __restrict__ fh,
                               const double* __restrict__ fhu, const double* __restrict__ fhv,
                               double dt, Physics ph, Forcing fo) {
  // cos / sin of the Coriolis rotation, correctly rounded once per block
  // (rki_kernel_fused.F90:211-214)
  __shared__ double rot[2];
  const bool has_cor = fabs(ph.coriolis_f) > 1.0e-20;
  if (threadIdx.x == 0) {
    double sn = 0.0, cs = 0.0;
    if (has_cor) cr_sincos(ph.coriolis_f * dt, sn, cs);
    rot[0] = cs;
    rot[1] = sn;
  }
  __syncthreads();
  const double n_sq = ph.manning_n * ph.manning_n;
  for (long long k = first();; k += stride()) {
    int i, j;
    if (!interior_cell(g, k, i, j)) break;
    const size_t q = g.at(i, j);
    double a = U.h[q], u = U.hu[q], v = U.hv[q];
    if (MODE == 1) {
      U0.h[q] = a;
      U0.hu[q] = u;
      U0.hv[q] = v;
    }
    a = a + dt * fh[q];
    u = u + dt * fhu[q];
    v = v + dt * fhv[q];
    protect(a, u, v);
    sources(a, u, v, &ph, dt, n_sq, rot[0], rot[1], has_cor, g, i, j, fo);
    if (MODE == 2) {
      a = 0.5 * (U0.h[q] + a);
      u = 0.5 * (U0.hu[q] + u);
      v = 0.5 * (U0.hv[q] + v);
      protect(a, u, v);
    }
    U.h[q] = a;
    U.hu[q] = u;
    U.hv[q] = v;
  }
}

// MODE 0: compute_update (U + dt F), 1: compute_ssp_combine (a_n U0 +
// (1 - a_n) U; compute_rk2_average is a_n = 1/2 written as 0.5 (U0 + U)),
// 2: compute_rk2_average; each followed by the clamp.
template <int MODE>
__global__ void k_update(Grid g, FieldSet U, FieldSet U0, const double* __restrict__ fh,
                         const double* __restrict__ fhu, const double* __restrict__ fhv,
                         double c) {
  for (long long k = first();; k += stride()) {
    int i, j;
    if (!interior_cell(g, k, i, j)) break;
    const size_t q = g.at(i, j);
    double a, u, v;
    if (MODE == 0) {
      a = U.h[q] + c * fh[q];
      u = U.hu[q] + c * fhu[q];
      v = U.hv[q] + c * fhv[q];
    } else if (MODE == 1) {
      const double a_prev = 1.0 - c;
      a = c * U0.h[q] + a_prev * U.h[q];
      u = c * U0.hu[q] + a_prev * U.hu[q];
      v = c * U0.hv[q] + a_prev * U.hv[q];
    } else {
      a = 0.5 * (U0.h[q] + U.h[q]);
      u = 0.5 * (U0.hu[q] + U.hu[q]);
      v = 0.5 * (U0.hv[q] + U.hv[q]);
    }
    protect(a, u, v);
    U.h[q] = a;
    U.hu[q] = u;
    U.hv[q] = v;
  }
}

// apply_friction (rki_kernel_friction.F90:16-113), both of its paths.
__global__ void k_friction(Grid g, FieldSet U, double dt, double manning_n, Forcing fo,
                           int forcing, int include_wind) {
  const bool has_friction = manning_n > 0.0;
  for (long long k = first();; k += stride()) {
    int i, j;
    if (!interior_cell(g, k, i, j)) break;
    const size_t q = g.at(i, j);
    const double hval = U.h[q];
    if (hval > kDry) {
      const double uu = U.hu[q] / hval;
      const double vv = U.hv[q] / hval;
      const double speed = sqrt(uu * uu + vv * vv);
      if (has_friction) {
        const double cf = kG * manning_n * manning_n / cr_pow_third(hval);
        const double den = 1.0 + dt * cf * speed / hval;
        U.hu[q] = U.hu[q] / den;
        U.hv[q] = U.hv[q] / den;
      }
      if (forcing) {
        if (include_wind) {
          U.hu[q] = U.hu[q] + dt * fo.wind_x[q] / kRho;
          U.hv[q] = U.hv[q] + dt * fo.wind_y[q] / kRho;
        }
        const double dpdx = (fo.atm[g.at(i + 1, j)] - fo.atm[g.at(i - 1, j)]) / (2.0 * g.dx);
        const double dpdy = (fo.atm[g.at(i, j + 1)] - fo.atm[g.at(i, j - 1)]) / (2.0 * g.dy);
        U.hu[q] = U.hu[q] - dt * hval * dpdx / kRho;
        U.hv[q] = U.hv[q] - dt * hval * dpdy / kRho;
      }
    }
    if (forcing) U.h[q] = U.h[q] + dt * fo.precip[q];
  }
}

// apply_coriolis (rki_kernel_friction.F90:115-152).
__global__ void k_coriolis(Grid g, const double* __restrict__ h, double* hu, double* hv,
                           double dt, double f) {
  __shared__ double rot[2];
  if (threadIdx.x == 0) cr_sincos(f * dt, rot[1], rot[0]);
  __syncthreads();
  const double cs = rot[0], sn = rot[1];
  for (long long k = first();; k += stride()) {
    int i, j;
    if (!interior_cell(g, k, i, j)) break;
    const size_t q = g.at(i, j);
    if (h[q] > kDry) {
      const double uo = hu[q], vo = hv[q];
      hu[q] = uo * cs + vo * sn;
      hv[q] = -(uo * sn) + vo * cs;
    }
  }
}

// apply_sponge (rki_kernel_sponge.F90:16-88).
__global__ void k_sponge(Grid g, FieldSet U, double dt, BcParams bc) {
  for (long long k = first();; k += stride()) {
    int i, j;
    if (!interior_cell(g, k, i, j)) break;
    const size_t q = g.at(i, j);
    double a = U.h[q], u = U.hu[q], v = U.hv[q];
    const double alpha = sponge_alpha(&bc, g, i, j);
    if (alpha > 0.0) {
      sponge(a, u, v, &bc, g, i, j, dt);
      U.h[q] = a;
      U.hu[q] = u;
      U.hv[q] = v;
    }
  }
}

// Edges [e0, e0 + gridDim.y), one thread per tangential position; the
// reference's single-call semantics (the stored Chapman surfaces are read).
__global__ void k_bc_api(Grid g, FieldSet U, double* b, BcParams bc, double time, double dt,
                         double* eo0, double* eo1, double* eo2, double* eo3, int e0) {
  const int w = e0 + (int)blockIdx.y;
  double* eo = w == 0 ? eo0 : w == 1 ? eo1 : w == 2 ? eo2 : eo3;
  fill_edge(g, &bc, b, U, nullptr, nullptr, nullptr, w, (int)(blockIdx.x * blockDim.x + threadIdx.x),
            time, dt, eo, false);
}

unsigned cell_blocks(const Grid& g) {
  const long long n = (long long)g.nx_phys() * g.ny_phys();
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  return (unsigned)(blocks < 1 ? 1 : blocks);
}

int finish(cudaError_t e) {
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    set_last_error(std::string("kernel entry point: ") + cudaGetErrorString(e));
    return -1;
  }
  return 0;
}

bool forcing_ok(int forcing_active, const double* wx, const double* wy, const double* atm,
                const double* pr) {
  return !forcing_active || (wx && wy && atm && pr);
}

bool bc_ok(const rkb_bc_params* p, BcParams& out) {
  if (!p) return false;
  out = BcParams{};
  for (int w = 0; w < 4; ++w) {
    if (p->type[w] < kWall || p->type[w] > kChapman) return false;
    if (p->type[w] == kChapman && !p->eta_old[w]) return false;
    out.type[w] = p->type[w];
  }
  if (p->n_tidal < 0 || p->n_tidal > kMaxTidal) return false;
  out.n_tidal = p->n_tidal;
  out.sponge_width = p->sponge_width;
  out.tidal_amplitude = p->tidal_amplitude;
  out.tidal_period = p->tidal_period;
  for (int n = 0; n < kMaxTidal; ++n) {
    out.amp[n] = p->tidal_amp[n];
    out.phase[n] = p->tidal_phase[n];
    out.omega[n] = p->tidal_omega[n];
  }
  out.inflow_velocity = p->inflow_velocity;
  out.discharge_flux = p->discharge_flux;
  out.clamped_elevation = p->clamped_elevation;
  out.sponge_strength = p->sponge_strength;
  out.sponge_h_ref = p->sponge_h_ref;
  return true;
}

FieldSet fs(double* h, double* hu, double* hv) { return FieldSet{h, hu, hv}; }
FieldSet cfs(const double* h, const double* hu, const double* hv) {
  return FieldSet{const_cast<double*>(h), const_cast<double*>(hu), const_cast<double*>(hv)};
}

template <int MODE>
int fused_update(double* h, double* hu, double* hv, double* h0, double* hu0, double* hv0,
                 const double* fh, const double* fhu, const double* fhv, int nxt, int nyt, int ng,
                 int ld, double dx, double dy, double dt, double manning_n, const double* wx,
                 const double* wy, const double* atm, const double* pr, double coriolis_f,
                 int forcing_active) {
  if (!grid_ok(nxt, nyt, ng, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv || !fh || !fhu || !fhv) return -2;
  if (MODE != 3 && (!h0 || !hu0 || !hv0)) return -2;
  if (!forcing_ok(forcing_active, wx, wy, atm, pr)) return -2;
  const Grid g = make_grid(nxt, nyt, ng, ld, dx, dy);
  Physics ph{};
  ph.manning_n = manning_n;
  ph.coriolis_f = coriolis_f;
  ph.forcing_active = forcing_active ? 1 : 0;
  const Forcing fo{wx, wy, atm, pr};
  k_fused_update<MODE><<<cell_blocks(g), 256>>>(g, fs(h, hu, hv), fs(h0, hu0, hv0), fh, fhu, fhv,
                                                 dt, ph, fo);
  return finish(cudaSuccess);
}

}  // namespace
}  // namespace rkb

extern "C" {

int rkb_fused_update_stage1(double* h, double* hu, double* hv, double* h0, double* hu0,
                            double* hv0, const double* flux_h, const double* flux_hu,
                            const double* flux_hv, int nx_total, int ny_total, int nghost, int ld,
                            double dx, double dy, double dt, double manning_n,
                            const double* wind_x, const double* wind_y, const double* atm,
                            const double* precip, double coriolis_f, int forcing_active) {
  return rkb::fused_update<1>(h, hu, hv, h0, hu0, hv0, flux_h, flux_hu, flux_hv, nx_total,
                              ny_total, nghost, ld, dx, dy, dt, manning_n, wind_x, wind_y, atm,
                              precip, coriolis_f, forcing_active);
}

int rkb_fused_update_stage2(double* h, double* hu, double* hv, const double* h0,
                            const double* hu0, const double* hv0, const double* flux_h,
                            const double* flux_hu, const double* flux_hv, int nx_total,
                            int ny_total, int nghost, int ld, double dx, double dy, double dt,
                            double manning_n, const double* wind_x, const double* wind_y,
                            const double* atm, const double* precip, double coriolis_f,
                            int forcing_active) {
  return rkb::fused_update<2>(h, hu, hv, const_cast<double*>(h0), const_cast<double*>(hu0),
                              const_cast<double*>(hv0), flux_h, flux_hu, flux_hv, nx_total,
                              ny_total, nghost, ld, dx, dy, dt, manning_n, wind_x, wind_y, atm,
                              precip, coriolis_f, forcing_active);
}

int rkb_fused_update_stage_generic(double* h, double* hu, double* hv, const double* flux_h,
                                   const double* flux_hu, const double* flux_hv, int nx_total,
                                   int ny_total, int nghost, int ld, double dx, double dy,
                                   double dt, double manning_n, const double* wind_x,
                                   const double* wind_y, const double* atm,
                                   const double* precip, double coriolis_f, int forcing_active) {
  return rkb::fused_update<3>(h, hu, hv, nullptr, nullptr, nullptr, flux_h, flux_hu, flux_hv,
                              nx_total, ny_total, nghost, ld, dx, dy, dt, manning_n, wind_x,
                              wind_y, atm, precip, coriolis_f, forcing_active);
}

int rkb_compute_update(double* h, double* hu, double* hv, const double* flux_h,
                       const double* flux_hu, const double* flux_hv, int nx_total, int ny_total,
                       int nghost, int ld, double dt) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld)) return -2;
  if (!h || !hu || !hv || !flux_h || !flux_hu || !flux_hv) return -2;
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, 1.0, 1.0);
  rkb::k_update<0><<<rkb::cell_blocks(g), 256>>>(g, rkb::fs(h, hu, hv), rkb::FieldSet{}, flux_h,
                                                  flux_hu, flux_hv, dt);
  return rkb::finish(cudaSuccess);
}

int rkb_compute_rk2_average(double* h, double* hu, double* hv, const double* h0,
                            const double* hu0, const double* hv0, int nx_total, int ny_total,
                            int nghost, int ld) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld)) return -2;
  if (!h || !hu || !hv || !h0 || !hu0 || !hv0) return -2;
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, 1.0, 1.0);
  rkb::k_update<2><<<rkb::cell_blocks(g), 256>>>(g, rkb::fs(h, hu, hv), rkb::cfs(h0, hu0, hv0),
                                                  nullptr, nullptr, nullptr, 0.0);
  return rkb::finish(cudaSuccess);
}

int rkb_compute_ssp_combine(double* h, double* hu, double* hv, const double* h0,
                            const double* hu0, const double* hv0, double a_n, int nx_total,
                            int ny_total, int nghost, int ld) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld)) return -2;
  if (!h || !hu || !hv || !h0 || !hu0 || !hv0) return -2;
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, 1.0, 1.0);
  rkb::k_update<1><<<rkb::cell_blocks(g), 256>>>(g, rkb::fs(h, hu, hv), rkb::cfs(h0, hu0, hv0),
                                                  nullptr, nullptr, nullptr, a_n);
  return rkb::finish(cudaSuccess);
}

int rkb_apply_friction(double* h, double* hu, double* hv, int nx_total, int ny_total, int nghost,
                       int ld, double dx, double dy, double dt, double manning_n,
                       const double* wind_x, const double* wind_y, const double* atm,
                       const double* precip, int forcing_active, int include_wind) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv) return -2;
  if (!rkb::forcing_ok(forcing_active, include_wind ? wind_x : atm, include_wind ? wind_y : atm,
                       atm, precip))
    return -2;
  if (!(manning_n > 0.0) && !forcing_active) return 0;  // the reference's early exit
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, dx, dy);
  const rkb::Forcing fo{wind_x, wind_y, atm, precip};
  rkb::k_friction<<<rkb::cell_blocks(g), 256>>>(g, rkb::fs(h, hu, hv), dt, manning_n, fo,
                                                forcing_active ? 1 : 0, include_wind ? 1 : 0);
  return rkb::finish(cudaSuccess);
}

int rkb_apply_coriolis(const double* h, double* hu, double* hv, int nx_total, int ny_total,
                       int nghost, int ld, double dt, double f) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld)) return -2;
  if (!h || !hu || !hv) return -2;
  if (fabs(f) < 1.0e-20) return 0;  // rki_kernel_friction.F90:131
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, 1.0, 1.0);
  rkb::k_coriolis<<<rkb::cell_blocks(g), 256>>>(g, h, hu, hv, dt, f);
  return rkb::finish(cudaSuccess);
}

int rkb_apply_boundary_conditions(double* h, double* hu, double* hv, double* b, int nx_total,
                                  int ny_total, int nghost, int ld, double dx, double dy,
                                  const rkb_bc_params* bc) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld) || !(dx > 0.0) || !(dy > 0.0)) return -2;
  if (!h || !hu || !hv || !b) return -2;
  rkb::BcParams p;
  if (!rkb::bc_ok(bc, p)) return -2;
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, dx, dy);
  const rkb::FieldSet U = rkb::fs(h, hu, hv);
  const int tpb = 128;
  // Opposite edges run in one launch only when neither reads cells the
  // other writes (an interior at least max(nghost, 2) wide); otherwise one
  // launch per edge, W, E, S, N as the reference orders them.
  const int wide = nghost > 2 ? nghost : 2;
  auto go = [&](int e0, int count, int n_tan) {
    const dim3 grid((unsigned)((n_tan + tpb - 1) / tpb), (unsigned)count);
    rkb::k_bc_api<<<grid, tpb>>>(g, U, b, p, bc->time, bc->dt, bc->eta_old[0], bc->eta_old[1],
                                 bc->eta_old[2], bc->eta_old[3], e0);
  };
  if (g.nx_phys() >= wide) {
    go(0, 2, g.nyt);
  } else {
    go(0, 1, g.nyt);
    go(1, 1, g.nyt);
  }
  if (g.ny_phys() >= wide) {
    go(2, 2, g.nxt);
  } else {
    go(2, 1, g.nxt);
    go(3, 1, g.nxt);
  }
  return rkb::finish(cudaSuccess);
}

int rkb_apply_sponge(double* h, double* hu, double* hv, int nx_total, int ny_total, int nghost,
                     int ld, double dt, const rkb_bc_params* bc) {
  if (!rkb::grid_ok(nx_total, ny_total, nghost, ld)) return -2;
  if (!h || !hu || !hv) return -2;
  rkb::BcParams p;
  if (!rkb::bc_ok(bc, p)) return -2;
  if (p.sponge_width <= 0 || !(p.sponge_strength > 0.0)) return 0;  // :41-46
  const rkb::Grid g = rkb::make_grid(nx_total, ny_total, nghost, ld, 1.0, 1.0);
  rkb::k_sponge<<<rkb::cell_blocks(g), 256>>>(g, rkb::fs(h, hu, hv), dt, p);
  return rkb::finish(cudaSuccess);
}

}  // extern "C"
