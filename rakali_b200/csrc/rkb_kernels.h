// Host-side launch interface of the B200 kernels (no torch types).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "rkb_common.cuh"

namespace rkb {

struct FieldSet {
  double* h;
  double* hu;
  double* hv;
};

struct Forcing {
  const double* wind_x;
  const double* wind_y;
  const double* atm;
  const double* precip;
};

struct FluxOut {
  double* flux_h;
  double* flux_hu;
  double* flux_hv;
  double* mflux_x;
  double* mflux_y;
};

// Tile shapes of the fused stage kernel (cells per block in x and y).
enum TileShape : int {
  kTile32x8 = 0, kTile32x16 = 1, kTile64x4 = 2, kTile16x16 = 3,  // shared-memory tiles
  kMarch64 = 4, kMarch32 = 5,  // warp-per-strip marching kernel, 64 / 32 rows per warp
  kNumTiles = 6
};
const char* tile_name(int tile);
void tile_dims(int tile, int& tx, int& ty);

// Everything one step needs; all pointers are device pointers.
struct StepArgs {
  Grid g;
  StepCtl* ctl;
  const Physics* phys;
  const BcParams* bc;
  FieldSet U0, U1, S;
  double* b;
  Forcing fo;
  double* partials;  // 4 * blocks_per_stage doubles
  double* eta_old[4];
  int tile;
  int hllc;
};

// Doubles of per-block partial storage the step kernels need.
size_t partials_doubles(const Grid& g, int tile);

// Set the shared-memory attributes of the stage kernels of one variant (call
// before capturing them in a graph).
cudaError_t configure_kernels(int tile, int hllc);

// Queue one SSP-RK2 step (4-6 launches) on `s`.  Every launch checks the
// device clock, so steps past the stop condition are no-ops.
cudaError_t launch_step(const StepArgs& a, cudaStream_t s);

// One stage kernel alone (stage 1 or 2), for per-kernel timing.
cudaError_t launch_stage_only(const StepArgs& a, int stage, cudaStream_t s);
// Kernel launches one step issues.
int launches_per_step(const StepArgs& a);

// Queue the CFL reduction of the current state (fills ctl->msx/msy).
cudaError_t launch_max_speed(const StepArgs& a, cudaStream_t s);

// Kernel-level entry points (device pointers, pitched arrays).
cudaError_t launch_flux(const Grid& g, int hllc, FieldSet in, const double* b, FluxOut out,
                        int tile, cudaStream_t s);
cudaError_t launch_bc(const StepArgs& a, int stage, cudaStream_t s);

}  // namespace rkb
