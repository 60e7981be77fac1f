// Host-side launch interface of the B200 kernels (no torch types).
#pragma once

#include <cstddef>
#include <cuda.h>  // CUtensorMap (the maps are encoded through the runtime's driver entry point)
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
  kTile32x8w = 6, kTile32x12w = 7,  // shared-memory tiles with two extra warps
  // tiles whose face loop takes exactly two rounds of 256 threads: 16x15
  // (511 faces) and 32x7 with one extra warp (487 faces)
  kTile16x15 = 8, kTile32x7w = 9,
  // 16x15 tiles loaded by TMA copies of their halo boxes (the plain 16x15
  // kernel runs where the maps cannot be encoded)
  kTile16x15t = 10,
  kNumTiles = 11
};
const char* tile_name(int tile);
void tile_dims(int tile, int& tx, int& ty);

// TMA maps (2D, FP64, pitched rows, zero fill outside) of the state buffers
// for the TMA-staged tile kernel: the halo box of a tile (TX + 6 by TY + 4:
// boxes start on an even column) over U0, U1 and S, the same box over the
// bed, and the box of the tile's cells (TX + 2 by TY) over U0 and U1 (U^n in
// stage 2).
struct alignas(64) TileMaps {
  CUtensorMap tile[3][3];   // [U0, U1, S][h, hu, hv]
  CUtensorMap bed;
  CUtensorMap cells[2][3];  // [U0, U1][h, hu, hv]
};

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
  int scheme;    // time scheme: 2 SSP-RK2 (fused stages), 1 euler, 3 rk3, 4 rk43
  int n_stages;  // stages of the generic schemes
  int plain;     // no forcing, Coriolis or sponge: the SSP-RK2 stages built without those terms
  const TileMaps* maps;    // HOST copy of the TMA maps of these buffers (null: none)
  long long wait_cycles;   // limit of the TMA tile kernel's waits (kWaitCyclesDefault)
};

// Encodes the TMA maps of a's buffers for the TMA-staged tile kernel.  0, or
// why that kernel cannot serve this grid: 1 rows not on 16-byte boundaries, 2 a misaligned buffer, 3 no encoder, 100 + a runtime
// error or 200 + an entry-point query result while finding the encoder,
// 1000 + the encoder's own result.
int encode_tile_maps(const StepArgs& a, TileMaps* m);

// Doubles of per-block partial storage the step kernels need.
size_t partials_doubles(const Grid& g, int tile);

// ---- FP32 surface form ----------------------------------------------------
// State (eta = h + b, hu, hv) in FP32, bed in FP64 (rkb_step_f32.cu).
struct FieldSet32 {
  float* eta;
  float* hu;
  float* hv;
};

// Pointers of the surface form are offset so that element (i, j) is
// p[i + j * g.pitch] and the first interior column of every row is
// 128-byte aligned; the pitch also covers the right halo of the last strip.
struct StepArgs32 {
  Grid g;              // surface-form layout (pitch in elements)
  StepCtl* ctl;
  const Physics* phys;
  const BcParams* bc;
  FieldSet32 U0, U1, S;
  double* b;           // bed, FP64, surface-form layout
  Forcing fo;          // FP64 forcing fields, depth-form layout (pitch fpitch)
  int fpitch;
  double* partials;
  double* eta_old[4];  // Chapman surfaces (FP64)
  int hllc;
  int plain;           // no forcing, Coriolis or sponge: the sweep built without those terms
  int cpl;             // columns per lane of the sweep (2 or 4)
  int rows;            // rows per warp sweep
  int nstrips, nrowblk;
  long long wait_cycles;  // limit of the waits for the bulk copies (kWaitCyclesDefault)
};

// Strips and row blocks of the sweep for `rows` rows per warp and `cpl`
// columns per lane (strips of 30 * cpl output columns).
void sweep_shape(const Grid& g, int rows, int cpl, int& nstrips, int& nrowblk);
// Columns of a row (counted from column 0) that the sweep's copies touch, for
// any supported cpl: the surface-form pitch must cover it.
size_t sweep_row_extent(const Grid& g);
// Rows per sweep so that one wave of resident warps covers the grid.
int auto_rows32(const Grid& g, int cpl);
// Partial-sum doubles for any cpl and rows >= `rows`.
size_t partials_doubles32(const Grid& g, int rows);
cudaError_t configure_kernels32();
int launches_per_step32(const StepArgs32& a);
cudaError_t launch_step32(const StepArgs32& a, cudaStream_t s);
cudaError_t launch_bc32(const StepArgs32& a, int stage, cudaStream_t s);
cudaError_t launch_stage32_only(const StepArgs32& a, int stage, cudaStream_t s);
cudaError_t launch_max_speed32(const StepArgs32& a, cudaStream_t s);
// Conversions between the FP64 depth form and the FP32 surface form (every
// cell, ghosts included); `bed_out` (may be null) receives the bed.
cudaError_t launch_to_surface(const Grid& g64, const Grid& g32, FieldSet src, const double* b64,
                              FieldSet32 dst, double* bed_out, cudaStream_t s);
cudaError_t launch_to_depth(const Grid& g32, const Grid& g64, FieldSet32 src, const double* b32,
                            FieldSet dst, double* bed_out, cudaStream_t s);

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

// ---- batches of independent simulations --------------------------------
// One launch per phase covers every simulation: `args` holds each
// simulation's StepArgs (device array) and `map` gives each block of the stage
// launch its simulation and its tile / warp-group index within it.  All
// simulations of a batch share the kernel variant (tile or columns per lane,
// HLL / HLLC) and are at least max(nghost, 2) cells wide.
struct BatchLaunch {
  const StepArgs* args;
  const int2* map;
  int n;        // simulations
  int blocks;   // blocks of one stage launch
  int max_nxt, max_nyt;
  int tile, hllc;
  int plain;  // every member plain (StepArgs::plain)
  const TileMaps* maps;  // device array: every member's TMA maps (null: not all encoded)
};
int batch_stage_blocks(const Grid& g, int tile);
cudaError_t configure_batch(int tile, int hllc);
cudaError_t launch_step_batch(const BatchLaunch& bl, cudaStream_t s);
cudaError_t launch_bc_batch(const BatchLaunch& bl, int stage, cudaStream_t s);
cudaError_t launch_stage_batch_only(const BatchLaunch& bl, int stage, cudaStream_t s);

struct BatchLaunch32 {
  const StepArgs32* args;
  const int2* map;
  int n;
  int blocks;
  int max_nxt, max_nyt;
  int cpl, hllc;
  int plain;  // every member plain (StepArgs32::plain)
};
int batch_sweep_blocks(const StepArgs32& a);
cudaError_t configure_batch32();
cudaError_t launch_step32_batch(const BatchLaunch32& bl, cudaStream_t s);
cudaError_t launch_stage32_batch(const BatchLaunch32& bl, int stage, cudaStream_t s);
cudaError_t launch_bc32_batch(const BatchLaunch32& bl, int stage, cudaStream_t s);

// Kernel-level entry points (device pointers, pitched arrays).
cudaError_t launch_flux(const Grid& g, int hllc, FieldSet in, const double* b, FluxOut out,
                        int tile, cudaStream_t s);
cudaError_t launch_bc(const StepArgs& a, int stage, cudaStream_t s);

}  // namespace rkb
