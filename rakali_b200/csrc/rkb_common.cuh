// Shared definitions for the B200 structured shallow-water step.
//
// Layout: every field is a pitched, column-major (Fortran order) array of
// nx_total x ny_total cells, ghosts included; element (i, j) (0-based) lives
// at a[i + j * pitch] with pitch >= nx_total a multiple of 32 elements, so
// every row starts on a 256-byte boundary.
//
// The FP64 path is compiled with --fmad=false and evaluates every expression
// in the reference's left-to-right order, so its results are bit-identical
// to the Fortran arithmetic wherever only +, -, *, / and sqrt are involved
// (IEEE-754 correctly rounded on both CPU and GPU).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rkb {

// src/core/rki_constants.F90:38-157
constexpr double kG = 9.80665;
constexpr double kRho = 1035.0;
constexpr double kDry = 1.0e-6;
constexpr double kThin = 1.0e-3;
constexpr double kFroude = 50.0;
// DESING_EPS = 1.5e-4; the reference folds DESING_EPS**4 at compile time.
constexpr double kEps4 = 5.062499999999998e-16;
constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kTwoPi = 6.283185307179586;
constexpr double kHalfG = 0.5 * kG;  // exact: halving is exact

constexpr int kMaxTidal = 10;

// Boundary tags, src/core/structured/rki_boundary_types.F90:19-36.
enum BcType : int {
  kWall = 1, kOpen = 2, kTidal = 3, kNested = 4, kInflow = 5,
  kDischarge = 6, kClamped = 7, kSponge = 8, kChapman = 9
};

struct Grid {
  int nxt, nyt, ng;  // totals including ghosts, ghost width
  int pitch;         // elements between consecutive j
  double dx, dy;
  __host__ __device__ int nx_phys() const { return nxt - 2 * ng; }
  __host__ __device__ int ny_phys() const { return nyt - 2 * ng; }
  __host__ __device__ size_t at(int i, int j) const { return (size_t)i + (size_t)j * (size_t)pitch; }
};

// Boundary parameters (bc_params_t, rki_boundary_types.F90:38-100), kept in
// device memory so setters can change them without re-capturing graphs.
struct BcParams {
  int type[4];  // west, east, south, north
  int n_tidal;
  int sponge_width;
  double tidal_amplitude, tidal_period;
  double amp[kMaxTidal], phase[kMaxTidal], omega[kMaxTidal];
  double inflow_velocity, discharge_flux, clamped_elevation;
  double sponge_strength, sponge_h_ref;
};

// Physics / time-control scalars (state_t + config_t fields the step reads).
struct Physics {
  double cfl, dt_fixed, t_end, ssp_coeff;
  double manning_n, coriolis_f;
  int cfl_interval;
  int forcing_active;
  int use_hllc;
  // time_scheme: 2 = SSP-RK2 (the fused two-stage path); 1 euler, 3 rk3,
  // 4 rk43 run the generic Shu-Osher stages (rki_timestepper.F90:60-100):
  // stage k updates with beta[k] dt at time t + c[k] dt, then (alpha[k] != 0)
  // blends alpha[k] U^n + (1 - alpha[k]) U.
  int scheme;
  int n_stages;
  int pad_;
  double alpha[4], beta[4], c[4];
};

// Device-resident clock and reductions of one simulation.  Fields marked
// (step) are written inside a step; the others change only at the end of a
// step (by the last block of the final stage kernel) or from the host.
struct StepCtl {
  double t;            // h%t_current
  double dt_prev;      // state%dt as of the start of the step
  double dt;           // (step) this step's dt
  double target;       // advance target (mode 0)
  double mass_out, mass_src;
  double precip_sum;   // sum of precipitation over the interior (host-set)
  double msx, msy;     // max over wet cells of (|u|+c) along x and y (current state)
  unsigned long long msx_next, msy_next;  // (step) atomicMax accumulators (bit patterns)
  int step_count;
  int cur;             // ping-pong buffer holding U^n
  int active;          // (step) 1 when this step runs
  int mode;            // 0: advance to target, 1: fixed step count
  int remaining;       // steps left in mode 1
  int ms_valid;        // msx/msy describe the current state
  unsigned int done_blocks;  // last-block counter of the final stage kernel
  unsigned int ms_done_blocks;
  int steps_run;       // steps executed since the host last cleared it
  int error;           // nonzero: kErrWait, kErrPhysics or kErrNonFinite
};

// StepCtl::error codes.  A step that sets one completes; the steps after it
// in the same graph chunk do not run (step_begin), and the host reports it.
constexpr int kErrWait = 1;       // a bounded device-side wait for a bulk or TMA copy gave up
constexpr int kErrPhysics = 2;    // a launch built without forcing / Coriolis / sponge met them
constexpr int kErrNonFinite = 3;  // the new state holds a NaN or an infinity

// Default limit of the device-side waits for bulk and TMA copies (FP32
// sweep, FP64 TMA-staged tiles; ~1 s at B200 clocks); the drain after a wait
// gave up always uses this one.
constexpr long long kWaitCyclesDefault = 2000000000ll;

// ---------------------------------------------------------------------------
// Small FP64 helpers in the reference's evaluation order.
// ---------------------------------------------------------------------------

// The pointwise helpers are templates on the real type T: the production
// FP64 kernels instantiate them with double; the FP32 adjoint with float.
// Every constant enters as T(c), so the double instances evaluate exactly the
// expressions written here.
template <typename T>
__host__ __device__ __forceinline__ T dmax(T a, T b) { return a > b ? a : b; }
template <typename T>
__host__ __device__ __forceinline__ T dmin(T a, T b) { return a < b ? a : b; }
// Fortran max(0, x) for non-NaN x.
template <typename T>
__host__ __device__ __forceinline__ T pos(T x) { return x > T(0) ? x : T(0); }

// minmod, rki_kernel_flux.F90:380-393
template <typename T>
__host__ __device__ __forceinline__ T minmod(T a, T b) {
  if (a * b <= T(0)) return T(0);
  return fabs(a) < fabs(b) ? a : b;
}

// Clamp + KP07 desingularisation + Froude backstop
// (rki_kernel_fused.F90:93-119 and :441-463).
template <typename T>
__host__ __device__ __forceinline__ void protect(T& h, T& u, T& v) {
  if (h < T(0)) {
    h = T(0); u = T(0); v = T(0);
  } else if (h < T(kDry)) {
    u = T(0); v = T(0);
  } else {
    T h2 = h * h;
    T h4 = h2 * h2;
    if (h4 < T(kEps4)) {
      T r = sqrt(h4 + T(kEps4));
      T uu = T(kSqrt2) * h * u / r;
      T vv = T(kSqrt2) * h * v / r;
      u = h * uu;
      v = h * vv;
    }
    T sp2 = (u * u + v * v) / (h * h);
    T fr2 = T(kFroude) * T(kFroude) * T(kG) * h;
    if (sp2 > fr2) {
      T sc = sqrt(fr2 / sp2);
      u = u * sc;
      v = v * sc;
    }
  }
}

// Wave speed terms of compute_timestep (rki_kernel_timestep.F90:52-66):
// returns (|u|_KP07 + sqrt(g h)) along x and y, before the division by dx/dy.
template <typename T>
__host__ __device__ __forceinline__ void wave_speed(T h, T hu, T hv, T& sx, T& sy) {
  sx = T(0);
  sy = T(0);
  if (h > T(kDry)) {
    T c = sqrt(T(kG) * h);
    T h2 = h * h;
    T den = sqrt(h2 * h2 + T(kEps4));
    T ua = fabs(hu) * T(kSqrt2) * h / den;
    T va = fabs(hv) * T(kSqrt2) * h / den;
    sx = ua + c;
    sy = va + c;
  }
}

// dt from the maximum wave speed (rki_kernel_timestep.F90:68-72), the SSP
// factor and the cap (rki_solver.F90:731-748).  Dividing the maxima by dx/dy
// once is exact: x -> fl(x/d) is monotone for d > 0.
__host__ __device__ inline double cfl_dt(double msx, double msy, const Grid& g, double cfl) {
  double ms = dmax(msx / g.dx, msy / g.dy);
  if (ms > 0.0) return cfl / ms;
  return cfl * dmin(g.dx, g.dy) / sqrt(kG * kDry);
}

// Non-negative doubles order like their bit patterns.
__device__ __forceinline__ void atomic_max_pos(unsigned long long* addr, double v) {
  if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

}  // namespace rkb
