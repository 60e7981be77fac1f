// FP64 kernels of the structured SSP-RK2 step (sm_100a).
//
// One step is eight launches, all reading their clock from the device-side
// StepCtl so a whole chunk of steps can be captured once in a CUDA graph:
//
//   bc_we / bc_sn (stage 1, time t)   ghost fill of U^n          rki_boundary.F90:40-218
//   stage<1>                          U^n -> U*                  rki_kernel_flux.F90 + rki_kernel_fused.F90:164-303
//   bc_we / bc_sn (stage 2, t + dt)   ghost fill of U*           (ghosts also copied into the U^{n+1} buffer)
//   stage<2>                          U*, U^n -> U^{n+1}         rki_kernel_fused.F90:305-471
//   close_part, close                 sums, budget, clock        rki_solver.F90:507-657
//
// The CFL reduction (rki_kernel_timestep.F90:16-74) is folded into the
// stage-2 epilogue; the first launch of the next step turns it into dt.
// The boundary mass-out sums (rki_solver.F90:507-537) are per-tile partials
// reduced in a fixed order by the two close kernels after stage 2.
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include "rkb_async.cuh"
#include "rkb_bc.cuh"
#include "rkb_cell.cuh"
#include "rkb_crmath.cuh"
#include "rkb_face.cuh"
#include "rkb_kernels.h"
#include "rkb_stepctl.cuh"

namespace rkb {

// ---------------------------------------------------------------------------
// Boundary conditions (rki_boundary.F90:40-552)
// ---------------------------------------------------------------------------

// Buffers of the generic Shu-Osher stages: stage k reads X_k and writes
// X_{k+1}; X_0 = U^n (buffer cur), the last stage writes buffer cur^1, and
// the others alternate with the scratch S so no stage writes its own input.
__device__ __forceinline__ FieldSet generic_out(const FieldSet& U0, const FieldSet& U1,
                                                const FieldSet& S, int k, int nst, int cur) {
  return ((nst - 1 - k) % 2 == 0) ? (cur ? U0 : U1) : S;
}
__device__ __forceinline__ FieldSet generic_in(const FieldSet& U0, const FieldSet& U1,
                                               const FieldSet& S, int k, int nst, int cur) {
  return k == 0 ? (cur ? U1 : U0) : generic_out(U0, U1, S, k - 1, nst, cur);
}

// One thread per tangential position t of edge w, looping over the ghost
// layers k (so the Chapman surface refresh of position t is race-free).
// Ghost values go to the stage's input buffer and, in RK2 stage 2 and the
// last generic stage, also to the buffer that receives U^{n+1} (its ghosts
// then hold the last fill, as the reference's single array does).  `stage` is
// 1 or 2 (SSP-RK2) or 10 + k (generic stage k, time t + c_k dt).  `writer`
// marks the one thread of the step's first boundary launch that publishes
// this step's active flag and dt.
//
// Narrow grids (an interior thinner than max(nghost, 2) in x or y): a ghost
// layer then mirrors a ghost of the opposite edge, so the values left by the
// previous fill matter.  The reference fills its single array once before
// computing dt (rki_solver.F90:719) and once per stage; for these grids the
// step runs that extra fill (stage 9: time t, the previous step's dt) and
// every stage's fill also writes the buffer the next stage reads, so each
// fill sees the ghosts the reference's array holds at that point.
__device__ __forceinline__ void bc_body(const StepArgs& a, int stage, int w, int t, bool writer) {
  const Grid& g = a.g;
  StepCtl* ctl = a.ctl;
  const BcParams* bc = a.bc;
  double* __restrict__ b = a.b;
  double dt;
  bool active = step_begin(ctl, a.phys, g, dt);
  if (writer) {
    ctl->active = active ? 1 : 0;
    ctl->dt = dt;
  }
  if (!active) return;
  const FieldSet U0 = a.U0, U1 = a.U1, S = a.S;

  const int cur = ctl->cur;
  const int wide = g.ng > 2 ? g.ng : 2;
  const bool narrow = g.nx_phys() < wide || g.ny_phys() < wide;
  double time;
  double dtb = dt;  // the dt this fill uses (Chapman)
  FieldSet F;
  double* h2 = nullptr;
  double* hu2 = nullptr;
  double* hv2 = nullptr;
  auto also = [&](const FieldSet& N) { h2 = N.h; hu2 = N.hu; hv2 = N.hv; };
  if (stage == 9) {  // the fill before dt (narrow grids only)
    time = ctl->t;
    dtb = ctl->dt_prev;
    F = cur ? U1 : U0;
  } else if (stage >= 10) {
    const int k = stage - 10, nst = a.phys->n_stages;
    time = ctl->t + a.phys->c[k] * dt;
    F = generic_in(U0, U1, S, k, nst, cur);
    if (k == nst - 1)
      also(cur ? U0 : U1);
    else if (narrow)
      also(generic_out(U0, U1, S, k, nst, cur));
  } else {
    time = stage == 1 ? ctl->t : ctl->t + dt;
    F = stage == 1 ? (cur ? U1 : U0) : S;
    if (stage == 2)
      also(cur ? U0 : U1);
    else if (narrow)
      also(S);
  }
  double* eo = a.eta_old[w];
  fill_edge(g, bc, b, F, h2, hu2, hv2, w, t, time, dtb, eo, stage == 1 || stage == 10);
}

// Edges [e0, e0 + gridDim.y) of one simulation.
__global__ void k_bc(StepArgs a, int stage, int e0, int first_launch) {
  bc_body(a, stage, e0 + (int)blockIdx.y, (int)(blockIdx.x * blockDim.x + threadIdx.x),
          first_launch && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0);
}

// The same edges of every simulation of a batch (blockIdx.z = simulation).
__global__ void k_bc_batch(const StepArgs* __restrict__ args, int stage, int e0, int first_launch) {
  __shared__ StepArgs sa;
  if (threadIdx.x == 0) sa = args[blockIdx.z];
  __syncthreads();
  bc_body(sa, stage, e0 + (int)blockIdx.y, (int)(blockIdx.x * blockDim.x + threadIdx.x),
          first_launch && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0);
}

// ---------------------------------------------------------------------------
// CFL reduction over the current state (used when no stage-2 epilogue has
// produced it yet: after create or after the host changed the state).
// ---------------------------------------------------------------------------

__global__ void k_max_speed(Grid g, StepCtl* ctl, FieldSet U0, FieldSet U1) {
  const FieldSet F = ctl->cur ? U1 : U0;
  const int nxp = g.nx_phys(), nyp = g.ny_phys();
  const long long n = (long long)nxp * nyp;
  double mx = 0.0, my = 0.0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int i = g.ng + (int)(k % nxp);
    const int j = g.ng + (int)(k / nxp);
    const size_t q = g.at(i, j);
    double sx, sy;
    wave_speed(F.h[q], F.hu[q], F.hv[q], sx, sy);
    if (sx > mx) mx = sx;
    if (sy > my) my = sy;
  }
  mx = warp_max(mx);
  my = warp_max(my);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&ctl->msx_next, mx);
    atomic_max_pos(&ctl->msy_next, my);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int done = atomicAdd(&ctl->ms_done_blocks, 1u);
    if (done == gridDim.x - 1) {
      __threadfence();
      volatile StepCtl* vc = ctl;
      ctl->msx = __longlong_as_double((long long)vc->msx_next);
      ctl->msy = __longlong_as_double((long long)vc->msy_next);
      ctl->msx_next = 0ull;
      ctl->msy_next = 0ull;
      ctl->ms_valid = 1;
      ctl->ms_done_blocks = 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// Fused stage kernel
// ---------------------------------------------------------------------------

// Shared-memory plan of one TX x TY tile (doubles):
//   tile  4 x (TX+4)(TY+4)   h, hu, hv, b with a 2-cell halo (eta = h + b is
//                            formed where it is read, with the same rounding)
//   fx    6 x (TX+1) TY      x-face fluxes + well-balanced terms
//   fy    6 x TX (TY+1)      y-face fluxes + well-balanced terms
//   old   3 x TX TY          U^n of the tile's cells (stage 2: the RK2 average)
// The limited slopes are not stored: each face computes the slopes of its
// two cells along its normal from the tile (every slope twice, the same
// expressions, so the same bits), which spares the slope arrays and a block
// barrier.
// Threads of a TX x TY tile with XW extra warps: the cells rounded up to
// whole warps, plus the extra warps.
constexpr int stage_threads(int tx, int ty, int xw) { return (tx * ty + 31) / 32 * 32 + 32 * xw; }

// TMA: the layout of the TMA-staged kernel.  Its boxes start on an even
// column (16 bytes), one column left of the tile when the ghost width is odd,
// so their rows are two columns wider (TX + 6 with the halo, TX + 2 for U^n)
// and the arrays are read from an offset of (ng & 1); every array starts on
// a 128-byte line, and the dynamic buffer carries 128 bytes of slack to
// align its start.
template <int TX, int TY, bool TMA = false>
struct StageSmem {
  static constexpr int TW = TX + 4 + (TMA ? 2 : 0), TH = TY + 4;  // tile row stride, rows
  static constexpr int NT = TW * TH;
  static constexpr int NTP = TMA ? (NT + 15) / 16 * 16 : NT;  // tile array stride
  static constexpr int NFX = (TX + 1) * TY;
  static constexpr int NFY = TX * (TY + 1);
  static constexpr int NC = TX * TY;                        // cells
  static constexpr int CW = TX + (TMA ? 2 : 0);             // U^n row stride
  static constexpr int NCP = TMA ? (CW * TY + 15) / 16 * 16 : NC;  // U^n array stride
  static constexpr int DOUBLES = 4 * NTP + 3 * NCP + 6 * NFX + 6 * NFY;
  static constexpr size_t BYTES = sizeof(double) * (size_t)DOUBLES + (TMA ? 128 : 0);
  static_assert(!TMA || TX % 2 == 0, "TMA boxes start on even columns");
};

// Shared-memory arrays of one stage block: tile (h, hu, hv, b with a 2-cell
// halo), U^n of the cells, x- and y-face terms.
struct StagePtrs {
  double *th, *tu, *tv, *tb, *oh, *ou, *ov, *fxa, *fya;
};

// The arrays where the copies land (TMA: 128-byte aligned).
template <int TX, int TY, bool TMA>
__device__ __forceinline__ StagePtrs stage_ptrs(double* base) {
  using SM = StageSmem<TX, TY, TMA>;
  // aligned by an element offset, not an integer cast, so that the compiler
  // still sees shared-memory pointers (shared loads, not generic ones)
  if (TMA) base += ((128u - (smem_u32(base) & 127u)) & 127u) / sizeof(double);
  StagePtrs p;
  p.th = base;
  p.tu = p.th + SM::NTP;
  p.tv = p.tu + SM::NTP;
  p.tb = p.tv + SM::NTP;
  p.oh = p.tb + SM::NTP;
  p.ou = p.oh + SM::NCP;
  p.ov = p.ou + SM::NCP;
  p.fxa = p.ov + SM::NCP;  // 6 arrays of NFX: fh, fqx, fqy, wbR, hL2, pL2
  p.fya = p.fxa + 6 * SM::NFX;
  return p;
}

// TMA copies of tile (bx, by) for the TMA-staged kernel (one thread): the
// halo box of h, hu, hv from field set `in_set` (0 U0, 1 U1, 2 S) and of the
// bed, and in stage 2 the cell box of U^n from `old_set`, all completing on
// `bar`.  The box x coordinates, ng + bx TX - 2 - (ng & 1) and that + 2, are
// even (TX is), which puts every box start on a 16-byte boundary.
template <int TX, int TY, int STAGE>
__device__ __forceinline__ void issue_tile(const TileMaps& tm, int in_set, int old_set,
                                           const Grid& g, unsigned bx, unsigned by,
                                           uint32_t bar, const StagePtrs& p) {
  using SM = StageSmem<TX, TY, true>;
  constexpr uint32_t kBox = 8u * SM::TW * SM::TH, kCells = 8u * SM::CW * TY;
  const int x = g.ng + (int)bx * TX - 2 - (g.ng & 1), y = g.ng + (int)by * TY - 2;
  fence_proxy_async();
  mbar_expect_tx(bar, 4 * kBox + (STAGE == 2 ? 3 * kCells : 0));
  tma_load_2d(smem_u32(p.th), &tm.tile[in_set][0], x, y, bar);
  tma_load_2d(smem_u32(p.tu), &tm.tile[in_set][1], x, y, bar);
  tma_load_2d(smem_u32(p.tv), &tm.tile[in_set][2], x, y, bar);
  tma_load_2d(smem_u32(p.tb), &tm.bed, x, y, bar);
  if (STAGE == 2) {
    tma_load_2d(smem_u32(p.oh), &tm.cells[old_set][0], x + 2, y + 2, bar);
    tma_load_2d(smem_u32(p.ou), &tm.cells[old_set][1], x + 2, y + 2, bar);
    tma_load_2d(smem_u32(p.ov), &tm.cells[old_set][2], x + 2, y + 2, bar);
  }
}



// STAGE 1: U^n (buffer cur) -> U* (scratch S).
// STAGE 2: U* (S) and U^n (buffer cur) -> U^{n+1} (buffer cur^1).
// STAGE 0: flux divergence only (kernel-level API): writes flux/mass-flux
//          arrays from `in`, no update.
// STAGE 3: generic Shu-Osher stage gk of an n-stage scheme
//          (rki_solver.F90:861-926): X_gk -> X_gk+1 with step beta_gk dt,
//          then the SSP combination with U^n when alpha_gk != 0.  The last
//          stage closes the step without the boundary mass budget.
// Tile (bx, by) of a gx x gy tiling of one simulation, with TX * TY + 32 XW
// threads: XW extra warps share the slope and face loops (so that no warp
// runs a third, mostly empty face round) and sit out the cell update.
// PLAIN: the build for stages without forcing, Coriolis or sponge terms
// (Manning friction only), chosen by the host from its copy of the physics.
// TMA: the tile arrays were filled by TMA copies the caller has waited for
// (the TMA-staged kernel, stages 1 and 2).
template <int TX, int TY, bool HLLC, int STAGE, int XW = 0, bool PLAIN = false, bool TMA = false>
__device__ __forceinline__ void stage_body(const Grid& g, StepCtl* ctl, const Physics* phys,
                                           const BcParams* bcp, const FieldSet& U0,
                                           const FieldSet& U1, const FieldSet& S,
                                           const double* __restrict__ b, const Forcing& fo,
                                           double* __restrict__ partials, const FluxOut& fl,
                                           unsigned bx, unsigned by, unsigned gx, unsigned gy,
                                           int gk = 0) {
  static_assert(!TMA || STAGE == 1 || STAGE == 2, "TMA staging serves the SSP-RK2 stages");
  using SM = StageSmem<TX, TY, TMA>;
  constexpr int TW = SM::TW;
  constexpr int NTH = stage_threads(TX, TY, XW);
  extern __shared__ double smem[];
  const StagePtrs P = stage_ptrs<TX, TY, TMA>(smem);
  const int xo = TMA ? (g.ng & 1) : 0;  // column of the tile's first x in the TMA boxes
  double* th = P.th + xo;
  double* tu = P.tu + xo;
  double* tv = P.tv + xo;
  double* tb = P.tb + xo;
  double* fxa = P.fxa;
  double* fya = P.fya;
  double* oh = P.oh + xo;  // U^n of the tile's cells (stage 2), rows SM::CW apart
  double* ou = P.ou + xo;
  double* ov = P.ov + xo;

  double dt = 0.0;
  int cur = 0;
  if (STAGE != 0) {
    if (!TMA && !ctl->active) return;  // the TMA-staged kernel checks before its first copy
    dt = ctl->dt;
    cur = ctl->cur;
  }
  const double step_dt = dt;
  const int nst = STAGE == 3 ? phys->n_stages : 0;
  if (STAGE == 3) dt = phys->beta[gk] * dt;  // the stage's own step
  const FieldSet in = STAGE == 3   ? generic_in(U0, U1, S, gk, nst, cur)
                      : STAGE == 2 ? S
                                   : (cur ? U1 : U0);

  const int tid = threadIdx.x;
  const int gx0 = g.ng + (int)bx * TX;  // first interior cell of the tile
  const int gy0 = g.ng + (int)by * TY;

  // Coriolis rotation of this stage, cos/sin(f dt), correctly rounded once
  // per block (rki_kernel_fused.F90:211-214)
  __shared__ double rot[2];
  if (STAGE != 0 && !PLAIN && tid == 0) {
    double sn = 0.0, cs = 0.0;
    if (fabs(phys->coriolis_f) > 1.0e-20) cr_sincos(phys->coriolis_f * dt, sn, cs);
    rot[0] = cs;
    rot[1] = sn;
  }

  // 1. tile load with halo (ghost cells come from the BC launches); the
  // TMA-staged kernel has its tile already
  for (int k = tid; !TMA && k < SM::NT; k += NTH) {
    const int x = k % TW, y = k / TW;
    const int gi = gx0 - 2 + x, gj = gy0 - 2 + y;
    double vh = 0.0, vu = 0.0, vv = 0.0, vb = 0.0;
    if (gi < g.nxt && gj < g.nyt) {
      const size_t q = g.at(gi, gj);
      vh = in.h[q]; vu = in.hu[q]; vv = in.hv[q]; vb = b[q];
    }
    th[k] = vh; tu[k] = vu; tv[k] = vv; tb[k] = vb;
  }
  if (STAGE == 2 && !TMA) {
    // U^n of the tile's cells for the RK2 average, loaded with the tile so
    // its latency passes during the face phase
    const FieldSet old = cur ? U1 : U0;
    for (int k = tid; k < SM::NC; k += NTH) {
      const int pi = gx0 + k % TX, pj = gy0 + k / TX;
      if (pi < g.nxt - g.ng && pj < g.nyt - g.ng) {
        const size_t q = g.at(pi, pj);
        oh[k] = old.h[q];
        ou[k] = old.hu[q];
        ov[k] = old.hv[q];
      }
    }
  }
  // The TMA-staged kernel's threads each waited for the tile copies, so only
  // the Coriolis terms written by thread 0 (full physics) need this barrier.
  if (!TMA || !PLAIN) __syncthreads();

  auto te = [&](int q) { return th[q] + tb[q]; };  // the surface eta = h + b
  // limited slope (eta, hu, hv) of tile cell q along the direction whose
  // neighbours are q - d and q + d
  auto slope_at = [&](int q, int d, double& se, double& su, double& sv) {
    cell_slope(th[q - d], th[q], th[q + d], te(q - d), te(q), te(q + d), tu[q - d], tu[q],
               tu[q + d], tv[q - d], tv[q], tv[q + d], se, su, sv);
  };

  // 2. faces, each evaluated once, with the slopes of its two cells.  In the
  // paired form (below) thread t takes x-face t in the first round and y-face
  // t in the second; otherwise faces go round-robin over the threads.
  constexpr bool kPaired = TMA && TX == 16 && TY == 15 && XW == 0;
  static_assert(!kPaired || (NTH == 256 && SM::NFX == 255 && SM::NFY == 256), "paired layout");
  auto face = [&](int k) {
    FaceOut o;
    if (k < SM::NFX) {
      const int c = k % (TX + 1), r = k / (TX + 1);  // face between c-1 and c
      const int qL = (r + 2) * TW + (c + 1), qR = qL + 1;
      double sLe, sLu, sLv, sRe, sRu, sRv;
      slope_at(qL, 1, sLe, sLu, sLv);
      slope_at(qR, 1, sRe, sRu, sRv);
      face_flux<0, HLLC>(te(qL) + 0.5 * sLe, tu[qL] + 0.5 * sLu, tv[qL] + 0.5 * sLv, tb[qL],
                         te(qR) - 0.5 * sRe, tu[qR] - 0.5 * sRu, tv[qR] - 0.5 * sRv, tb[qR], o);
      fxa[k] = o.fh;
      fxa[SM::NFX + k] = o.fqx;
      fxa[2 * SM::NFX + k] = o.fqy;
      fxa[3 * SM::NFX + k] = o.wbR;
      fxa[4 * SM::NFX + k] = o.hL2;
      fxa[5 * SM::NFX + k] = o.pL2;
    } else {
      const int kk = k - SM::NFX;
      const int c = kk % TX, r = kk / TX;  // face between rows r-1 and r
      const int qB = (r + 1) * TW + (c + 2), qT = qB + TW;
      double sBe, sBu, sBv, sTe, sTu, sTv;
      slope_at(qB, TW, sBe, sBu, sBv);
      slope_at(qT, TW, sTe, sTu, sTv);
      face_flux<1, HLLC>(te(qB) + 0.5 * sBe, tu[qB] + 0.5 * sBu, tv[qB] + 0.5 * sBv, tb[qB],
                         te(qT) - 0.5 * sTe, tu[qT] - 0.5 * sTu, tv[qT] - 0.5 * sTv, tb[qT], o);
      fya[kk] = o.fh;
      fya[SM::NFY + kk] = o.fqx;
      fya[2 * SM::NFY + kk] = o.fqy;
      fya[3 * SM::NFY + kk] = o.wbR;
      fya[4 * SM::NFY + kk] = o.hL2;
      fya[5 * SM::NFY + kk] = o.pL2;
    }
  };
  if (kPaired) {
    if (tid < SM::NFX) face(tid);
    face(SM::NFX + tid);
    // The cells of warp w (rows 2w, 2w+1) read x-faces 34w .. 34w+33 and
    // y-faces 32w .. 32w+47: faces of warps w and w+1 only, and warp 7 reads
    // its own.  So instead of a block barrier, warp w+1 arrives on named
    // barrier w+1 (64 threads) and warp w waits on it; warp 7 orders its own
    // lanes.  Every warp reaches this point (the early exits above are
    // block-uniform), so each barrier gets its 64 threads.
    const int w = tid >> 5;
    __syncwarp();
    if (w > 0) named_arrive(w, 64);
    if (w < NTH / 32 - 1)
      named_sync(w + 1, 64);
    else
      __syncwarp();
  } else {
    for (int k = tid; k < SM::NFX + SM::NFY; k += NTH) face(k);
    __syncthreads();
  }

  // 3. cell update: one cell per thread (the extra warps repeat cell 0 and
  // store nothing)
  const int tc = tid < TX * TY ? tid : 0;
  const int c = tc % TX, r = tc / TX;
  const int i = gx0 + c, j = gy0 + r;
  const bool valid = tid < TX * TY && i < g.nxt - g.ng && j < g.nyt - g.ng;
  const int fl_ = r * (TX + 1) + c, fr_ = fl_ + 1;
  const int fb_ = r * TX + c, ft_ = fb_ + TX;
  const double dx = g.dx, dy = g.dy;
  const double o_fh = -((fxa[fr_] - fxa[fl_]) / dx) - (fya[ft_] - fya[fb_]) / dy;
  const double o_fhu =
      -((fxa[SM::NFX + fr_] - fxa[SM::NFX + fl_]) / dx) -
      (fya[SM::NFY + ft_] - fya[SM::NFY + fb_]) / dy -
      kHalfG * (fxa[3 * SM::NFX + fl_] - fxa[4 * SM::NFX + fr_] + fxa[5 * SM::NFX + fr_]) / dx;
  const double o_fhv =
      -((fxa[2 * SM::NFX + fr_] - fxa[2 * SM::NFX + fl_]) / dx) -
      (fya[2 * SM::NFY + ft_] - fya[2 * SM::NFY + fb_]) / dy -
      kHalfG * (fya[3 * SM::NFY + fb_] - fya[4 * SM::NFY + ft_] + fya[5 * SM::NFY + ft_]) / dy;

  double part = 0.0, sponge_d = 0.0, wsx = 0.0, wsy = 0.0;
  bool bad = false;  // the new state of this cell is not finite
  if (valid) {
    const size_t q = g.at(i, j);
    if (STAGE == 0) {
      fl.flux_h[q] = o_fh;
      fl.flux_hu[q] = o_fhu;
      fl.flux_hv[q] = o_fhv;
      if (fl.mflux_x) {
        fl.mflux_x[q] = fxa[fr_];
        if (i == g.ng) fl.mflux_x[q - 1] = fxa[fl_];
      }
      if (fl.mflux_y) {
        fl.mflux_y[q] = fya[ft_];
        if (j == g.ng) fl.mflux_y[q - g.pitch] = fya[fb_];
      }
    } else {
      const int qc = (r + 2) * TW + (c + 2);
      double a = th[qc], u = tu[qc], v = tv[qc];
      a = a + dt * o_fh;
      u = u + dt * o_fhu;
      v = v + dt * o_fhv;
      protect(a, u, v);
      const double n_sq = phys->manning_n * phys->manning_n;
      if (PLAIN) {
        sources_plain(a, u, v, phys->manning_n, dt, n_sq);
      } else {
        const bool has_cor = fabs(phys->coriolis_f) > 1.0e-20;
        sources(a, u, v, phys, dt, n_sq, rot[0], rot[1], has_cor, g, i, j, fo);
      }
      FieldSet out;
      if (STAGE == 1) {
        out = S;
      } else if (STAGE == 3) {
        out = generic_out(U0, U1, S, gk, nst, cur);
        // SSP combination with U^n and its clamp (rki_kernel_update.F90:152-208)
        const double an = phys->alpha[gk];
        if (an != 0.0) {
          const FieldSet old = cur ? U1 : U0;
          const double ap = 1.0 - an;
          a = an * old.h[q] + ap * a;
          u = an * old.hu[q] + ap * u;
          v = an * old.hv[q] + ap * v;
          protect(a, u, v);
        }
      } else {
        // RK2 average with U^n and the second clamp (rki_kernel_fused.F90:435-463)
        out = cur ? U0 : U1;
        const int qn = r * SM::CW + c;  // U^n of this cell
        a = 0.5 * (oh[qn] + a);
        u = 0.5 * (ou[qn] + u);
        v = 0.5 * (ov[qn] + v);
        protect(a, u, v);
      }
      const double h_pre_sponge = a;
      if (!PLAIN) sponge(a, u, v, bcp, g, i, j, dt);
      out.h[q] = a;
      out.hu[q] = u;
      out.hv[q] = v;
      part = o_fh;
      sponge_d = PLAIN ? 0.0 : a - h_pre_sponge;
      if (STAGE == 2 || (STAGE == 3 && gk == nst - 1)) {
        wave_speed(a, u, v, wsx, wsy);
        bad = !isfinite(a + u + v);
      }
    }
  }
  if (STAGE == 0) return;
  if (STAGE == 3 && gk != nst - 1) return;  // block-uniform

  // 4. block partials (fixed order) and the CFL maxima of the new state
  constexpr bool kBudget = STAGE != 3;
  if (STAGE != 1) {
    wsx = warp_max(wsx);
    wsy = warp_max(wsy);
    bad = __any_sync(0xffffffffu, bad);
    if ((tid & 31) == 0) {
      atomic_max_pos(&ctl->msx_next, wsx);
      atomic_max_pos(&ctl->msy_next, wsy);
      if (bad) atomicExch(&ctl->error, kErrNonFinite);
    }
  }
  const unsigned int nblocks = gx * gy;
  if (kBudget) {
    part = warp_sum(part);
    sponge_d = warp_sum(sponge_d);
    __shared__ double red[2][NTH / 32];
    if ((tid & 31) == 0) {
      red[0][tid >> 5] = part;
      red[1][tid >> 5] = sponge_d;
    }
    __syncthreads();
    const unsigned int bid = by * gx + bx;
    if (tid == 0) {
      double s0 = 0.0, s1 = 0.0;
      for (int w = 0; w < NTH / 32; ++w) {
        s0 = s0 + red[0][w];
        s1 = s1 + red[1][w];
      }
      double* P = partials + (size_t)(STAGE - 1) * 2 * nblocks;
      P[bid] = s0;
      P[nblocks + bid] = s1;
    }
  }
  // 5. the step is closed by k_close, launched right after this stage: a
  // grid-wide "last block" counter would hold every block for an atomic
  // round trip and leave the closing sums to one block at the tail
  (void)step_dt;
  (void)cur;
}

// Close a step after its last stage kernel (one block): the fixed-order sums
// of the per-block partials, the mass budget, the CFL maxima and the clock.
__global__ void __launch_bounds__(1024)
    k_close(Grid g, StepCtl* ctl, const Physics* phys, double* partials, unsigned int nblocks,
            int budget) {
  if (!ctl->active) return;
  finalize_step(g, ctl, phys, partials, nblocks, ctl->dt, ctl->cur, budget != 0);
}

// First level of the close, before k_close: block b of the kCloseBlocks sums
// its contiguous share of each of the four per-tile partial arrays (nparts
// long, one after the other) in a fixed order into out[s * gridDim.x + b].
// One block alone reads the tens of thousands of partials of a large grid at
// the latency of its own loads (45 us a step at 4096^2).
__global__ void __launch_bounds__(256)
    k_close_part(const StepCtl* ctl, const double* __restrict__ partials, unsigned int nparts,
                 double* __restrict__ out) {
  if (!ctl->active) return;
  const unsigned int per = (nparts + gridDim.x - 1) / gridDim.x;
  const unsigned int k0 = blockIdx.x * per;
  const unsigned int k1 = k0 + per < nparts ? k0 + per : nparts;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (unsigned int k = k0 + threadIdx.x; k < k1; k += blockDim.x)
    for (int s = 0; s < 4; ++s) acc[s] = acc[s] + __ldcg(partials + (size_t)s * nparts + k);
  __shared__ double red[4][8];
  for (int s = 0; s < 4; ++s) {
    const double w = warp_sum(acc[s]);
    if ((threadIdx.x & 31) == 0) red[s][threadIdx.x >> 5] = w;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t = t + red[threadIdx.x][w];
    out[threadIdx.x * gridDim.x + blockIdx.x] = t;
  }
}

// The same for every simulation of a batch (blockIdx.x = simulation), tiles
// of tx x ty cells.
__global__ void __launch_bounds__(1024)
    k_close_batch(const StepArgs* __restrict__ args, int tx, int ty) {
  __shared__ StepArgs sa;
  if (threadIdx.x == 0) sa = args[blockIdx.x];
  __syncthreads();
  if (!sa.ctl->active) return;
  const unsigned int nb = (unsigned)((sa.g.nx_phys() + tx - 1) / tx) *
                          (unsigned)((sa.g.ny_phys() + ty - 1) / ty);
  finalize_step(sa.g, sa.ctl, sa.phys, sa.partials, nb, sa.ctl->dt, sa.ctl->cur, true);
}

// The host picks the PLAIN build from its copy of the physics; a launch whose
// device-side physics disagree computes nothing and reports kErrPhysics (the
// host then fails the step).  Every block sees the same physics, so either
// all blocks return here or none does.
__device__ __forceinline__ bool plain_mismatch64(StepCtl* ctl, const Physics* phys,
                                                 const BcParams* bcp) {
  if (plain_physics(*phys, *bcp)) return false;
  if (threadIdx.x == 0) atomicExch(&ctl->error, kErrPhysics);
  return true;
}

// Resident blocks per SM the stage kernels are built for: 32 warps per SM,
// i.e. 64 registers a thread (4 blocks of 256 threads, 8 of 128, 3 of 320, 2
// of 448 and 512).  Left free, the compiler gives the stages more registers
// than that occupancy allows.  `forty`: 40 warps (48 registers) where the
// tile's shared memory, with the 1 KB each block reserves, holds that many
// blocks in the SM's 228 KB; the plain-physics stage 1 is built so (48
// registers and a few spilled bytes, measured 3% faster with 256-thread
// tiles).  Stage 2 holds U^n as well and measured 1% slower so, and the
// full-physics build spills several times more: both keep 32 warps.
constexpr int stage_blocks_per_sm(int threads, int smem_bytes = 0, bool forty = false) {
  const int warps = (threads + 31) / 32;
  const int fit = smem_bytes > 0 ? 228 * 1024 / (smem_bytes + 128 + 1024) : 0;
  if (forty && fit * warps >= 40) return 40 / warps;
  return 32 / warps > 0 ? 32 / warps : 1;
}

template <int TX, int TY, bool HLLC, int STAGE, int XW = 0, bool PLAIN = false>
__global__ void __launch_bounds__(stage_threads(TX, TY, XW),
                                  stage_blocks_per_sm(stage_threads(TX, TY, XW),
                                                      (int)StageSmem<TX, TY>::BYTES,
                                                      STAGE == 1 && PLAIN))
    k_stage(Grid g, StepCtl* ctl, const Physics* phys, const BcParams* bcp, FieldSet U0,
            FieldSet U1, FieldSet S, const double* __restrict__ b, Forcing fo,
            double* __restrict__ partials, FluxOut fl, int gk) {
  if (PLAIN && plain_mismatch64(ctl, phys, bcp)) return;
  // one-dimensional grid over the gx x gy tiles (no limit on the row count)
  const unsigned gx = (unsigned)((g.nx_phys() + TX - 1) / TX);
  stage_body<TX, TY, HLLC, STAGE, XW, PLAIN>(g, ctl, phys, bcp, U0, U1, S, b, fo, partials, fl,
                                             blockIdx.x % gx, blockIdx.x / gx, gx,
                                             gridDim.x / gx, gk);
}

// Every simulation of a batch in one launch: map[blockIdx.x] = (simulation,
// tile index within that simulation's tiling).
template <int TX, int TY, bool HLLC, int STAGE, int XW = 0, bool PLAIN = false>
__global__ void __launch_bounds__(stage_threads(TX, TY, XW),
                                  stage_blocks_per_sm(stage_threads(TX, TY, XW),
                                                      (int)StageSmem<TX, TY>::BYTES,
                                                      STAGE == 1 && PLAIN))
    k_stage_batch(const StepArgs* __restrict__ args, const int2* __restrict__ map) {
  __shared__ StepArgs sa;
  const int2 m = map[blockIdx.x];
  if (threadIdx.x == 0) sa = args[m.x];
  __syncthreads();
  if (PLAIN && plain_mismatch64(sa.ctl, sa.phys, sa.bc)) return;
  const unsigned gx = (unsigned)((sa.g.nx_phys() + TX - 1) / TX);
  const unsigned gy = (unsigned)((sa.g.ny_phys() + TY - 1) / TY);
  const FluxOut none{};
  stage_body<TX, TY, HLLC, STAGE, XW, PLAIN>(sa.g, sa.ctl, sa.phys, sa.bc, sa.U0, sa.U1, sa.S,
                                             sa.b, sa.fo, sa.partials, none, (unsigned)m.y % gx,
                                             (unsigned)m.y / gx, gx, gy);
}

// TMA-staged SSP-RK2 stage (STAGE 1 or 2) on TX x TY tiles: thread 0 loads
// the tile's halo boxes (and in stage 2 its U^n) with TMA copies completing
// on the block's mbarrier, which every thread waits on; the rest is k_stage.
// A wait that runs out of `limit` cycles marks the step (kErrWait), waits
// for the copies in flight with the default limit and ends the block.
// Without the load loop, stage 2 also runs faster at 40 warps per SM (48
// registers, 20-70 spilled bytes): 1.79 -> 1.76 ms at 4096^2.  (A persistent
// form, each block walking a list of tiles and loading the next while it
// updated the current one, measured 9% slower.)
template <int TX, int TY, bool HLLC, int STAGE, bool PLAIN = false>
__global__ void __launch_bounds__(stage_threads(TX, TY, 0),
                                  stage_blocks_per_sm(stage_threads(TX, TY, 0),
                                                      (int)StageSmem<TX, TY, true>::BYTES,
                                                      PLAIN))
    k_stage_tma(Grid g, StepCtl* ctl, const Physics* phys, const BcParams* bcp, FieldSet U0,
                FieldSet U1, FieldSet S, const double* __restrict__ b, Forcing fo,
                double* __restrict__ partials, long long limit, const __grid_constant__ TileMaps tm) {
  if (PLAIN && plain_mismatch64(ctl, phys, bcp)) return;
  if (!ctl->active) return;
  const int cur = ctl->cur;
  const unsigned gx = (unsigned)((g.nx_phys() + TX - 1) / TX);
  const unsigned bx = blockIdx.x % gx, by = blockIdx.x / gx;
  extern __shared__ double smem[];
  __shared__ __align__(8) unsigned long long bar_word;
  const uint32_t bar = smem_u32(&bar_word);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    issue_tile<TX, TY, STAGE>(tm, STAGE == 2 ? 2 : cur, cur, g, bx, by, bar,
                              stage_ptrs<TX, TY, true>(smem));
  }
  __syncthreads();
  const bool ok = mbar_wait(bar, 0, limit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(&ctl->error, kErrWait);
    mbar_wait(bar, 0, kWaitCyclesDefault);  // the copies still in flight
    return;
  }
  stage_body<TX, TY, HLLC, STAGE, 0, PLAIN, true>(g, ctl, phys, bcp, U0, U1, S, b, fo, partials,
                                                  FluxOut{}, bx, by, gx, gridDim.x / gx);
}

// The TMA-staged stage for every simulation of a batch (blocks as in
// k_stage_batch): member m's tiles come through its own maps, maps[m], in
// global memory.
template <int TX, int TY, bool HLLC, int STAGE, bool PLAIN = false>
__global__ void __launch_bounds__(stage_threads(TX, TY, 0),
                                  stage_blocks_per_sm(stage_threads(TX, TY, 0),
                                                      (int)StageSmem<TX, TY, true>::BYTES, PLAIN))
    k_stage_batch_tma(const StepArgs* __restrict__ args, const int2* __restrict__ map,
                      const TileMaps* __restrict__ maps) {
  __shared__ StepArgs sa;
  const int2 m = map[blockIdx.x];
  if (threadIdx.x == 0) sa = args[m.x];
  __syncthreads();
  if (PLAIN && plain_mismatch64(sa.ctl, sa.phys, sa.bc)) return;
  if (!sa.ctl->active) return;
  const int cur = sa.ctl->cur;
  const unsigned gx = (unsigned)((sa.g.nx_phys() + TX - 1) / TX);
  const unsigned gy = (unsigned)((sa.g.ny_phys() + TY - 1) / TY);
  const unsigned bx = (unsigned)m.y % gx, by = (unsigned)m.y / gx;
  extern __shared__ double smem[];
  __shared__ __align__(8) unsigned long long bar_word;
  const uint32_t bar = smem_u32(&bar_word);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    issue_tile<TX, TY, STAGE>(maps[m.x], STAGE == 2 ? 2 : cur, cur, sa.g, bx, by, bar,
                              stage_ptrs<TX, TY, true>(smem));
  }
  __syncthreads();
  const bool ok = mbar_wait(bar, 0, sa.wait_cycles > 0 ? sa.wait_cycles : kWaitCyclesDefault);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(&sa.ctl->error, kErrWait);
    mbar_wait(bar, 0, kWaitCyclesDefault);  // the copies still in flight
    return;
  }
  const FluxOut none{};
  stage_body<TX, TY, HLLC, STAGE, 0, PLAIN, true>(sa.g, sa.ctl, sa.phys, sa.bc, sa.U0, sa.U1, sa.S,
                                                  sa.b, sa.fo, sa.partials, none, bx, by, gx, gy);
}

// ---------------------------------------------------------------------------
// Marching stage kernel: one warp per 28-column strip, stepping up the rows.
// ---------------------------------------------------------------------------
//
// Lane l of a warp owns column x0 - 2 + l; lanes 2..29 produce output cells,
// lanes 0, 1, 30, 31 carry the x halo.  Each iteration handles one row j:
// the y-face above it (the one below was computed in the previous
// iteration), the x-face left of every lane (the right face comes from the
// next lane by shuffle), then the cell update.  No shared memory and no
// block barriers on the data path; each face is evaluated once except the
// strip-boundary ones (x: 1 in 29, y: 1 per ROWS rows).

constexpr int kMarchWarps = 4;   // strips per block
constexpr int kMarchCols = 28;   // output columns per strip

struct RowVals {
  double h, u, v, b;
};

__device__ __forceinline__ RowVals load_row(const FieldSet& F, const double* __restrict__ b,
                                            const Grid& g, int gi, int j, bool col_in) {
  RowVals r{0.0, 0.0, 0.0, 0.0};
  if (col_in) {
    const size_t q = g.at(gi, j);
    r.h = F.h[q];
    r.u = F.hu[q];
    r.v = F.hv[q];
    r.b = b[q];
  }
  return r;
}

__device__ __forceinline__ void yslope(const RowVals& m, const RowVals& c, const RowVals& p,
                                       double& se, double& su, double& sv) {
  cell_slope(m.h, c.h, p.h, m.h + m.b, c.h + c.b, p.h + p.b, m.u, c.u, p.u, m.v, c.v, p.v, se,
             su, sv);
}

template <bool HLLC>
__device__ __forceinline__ void yface(const RowVals& lo, double sle, double slu, double slv,
                                      const RowVals& hi, double she, double shu, double shv,
                                      FaceOut& o) {
  face_flux<1, HLLC>(lo.h + lo.b + 0.5 * sle, lo.u + 0.5 * slu, lo.v + 0.5 * slv, lo.b,
                     hi.h + hi.b - 0.5 * she, hi.u - 0.5 * shu, hi.v - 0.5 * shv, hi.b, o);
}

template <bool HLLC, int STAGE, int ROWS>
__global__ void __launch_bounds__(kMarchWarps * 32, 4)
    k_march(Grid g, StepCtl* ctl, const Physics* phys, const BcParams* bcp, FieldSet U0,
            FieldSet U1, FieldSet S, const double* __restrict__ b, Forcing fo,
            double* __restrict__ partials) {
  if (!ctl->active) return;
  const double dt = ctl->dt;
  const int cur = ctl->cur;
  const FieldSet in = STAGE == 2 ? S : (cur ? U1 : U0);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int strip = blockIdx.x * kMarchWarps + warp;
  const int x0 = g.ng + strip * kMarchCols;
  const int gi = x0 - 2 + lane;
  const int y0 = g.ng + blockIdx.y * ROWS;
  const int yend = min(y0 + ROWS, g.nyt - g.ng);
  const bool col_in = gi < g.nxt;
  const bool out_lane = lane >= 2 && lane < 2 + kMarchCols && gi < g.nxt - g.ng;
  const double dx = g.dx, dy = g.dy;
  const double n_sq = phys->manning_n * phys->manning_n;
  const bool has_cor = fabs(phys->coriolis_f) > 1.0e-20;
  double cosf = 0.0, sinf = 0.0;
  if (has_cor) cr_sincos(phys->coriolis_f * dt, sinf, cosf);

  double part = 0.0, sponge_d = 0.0, wsx = 0.0, wsy = 0.0;
  if (x0 < g.nxt - g.ng && y0 < yend) {  // warp-uniform
    // prologue: rows y0-2 .. y0+1, slopes of y0-1 and y0, face y0-1/2
    RowVals A = load_row(in, b, g, gi, y0 - 2, col_in);
    RowVals B = load_row(in, b, g, gi, y0 - 1, col_in);
    RowVals C = load_row(in, b, g, gi, y0, col_in);
    RowVals D = load_row(in, b, g, gi, y0 + 1, col_in);
    double sBe, sBu, sBv, sCe, sCu, sCv;
    yslope(A, B, C, sBe, sBu, sBv);
    yslope(B, C, D, sCe, sCu, sCv);
    FaceOut bot;
    yface<HLLC>(B, sBe, sBu, sBv, C, sCe, sCu, sCv, bot);
    RowVals E = load_row(in, b, g, gi, y0 + 2, col_in);
    for (int j = y0; j < yend; ++j) {
      // prefetch row j+3 (stays inside the array: j + 3 <= nyt - ng + 2)
      RowVals Fn{0.0, 0.0, 0.0, 0.0};
      if (j + 1 < yend) Fn = load_row(in, b, g, gi, j + 3, col_in);
      double old_h = 0.0, old_u = 0.0, old_v = 0.0;
      size_t q = 0;
      if (out_lane) {
        q = g.at(gi, j);
        if (STAGE == 2) {
          const FieldSet old = cur ? U1 : U0;
          old_h = old.h[q];
          old_u = old.hu[q];
          old_v = old.hv[q];
        }
      }
      // y-face above row j
      double sDe, sDu, sDv;
      yslope(C, D, E, sDe, sDu, sDv);
      FaceOut top;
      yface<HLLC>(C, sCe, sCu, sCv, D, sDe, sDu, sDv, top);
      // x-slope of this lane's cell in row j (neighbours by shuffle)
      const double ec = C.h + C.b;
      const double hm = __shfl_up_sync(0xffffffffu, C.h, 1);
      const double hp = __shfl_down_sync(0xffffffffu, C.h, 1);
      const double em = __shfl_up_sync(0xffffffffu, ec, 1);
      const double ep = __shfl_down_sync(0xffffffffu, ec, 1);
      const double um = __shfl_up_sync(0xffffffffu, C.u, 1);
      const double up = __shfl_down_sync(0xffffffffu, C.u, 1);
      const double vm = __shfl_up_sync(0xffffffffu, C.v, 1);
      const double vp = __shfl_down_sync(0xffffffffu, C.v, 1);
      double sxe, sxu, sxv;
      cell_slope(hm, C.h, hp, em, ec, ep, um, C.u, up, vm, C.v, vp, sxe, sxu, sxv);
      // x-face left of this lane: left state = previous lane reconstructed right
      const double re = ec + 0.5 * sxe, ru = C.u + 0.5 * sxu, rv = C.v + 0.5 * sxv;
      const double le = __shfl_up_sync(0xffffffffu, re, 1);
      const double lu = __shfl_up_sync(0xffffffffu, ru, 1);
      const double lv = __shfl_up_sync(0xffffffffu, rv, 1);
      const double lb = __shfl_up_sync(0xffffffffu, C.b, 1);
      FaceOut xf;
      face_flux<0, HLLC>(le, lu, lv, lb, ec - 0.5 * sxe, C.u - 0.5 * sxu, C.v - 0.5 * sxv, C.b,
                         xf);
      const double r_fh = __shfl_down_sync(0xffffffffu, xf.fh, 1);
      const double r_fx = __shfl_down_sync(0xffffffffu, xf.fqx, 1);
      const double r_fy = __shfl_down_sync(0xffffffffu, xf.fqy, 1);
      const double r_h2 = __shfl_down_sync(0xffffffffu, xf.hL2, 1);
      const double r_p2 = __shfl_down_sync(0xffffffffu, xf.pL2, 1);
      if (out_lane) {
        const double o_fh = -((r_fh - xf.fh) / dx) - (top.fh - bot.fh) / dy;
        const double o_fhu = -((r_fx - xf.fqx) / dx) - (top.fqx - bot.fqx) / dy -
                             kHalfG * (xf.wbR - r_h2 + r_p2) / dx;
        const double o_fhv = -((r_fy - xf.fqy) / dx) - (top.fqy - bot.fqy) / dy -
                             kHalfG * (bot.wbR - top.hL2 + top.pL2) / dy;
        double a = C.h, u = C.u, v = C.v;
        a = a + dt * o_fh;
        u = u + dt * o_fhu;
        v = v + dt * o_fhv;
        protect(a, u, v);
        sources(a, u, v, phys, dt, n_sq, cosf, sinf, has_cor, g, gi, j, fo);
        FieldSet out;
        if (STAGE == 1) {
          out = S;
        } else {
          out = cur ? U0 : U1;
          a = 0.5 * (old_h + a);
          u = 0.5 * (old_u + u);
          v = 0.5 * (old_v + v);
          protect(a, u, v);
        }
        const double h_pre_sponge = a;
        sponge(a, u, v, bcp, g, gi, j, dt);
        out.h[q] = a;
        out.hu[q] = u;
        out.hv[q] = v;
        part = part + o_fh;
        sponge_d = sponge_d + (a - h_pre_sponge);
        if (STAGE == 2) {
          double sx, sy;
          wave_speed(a, u, v, sx, sy);
          if (sx > wsx) wsx = sx;
          if (sy > wsy) wsy = sy;
        }
      }
      // rotate the row window
      C = D;
      D = E;
      E = Fn;
      sCe = sDe;
      sCu = sDu;
      sCv = sDv;
      bot = top;
    }
  }

  // per-warp partials (fixed order) and the CFL maxima of the new state
  part = warp_sum(part);
  sponge_d = warp_sum(sponge_d);
  const unsigned int nblocks = gridDim.x * gridDim.y;
  const unsigned int nw = nblocks * kMarchWarps;
  const unsigned int wid = (blockIdx.y * gridDim.x + blockIdx.x) * kMarchWarps + warp;
  if (STAGE == 2) {
    wsx = warp_max(wsx);
    wsy = warp_max(wsy);
  }
  if (lane == 0) {
    double* P = partials + (size_t)(STAGE - 1) * 2 * nw;
    P[wid] = part;
    P[nw + wid] = sponge_d;
    if (STAGE == 2) {
      atomic_max_pos(&ctl->msx_next, wsx);
      atomic_max_pos(&ctl->msy_next, wsy);
    }
  }
  if (STAGE != 2) return;
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&ctl->done_blocks, 1u) == nblocks - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_step(g, ctl, phys, partials, nw, dt, cur);
}

}  // namespace rkb

// ---------------------------------------------------------------------------
// Host launch wrappers
// ---------------------------------------------------------------------------

namespace rkb {

const char* tile_name(int tile) {
  switch (tile) {
    case kTile32x8: return "32x8";
    case kTile32x16: return "32x16";
    case kTile64x4: return "64x4";
    case kTile16x16: return "16x16";
    case kTile32x8w: return "32x8+2w";
    case kTile32x12w: return "32x12+2w";
    case kTile16x15: return "16x15";
    case kTile32x7w: return "32x7+1w";
    case kTile16x15t: return "16x15 TMA";
    case kMarch64: return "march28x64";
    default: return "march28x32";
  }
}

void tile_dims(int tile, int& tx, int& ty) {
  switch (tile) {
    case kTile32x8: tx = 32; ty = 8; break;
    case kTile32x16: tx = 32; ty = 16; break;
    case kTile64x4: tx = 64; ty = 4; break;
    case kTile16x16: tx = 16; ty = 16; break;
    case kTile32x8w: tx = 32; ty = 8; break;
    case kTile32x12w: tx = 32; ty = 12; break;
    case kTile16x15: tx = 16; ty = 15; break;
    case kTile32x7w: tx = 32; ty = 7; break;
    case kTile16x15t: tx = 16; ty = 15; break;
    case kMarch64: tx = kMarchCols * kMarchWarps; ty = 64; break;
    default: tx = kMarchCols * kMarchWarps; ty = 32; break;
  }
}

static bool is_march(int tile) { return tile == kMarch64 || tile == kMarch32; }

static dim3 stage_grid(const Grid& g, int tile) {
  int tx, ty;
  tile_dims(tile, tx, ty);
  return dim3((unsigned)((g.nx_phys() + tx - 1) / tx), (unsigned)((g.ny_phys() + ty - 1) / ty));
}

// Blocks of the close's first level (k_close_part).
constexpr unsigned int kCloseBlocks = 148;

size_t partials_doubles(const Grid& g, int tile) {
  dim3 d = stage_grid(g, tile);
  const size_t parts = (size_t)d.x * (size_t)d.y * (is_march(tile) ? kMarchWarps : 1);
  return 4 * parts + 4 * kCloseBlocks;  // + the first level of the close
}

template <int TX, int TY, bool HLLC, int STAGE, int XW = 0>
static cudaError_t launch_stage_t(const StepArgs& a, FluxOut fl, cudaStream_t s, int gk) {
  using SM = StageSmem<TX, TY>;
  // the plain-physics build serves the SSP-RK2 stages
  constexpr bool kRk2 = STAGE == 1 || STAGE == 2;
  auto kern = (kRk2 && a.plain) ? k_stage<TX, TY, HLLC, STAGE, XW, kRk2>
                                : k_stage<TX, TY, HLLC, STAGE, XW, false>;
  const dim3 d = stage_grid(a.g, a.tile);
  kern<<<d.x * d.y, stage_threads(TX, TY, XW), SM::BYTES, s>>>(a.g, a.ctl, a.phys, a.bc, a.U0, a.U1, a.S,
                                                       a.b, a.fo, a.partials, fl, gk);
  return cudaGetLastError();
}

// The TMA-staged kernel: one block per tile.
template <int TX, int TY, bool HLLC, int STAGE>
static cudaError_t launch_stage_tma_t(const StepArgs& a, cudaStream_t s) {
  using SM = StageSmem<TX, TY, true>;
  auto kern = a.plain ? k_stage_tma<TX, TY, HLLC, STAGE, true> : k_stage_tma<TX, TY, HLLC, STAGE, false>;
  const dim3 d = stage_grid(a.g, a.tile);
  const long long limit = a.wait_cycles > 0 ? a.wait_cycles : kWaitCyclesDefault;
  kern<<<d.x * d.y, stage_threads(TX, TY, 0), SM::BYTES, s>>>(
      a.g, a.ctl, a.phys, a.bc, a.U0, a.U1, a.S, a.b, a.fo, a.partials, limit, *a.maps);
  return cudaGetLastError();
}

template <bool HLLC, int STAGE, int ROWS>
static cudaError_t launch_march_t(const StepArgs& a, cudaStream_t s) {
  dim3 grid = stage_grid(a.g, a.tile);
  k_march<HLLC, STAGE, ROWS><<<grid, kMarchWarps * 32, 0, s>>>(a.g, a.ctl, a.phys, a.bc, a.U0,
                                                              a.U1, a.S, a.b, a.fo, a.partials);
  return cudaGetLastError();
}

template <int TX, int TY, bool HLLC>
static cudaError_t configure_tma_t() {
  const int bytes = (int)StageSmem<TX, TY, true>::BYTES;
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_stage_tma<TX, TY, HLLC, 1, false>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_tma<TX, TY, HLLC, 2, false>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_tma<TX, TY, HLLC, 1, true>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_tma<TX, TY, HLLC, 2, true>, attr, bytes);
  return e;
}

template <int TX, int TY, bool HLLC, int XW = 0>
static cudaError_t configure_t() {
  cudaError_t e = cudaSuccess;
  const int bytes = (int)StageSmem<TX, TY>::BYTES;
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 0, XW>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 1, XW>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 2, XW>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 3, XW>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 1, XW, true>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage<TX, TY, HLLC, 2, XW, true>, attr, bytes);
  return e;
}

cudaError_t configure_kernels(int tile, int hllc) {
  const bool h = hllc != 0;
  switch (tile) {
    case kTile32x8: return h ? configure_t<32, 8, true>() : configure_t<32, 8, false>();
    case kTile32x16: return h ? configure_t<32, 16, true>() : configure_t<32, 16, false>();
    case kTile64x4: return h ? configure_t<64, 4, true>() : configure_t<64, 4, false>();
    case kTile16x16: return h ? configure_t<16, 16, true>() : configure_t<16, 16, false>();
    case kTile32x8w: return h ? configure_t<32, 8, true, 2>() : configure_t<32, 8, false, 2>();
    case kTile32x12w: return h ? configure_t<32, 12, true, 2>() : configure_t<32, 12, false, 2>();
    case kTile16x15: return h ? configure_t<16, 15, true>() : configure_t<16, 15, false>();
    case kTile32x7w: return h ? configure_t<32, 7, true, 1>() : configure_t<32, 7, false, 1>();
    case kTile16x15t: {
      // the plain 16x15 kernel serves the other stages and grids without maps
      const cudaError_t e = h ? configure_t<16, 15, true>() : configure_t<16, 15, false>();
      if (e != cudaSuccess) return e;
      return h ? configure_tma_t<16, 15, true>() : configure_tma_t<16, 15, false>();
    }
    // marching kernels use no dynamic shared memory; the generic stages run
    // on 32x16 tiles under them
    default: return h ? configure_t<32, 16, true>() : configure_t<32, 16, false>();
  }
}

// The close of a step whose last stage ran on shared-memory tiles.
// With the boundary budget, k_close_part first reduces the per-tile partials
// to kCloseBlocks per array (stored after them), which k_close then sums.
static cudaError_t launch_close(const StepArgs& a, bool budget, cudaStream_t s) {
  const dim3 d = stage_grid(a.g, a.tile);
  const unsigned int nparts = d.x * d.y;
  if (!budget) {
    k_close<<<1, 1024, 0, s>>>(a.g, a.ctl, a.phys, a.partials, nparts, 0);
    return cudaGetLastError();
  }
  double* first = a.partials + 4 * (size_t)nparts;
  k_close_part<<<kCloseBlocks, 256, 0, s>>>(a.ctl, a.partials, nparts, first);
  k_close<<<1, 1024, 0, s>>>(a.g, a.ctl, a.phys, first, kCloseBlocks, 1);
  return cudaGetLastError();
}

template <int STAGE>
static cudaError_t launch_stage(const StepArgs& a, FluxOut fl, cudaStream_t s, int gk = 0) {
  const bool h = a.hllc != 0;
  switch (a.tile) {
    case kTile32x8:
      return h ? launch_stage_t<32, 8, true, STAGE>(a, fl, s, gk) : launch_stage_t<32, 8, false, STAGE>(a, fl, s, gk);
    case kTile32x16:
      return h ? launch_stage_t<32, 16, true, STAGE>(a, fl, s, gk) : launch_stage_t<32, 16, false, STAGE>(a, fl, s, gk);
    case kTile64x4:
      return h ? launch_stage_t<64, 4, true, STAGE>(a, fl, s, gk) : launch_stage_t<64, 4, false, STAGE>(a, fl, s, gk);
    case kTile16x16:
      return h ? launch_stage_t<16, 16, true, STAGE>(a, fl, s, gk) : launch_stage_t<16, 16, false, STAGE>(a, fl, s, gk);
    case kTile32x8w:
      return h ? launch_stage_t<32, 8, true, STAGE, 2>(a, fl, s, gk) : launch_stage_t<32, 8, false, STAGE, 2>(a, fl, s, gk);
    case kTile32x12w:
      return h ? launch_stage_t<32, 12, true, STAGE, 2>(a, fl, s, gk) : launch_stage_t<32, 12, false, STAGE, 2>(a, fl, s, gk);
    case kTile16x15:
      return h ? launch_stage_t<16, 15, true, STAGE>(a, fl, s, gk) : launch_stage_t<16, 15, false, STAGE>(a, fl, s, gk);
    case kTile32x7w:
      return h ? launch_stage_t<32, 7, true, STAGE, 1>(a, fl, s, gk) : launch_stage_t<32, 7, false, STAGE, 1>(a, fl, s, gk);
    case kTile16x15t:
      if constexpr (STAGE == 1 || STAGE == 2) {
        if (a.maps)
          return h ? launch_stage_tma_t<16, 15, true, STAGE>(a, s) : launch_stage_tma_t<16, 15, false, STAGE>(a, s);
      }
      return h ? launch_stage_t<16, 15, true, STAGE>(a, fl, s, gk) : launch_stage_t<16, 15, false, STAGE>(a, fl, s, gk);
    default:
      break;
  }
  if (STAGE == 0 || STAGE == 3) return cudaErrorInvalidValue;  // tiled kernels only
  constexpr int ST = STAGE == 1 ? 1 : 2;
  if (a.tile == kMarch64)
    return h ? launch_march_t<true, ST, 64>(a, s) : launch_march_t<false, ST, 64>(a, s);
  return h ? launch_march_t<true, ST, 32>(a, s) : launch_march_t<false, ST, 32>(a, s);
}

static bool narrow_grid(const Grid& g) {
  const int wide = g.ng > 2 ? g.ng : 2;
  return g.nx_phys() < wide || g.ny_phys() < wide;
}

// One boundary fill; `first`: this launch opens the step (publishes dt).
static cudaError_t launch_bc_pass(const StepArgs& a, int stage, bool first_pass,
                                  cudaStream_t s) {
  const Grid& g = a.g;
  const int tpb = 128;
  // Opposite edges may run in one launch only when neither reads cells the
  // other writes, i.e. when the interior is at least max(nghost, 2) wide.
  const bool pair_x = g.nx_phys() >= (g.ng > 2 ? g.ng : 2);
  const bool pair_y = g.ny_phys() >= (g.ng > 2 ? g.ng : 2);
  int first = first_pass ? 1 : 0;
  auto go = [&](int e0, int count, int n_tan) {
    dim3 grid((unsigned)((n_tan + tpb - 1) / tpb), (unsigned)count);
    k_bc<<<grid, tpb, 0, s>>>(a, stage, e0, first);
    first = 0;
  };
  if (pair_x) {
    go(0, 2, g.nyt);
  } else {
    go(0, 1, g.nyt);
    go(1, 1, g.nyt);
  }
  if (pair_y) {
    go(2, 2, g.nxt);
  } else {
    go(2, 1, g.nxt);
    go(3, 1, g.nxt);
  }
  return cudaGetLastError();
}

// The fill of a stage; a narrow grid's step opens with the fill before dt.
cudaError_t launch_bc(const StepArgs& a, int stage, cudaStream_t s) {
  const bool opens = stage == 1 || stage == 10;
  if (opens && narrow_grid(a.g)) {
    const cudaError_t e = launch_bc_pass(a, 9, true, s);
    if (e != cudaSuccess) return e;
    return launch_bc_pass(a, stage, false, s);
  }
  return launch_bc_pass(a, stage, opens, s);
}

// Generic Shu-Osher schemes (euler, rk3, rk43): per stage k a boundary fill
// at t + c_k dt and one stage<3> launch; the marching tiles have no generic
// form, so those stages run on 32x16 tiles.
static cudaError_t launch_step_generic(const StepArgs& a, cudaStream_t s) {
  FluxOut none{};
  StepArgs ga = a;
  if (is_march(ga.tile)) ga.tile = kTile32x16;
  for (int k = 0; k < a.n_stages; ++k) {
    cudaError_t e = launch_bc(ga, 10 + k, s);
    if (e != cudaSuccess) return e;
    e = launch_stage<3>(ga, none, s, k);
    if (e != cudaSuccess) return e;
  }
  return launch_close(ga, false, s);  // the generic schemes keep no boundary budget
}

cudaError_t launch_step(const StepArgs& a, cudaStream_t s) {
  if (a.scheme != 2) return launch_step_generic(a, s);
  FluxOut none{};
  cudaError_t e = launch_bc(a, 1, s);
  if (e != cudaSuccess) return e;
  e = launch_stage<1>(a, none, s);
  if (e != cudaSuccess) return e;
  e = launch_bc(a, 2, s);
  if (e != cudaSuccess) return e;
  e = launch_stage<2>(a, none, s);
  if (e != cudaSuccess || is_march(a.tile)) return e;  // marching kernels close the step themselves
  return launch_close(a, true, s);
}

// Stage 2 includes the close of the step.
cudaError_t launch_stage_only(const StepArgs& a, int stage, cudaStream_t s) {
  FluxOut none{};
  if (stage == 1) return launch_stage<1>(a, none, s);
  const cudaError_t e = launch_stage<2>(a, none, s);
  if (e != cudaSuccess || is_march(a.tile)) return e;
  return launch_close(a, true, s);
}

// ---- TMA maps of the state buffers ----

// The driver's tensor-map encoder through the runtime (no link against the
// driver library); *status: 0, or 100 + the runtime error, or 200 + the
// entry-point query result.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder(int* status) {
  static int st = 0;
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    const cudaError_t e =
        cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q);
    if (e != cudaSuccess) {
      st = 100 + (int)e;
      p = nullptr;
    } else if (q != cudaDriverEntryPointSuccess) {
      st = 200 + (int)q;
      p = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  *status = st;
  return fn;
}

// One FP64 field of g's layout (nxt x nyt elements, rows `pitch` apart),
// boxes of bw x bh elements, zeros outside; 0 or 1000 + the driver's result.
static int encode_field(PFN_cuTensorMapEncodeTiled_v12000 enc, CUtensorMap* m,
                        const double* base, const Grid& g, int bw, int bh) {
  if (((uintptr_t)base & 15) != 0) return 2;
  cuuint64_t dims[2] = {(cuuint64_t)g.nxt, (cuuint64_t)g.nyt};
  cuuint64_t strides[1] = {(cuuint64_t)g.pitch * sizeof(double)};
  cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  cuuint32_t estride[2] = {1, 1};
  const CUresult r =
      enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(base), dims, strides, box,
          estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : 1000 + (int)r;
}

int encode_tile_maps(const StepArgs& a, TileMaps* m) {
  const Grid& g = a.g;
  // rows must start on 16-byte boundaries (the boxes' x starts are even)
  if ((g.pitch * sizeof(double)) % 16 != 0 || g.nx_phys() < 1 || g.ny_phys() < 1) return 1;
  int st = 0;
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder(&st);
  if (!enc) return st != 0 ? st : 3;
  using SM = StageSmem<16, 15, true>;  // kTile16x15t
  const FieldSet sets[3] = {a.U0, a.U1, a.S};
  for (int k = 0; k < 3; ++k) {
    const double* f[3] = {sets[k].h, sets[k].hu, sets[k].hv};
    for (int c = 0; c < 3; ++c) {
      if ((st = encode_field(enc, &m->tile[k][c], f[c], g, SM::TW, SM::TH)) != 0) return st;
      if (k < 2 && (st = encode_field(enc, &m->cells[k][c], f[c], g, SM::CW, 15)) != 0) return st;
    }
  }
  return encode_field(enc, &m->bed, a.b, g, SM::TW, SM::TH);
}

int launches_per_step(const StepArgs& a) {
  const Grid& g = a.g;
  const int need = g.ng > 2 ? g.ng : 2;
  const int bc = (g.nx_phys() >= need ? 1 : 2) + (g.ny_phys() >= need ? 1 : 2);
  const int pre = narrow_grid(g) ? bc : 0;
  if (a.scheme != 2) return a.n_stages * (bc + 1) + pre + 1;  // + the close
  return 2 * bc + 2 + pre + (is_march(a.tile) ? 0 : 2);  // + the close's two levels
}

cudaError_t launch_max_speed(const StepArgs& a, cudaStream_t s) {
  const long long n = (long long)a.g.nx_phys() * a.g.ny_phys();
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  k_max_speed<<<(unsigned)blocks, 256, 0, s>>>(a.g, a.ctl, a.U0, a.U1);
  return cudaGetLastError();
}

// ---- batches: every simulation of a batch in one launch per phase ----

int batch_stage_blocks(const Grid& g, int tile) {
  const dim3 d = stage_grid(g, tile);
  return (int)(d.x * d.y);
}

template <int TX, int TY, bool HLLC, int XW = 0>
static cudaError_t configure_batch_t() {
  const int bytes = (int)StageSmem<TX, TY>::BYTES;
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_stage_batch<TX, TY, HLLC, 1, XW>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_batch<TX, TY, HLLC, 2, XW>, attr, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_stage_batch<TX, TY, HLLC, 1, XW, true>, attr, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_stage_batch<TX, TY, HLLC, 2, XW, true>, attr, bytes);
  return e;
}

template <int TX, int TY, bool HLLC>
static cudaError_t configure_batch_tma_t() {
  const int bytes = (int)StageSmem<TX, TY, true>::BYTES;
  const auto attr = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_stage_batch_tma<TX, TY, HLLC, 1>, attr, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stage_batch_tma<TX, TY, HLLC, 2>, attr, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_stage_batch_tma<TX, TY, HLLC, 1, true>, attr, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_stage_batch_tma<TX, TY, HLLC, 2, true>, attr, bytes);
  return e;
}

cudaError_t configure_batch(int tile, int hllc) {
  const bool h = hllc != 0;
  switch (tile) {
    case kTile32x8: return h ? configure_batch_t<32, 8, true>() : configure_batch_t<32, 8, false>();
    case kTile32x16: return h ? configure_batch_t<32, 16, true>() : configure_batch_t<32, 16, false>();
    case kTile64x4: return h ? configure_batch_t<64, 4, true>() : configure_batch_t<64, 4, false>();
    case kTile16x16: return h ? configure_batch_t<16, 16, true>() : configure_batch_t<16, 16, false>();
    case kTile32x8w: return h ? configure_batch_t<32, 8, true, 2>() : configure_batch_t<32, 8, false, 2>();
    case kTile32x12w: return h ? configure_batch_t<32, 12, true, 2>() : configure_batch_t<32, 12, false, 2>();
    case kTile16x15: return h ? configure_batch_t<16, 15, true>() : configure_batch_t<16, 15, false>();
    case kTile32x7w: return h ? configure_batch_t<32, 7, true, 1>() : configure_batch_t<32, 7, false, 1>();
    case kTile16x15t: {
      // the plain 16x15 kernel serves batches whose maps are not all encoded
      const cudaError_t e =
          h ? configure_batch_t<16, 15, true>() : configure_batch_t<16, 15, false>();
      if (e != cudaSuccess) return e;
      return h ? configure_batch_tma_t<16, 15, true>() : configure_batch_tma_t<16, 15, false>();
    }
    default: return cudaErrorInvalidValue;  // batches use the shared-memory tiles
  }
}

template <int TX, int TY, bool HLLC, int STAGE, int XW = 0>
static cudaError_t launch_stage_batch_t(const BatchLaunch& bl, cudaStream_t s) {
  auto kern = bl.plain ? k_stage_batch<TX, TY, HLLC, STAGE, XW, true>
                       : k_stage_batch<TX, TY, HLLC, STAGE, XW, false>;
  kern<<<(unsigned)bl.blocks, stage_threads(TX, TY, XW), StageSmem<TX, TY>::BYTES, s>>>(bl.args,
                                                                                      bl.map);
  return cudaGetLastError();
}

template <int TX, int TY, bool HLLC, int STAGE>
static cudaError_t launch_stage_batch_tma_t(const BatchLaunch& bl, cudaStream_t s) {
  auto kern = bl.plain ? k_stage_batch_tma<TX, TY, HLLC, STAGE, true>
                       : k_stage_batch_tma<TX, TY, HLLC, STAGE, false>;
  kern<<<(unsigned)bl.blocks, stage_threads(TX, TY, 0), StageSmem<TX, TY, true>::BYTES, s>>>(
      bl.args, bl.map, bl.maps);
  return cudaGetLastError();
}

template <int STAGE>
static cudaError_t launch_stage_batch(const BatchLaunch& bl, cudaStream_t s) {
  const bool h = bl.hllc != 0;
  switch (bl.tile) {
    case kTile32x8:
      return h ? launch_stage_batch_t<32, 8, true, STAGE>(bl, s) : launch_stage_batch_t<32, 8, false, STAGE>(bl, s);
    case kTile32x16:
      return h ? launch_stage_batch_t<32, 16, true, STAGE>(bl, s) : launch_stage_batch_t<32, 16, false, STAGE>(bl, s);
    case kTile64x4:
      return h ? launch_stage_batch_t<64, 4, true, STAGE>(bl, s) : launch_stage_batch_t<64, 4, false, STAGE>(bl, s);
    case kTile16x16:
      return h ? launch_stage_batch_t<16, 16, true, STAGE>(bl, s) : launch_stage_batch_t<16, 16, false, STAGE>(bl, s);
    case kTile32x8w:
      return h ? launch_stage_batch_t<32, 8, true, STAGE, 2>(bl, s) : launch_stage_batch_t<32, 8, false, STAGE, 2>(bl, s);
    case kTile32x12w:
      return h ? launch_stage_batch_t<32, 12, true, STAGE, 2>(bl, s) : launch_stage_batch_t<32, 12, false, STAGE, 2>(bl, s);
    case kTile16x15:
      return h ? launch_stage_batch_t<16, 15, true, STAGE>(bl, s) : launch_stage_batch_t<16, 15, false, STAGE>(bl, s);
    case kTile32x7w:
      return h ? launch_stage_batch_t<32, 7, true, STAGE, 1>(bl, s) : launch_stage_batch_t<32, 7, false, STAGE, 1>(bl, s);
    case kTile16x15t:
      if (bl.maps)
        return h ? launch_stage_batch_tma_t<16, 15, true, STAGE>(bl, s) : launch_stage_batch_tma_t<16, 15, false, STAGE>(bl, s);
      return h ? launch_stage_batch_t<16, 15, true, STAGE>(bl, s) : launch_stage_batch_t<16, 15, false, STAGE>(bl, s);
    default:
      return cudaErrorInvalidValue;
  }
}

// W/E edges of every simulation, then S/N (every simulation of a batch is at
// least max(nghost, 2) cells wide, so opposite edges never overlap).
cudaError_t launch_bc_batch(const BatchLaunch& bl, int stage, cudaStream_t s) {
  const int tpb = 128;
  const dim3 gx((unsigned)((bl.max_nyt + tpb - 1) / tpb), 2, (unsigned)bl.n);
  k_bc_batch<<<gx, tpb, 0, s>>>(bl.args, stage, 0, stage == 1 ? 1 : 0);
  const dim3 gy((unsigned)((bl.max_nxt + tpb - 1) / tpb), 2, (unsigned)bl.n);
  k_bc_batch<<<gy, tpb, 0, s>>>(bl.args, stage, 2, 0);
  return cudaGetLastError();
}

static cudaError_t launch_close_batch(const BatchLaunch& bl, cudaStream_t s) {
  int tx, ty;
  tile_dims(bl.tile, tx, ty);
  k_close_batch<<<(unsigned)bl.n, 1024, 0, s>>>(bl.args, tx, ty);
  return cudaGetLastError();
}

// Stage 2 includes the close of every member's step.
cudaError_t launch_stage_batch_only(const BatchLaunch& bl, int stage, cudaStream_t s) {
  if (stage == 1) return launch_stage_batch<1>(bl, s);
  const cudaError_t e = launch_stage_batch<2>(bl, s);
  return e == cudaSuccess ? launch_close_batch(bl, s) : e;
}

cudaError_t launch_step_batch(const BatchLaunch& bl, cudaStream_t s) {
  cudaError_t e = launch_bc_batch(bl, 1, s);
  if (e == cudaSuccess) e = launch_stage_batch<1>(bl, s);
  if (e == cudaSuccess) e = launch_bc_batch(bl, 2, s);
  if (e == cudaSuccess) e = launch_stage_batch<2>(bl, s);
  if (e == cudaSuccess) e = launch_close_batch(bl, s);
  return e;
}

cudaError_t launch_flux(const Grid& g, int hllc, FieldSet in, const double* b, FluxOut out,
                        int tile, cudaStream_t s) {
  StepArgs a{};
  a.g = g;
  a.U0 = in;
  a.U1 = in;
  a.S = in;
  a.b = const_cast<double*>(b);
  a.tile = tile;
  a.hllc = hllc;
  cudaError_t e = configure_kernels(tile, hllc);
  if (e != cudaSuccess) return e;
  return launch_stage<0>(a, out, s);
}

}  // namespace rkb
