// Adjoint of the structured step for gauge-misfit gradients, over a batch of
// equally sized simulations (members), templated on the real type T.
//
// J_m(b, n) = sum over steps k = 1..N and gauge cells g of member m of
// (eta_g^k - obs_g^k)^2 for the SSP-RK2 step of rki_solver.F90:659-815 with
// wall boundaries, HLL or HLLC fluxes and Manning friction with a per-cell n
// field, on a fixed dt sequence per member (recorded once from CFL steps and
// replayed, so J is a piecewise-smooth function of b and n).  Gradients
// dJ_m/db_m and dJ_m/dn_m come from hand-written reverse kernels:
//
//   forward, per stage:  slopes -> faces -> cells          (taped: slopes, face outputs)
//   reverse, per stage:  cells -> faces -> reconstruction -> slope gather -> walls
//
// Every reverse kernel gathers (each output element is written by one thread),
// so there are no atomics and the gradient is deterministic.  States are
// checkpointed every K ~ sqrt(N) steps and recomputed segment by segment;
// given a state budget (set_state_budget), a gradient run instead keeps every
// state U^0..U^N in device memory when they fit (12.7 GB for 1024^2 FP64 over
// 500 steps) and the reverse sweep reads U^k directly.  Both give the same
// bits.
// Each launch covers every member (blockIdx.z = member; member m's arrays start
// m * ms elements after member 0's).
//
// T = double (rkb_adjoint.cu, --fmad=false): the forward kernels evaluate the
// reference's expressions in its order, like rkb_step_f64.cu, so with a
// uniform n field equal to the scalar manning_n the trajectory is
// bit-identical to the production step.  T = float (rkb_adjoint32.cu): the
// same scheme in FP32 arithmetic; the misfit and the domain mass are summed
// in FP64.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "rkb_adjoint.cuh"
#include "rkb_async.cuh"
#include "rkb_kernels.h"

namespace rkb {

// Precision-independent interface of one adjoint batch (the C ABI's handle).
class AdjointBase {
 public:
  virtual ~AdjointBase() {}
  virtual int set_obs(const double* obs) = 0;   // [step][member][gauge]
  virtual int set_dt(const double* dts) = 0;    // [member][step]
  virtual void get_dt(double* dts) const = 0;
  virtual int forward(const double* b, const double* n, double n_scalar, bool record, double* J,
                      double* eta_out) = 0;
  virtual int gradient(const double* b, const double* n, double n_scalar, double* J,
                       double* gb_out, double* gn_out) = 0;
  // 1 once a gradient run kept every state, else K ~ sqrt(N).
  virtual int checkpoint_interval() const = 0;
  // Bytes the gradient may allocate to keep every state: < 0 half the free
  // device memory at the next gradient run, 0 never (sqrt(N) checkpoints
  // and recomputation only, the default).  Frees a kept-state allocation
  // above it.
  virtual void set_state_budget(long long bytes) = 0;
  virtual double last_ms() = 0;
  virtual int members() const = 0;
  virtual int precision() const = 0;
  virtual void mass(double* out) const = 0;     // [2][member]: initial, after the last forward
  // Frozen slopes: gradients of the step with its limited slopes held at
  // their current values (an approximation that stays bounded over long
  // windows where the exact derivative of the limiter does not).
  virtual void set_frozen_slopes(bool on) = 0;
};

// Factories (one per precision, each in its own translation unit).
AdjointBase* make_adjoint64(int nm, int nx, int ny, int ng, double dx, double dy, double cfl,
                            int hllc, int nsteps, const double* h0, const double* hu0,
                            const double* hv0, const int* gi, const int* gj, int ngauge,
                            std::string& err, int& rc);
AdjointBase* make_adjoint32(int nm, int nx, int ny, int ng, double dx, double dy, double cfl,
                            int hllc, int nsteps, const double* h0, const double* hu0,
                            const double* hv0, const int* gi, const int* gj, int ngauge,
                            std::string& err, int& rc);

namespace adj {

constexpr int kBX = 32, kBY = 8;

template <typename T>
struct Fields {
  T* h;
  T* hu;
  T* hv;
};

template <typename T>
struct Tape {
  T* s[6];   // x-slopes (eta, hu, hv), y-slopes (eta, hu, hv)
  T* fx[6];  // x-face i-1/2 at (i, j): fh, fqx, fqy, wbR, hL2, pL2
  T* fy[6];  // y-face j-1/2 at (i, j)
  T* od[3];  // flux divergence of the cell (stage 1, written by k_cells)
};

template <typename T>
struct Rev {
  T* go[3];   // adjoint of the cell's flux divergence (o_fh, o_fhu, o_fhv)
  T* ga[3];   // direct adjoint of the stage input at interior cells (a = h + dt o)
  T* gfx[8];  // x-face input adjoints (eL, qxL, qyL, bL, eR, qxR, qyR, bR)
  T* gfy[8];
};

__device__ __forceinline__ bool in_box(int i, int j, int i0, int i1, int j0, int j1) {
  return i >= i0 && i <= i1 && j >= j0 && j <= j1;
}

__device__ __forceinline__ size_t member_base(size_t ms) { return (size_t)blockIdx.z * ms; }

// ---- forward ------------------------------------------------------------------

// Wall ghosts (rki_boundary.F90:220-291), W/E (pass 0) or S/N (pass 1).
template <typename T>
__global__ void k_walls(Grid g, size_t ms, Fields<T> V, T* __restrict__ b, int pass) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int side = blockIdx.y;  // 0: west / south, 1: east / north
  const int n_tan = pass == 0 ? g.nyt : g.nxt;
  if (t >= n_tan) return;
  const size_t zb = member_base(ms);
  for (int k = 1; k <= g.ng; ++k) {
    int ig, jg, im, jm;
    if (pass == 0) {
      jg = jm = t;
      ig = side == 0 ? g.ng - k : g.nxt - g.ng + k - 1;
      im = side == 0 ? g.ng + k - 1 : g.nxt - g.ng - k;
    } else {
      ig = im = t;
      jg = side == 0 ? g.ng - k : g.nyt - g.ng + k - 1;
      jm = side == 0 ? g.ng + k - 1 : g.nyt - g.ng - k;
    }
    const size_t q = g.at(ig, jg) + zb, m = g.at(im, jm) + zb;
    const T bm = b[m];
    b[q] = bm;
    V.h[q] = pos(V.h[m] + bm - bm);
    if (pass == 0) { V.hu[q] = -V.hu[m]; V.hv[q] = V.hv[m]; }
    else { V.hv[q] = -V.hv[m]; V.hu[q] = V.hu[m]; }
  }
}

template <typename T>
__global__ void k_slopes(Grid g, size_t ms, Fields<T> V, const T* __restrict__ b, Tape<T> Tp) {
  const int i = g.ng - 1 + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng - 1 + blockIdx.y * kBY + threadIdx.x / kBX;
  const int ie = g.nxt - g.ng, je = g.nyt - g.ng;
  if (i > ie || j > je) return;
  const size_t c = g.at(i, j) + member_base(ms);
  auto eta = [&](size_t q) { return V.h[q] + b[q]; };
  if (j >= g.ng && j < je) {  // x-slope
    const size_t m = c - 1, p = c + 1;
    cell_slope(V.h[m], V.h[c], V.h[p], eta(m), eta(c), eta(p), V.hu[m], V.hu[c], V.hu[p], V.hv[m],
               V.hv[c], V.hv[p], Tp.s[0][c], Tp.s[1][c], Tp.s[2][c]);
  }
  if (i >= g.ng && i < ie) {  // y-slope
    const size_t m = c - g.pitch, p = c + g.pitch;
    cell_slope(V.h[m], V.h[c], V.h[p], eta(m), eta(c), eta(p), V.hu[m], V.hu[c], V.hu[p], V.hv[m],
               V.hv[c], V.hv[p], Tp.s[3][c], Tp.s[4][c], Tp.s[5][c]);
  }
}

// Reconstructed left / right states of x-face (i-1/2, j) or y-face (i, j-1/2).
template <typename T>
struct FaceIn {
  T eL, qxL, qyL, bL, eR, qxR, qyR, bR;
};

template <typename T>
__device__ __forceinline__ FaceIn<T> face_in(const Fields<T>& V, const T* __restrict__ b,
                                             const Tape<T>& Tp, size_t qL, size_t qR, int dir) {
  const int o = dir == 0 ? 0 : 3;
  FaceIn<T> f;
  f.eL = (V.h[qL] + b[qL]) + T(0.5) * Tp.s[o][qL];
  f.qxL = V.hu[qL] + T(0.5) * Tp.s[o + 1][qL];
  f.qyL = V.hv[qL] + T(0.5) * Tp.s[o + 2][qL];
  f.bL = b[qL];
  f.eR = (V.h[qR] + b[qR]) - T(0.5) * Tp.s[o][qR];
  f.qxR = V.hu[qR] - T(0.5) * Tp.s[o + 1][qR];
  f.qyR = V.hv[qR] - T(0.5) * Tp.s[o + 2][qR];
  f.bR = b[qR];
  return f;
}

template <typename T, bool HLLC>
__global__ void k_faces(Grid g, size_t ms, Fields<T> V, const T* __restrict__ b, Tape<T> Tp) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  const int ie = g.nxt - g.ng, je = g.nyt - g.ng;
  if (i > ie || j > je) return;
  const size_t c = g.at(i, j) + member_base(ms);
  if (j < je) {  // x-face between (i-1, j) and (i, j)
    const FaceIn<T> f = face_in(V, b, Tp, c - 1, c, 0);
    FaceOutT<T> o;
    face_flux<0, HLLC>(f.eL, f.qxL, f.qyL, f.bL, f.eR, f.qxR, f.qyR, f.bR, o);
    Tp.fx[0][c] = o.fh; Tp.fx[1][c] = o.fqx; Tp.fx[2][c] = o.fqy;
    Tp.fx[3][c] = o.wbR; Tp.fx[4][c] = o.hL2; Tp.fx[5][c] = o.pL2;
  }
  if (i < ie) {  // y-face between (i, j-1) and (i, j)
    const FaceIn<T> f = face_in(V, b, Tp, c - g.pitch, c, 1);
    FaceOutT<T> o;
    face_flux<1, HLLC>(f.eL, f.qxL, f.qyL, f.bL, f.eR, f.qxR, f.qyR, f.bR, o);
    Tp.fy[0][c] = o.fh; Tp.fy[1][c] = o.fqx; Tp.fy[2][c] = o.fqy;
    Tp.fy[3][c] = o.wbR; Tp.fy[4][c] = o.hL2; Tp.fy[5][c] = o.pL2;
  }
}

// Flux divergence of interior cell c in k_stage's expression order.
template <typename T>
__device__ __forceinline__ void divergence(const Grid& g, const Tape<T>& Tp, size_t c, T& ofh,
                                           T& ofhu, T& ofhv) {
  const size_t r = c + 1, t = c + g.pitch;
  const T dx = T(g.dx), dy = T(g.dy);
  ofh = -((Tp.fx[0][r] - Tp.fx[0][c]) / dx) - (Tp.fy[0][t] - Tp.fy[0][c]) / dy;
  ofhu = -((Tp.fx[1][r] - Tp.fx[1][c]) / dx) - (Tp.fy[1][t] - Tp.fy[1][c]) / dy -
         T(kHalfG) * (Tp.fx[3][c] - Tp.fx[4][r] + Tp.fx[5][r]) / dx;
  ofhv = -((Tp.fx[2][r] - Tp.fx[2][c]) / dx) - (Tp.fy[2][t] - Tp.fy[2][c]) / dy -
         T(kHalfG) * (Tp.fy[3][c] - Tp.fy[4][t] + Tp.fy[5][t]) / dy;
}

// Cell update of stage 1 (out = protect(sources(V + dt L))) or stage 2 (RK2
// average with the base state and the second clamp); dts[m] = member m's dt.
template <typename T>
__global__ void k_cells(Grid g, size_t ms, Fields<T> V, Fields<T> base, const T* __restrict__ nf,
                        Tape<T> Tp, const double* __restrict__ dts, int stage, Fields<T> out) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  if (i >= g.nxt - g.ng || j >= g.nyt - g.ng) return;
  const size_t c = g.at(i, j) + member_base(ms);
  const T dt = T(dts[blockIdx.z]);
  T ofh, ofhu, ofhv;
  divergence(g, Tp, c, ofh, ofhu, ofhv);
  Tp.od[0][c] = ofh;  // for k_cells_adj<T, 1>
  Tp.od[1][c] = ofhu;
  Tp.od[2][c] = ofhv;
  T a = V.h[c], u = V.hu[c], v = V.hv[c];
  a = a + dt * ofh;
  u = u + dt * ofhu;
  v = v + dt * ofhv;
  protect(a, u, v);
  friction(a, u, v, nf[c], dt);
  if (stage == 2) {
    a = T(0.5) * (base.h[c] + a);
    u = T(0.5) * (base.hu[c] + u);
    v = T(0.5) * (base.hv[c] + v);
    protect(a, u, v);
  }
  out.h[c] = a;
  out.hu[c] = u;
  out.hv[c] = v;
}

// One forward stage in one launch, for the steps whose slopes and face values
// the reverse sweep does not read (the checkpointing pass and the segment
// recomputes): a kBX x kBY tile of cells with a 2-cell halo in shared memory,
// then the limited slopes, the faces (each once) and the cell update of
// k_slopes / k_faces / k_cells, with the same device functions in the same
// expression order, so the trajectory is the taped kernels' bit for bit.
// Tile of the fused kernel: 16 x 15 cells on 256 threads, so that its 255
// x-faces and 256 y-faces take exactly two rounds; the limited slopes are
// computed where a face needs them (each slope twice, by the same
// expressions, so the same bits), which spares slope arrays and a barrier.
constexpr int kFX = 16, kFY = 15, kFThreads = 256;

template <typename T>
struct FusedSmem {
  static constexpr int TX = kFX, TY = kFY, TW = TX + 4, NT = TW * (TY + 4);
  static constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
  static constexpr size_t BYTES = sizeof(T) * (4 * (size_t)NT + 6 * NFX + 6 * NFY);
};

// Five blocks per SM (48 registers a thread in FP64, 8 bytes spilled):
// measured 4% faster than four blocks of 56 registers.
template <typename T, bool HLLC>
__global__ void __launch_bounds__(kFThreads, 5)
    k_stage_fused(Grid g, size_t ms, Fields<T> V, Fields<T> base, const T* __restrict__ b,
                  const T* __restrict__ nf, const double* __restrict__ dts, int stage,
                  Fields<T> out) {
  using SM = FusedSmem<T>;
  constexpr int TX = SM::TX, TY = SM::TY, TW = SM::TW, NTH = kFThreads;
  extern __shared__ __align__(16) unsigned char fused_smem[];
  T* th = reinterpret_cast<T*>(fused_smem);
  T* tu = th + SM::NT;
  T* tv = tu + SM::NT;
  T* tb = tv + SM::NT;
  T* fx = tb + SM::NT;       // 6 x NFX: x-face (c-1 | c) outputs, c = 0 .. TX
  T* fy = fx + 6 * SM::NFX;  // 6 x NFY: y-face (r-1 | r) outputs, r = 0 .. TY
  const int tid = threadIdx.x;
  const size_t zb = member_base(ms);
  const int gx0 = g.ng + (int)blockIdx.x * TX, gy0 = g.ng + (int)blockIdx.y * TY;

  for (int k = tid; k < SM::NT; k += NTH) {
    const int gi = gx0 - 2 + k % TW, gj = gy0 - 2 + k / TW;
    T vh = T(0), vu = T(0), vv = T(0), vb = T(0);
    if (gi < g.nxt && gj < g.nyt) {
      const size_t q = g.at(gi, gj) + zb;
      vh = V.h[q];
      vu = V.hu[q];
      vv = V.hv[q];
      vb = b[q];
    }
    th[k] = vh;
    tu[k] = vu;
    tv[k] = vv;
    tb[k] = vb;
  }
  __syncthreads();

  auto eta = [&](int q) { return th[q] + tb[q]; };
  // limited slope (eta, hu, hv) of tile cell q between q - d and q + d
  auto slope_at = [&](int q, int d, T& se, T& su, T& sv) {
    cell_slope(th[q - d], th[q], th[q + d], eta(q - d), eta(q), eta(q + d), tu[q - d], tu[q],
               tu[q + d], tv[q - d], tv[q], tv[q + d], se, su, sv);
  };
  // thread t takes x-face t, then y-face t
  static_assert(NTH == 256 && SM::NFX == 255 && SM::NFY == 256, "face layout");
  auto face = [&](int k) {
    FaceOutT<T> o;
    if (k < SM::NFX) {
      const int c = k % (TX + 1), r = k / (TX + 1);
      const int qL = (r + 2) * TW + (c + 1), qR = qL + 1;
      T sLe, sLu, sLv, sRe, sRu, sRv;
      slope_at(qL, 1, sLe, sLu, sLv);
      slope_at(qR, 1, sRe, sRu, sRv);
      face_flux<0, HLLC>(eta(qL) + T(0.5) * sLe, tu[qL] + T(0.5) * sLu, tv[qL] + T(0.5) * sLv,
                         tb[qL], eta(qR) - T(0.5) * sRe, tu[qR] - T(0.5) * sRu,
                         tv[qR] - T(0.5) * sRv, tb[qR], o);
      T* f = fx + k;
      f[0] = o.fh;
      f[SM::NFX] = o.fqx;
      f[2 * SM::NFX] = o.fqy;
      f[3 * SM::NFX] = o.wbR;
      f[4 * SM::NFX] = o.hL2;
      f[5 * SM::NFX] = o.pL2;
    } else {
      const int kk = k - SM::NFX;
      const int c = kk % TX, r = kk / TX;
      const int qB = (r + 1) * TW + (c + 2), qT = qB + TW;
      T sBe, sBu, sBv, sTe, sTu, sTv;
      slope_at(qB, TW, sBe, sBu, sBv);
      slope_at(qT, TW, sTe, sTu, sTv);
      face_flux<1, HLLC>(eta(qB) + T(0.5) * sBe, tu[qB] + T(0.5) * sBu, tv[qB] + T(0.5) * sBv,
                         tb[qB], eta(qT) - T(0.5) * sTe, tu[qT] - T(0.5) * sTu,
                         tv[qT] - T(0.5) * sTv, tb[qT], o);
      T* f = fy + kk;
      f[0] = o.fh;
      f[SM::NFY] = o.fqx;
      f[2 * SM::NFY] = o.fqy;
      f[3 * SM::NFY] = o.wbR;
      f[4 * SM::NFY] = o.hL2;
      f[5 * SM::NFY] = o.pL2;
    }
  };
  if (tid < SM::NFX) face(tid);
  face(SM::NFX + tid);
  // The cells of warp w read the faces of warps w and w+1 only (warp 7 its
  // own): warp w+1 arrives on named barrier w+1 and warp w waits on it.
  // Every warp gets here (no exit above).
  {
    const int w = tid >> 5;
    __syncwarp();
    if (w > 0) named_arrive(w, 64);
    if (w < NTH / 32 - 1)
      named_sync(w + 1, 64);
    else
      __syncwarp();
  }

  if (tid >= TX * TY) return;  // the 16 threads beyond the tile's cells only took faces
  const int cx = tid % TX, cy = tid / TX;
  const int i = gx0 + cx, j = gy0 + cy;
  if (i >= g.nxt - g.ng || j >= g.nyt - g.ng) return;
  // divergence() on the tile's faces
  const int l = cy * (TX + 1) + cx, r = l + 1, bo = cy * TX + cx, to = bo + TX;
  const T dx = T(g.dx), dy = T(g.dy);
  const T ofh = -((fx[r] - fx[l]) / dx) - (fy[to] - fy[bo]) / dy;
  const T ofhu = -((fx[SM::NFX + r] - fx[SM::NFX + l]) / dx) -
                 (fy[SM::NFY + to] - fy[SM::NFY + bo]) / dy -
                 T(kHalfG) * (fx[3 * SM::NFX + l] - fx[4 * SM::NFX + r] + fx[5 * SM::NFX + r]) / dx;
  const T ofhv = -((fx[2 * SM::NFX + r] - fx[2 * SM::NFX + l]) / dx) -
                 (fy[2 * SM::NFY + to] - fy[2 * SM::NFY + bo]) / dy -
                 T(kHalfG) * (fy[3 * SM::NFY + bo] - fy[4 * SM::NFY + to] + fy[5 * SM::NFY + to]) / dy;
  // k_cells
  const size_t c = g.at(i, j) + zb;
  const T dt = T(dts[blockIdx.z]);
  const int qc = (cy + 2) * TW + (cx + 2);
  T a = th[qc], u = tu[qc], v = tv[qc];
  a = a + dt * ofh;
  u = u + dt * ofhu;
  v = v + dt * ofhv;
  protect(a, u, v);
  friction(a, u, v, nf[c], dt);
  if (stage == 2) {
    // the base is read only at the cell this thread writes: out may alias it
    a = T(0.5) * (base.h[c] + a);
    u = T(0.5) * (base.hu[c] + u);
    v = T(0.5) * (base.hv[c] + v);
    protect(a, u, v);
  }
  out.h[c] = a;
  out.hu[c] = u;
  out.hv[c] = v;
}

// CFL maxima of a state (same wave speed and reduction as the step), per
// member: mx[2 m], mx[2 m + 1] (FP64 bit patterns of non-negative values).
template <typename T>
__global__ void k_speeds(Grid g, size_t ms, Fields<T> V, unsigned long long* mx) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  T sx = T(0), sy = T(0);
  if (i < g.nxt - g.ng && j < g.nyt - g.ng) {
    const size_t c = g.at(i, j) + member_base(ms);
    wave_speed(V.h[c], V.hu[c], V.hv[c], sx, sy);
  }
  for (int o = 16; o > 0; o >>= 1) {
    sx = dmax(sx, (T)__shfl_xor_sync(0xffffffffu, sx, o));
    sy = dmax(sy, (T)__shfl_xor_sync(0xffffffffu, sy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&mx[2 * blockIdx.z], (double)sx);
    atomic_max_pos(&mx[2 * blockIdx.z + 1], (double)sy);
  }
}

// Gauge residuals eta - obs of one step; gq holds each gauge's cell index
// with its member's offset, r and obs are [member][gauge] for this step.
template <typename T>
__global__ void k_gauges(Fields<T> V, const T* __restrict__ b, const long long* __restrict__ gq,
                         const double* __restrict__ obs, int n, double* r) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t q = (size_t)gq[k];
  r[k] = (double)(V.h[q] + b[q]) - obs[k];
}

// FP64 sums of the interior depth, one per member (mass[m] += ...).
template <typename T>
__global__ void k_mass(Grid g, size_t ms, const T* __restrict__ h, double* mass) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  double s = 0.0;
  if (i < g.nxt - g.ng && j < g.nyt - g.ng) s = (double)h[g.at(i, j) + member_base(ms)];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&mass[blockIdx.z], s);
}

// ---- reverse ------------------------------------------------------------------

// Cells: output adjoint gout -> divergence adjoint go, direct input adjoint
// ga (a = h + dt o), base adjoint (stage 2), n adjoint.  STAGE is a template
// argument so that stage 1, which needs no post-friction state (no RK2
// average), does not recompute the forward friction.
template <typename T, int STAGE>
__global__ void __launch_bounds__(kBX * kBY, 4)
    k_cells_adj(Grid g, size_t ms, Fields<T> V, Fields<T> base,
                            const T* __restrict__ nf, Tape<T> Tp, const double* __restrict__ dts,
                            Fields<T> gout, Rev<T> R, Fields<T> gbase,
                            T* __restrict__ gn) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  if (i >= g.nxt - g.ng || j >= g.nyt - g.ng) return;
  const size_t c = g.at(i, j) + member_base(ms);
  const T dt = T(dts[blockIdx.z]);
  T ofh, ofhu, ofhv;
  if (STAGE == 1) {  // taped by k_cells, the same bits
    ofh = Tp.od[0][c];
    ofhu = Tp.od[1][c];
    ofhv = Tp.od[2][c];
  } else {
    divergence(g, Tp, c, ofh, ofhu, ofhv);
  }
  // forward with intermediates
  const T a0 = V.h[c] + dt * ofh, u0 = V.hu[c] + dt * ofhu, v0 = V.hv[c] + dt * ofhv;
  T a1 = a0, u1 = u0, v1 = v0;
  protect(a1, u1, v1);
  T a2 = a1, u2 = u1, v2 = v1;
  friction(a2, u2, v2, nf[c], dt);
  T ga = gout.h[c], gu = gout.hu[c], gv = gout.hv[c];
  if (STAGE == 2) {
    const T ap = T(0.5) * (base.h[c] + a2), up = T(0.5) * (base.hu[c] + u2),
            vp = T(0.5) * (base.hv[c] + v2);
    protect_adj(ap, up, vp, ga, gu, gv);
    gbase.h[c] = T(0.5) * ga;
    gbase.hu[c] = T(0.5) * gu;
    gbase.hv[c] = T(0.5) * gv;
    ga *= T(0.5);
    gu *= T(0.5);
    gv *= T(0.5);
  }
  T gnc = T(0);
  friction_adj(a1, u1, v1, nf[c], dt, ga, gu, gv, gnc);
  gn[c] += gnc;
  protect_adj(a0, u0, v0, ga, gu, gv);
  R.ga[0][c] = ga;
  R.ga[1][c] = gu;
  R.ga[2][c] = gv;
  R.go[0][c] = dt * ga;
  R.go[1][c] = dt * gu;
  R.go[2][c] = dt * gv;
}

// Faces: divergence adjoints of the two adjacent cells -> face output
// adjoints -> adjoints of the reconstructed inputs.
// Occupancy floors: left free, the FP64 instance of k_faces_adj takes 126-138
// registers (two blocks per SM) and waits on FP64 latency; three blocks with
// a few spilled registers run faster.
template <typename T, bool HLLC>
__global__ void __launch_bounds__(kBX * kBY, 3)
    k_faces_adj(Grid g, size_t ms, Fields<T> V, const T* __restrict__ b, Tape<T> Tp, Rev<T> R) {
  const int i = g.ng + blockIdx.x * kBX + threadIdx.x % kBX;
  const int j = g.ng + blockIdx.y * kBY + threadIdx.x / kBX;
  const int ie = g.nxt - g.ng, je = g.nyt - g.ng;
  if (i > ie || j > je) return;
  const size_t zb = member_base(ms);
  const size_t c = g.at(i, j) + zb;
  // R.go is written at interior cells only (k_cells_adj) and was zeroed at
  // creation, so the ghost ring around the interior reads as zero: the
  // neighbours (i-1, j), (i, j), (i, j-1) need no bounds test
  auto go = [&](int k, int ii, int jj) { return R.go[k][g.at(ii, jj) + zb]; };
  // the divergence's divisions by dx and dy, as products with the
  // reciprocals: they only scale adjoints
  if (j < je) {
    const T rdx = T(1) / T(g.dx);
    const T lh = go(0, i - 1, j), lu = go(1, i - 1, j), lv = go(2, i - 1, j);
    const T rh = go(0, i, j), ru = go(1, i, j), rv = go(2, i, j);
    const T gout[6] = {(-lh + rh) * rdx, (-lu + ru) * rdx, (-lv + rv) * rdx,
                       -T(kHalfG) * ru * rdx, T(kHalfG) * lu * rdx, -T(kHalfG) * lu * rdx};
    const FaceIn<T> f = face_in(V, b, Tp, c - 1, c, 0);
    T gin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    face_adj<0, HLLC>(f.eL, f.qxL, f.qyL, f.bL, f.eR, f.qxR, f.qyR, f.bR, gout, gin);
    for (int k = 0; k < 8; ++k) R.gfx[k][c] = gin[k];
  }
  if (i < ie) {
    const T rdy = T(1) / T(g.dy);
    const T bh = go(0, i, j - 1), bu = go(1, i, j - 1), bv = go(2, i, j - 1);
    const T th = go(0, i, j), tu = go(1, i, j), tv = go(2, i, j);
    const T gout[6] = {(-bh + th) * rdy, (-bu + tu) * rdy, (-bv + tv) * rdy,
                       -T(kHalfG) * tv * rdy, T(kHalfG) * bv * rdy, -T(kHalfG) * bv * rdy};
    const FaceIn<T> f = face_in(V, b, Tp, c - g.pitch, c, 1);
    T gin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    face_adj<1, HLLC>(f.eL, f.qxL, f.qyL, f.bL, f.eR, f.qxR, f.qyR, f.bR, gout, gin);
    for (int k = 0; k < 8; ++k) R.gfy[k][c] = gin[k];
  }
}

// Reconstruction adjoint of cell (i, j) (global index c): the face input
// adjoints of its four faces -> the direct adjoints gd of its eta, hu, hv, b
// and the adjoints gs of its six limited slopes, with the minmod branch of
// each slope (2 bits per slope) in ch.  Cells of [ng-1, ie] x [ng-1, je].
template <typename T>
__device__ __forceinline__ void recon_cell(const Grid& g, const Fields<T>& V,
                                           const T* __restrict__ b, const Rev<T>& R, size_t c,
                                           int i, int j, T (&gs)[6], T (&gd)[4], int& ch) {
  const int ie = g.nxt - g.ng, je = g.nyt - g.ng;
  T de = T(0), du = T(0), dv = T(0), db = T(0);
  ch = 0;
  auto eta = [&](size_t q) { return V.h[q] + b[q]; };
  for (int dir = 0; dir < 2; ++dir) {
    const int o = dir == 0 ? 0 : 3;
    gs[o] = gs[o + 1] = gs[o + 2] = T(0);
    const bool in_range = dir == 0 ? (j >= g.ng && j < je) : (i >= g.ng && i < ie);
    if (!in_range) continue;
    const int lo = dir == 0 ? i : j, hi = dir == 0 ? ie : je;
    const size_t step = dir == 0 ? 1 : (size_t)g.pitch;
    T* const* gf = dir == 0 ? R.gfx : R.gfy;
    // right/top face of c is stored at c + step (exists if lo + 1 <= hi),
    // left/bottom face at c (exists if lo >= ng)
    T gr[8] = {0, 0, 0, 0, 0, 0, 0, 0}, gl[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (lo + 1 <= hi)
      for (int k = 0; k < 8; ++k) gr[k] = gf[k][c + step];
    if (lo >= g.ng)
      for (int k = 0; k < 8; ++k) gl[k] = gf[k][c];
    // eL = eta + s/2 on the right face, eR = eta - s/2 on the left face
    de += gr[0] + gl[4];
    du += gr[1] + gl[5];
    dv += gr[2] + gl[6];
    db += gr[3] + gl[7];
    gs[o] = T(0.5) * (gr[0] - gl[4]);
    gs[o + 1] = T(0.5) * (gr[1] - gl[5]);
    gs[o + 2] = T(0.5) * (gr[2] - gl[6]);
    // minmod branches (cell_slope: zero near dry cells)
    const size_t m = c - step, p = c + step;
    if (!(V.h[c] < T(kThin) || V.h[m] < T(kDry) || V.h[p] < T(kDry))) {
      const int c0 = minmod_choice(eta(c) - eta(m), eta(p) - eta(c));
      const int c1 = minmod_choice(V.hu[c] - V.hu[m], V.hu[p] - V.hu[c]);
      const int c2 = minmod_choice(V.hv[c] - V.hv[m], V.hv[p] - V.hv[c]);
      ch |= (c0 | (c1 << 2) | (c2 << 4)) << (dir * 6);
    }
  }
  gd[0] = de;
  gd[1] = du;
  gd[2] = dv;
  gd[3] = db;
}

// Reconstruction adjoint and slope gather in one launch.  Block (bx, by)
// gathers the kBX x kBY cells from (ng-2 + bx kBX, ng-2 + by kBY): every cell
// collects the slope adjoints of itself and its neighbours (minmod branch a =
// q_c - q_{c-1}, b = q_{c+1} - q_c), plus the direct reconstruction and
// cell-update adjoints.  The reconstruction adjoints of the block's cells and
// a one-cell ring around them are computed first into shared memory (the
// ring's recomputed by both neighbouring blocks, the same bits).  gV receives
// the adjoint of the stage input (all cells, ghosts included); gb
// accumulates the bed's.  frozen: the limited slopes are held constant (their
// adjoints are dropped), the derivative of the step with the slopes of the
// current state frozen.
constexpr int kRW = kBX + 2, kRH = kBY + 2, kRN = kRW * kRH;

template <typename T>
__global__ void __launch_bounds__(kBX * kBY)
    k_recon_gather_adj(Grid g, size_t ms, Fields<T> V, const T* __restrict__ b, Rev<T> R,
                       Fields<T> gV, T* __restrict__ gb, int frozen, Fields<T> gadd) {
  __shared__ T s_gs[6][kRN];
  __shared__ T s_gd[4][kRN];
  __shared__ int s_ch[kRN];
  const int ie = g.nxt - g.ng, je = g.nyt - g.ng;
  const size_t zb = member_base(ms);
  const int i0 = g.ng - 2 + (int)blockIdx.x * kBX, j0 = g.ng - 2 + (int)blockIdx.y * kBY;
  // recon cells: [ng-1, ie] x [ng-1, je]
  auto rc = [&](int ii, int jj) { return in_box(ii, jj, g.ng - 1, ie, g.ng - 1, je); };
  for (int k = threadIdx.x; k < kRN; k += kBX * kBY) {
    const int ii = i0 - 1 + k % kRW, jj = j0 - 1 + k / kRW;
    T gs[6] = {0, 0, 0, 0, 0, 0}, gd[4] = {0, 0, 0, 0};
    int ch = 0;
    if (rc(ii, jj)) recon_cell(g, V, b, R, g.at(ii, jj) + zb, ii, jj, gs, gd, ch);
    for (int q = 0; q < 6; ++q) s_gs[q][k] = gs[q];
    for (int q = 0; q < 4; ++q) s_gd[q][k] = gd[q];
    s_ch[k] = ch;
  }
  __syncthreads();

  const int tx = threadIdx.x % kBX, ty = threadIdx.x / kBX;
  const int i = i0 + tx, j = j0 + ty;
  if (i > ie + 1 || j > je + 1) return;
  const size_t c = g.at(i, j) + zb;
  const int t = (ty + 1) * kRW + (tx + 1);  // this cell in the shared arrays
  // slope ranges: x-slopes on [ng-1, ie] x [ng, je-1], y-slopes on [ng, ie-1] x [ng-1, je]
  auto xs = [&](int ii, int jj) { return in_box(ii, jj, g.ng - 1, ie, g.ng, je - 1); };
  auto ys = [&](int ii, int jj) { return in_box(ii, jj, g.ng, ie - 1, g.ng - 1, je); };
  T acc[3] = {T(0), T(0), T(0)};
  for (int dir = 0; dir < 2 && !frozen; ++dir) {
    const int di = dir == 0 ? 1 : 0, dj = dir == 0 ? 0 : 1;
    const int dt = dir == 0 ? 1 : kRW;
    auto has = [&](int ii, int jj) { return dir == 0 ? xs(ii, jj) : ys(ii, jj); };
    for (int v = 0; v < 3; ++v) {
      const int o = dir * 3 + v;
      const int sh = dir * 6 + 2 * v;
      T s = T(0);
      if (has(i, j)) {
        const int chc = (s_ch[t] >> sh) & 3;
        if (chc == 1) s += s_gs[o][t];
        else if (chc == 2) s -= s_gs[o][t];
      }
      if (has(i + di, j + dj)) {  // neighbour above chose a = q_{c+1} - q_c
        if (((s_ch[t + dt] >> sh) & 3) == 1) s -= s_gs[o][t + dt];
      }
      if (has(i - di, j - dj)) {  // neighbour below chose b = q_c - q_{c-1}
        if (((s_ch[t - dt] >> sh) & 3) == 2) s += s_gs[o][t - dt];
      }
      acc[v] += s;
    }
  }
  T ge = acc[0], gu = acc[1], gv = acc[2], gbb = T(0);
  if (rc(i, j)) {
    ge += s_gd[0][t];
    gu += s_gd[1][t];
    gv += s_gd[2][t];
    gbb += s_gd[3][t];
  }
  T gh = ge;  // eta = h + b
  gbb += ge;
  if (i >= g.ng && i < ie && j >= g.ng && j < je) {
    gh += R.ga[0][c];
    gu += R.ga[1][c];
    gv += R.ga[2][c];
    if (gadd.h) {  // stage 1: the RK2 base adjoint of stage 2 (U^k enters both stages)
      gh += gadd.h[c];
      gu += gadd.hu[c];
      gv += gadd.hv[c];
    }
  }
  gV.h[c] = gh;
  gV.hu[c] = gu;
  gV.hv[c] = gv;
  gb[c] += gbb;
}

// Wall ghosts, reversed: a ghost's adjoint moves to the cell it mirrors
// (normal momentum with a sign change); run S/N (pass 1) before W/E (pass 0).
// With `bed`, fold the bed adjoint instead of the state's.
template <typename T>
__global__ void k_walls_adj(Grid g, size_t ms, Fields<T> V, Fields<T> gV, T* __restrict__ gb,
                            int pass, int bed) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int side = blockIdx.y;
  const int n_tan = pass == 0 ? g.nyt : g.nxt;
  if (t >= n_tan) return;
  const size_t zb = member_base(ms);
  // forward order k = 1..ng; mirrors are interior or earlier-filled cells, so
  // reverse k = ng..1
  for (int k = g.ng; k >= 1; --k) {
    int ig, jg, im, jm;
    if (pass == 0) {
      jg = jm = t;
      ig = side == 0 ? g.ng - k : g.nxt - g.ng + k - 1;
      im = side == 0 ? g.ng + k - 1 : g.nxt - g.ng - k;
    } else {
      ig = im = t;
      jg = side == 0 ? g.ng - k : g.nyt - g.ng + k - 1;
      jm = side == 0 ? g.ng + k - 1 : g.nyt - g.ng - k;
    }
    const size_t q = g.at(ig, jg) + zb, m = g.at(im, jm) + zb;
    if (bed) {
      gb[m] += gb[q];
      gb[q] = T(0);
      continue;
    }
    if (V.h[m] > T(0)) gV.h[m] += gV.h[q];  // h_g = max(0, h_m)
    gV.h[q] = T(0);
    if (pass == 0) {
      gV.hu[m] -= gV.hu[q];
      gV.hv[m] += gV.hv[q];
    } else {
      gV.hv[m] -= gV.hv[q];
      gV.hu[m] += gV.hu[q];
    }
    gV.hu[q] = T(0);
    gV.hv[q] = T(0);
  }
}

template <typename T>
__global__ void k_gauges_adj(const long long* __restrict__ gq, const double* __restrict__ r, int n,
                             Fields<T> lam, T* __restrict__ gb) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const size_t q = (size_t)gq[k];
  lam.h[q] += T(2.0 * r[k]);  // gauges are distinct cells: no two threads share q
  gb[q] += T(2.0 * r[k]);
}

// ---------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------

#define ADJ_TRY(expr)                      \
  do {                                     \
    cudaError_t e_ = (expr);               \
    if (e_ != cudaSuccess) return -1;      \
  } while (0)

template <typename T>
class Adjoint final : public AdjointBase {
 public:
  ~Adjoint() override {
    for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
    if (all_mem_) cudaFree(all_mem_);
    if (mem_) cudaFree(mem_);
    if (obs_d_) cudaFree(obs_d_);
    if (stream_) cudaStreamDestroy(stream_);
  }

  // nm members of nx x ny interior cells; h0, hu0, hv0: [member][nx * ny]
  // F-order (hu0, hv0 may be null: zero); gi, gj: [member][ngauge].
  int create(int nm, int nx, int ny, int ng, double dx, double dy, double cfl, int hllc,
             int nsteps, const double* h0, const double* hu0, const double* hv0, const int* gi,
             const int* gj, int ngauge, std::string& err) {
    if (nm < 1 || nx < 2 || ny < 2 || ng < 2 || nsteps < 1 || ngauge < 0 || !h0 ||
        (ngauge > 0 && (!gi || !gj))) {
      err = "invalid sizes";
      return -2;
    }
    if ((ny + 2 * ng + kBY - 1) / kBY > 65535 || nm > 65535) {
      err = "the adjoint supports at most 524000 rows and 65535 members";
      return -2;
    }
    if (nx < ng || ny < ng) {  // one wall fill per stage: ghosts must mirror interior cells
      err = "the adjoint needs an interior at least nghost cells wide in x and y";
      return -2;
    }
    if (cudaFuncSetAttribute(k_stage_fused<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)FusedSmem<T>::BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(k_stage_fused<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)FusedSmem<T>::BYTES) != cudaSuccess) {
      err = "cannot configure the fused forward kernel";
      return -1;
    }
    nm_ = nm;
    g_.ng = ng;
    g_.nxt = nx + 2 * ng;
    g_.nyt = ny + 2 * ng;
    g_.pitch = (g_.nxt + 31) / 32 * 32;
    g_.dx = dx;
    g_.dy = dy;
    ms_ = (size_t)g_.pitch * g_.nyt;
    cfl_ = cfl;
    hllc_ = hllc;
    nsteps_ = nsteps;
    ngauge_ = ngauge;
    std::vector<long long> gq((size_t)nm * ngauge);
    for (int m = 0; m < nm; ++m)
      for (int k = 0; k < ngauge; ++k) {
        const int a = gi[(size_t)m * ngauge + k], c = gj[(size_t)m * ngauge + k];
        if (a < 0 || a >= nx || c < 0 || c >= ny) {
          err = "gauge outside the interior";
          return -2;
        }
        long long& q = gq[(size_t)m * ngauge + k];
        q = (long long)(g_.at(a + ng, c + ng) + (size_t)m * ms_);
        for (int p = 0; p < k; ++p)
          if (gq[(size_t)m * ngauge + p] == q) {
            err = "gauges must be distinct cells";
            return -2;
          }
      }
    K_ = std::max(1, (int)std::ceil(std::sqrt((double)nsteps)));
    nck_ = (nsteps + K_ - 1) / K_ + 1;
    if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) return -1;
    const size_t f = ms_ * (size_t)nm;  // elements of one batched field
    // fields: b, n; U, Us, lam, lam*, gbase, gV (3 each); gb, gn; tapes
    // (2 x 21); reverse scratch (3+3+8+8); checkpoints; segment states
    nfields_ = 2 + 6 * 3 + 2 + 2 * 21 + (3 + 3 + 8 + 8) + 3 * (size_t)nck_ +
               3 * (size_t)(K_ + 1);
    const size_t fbytes = (f * sizeof(T) + 255) / 256 * 256;
    const size_t nres = (size_t)nsteps * nm * ngauge;
    const size_t bytes = nfields_ * fbytes + 8 * nres + 8 * (size_t)nm * ngauge +
                         16 * (size_t)nm + 8 * (size_t)nsteps * nm + 16 * (size_t)nm + 1024;
    if (cudaMalloc(&mem_, bytes) != cudaSuccess) {
      mem_ = nullptr;
      err = "device allocation failed (" + std::to_string(bytes >> 20) + " MiB)";
      return -1;
    }
    ADJ_TRY(cudaMemsetAsync(mem_, 0, bytes, stream_));
    char* p = (char*)mem_;
    auto take = [&]() { T* q = (T*)p; p += fbytes; return q; };
    auto takeset = [&]() { Fields<T> s{take(), take(), take()}; return s; };
    b_ = take();
    nf_ = take();
    U_ = takeset();
    Us_ = takeset();
    lam_ = takeset();
    lams_ = takeset();
    gbase_ = takeset();
    gV_ = takeset();
    gb_ = take();
    gn_ = take();
    for (Tape<T>* t : {&t1_, &t2_}) {
      for (auto& x : t->s) x = take();
      for (auto& x : t->fx) x = take();
      for (auto& x : t->fy) x = take();
      for (auto& x : t->od) x = take();
    }
    for (auto& x : R_.go) x = take();
    for (auto& x : R_.ga) x = take();
    for (auto& x : R_.gfx) x = take();
    for (auto& x : R_.gfy) x = take();
    ck_.resize(nck_);
    for (auto& c : ck_) c = takeset();
    seg_.resize(K_ + 1);
    for (auto& c : seg_) c = takeset();
    r_ = (double*)p;
    p += 8 * nres;
    gq_ = (long long*)p;
    p += 8 * (size_t)nm * ngauge;
    mx_ = (unsigned long long*)p;
    p += 16 * (size_t)nm;
    dts_d_ = (double*)p;
    p += 8 * (size_t)nsteps * nm;
    mass_d_ = (double*)p;
    if (ngauge > 0)
      ADJ_TRY(cudaMemcpyAsync(gq_, gq.data(), sizeof(long long) * gq.size(), cudaMemcpyHostToDevice,
                              stream_));
    // initial state: interior from the caller
    Fields<T>& c0 = ck_[0];
    const double* src[3] = {h0, hu0, hv0};
    T* dst[3] = {c0.h, c0.hu, c0.hv};
    for (int k = 0; k < 3; ++k)
      if (upload_interior(dst[k], src[k], 0.0) != 0) return -1;
    dts_.assign((size_t)nsteps * nm, 0.0);
    obs_.assign(nres, 0.0);
    mass_.assign(2 * (size_t)nm, 0.0);
    return 0;
  }

  int set_obs(const double* obs) override {
    std::memcpy(obs_.data(), obs, obs_.size() * sizeof(double));
    obs_dev_dirty_ = true;
    return 0;
  }
  int set_dt(const double* dts) override {  // [member][step]
    for (int m = 0; m < nm_; ++m)
      for (int k = 0; k < nsteps_; ++k) dts_[(size_t)k * nm_ + m] = dts[(size_t)m * nsteps_ + k];
    have_dt_ = true;
    return upload_dts();
  }
  void get_dt(double* dts) const override {
    for (int m = 0; m < nm_; ++m)
      for (int k = 0; k < nsteps_; ++k) dts[(size_t)m * nsteps_ + k] = dts_[(size_t)k * nm_ + m];
  }
  int members() const override { return nm_; }
  int precision() const override { return sizeof(T) == 8 ? 64 : 32; }
  void mass(double* out) const override { std::memcpy(out, mass_.data(), mass_.size() * 8); }
  void set_frozen_slopes(bool on) override { frozen_ = on; }

  // Forward run.  record: dt from the CFL condition of each state (stored);
  // else the stored dt sequence.  J[m] and, optionally, the gauge surfaces
  // ([step][member][gauge]) are returned.
  int forward(const double* b, const double* n, double n_scalar, bool record, double* J,
              double* eta_out) override {
    if (!record && !have_dt_) return -2;
    if (upload_params(b, n, n_scalar) != 0) return -1;
    if (domain_mass(ck_[0], 0) != 0) return -1;
    if (mark(0) != 0) return -1;
    if (copy(U_, ck_[0]) != 0) return -1;
    for (int k = 0; k < nsteps_; ++k) {
      if (record) {
        if (cfl_step(U_, k) != 0) return -1;
      }
      if (step(U_, U_, k) != 0) return -1;
      gauges(k, U_);
    }
    if (record) have_dt_ = true;
    if (mark(1) != 0) return -1;
    if (domain_mass(U_, 1) != 0) return -1;
    return finish_misfit(J, eta_out);
  }

  // J and its gradient with respect to the interior bed and n field.
  int gradient(const double* b, const double* n, double n_scalar, double* J, double* gb_out,
               double* gn_out) override {
    if (!have_dt_) return -2;
    if (upload_params(b, n, n_scalar) != 0) return -1;
    const size_t fb = ms_ * nm_ * sizeof(T);
    const bool all = keep_all_states();
    if (mark(0) != 0) return -1;
    if (all) {
      // forward keeping every state
      if (copy(all_[0], ck_[0]) != 0) return -1;
      for (int k = 0; k < nsteps_; ++k) {
        if (step(all_[k], all_[k + 1], k) != 0) return -1;
        gauges(k, all_[k + 1]);
      }
    } else {
      // forward with checkpoints
      if (copy(U_, ck_[0]) != 0) return -1;
      for (int k = 0; k < nsteps_; ++k) {
        if (step(U_, U_, k) != 0) return -1;
        gauges(k, U_);
        if ((k + 1) % K_ == 0 && (k + 1) / K_ < nck_)
          if (copy(ck_[(k + 1) / K_], U_) != 0) return -1;
      }
    }
    // reverse
    ADJ_TRY(cudaMemsetAsync(lam_.h, 0, fb, stream_));
    ADJ_TRY(cudaMemsetAsync(lam_.hu, 0, fb, stream_));
    ADJ_TRY(cudaMemsetAsync(lam_.hv, 0, fb, stream_));
    ADJ_TRY(cudaMemsetAsync(gb_, 0, fb, stream_));
    ADJ_TRY(cudaMemsetAsync(gn_, 0, fb, stream_));
    const int nseg = all ? 0 : (nsteps_ + K_ - 1) / K_;
    const int ng = nm_ * ngauge_;
    for (int k = all ? nsteps_ - 1 : -1; k >= 0; --k) {
      if (ng > 0)  // misfit at U^{k+1}
        k_gauges_adj<T><<<(ng + 127) / 128, 128, 0, stream_>>>(gq_, r_ + (size_t)k * ng, ng,
                                                               lam_, gb_);
      if (step_adj(all_[k], k, true) != 0) return -1;  // every kept U^k went through step()
    }
    for (int s = nseg - 1; s >= 0; --s) {
      const int k0 = s * K_, k1 = std::min(nsteps_, k0 + K_);
      if (copy(seg_[0], ck_[s]) != 0) return -1;
      for (int k = k0; k < k1 - 1; ++k)
        if (step(seg_[k - k0], seg_[k - k0 + 1], k) != 0) return -1;
      for (int k = k1 - 1; k >= k0; --k) {
        // misfit at U^{k+1}
        if (ng > 0)
          k_gauges_adj<T><<<(ng + 127) / 128, 128, 0, stream_>>>(gq_, r_ + (size_t)k * ng, ng,
                                                                 lam_, gb_);
        // the segment's last state was not the input of a recomputed step
        if (step_adj(seg_[k - k0], k, k < k1 - 1) != 0) return -1;
      }
    }
    // bed ghosts mirror interior cells: fold their adjoints in (S/N then W/E)
    walls_adj(gV_, true);
    if (mark(1) != 0) return -1;
    if (finish_misfit(J, nullptr) != 0) return -1;
    if (download_interior(gb_out, gb_) != 0) return -1;
    return download_interior(gn_out, gn_);
  }

  int checkpoint_interval() const override { return kept_all_ ? 1 : K_; }
  void set_state_budget(long long bytes) override {
    budget_ = bytes;
    if (all_mem_ && bytes >= 0 && (long long)all_bytes() > bytes) {
      cudaFree(all_mem_);
      all_mem_ = nullptr;
      all_.clear();
      kept_all_ = false;
    }
  }
  // Device milliseconds of the last forward / gradient run (CUDA events on
  // the adjoint's stream, from the initial state to the last kernel).
  double last_ms() override {
    float f = 0.0f;
    if (!ev_[0] || cudaEventSynchronize(ev_[1]) != cudaSuccess ||
        cudaEventElapsedTime(&f, ev_[0], ev_[1]) != cudaSuccess)
      return -1.0;
    return f;
  }

 private:
  int mark(int k) {
    if (!ev_[k] && cudaEventCreate(&ev_[k]) != cudaSuccess) return -1;
    return cudaEventRecord(ev_[k], stream_) == cudaSuccess ? 0 : -1;
  }
  cudaEvent_t ev_[2] = {nullptr, nullptr};

  dim3 blocks(int x0, int x1, int y0, int y1) const {  // cover [x0, x1] x [y0, y1], all members
    return dim3((unsigned)((x1 - x0 + kBX) / kBX), (unsigned)((y1 - y0 + kBY) / kBY),
                (unsigned)nm_);
  }
  dim3 interior() const { return blocks(g_.ng, g_.nxt - g_.ng - 1, g_.ng, g_.nyt - g_.ng - 1); }
  const double* dt_of(int k) const { return dts_d_ + (size_t)k * nm_; }

  const double* obs_dev() {
    if (obs_dev_dirty_) {
      if (!obs_d_) cudaMalloc(&obs_d_, obs_.size() * sizeof(double) + 8);
      cudaMemcpyAsync(obs_d_, obs_.data(), obs_.size() * sizeof(double), cudaMemcpyHostToDevice,
                      stream_);
      obs_dev_dirty_ = false;
    }
    return obs_d_;
  }

  int upload_dts() {
    ADJ_TRY(cudaMemcpyAsync(dts_d_, dts_.data(), dts_.size() * sizeof(double),
                            cudaMemcpyHostToDevice, stream_));
    return cudaStreamSynchronize(stream_) == cudaSuccess ? 0 : -1;
  }

  // [member][nx * ny] F-order host values (null: `fill`) -> interior cells of
  // a batched field (ghosts zero).
  int upload_interior(T* dst, const double* src, double fill) {
    const int nx = g_.nx_phys(), ny = g_.ny_phys();
    std::vector<T> tmp(ms_);
    for (int m = 0; m < nm_; ++m) {
      std::fill(tmp.begin(), tmp.end(), T(0));
      const double* s = src ? src + (size_t)m * nx * ny : nullptr;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          tmp[g_.at(i + g_.ng, j + g_.ng)] = T(s ? s[(size_t)i + (size_t)j * nx] : fill);
      ADJ_TRY(cudaMemcpyAsync(dst + (size_t)m * ms_, tmp.data(), ms_ * sizeof(T),
                              cudaMemcpyHostToDevice, stream_));
      ADJ_TRY(cudaStreamSynchronize(stream_));  // tmp is reused
    }
    return 0;
  }

  int download_interior(double* dst, const T* src) {
    const int nx = g_.nx_phys(), ny = g_.ny_phys();
    std::vector<T> tmp(ms_);
    for (int m = 0; m < nm_; ++m) {
      ADJ_TRY(cudaMemcpyAsync(tmp.data(), src + (size_t)m * ms_, ms_ * sizeof(T),
                              cudaMemcpyDeviceToHost, stream_));
      ADJ_TRY(cudaStreamSynchronize(stream_));
      double* d = dst + (size_t)m * nx * ny;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          d[(size_t)i + (size_t)j * nx] = (double)tmp[g_.at(i + g_.ng, j + g_.ng)];
    }
    return 0;
  }

  int upload_params(const double* b, const double* n, double n_scalar) {
    if (upload_interior(b_, b, 0.0) != 0) return -1;
    return upload_interior(nf_, n, n_scalar);
  }

  int copy(Fields<T>& dst, const Fields<T>& src) {
    const size_t bytes = ms_ * nm_ * sizeof(T);
    ADJ_TRY(cudaMemcpyAsync(dst.h, src.h, bytes, cudaMemcpyDeviceToDevice, stream_));
    ADJ_TRY(cudaMemcpyAsync(dst.hu, src.hu, bytes, cudaMemcpyDeviceToDevice, stream_));
    ADJ_TRY(cudaMemcpyAsync(dst.hv, src.hv, bytes, cudaMemcpyDeviceToDevice, stream_));
    return 0;
  }

  // Gauge residuals of step k from its new state V (= U^{k+1}).
  void gauges(int k, const Fields<T>& V) {
    const int ng = nm_ * ngauge_;
    if (ng > 0)
      k_gauges<T><<<(ng + 127) / 128, 128, 0, stream_>>>(V, b_, gq_, obs_dev() + (size_t)k * ng,
                                                         ng, r_ + (size_t)k * ng);
  }

  size_t all_bytes() const {
    const size_t fbytes = (ms_ * nm_ * sizeof(T) + 255) / 256 * 256;
    return 3 * fbytes * (size_t)(nsteps_ + 1);
  }

  // Every state U^0..U^N in device memory, allocated at the first gradient
  // run that the budget allows (kept for later runs); false: checkpoints.
  bool keep_all_states() {
    kept_all_ = false;
    if (budget_ == 0) return false;
    if (!all_mem_) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return false;
      const size_t limit = budget_ < 0 ? free_b / 2 : (size_t)budget_;
      if (all_bytes() > limit) return false;
      if (cudaMalloc(&all_mem_, all_bytes()) != cudaSuccess) {
        all_mem_ = nullptr;
        cudaGetLastError();  // the failed allocation is not an error of the run
        return false;
      }
      // zero, like the checkpoint buffers: cells no kernel writes (row
      // padding, corners) then hold the same values in both modes
      if (cudaMemsetAsync(all_mem_, 0, all_bytes(), stream_) != cudaSuccess) return false;
      const size_t fbytes = (ms_ * nm_ * sizeof(T) + 255) / 256 * 256;
      char* p = (char*)all_mem_;
      all_.resize((size_t)nsteps_ + 1);
      for (auto& st : all_) {
        st = Fields<T>{(T*)p, (T*)(p + fbytes), (T*)(p + 2 * fbytes)};
        p += 3 * fbytes;
      }
    }
    kept_all_ = true;
    return true;
  }

  // Per-member J = sum of squared residuals (FP64) and the gauge surfaces.
  int finish_misfit(double* J, double* eta_out) {
    const size_t nres = (size_t)nsteps_ * nm_ * ngauge_;
    std::vector<double> r(nres);
    if (nres > 0)
      ADJ_TRY(cudaMemcpyAsync(r.data(), r_, nres * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    ADJ_TRY(cudaStreamSynchronize(stream_));
    for (int m = 0; m < nm_; ++m) {
      double acc = 0.0;
      for (int k = 0; k < nsteps_; ++k)
        for (int q = 0; q < ngauge_; ++q) {
          const double x = r[((size_t)k * nm_ + m) * ngauge_ + q];
          acc += x * x;
        }
      J[m] = acc;
    }
    if (eta_out)
      for (size_t k = 0; k < nres; ++k) eta_out[k] = r[k] + obs_[k];
    return 0;
  }

  int domain_mass(const Fields<T>& V, int which) {
    ADJ_TRY(cudaMemsetAsync(mass_d_, 0, sizeof(double) * nm_, stream_));
    k_mass<T><<<interior(), kBX * kBY, 0, stream_>>>(g_, ms_, V.h, mass_d_);
    ADJ_TRY(cudaMemcpyAsync(mass_.data() + (size_t)which * nm_, mass_d_, sizeof(double) * nm_,
                            cudaMemcpyDeviceToHost, stream_));
    return 0;
  }

  void walls(Fields<T> V) {
    const int tpb = 128;
    k_walls<T><<<dim3((unsigned)((g_.nyt + tpb - 1) / tpb), 2, (unsigned)nm_), tpb, 0, stream_>>>(
        g_, ms_, V, b_, 0);
    k_walls<T><<<dim3((unsigned)((g_.nxt + tpb - 1) / tpb), 2, (unsigned)nm_), tpb, 0, stream_>>>(
        g_, ms_, V, b_, 1);
  }

  void walls_adj(Fields<T> V, bool bed) {
    const int tpb = 128;
    k_walls_adj<T><<<dim3((unsigned)((g_.nxt + tpb - 1) / tpb), 2, (unsigned)nm_), tpb, 0,
                     stream_>>>(g_, ms_, V, gV_, gb_, 1, bed ? 1 : 0);
    k_walls_adj<T><<<dim3((unsigned)((g_.nyt + tpb - 1) / tpb), 2, (unsigned)nm_), tpb, 0,
                     stream_>>>(g_, ms_, V, gV_, gb_, 0, bed ? 1 : 0);
  }

  void tape(Fields<T> V, Tape<T>& Tp) {
    const int ie = g_.nxt - g_.ng, je = g_.nyt - g_.ng;
    k_slopes<T><<<blocks(g_.ng - 1, ie, g_.ng - 1, je), kBX * kBY, 0, stream_>>>(g_, ms_, V, b_, Tp);
    if (hllc_)
      k_faces<T, true><<<blocks(g_.ng, ie, g_.ng, je), kBX * kBY, 0, stream_>>>(g_, ms_, V, b_, Tp);
    else
      k_faces<T, false><<<blocks(g_.ng, ie, g_.ng, je), kBX * kBY, 0, stream_>>>(g_, ms_, V, b_, Tp);
  }

  // Step k: U -> out, one fused launch per stage (no tapes).  out may alias
  // U: stage 2 reads the RK2 base only at the cell it writes, and its
  // neighbours come from the stage-1 result.
  int step(Fields<T> U, Fields<T> out, int k) {
    walls(U);
    fused_stage(U, U, 1, Us_, k);
    walls(Us_);
    fused_stage(Us_, U, 2, out, k);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  void fused_stage(Fields<T> V, Fields<T> base, int stage, Fields<T> out, int k) {
    const size_t smem = FusedSmem<T>::BYTES;
    const dim3 tiles((unsigned)((g_.nx_phys() + kFX - 1) / kFX),
                     (unsigned)((g_.ny_phys() + kFY - 1) / kFY), (unsigned)nm_);
    if (hllc_)
      k_stage_fused<T, true><<<tiles, kFThreads, smem, stream_>>>(g_, ms_, V, base, b_, nf_,
                                                                       dt_of(k), stage, out);
    else
      k_stage_fused<T, false><<<tiles, kFThreads, smem, stream_>>>(g_, ms_, V, base, b_, nf_,
                                                                        dt_of(k), stage, out);
  }

  // dt of step k for every member from the CFL condition of U (recorded).
  int cfl_step(Fields<T> U, int k) {
    std::vector<unsigned long long> h(2 * (size_t)nm_);
    ADJ_TRY(cudaMemsetAsync(mx_, 0, h.size() * sizeof(unsigned long long), stream_));
    k_speeds<T><<<interior(), kBX * kBY, 0, stream_>>>(g_, ms_, U, mx_);
    ADJ_TRY(cudaMemcpyAsync(h.data(), mx_, h.size() * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, stream_));
    ADJ_TRY(cudaStreamSynchronize(stream_));
    for (int m = 0; m < nm_; ++m) {
      double sx, sy;
      std::memcpy(&sx, &h[2 * (size_t)m], 8);
      std::memcpy(&sy, &h[2 * (size_t)m + 1], 8);
      dts_[(size_t)k * nm_ + m] = cfl_dt(sx, sy, g_, cfl_);
    }
    ADJ_TRY(cudaMemcpyAsync(dts_d_ + (size_t)k * nm_, dts_.data() + (size_t)k * nm_,
                            sizeof(double) * nm_, cudaMemcpyHostToDevice, stream_));
    return cudaStreamSynchronize(stream_) == cudaSuccess ? 0 : -1;  // host row reused next step
  }

  // Reverse of one stage: gout (adjoint of the stage output, interior) ->
  // gV_ (adjoint of the stage input after the wall fold), gbase_ (stage 2).
  int stage_adj(Fields<T> V, Fields<T> base, Tape<T>& Tp, int k, int stage, Fields<T> gout) {
    const int ie = g_.nxt - g_.ng, je = g_.nyt - g_.ng;
    if (g_.ng > 2) {  // the gather writes layers ng-2 .. nxt-ng+1: all of them when ng = 2
      const size_t fb = ms_ * nm_ * sizeof(T);
      ADJ_TRY(cudaMemsetAsync(gV_.h, 0, fb, stream_));
      ADJ_TRY(cudaMemsetAsync(gV_.hu, 0, fb, stream_));
      ADJ_TRY(cudaMemsetAsync(gV_.hv, 0, fb, stream_));
    }
    if (stage == 2)
      k_cells_adj<T, 2><<<interior(), kBX * kBY, 0, stream_>>>(g_, ms_, V, base, nf_, Tp,
                                                              dt_of(k), gout, R_, gbase_, gn_);
    else
      k_cells_adj<T, 1><<<interior(), kBX * kBY, 0, stream_>>>(g_, ms_, V, base, nf_, Tp,
                                                              dt_of(k), gout, R_, gbase_, gn_);
    if (hllc_)
      k_faces_adj<T, true><<<blocks(g_.ng, ie, g_.ng, je), kBX * kBY, 0, stream_>>>(g_, ms_, V, b_,
                                                                                    Tp, R_);
    else
      k_faces_adj<T, false><<<blocks(g_.ng, ie, g_.ng, je), kBX * kBY, 0, stream_>>>(g_, ms_, V,
                                                                                     b_, Tp, R_);
    k_recon_gather_adj<T><<<blocks(g_.ng - 2, ie + 1, g_.ng - 2, je + 1), kBX * kBY, 0,
                            stream_>>>(g_, ms_, V, b_, R_, gV_, gb_, frozen_ ? 1 : 0,
                                       stage == 1 ? gbase_ : Fields<T>{});
    walls_adj(V, false);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  // Reverse of step k from U (= U^k): lam_ (adjoint of U^{k+1}) -> lam_
  // (adjoint of U^k).  Recomputes U* and both tapes.  `walled`: U's wall
  // ghosts were filled from its interior already (a forward step() took it as
  // its input), so the fill, which would write the same values, is skipped.
  int step_adj(Fields<T> U, int k, bool walled) {
    if (!walled) walls(U);
    tape(U, t1_);
    k_cells<T><<<interior(), kBX * kBY, 0, stream_>>>(g_, ms_, U, U, nf_, t1_, dt_of(k), 1, Us_);
    walls(Us_);
    tape(Us_, t2_);
    if (stage_adj(Us_, U, t2_, k, 2, lam_) != 0) return -1;  // gV_ = adjoint of U*
    std::swap(lams_, gV_);  // three distinct buffers: renaming replaces the copies
    // gV_ = adjoint of U^k: stage 1's, with stage 2's RK2 base adjoint added in the gather
    if (stage_adj(U, U, t1_, k, 1, lams_) != 0) return -1;
    std::swap(lam_, gV_);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
  }

  Grid g_{};
  size_t ms_ = 0;
  int nm_ = 1;
  double cfl_ = 0.45;
  int hllc_ = 0, nsteps_ = 0, ngauge_ = 0, K_ = 1, nck_ = 1;
  // every state of a gradient run (keep_all_states)
  void* all_mem_ = nullptr;
  std::vector<Fields<T>> all_;
  long long budget_ = 0;
  bool kept_all_ = false;
  size_t nfields_ = 0;
  cudaStream_t stream_ = nullptr;
  void* mem_ = nullptr;
  T *b_ = nullptr, *nf_ = nullptr, *gb_ = nullptr, *gn_ = nullptr;
  double* r_ = nullptr;
  double* obs_d_ = nullptr;
  double* dts_d_ = nullptr;
  double* mass_d_ = nullptr;
  unsigned long long* mx_ = nullptr;
  long long* gq_ = nullptr;
  Fields<T> U_{}, Us_{}, lam_{}, lams_{}, gbase_{}, gV_{};
  Tape<T> t1_{}, t2_{};
  Rev<T> R_{};
  std::vector<Fields<T>> ck_, seg_;
  std::vector<double> dts_, obs_, mass_;  // dts_: [step][member]
  bool have_dt_ = false, obs_dev_dirty_ = true;
  bool frozen_ = false;
};

#undef ADJ_TRY

template <typename T>
AdjointBase* make_adjoint(int nm, int nx, int ny, int ng, double dx, double dy, double cfl,
                          int hllc, int nsteps, const double* h0, const double* hu0,
                          const double* hv0, const int* gi, const int* gj, int ngauge,
                          std::string& err, int& rc) {
  auto* a = new Adjoint<T>();
  rc = a->create(nm, nx, ny, ng, dx, dy, cfl, hllc, nsteps, h0, hu0, hv0, gi, gj, ngauge, err);
  if (rc != 0) {
    delete a;
    return nullptr;
  }
  return a;
}

}  // namespace adj
}  // namespace rkb
