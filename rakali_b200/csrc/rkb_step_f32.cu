// FP32 surface form of the structured SSP-RK2 step (sm_100a).
//
// State: the free surface eta = h + b and the momenta hu, hv in FP32; the bed
// b in FP64.  Same scheme and step structure as the FP64 kernels
// (rki_kernel_flux.F90:104-783, rki_kernel_fused.F90:164-471,
// rki_boundary.F90:40-552, rki_kernel_timestep.F90:16-74), with:
//
//  * every difference against the bed in FP64: the depth h = eta - b of a
//    cell, the reconstructed depths eta_face - b_cell and the Audusse
//    hydrostatic depths eta_face - max(b_L, b_R); the wet/dry threshold tests
//    are made on those FP64 values;
//  * the domain sums (mass budget partials) in FP64;
//  * the rest (slopes, Riemann fluxes, update, friction) in FP32.
//
// The momentum update never subtracts two hydrostatic pressures g/2 h^2: each
// face returns its flux in excess of the left hydrostatic pressure and the
// pressure jump g/2 (dh_hyd)(h_hyd,L + h_hyd,R) with dh_hyd an FP64
// difference, and each cell adds its own reconstruction term g h s (s = the
// limited surface slope); see face().  Lake at rest is exact: a flat wet
// surface has zero slopes, both sides of a face then have the same
// hydrostatic depth, so the jump, the excess flux and the cell term are all
// exactly zero.  Dry cells store the bed rounded down (eta <= b), so they
// read back as h <= 0.
//
// Data movement: one warp sweeps a strip of 30 C columns (C = 2 or 4 columns
// per lane) up a range of rows; lanes 0..29 own the output columns, lane 30
// the C columns right of the strip and lane 31 those left of it, so the lanes
// form a ring and x-neighbours are plain shuffles.  Rows arrive through a
// per-warp ring of shared-memory slots filled by 1D bulk asynchronous copies
// (cp.async.bulk, completion on an mbarrier); y-neighbours stay in
// registers.  No block barrier on the data path.  Every wait is bounded in
// time; a wait that gives up sets StepCtl::error.  A lane's columns are
// processed in pairs on packed FP32 arithmetic.
#include <cstdint>

#include "rkb_async.cuh"
#include "rkb_crmath.cuh"
#include "rkb_kernels.h"
#include "rkb_stepctl.cuh"

namespace rkb {
namespace {

constexpr float kGf = 9.80665f;
constexpr float kHalfGf = 0.5f * kGf;
constexpr float kDryF = 1.0e-6f;
constexpr float kEps4F = 5.062499999999998e-16f;
constexpr float kSqrt2F = 1.41421356f;
constexpr float kFroude2G = 50.0f * 50.0f * kGf;
constexpr unsigned kFull = 0xffffffffu;

// Strip geometry and shared-memory ring.  With C columns per lane, lanes
// 0..29 own the strip's 30 C output columns, lane 30 the C columns right of
// the strip and lane 31 the C columns left of it: the 32 lanes form a ring of
// consecutive column groups (31 -> 0 -> 1 -> ... -> 30), so neighbour
// exchanges are plain shuffles and every lane runs the same code.
constexpr int kWarps = 4;  // warps (strips) per block
constexpr int kNbuf = 5;   // ring slots per warp
template <int C>
struct Lay {
  static constexpr int kStrip = 30 * C;                     // output columns
  static constexpr int kSeg = (4 + 31 * C + 3) / 4 * 4;     // copied: [x0 - 4, x0 - 4 + kSeg)
  // slot layout (bytes): eta, hu, hv (FP32, kSeg), b (FP64, kSeg); stage 2
  // adds the RK2 save eta, hu, hv of the output columns (FP32, kStrip)
  static constexpr int kOffE = 0;
  static constexpr int kOffU = kOffE + 4 * kSeg;
  static constexpr int kOffV = kOffU + 4 * kSeg;
  static constexpr int kOffB = kOffV + 4 * kSeg;
  static constexpr int kOffOE = kOffB + 8 * kSeg;
  static constexpr int kOffOU = kOffOE + 4 * kStrip;
  static constexpr int kOffOV = kOffOU + 4 * kStrip;
  static constexpr int kSlot1 = kOffOE;
  static constexpr int kSlot2 = kOffOV + 4 * kStrip;
  static_assert(kStrip % 4 == 0 && kSeg % 4 == 0 && kSlot2 % 16 == 0,
                "bulk copies need 16-byte aligned rows and slots");
  static constexpr int slot(int stage) { return stage == 2 ? kSlot2 : kSlot1; }
};

// ---------------------------------------------------------------------------
// PTX helpers: approximate FP32 math (bulk copies and mbarriers: rkb_async.cuh)
// ---------------------------------------------------------------------------

__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Surface value of depth h over bed b; a dry cell stores the bed rounded
// down so that it reads back as h <= 0.
__device__ __forceinline__ float surface_of(double h, double b) {
  return h > 0.0 ? __double2float_rn(h + b) : __double2float_rd(b);
}

// minmod(a, b) (rki_kernel_flux.F90:380-393) as the median of (a, b, 0): 0
// when the signs differ or one is 0, else the value of smaller magnitude.
__device__ __forceinline__ float minmodf(float a, float b) {
  return fmaxf(fminf(a, b), fminf(fmaxf(a, b), 0.0f));
}

struct Slope {
  float e, u, v;
};

// Limited slope (rki_kernel_flux.F90:159-181): zero unless the cell is thick
// and both neighbours are wet.
__device__ __forceinline__ Slope slope(unsigned fm, unsigned fc, unsigned fp, float em, float ec,
                                       float ep, float um, float uc, float up, float vm, float vc,
                                       float vp) {
  const bool on = (fc & 2u) && (fm & 1u) && (fp & 1u);
  return Slope{on ? minmodf(ec - em, ep - ec) : 0.0f, on ? minmodf(uc - um, up - uc) : 0.0f,
               on ? minmodf(vc - vm, vp - vc) : 0.0f};
}

// Faces.  The Audusse hydrostatic depths max(0, eta - max(b_L, b_R))
// (rki_kernel_flux.F90:186-224) are FP64 differences: they are what keeps a
// lake at rest at rest, and in FP64 a dry island whose top lies a hair above
// the lake surface gets exactly zero depth on both sides of its shore faces.
//
// The reference hands each cell the face flux F together with its
// well-balanced terms, F - Q(h_hyd) + Q(h_face) with Q(h) = g/2 h^2
// (rki_kernel_flux.F90:361-369).  In FP32 those are differences of numbers of
// size g/2 h^2 (~490 in 10 m of water) whose rounding swamps the pressure
// gradient, so the same sums are regrouped to subtract only small numbers:
//
//   en = F - Q(h_hyd,L)                  flux in excess of the left hydrostatic pressure
//   dq = Q(h_hyd,R) - Q(h_hyd,L) = g/2 dy (h_hyd,L + h_hyd,R)
//
// with dy = h_hyd,R - h_hyd,L = eta_R - eta_L while both sides are wet (the
// bed cancels), else the difference of the clipped depths.  A cell with faces
// l, r then gets  en_r - en_l + dq_l + [Q(h_face,r) - Q(h_face,l)], the
// bracket being its own reconstruction term (cell_pressure).  At rest both
// surfaces are equal, so dy, dq, the fluxes and the cell term are exactly 0.
struct FaceF {
  float fh, en, dq, ft;
};

// Packed FP32 pairs (add / mul / fma on two lanes of a 64-bit register).
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 splat(float x) { return make_float2(x, x); }

struct FaceF2 {
  float2 fh, en, dq, ft;
};

// Two independent faces at once (two columns of a lane, or two neighbouring
// x-faces), each as described above: the FP64 depths and tests and the
// reciprocal / square-root approximations per face, the FP32 arithmetic on
// packed pairs (FADD2 / FMUL2 / FFMA2).  Per face: n = normal momentum, t =
// tangential momentum, hL / hR the reconstructed depths max(0, h_cell +- s/2),
// bL / bR the cell beds.
template <bool HLLC>
__device__ __forceinline__ FaceF2 face2(float2 eL, float2 nL, float2 tL, float2 hL, double bL0,
                                        double bL1, float2 eR, float2 nR, float2 tR, float2 hR,
                                        double bR0, double bR1) {
  const double bm0 = bL0 > bR0 ? bL0 : bR0, bm1 = bL1 > bR1 ? bL1 : bR1;
  const double yl0 = pos((double)eL.x - bm0), yl1 = pos((double)eL.y - bm1);
  const double yr0 = pos((double)eR.x - bm0), yr1 = pos((double)eR.y - bm1);
  const float2 yl = make_float2(__double2float_rn(yl0), __double2float_rn(yl1));
  const float2 yr = make_float2(__double2float_rn(yr0), __double2float_rn(yr1));
  const float2 de = sub2(eR, eL), dyy = sub2(yr, yl);
  const float2 dy = make_float2((yl.x > 0.0f && yr.x > 0.0f) ? de.x : dyy.x,
                                (yl.y > 0.0f && yr.y > 0.0f) ? de.y : dyy.y);
  const bool wl0 = yl0 > kDry, wl1 = yl1 > kDry, wr0 = yr0 > kDry, wr1 = yr1 > kDry;
  const float2 rl = make_float2(hL.x > kDryF ? rcp_approx(hL.x) : 0.0f,
                                hL.y > kDryF ? rcp_approx(hL.y) : 0.0f);
  const float2 rr = make_float2(hR.x > kDryF ? rcp_approx(hR.x) : 0.0f,
                                hR.y > kDryF ? rcp_approx(hR.y) : 0.0f);
  const float2 ul = mul2(nL, rl), vl = mul2(tL, rl), ur = mul2(nR, rr), vr = mul2(tR, rr);
  const float2 qnl = mul2(yl, ul), qtl = mul2(yl, vl), qnr = mul2(yr, ur), qtr = mul2(yr, vr);
  const float2 ml = make_float2(wl0 ? 1.0f : 0.0f, wl1 ? 1.0f : 0.0f);
  const float2 mr = make_float2(wr0 ? 1.0f : 0.0f, wr1 ? 1.0f : 0.0f);
  const float2 unl = mul2(ul, ml), utl = mul2(vl, ml), unr = mul2(ur, mr), utr = mul2(vr, mr);
  const float2 gl = mul2(splat(kGf), yl), gr = mul2(splat(kGf), yr);
  const float2 al = make_float2(sqrt_approx(gl.x), sqrt_approx(gl.y));
  const float2 ar = make_float2(sqrt_approx(gr.x), sqrt_approx(gr.y));
  const float2 a1 = sub2(unl, al), a2 = sub2(unr, ar), b1 = add2(unl, al), b2 = add2(unr, ar);
  const float2 c1 = fma2(splat(-2.0f), ar, unr), c2 = fma2(splat(2.0f), al, unl);
  const float2 sl = make_float2(!wr0 ? a1.x : (!wl0 ? c1.x : fminf(a1.x, a2.x)),
                                !wr1 ? a1.y : (!wl1 ? c1.y : fminf(a1.y, a2.y)));
  const float2 sr = make_float2(!wr0 ? c2.x : (!wl0 ? b2.x : fmaxf(b1.x, b2.x)),
                                !wr1 ? c2.y : (!wl1 ? b2.y : fmaxf(b1.y, b2.y)));
  FaceF2 o;
  o.dq = mul2(mul2(splat(kHalfGf), dy), add2(yl, yr));
  const float2 ln = mul2(qnl, unl), rn = mul2(qnr, unr);
  const float2 lt = mul2(qnl, utl), rt = mul2(qnr, utr);
  const float2 w = sub2(sr, sl);
  const float2 inv = make_float2(rcp_approx(w.x), rcp_approx(w.y));
  const float2 nsl = neg2(sl), nsr = neg2(sr);
  const float2 dqn = sub2(qnr, qnl);
  // F = F_L - s_L (F_R - F_L - s_R (U_R - U_L)) / (s_R - s_L)
  const float2 mfh = fma2(mul2(nsl, fma2(nsr, dy, dqn)), inv, qnl);
  const float2 men = fma2(mul2(nsl, fma2(nsr, dqn, add2(sub2(rn, ln), o.dq))), inv, ln);
  float2 mft;
  if (!HLLC) {
    mft = fma2(mul2(nsl, fma2(nsr, sub2(qtr, qtl), sub2(rt, lt))), inv, lt);
  } else {
    const float2 den = sub2(mul2(yr, sub2(unr, sr)), mul2(yl, sub2(unl, sl)));
    const float2 num = sub2(mul2(mul2(sl, yr), sub2(unr, sr)), mul2(mul2(sr, yl), sub2(unl, sl)));
    const float2 avg = mul2(splat(0.5f), add2(unl, unr));
    const float ss0 = fabsf(den.x) > kDryF ? num.x * rcp_approx(den.x) : avg.x;
    const float ss1 = fabsf(den.y) > kDryF ? num.y * rcp_approx(den.y) : avg.y;
    mft = mul2(mfh, make_float2(ss0 >= 0.0f ? utl.x : utr.x, ss1 >= 0.0f ? utl.y : utr.y));
  }
  const float2 rnq = add2(rn, o.dq);
  const bool up0 = sl.x >= 0.0f, dn0 = sr.x <= 0.0f, up1 = sl.y >= 0.0f, dn1 = sr.y <= 0.0f;
  o.fh = make_float2(up0 ? qnl.x : (dn0 ? qnr.x : mfh.x), up1 ? qnl.y : (dn1 ? qnr.y : mfh.y));
  o.en = make_float2(up0 ? ln.x : (dn0 ? rnq.x : men.x), up1 ? ln.y : (dn1 ? rnq.y : men.y));
  o.ft = make_float2(up0 ? lt.x : (dn0 ? rt.x : mft.x), up1 ? lt.y : (dn1 ? rt.y : mft.y));
  return o;
}

// Q(h_face,r) - Q(h_face,l) of a cell of depth hc whose limited surface slope
// is s: its reconstructed depths are hc + s/2 and hc - s/2 (clipped at 0), so
// the difference is g hc s unless a face depth is clipped.
__device__ __forceinline__ float cell_pressure(float hc, float s) {
  const float a = hc + 0.5f * s, c = hc - 0.5f * s;
  if (a >= 0.0f && c >= 0.0f) return kGf * hc * s;
  const float pa = fmaxf(a, 0.0f), pc = fmaxf(c, 0.0f);
  return kHalfGf * (pa - pc) * (pa + pc);
}

// The cell update below rounds every FP32 operation explicitly (the _rn
// intrinsics are never contracted or regrouped), so every build of the sweep
// (with or without the optional source terms, single or batched) gives the
// same bits.
__device__ __forceinline__ float sq_sum(float a, float b) { return __fmaf_rn(a, a, __fmul_rn(b, b)); }

// Clamp + KP07 + Froude backstop (rki_kernel_fused.F90:93-119) with the
// threshold tests on the FP64 depth; returns that depth.
__device__ __forceinline__ double protect(float& e, float& hu, float& hv, double b, float& h) {
  const double hd = (double)e - b;
  const bool neg = hd < 0.0, wet = hd >= kDry;
  h = neg ? 0.0f : __double2float_rn(hd);
  e = neg ? __double2float_rd(b) : e;
  hu = wet ? hu : 0.0f;
  hv = wet ? hv : 0.0f;
  const float h2 = __fmul_rn(h, h);
  const float h4 = __fmul_rn(h2, h2);
  const float q2 = sq_sum(hu, hv);
  const float lim = __fmul_rn(__fmul_rn(kFroude2G, h), h2);  // (Fr_max^2 g h) h^2
  if (wet && (h4 < kEps4F || q2 > lim)) {  // rare: KP07 and / or the Froude backstop
    if (h4 < kEps4F) {
      const float f = __fmul_rn(__fmul_rn(kSqrt2F, h2), rsqrt_approx(__fadd_rn(h4, kEps4F)));
      hu = __fmul_rn(hu, f);
      hv = __fmul_rn(hv, f);
    }
    const float q2b = sq_sum(hu, hv);
    if (q2b > lim) {
      const float sc = __fmul_rn(sqrt_approx(lim), rsqrt_approx(q2b));
      hu = __fmul_rn(hu, sc);
      hv = __fmul_rn(hv, sc);
    }
  }
  return neg ? 0.0 : hd;
}

// (|u| + c) along x and y with the KP07 velocity (rki_kernel_timestep.F90:52-66).
__device__ __forceinline__ void wave_speed32(double hd, float h, float hu, float hv, float& sx,
                                             float& sy) {
  sx = 0.0f;
  sy = 0.0f;
  if (hd > kDry) {  // the stage-2 epilogue's terms, rounded the same way
    const float c = sqrt_approx(__fmul_rn(kGf, h));
    const float h2 = __fmul_rn(h, h);
    const float f = __fmul_rn(__fmul_rn(kSqrt2F, h), rsqrt_approx(__fmaf_rn(h2, h2, kEps4F)));
    sx = __fmaf_rn(fabsf(hu), f, c);
    sy = __fmaf_rn(fabsf(hv), f, c);
  }
}

template <int C>
struct Row {
  float e[C], u[C], v[C];
  float h[C];     // cell depth (FP64 difference, rounded)
  double b[C];
  unsigned f[C];  // bit 0: h >= DRY_THRESHOLD, bit 1: h >= THIN_THRESHOLD (FP64 tests)
};

template <int C>
__device__ __forceinline__ void ld_f(const unsigned char* p, float (&o)[C]) {
  if (C == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    o[0] = t.x; o[1] = t.y; o[2 % C] = t.z; o[3 % C] = t.w;
  } else {
    const float2 t = *reinterpret_cast<const float2*>(p);
    o[0] = t.x; o[1] = t.y;
  }
}

template <int C>
__device__ __forceinline__ void ld_d(const unsigned char* p, double (&o)[C]) {
#pragma unroll
  for (int k = 0; k < C; k += 2) {
    const double2 t = *reinterpret_cast<const double2*>(p + 8 * k);
    o[k] = t.x;
    o[k + 1] = t.y;
  }
}

// This lane's C columns of a row from its ring slot (`base` = first column's
// index in the copied segment).
template <int C>
__device__ __forceinline__ void read_row(const unsigned char* slot, int base, Row<C>& r) {
  using L = Lay<C>;
  ld_f<C>(slot + L::kOffE + 4 * base, r.e);
  ld_f<C>(slot + L::kOffU + 4 * base, r.u);
  ld_f<C>(slot + L::kOffV + 4 * base, r.v);
  ld_d<C>(slot + L::kOffB + 8 * base, r.b);
#pragma unroll
  for (int k = 0; k < C; ++k) {
    const double hd = (double)r.e[k] - r.b[k];
    r.h[k] = __double2float_rn(hd);
    r.f[k] = (hd >= kDry ? 1u : 0u) | (hd >= kThin ? 2u : 0u);
  }
}

template <int C>
__device__ __forceinline__ void yslopes(const Row<C>& m, const Row<C>& c, const Row<C>& p,
                                        Slope (&s)[C]) {
#pragma unroll
  for (int k = 0; k < C; ++k)
    s[k] = slope(m.f[k], c.f[k], p.f[k], m.e[k], c.e[k], p.e[k], m.u[k], c.u[k], p.u[k], m.v[k],
                 c.v[k], p.v[k]);
}

// y-faces between rows lo and hi (normal momentum hv, tangential hu).
template <bool HLLC, int C>
__device__ __forceinline__ void yfaces(const Row<C>& lo, const Slope (&sl)[C], const Row<C>& hi,
                                       const Slope (&sh)[C], FaceF (&f)[C]) {
  const float2 half = splat(0.5f), nhalf = splat(-0.5f);
#pragma unroll
  for (int k = 0; k < C; k += 2) {  // columns k, k + 1 as one pair
    auto p = [&](float a, float b) { return make_float2(a, b); };
    const float2 hlo = fma2(half, p(sl[k].e, sl[k + 1].e), p(lo.h[k], lo.h[k + 1]));
    const float2 hhi = fma2(nhalf, p(sh[k].e, sh[k + 1].e), p(hi.h[k], hi.h[k + 1]));
    const FaceF2 o = face2<HLLC>(
        fma2(half, p(sl[k].e, sl[k + 1].e), p(lo.e[k], lo.e[k + 1])),
        fma2(half, p(sl[k].v, sl[k + 1].v), p(lo.v[k], lo.v[k + 1])),
        fma2(half, p(sl[k].u, sl[k + 1].u), p(lo.u[k], lo.u[k + 1])),
        p(fmaxf(hlo.x, 0.0f), fmaxf(hlo.y, 0.0f)), lo.b[k], lo.b[k + 1],
        fma2(nhalf, p(sh[k].e, sh[k + 1].e), p(hi.e[k], hi.e[k + 1])),
        fma2(nhalf, p(sh[k].v, sh[k + 1].v), p(hi.v[k], hi.v[k + 1])),
        fma2(nhalf, p(sh[k].u, sh[k + 1].u), p(hi.u[k], hi.u[k + 1])),
        p(fmaxf(hhi.x, 0.0f), fmaxf(hhi.y, 0.0f)), hi.b[k], hi.b[k + 1]);
    f[k] = FaceF{o.fh.x, o.en.x, o.dq.x, o.ft.x};
    f[k + 1] = FaceF{o.fh.y, o.en.y, o.dq.y, o.ft.y};
  }
}

// What a cell keeps of the face below it: mass flux, tangential (hu) flux,
// excess normal flux and hydrostatic pressure jump.
struct BotFace {
  float fh, ft, en, dq;
};

template <int C>
__device__ __forceinline__ void st_f(float* p, const float (&v)[C]) {
  if (C == 4)
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2 % C], v[3 % C]);
  else
    *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
}

// ---------------------------------------------------------------------------
// Stage kernel
// ---------------------------------------------------------------------------
// A field pointer at its point of use.  Batches keep a member's arguments in
// shared memory and read each pointer from there when it is needed (held in
// registers across the row loop they make the kernel spill); single
// simulations use the kernel-parameter copy.
template <bool BATCH, typename T>
__device__ __forceinline__ T* use_ptr(T* const& p) {
  if constexpr (!BATCH) {
    return p;
  } else {
    unsigned long long v;
    asm volatile("ld.shared.u64 %0, [%1];" : "=l"(v) : "r"(smem_u32(&p)));
    return reinterpret_cast<T*>(v);
  }
}

// The same for an int of the arguments (grid pitch and extents).
template <bool BATCH>
__device__ __forceinline__ int use_int(const int& p) {
  if constexpr (!BATCH) {
    return p;
  } else {
    int v;
    asm volatile("ld.shared.s32 %0, [%1];" : "=r"(v) : "r"(smem_u32(&p)));
    return v;
  }
}

template <bool BATCH>
__device__ __forceinline__ long long use_ll(const long long& p) {
  if constexpr (!BATCH) {
    return p;
  } else {
    long long v;
    asm volatile("ld.shared.s64 %0, [%1];" : "=l"(v) : "r"(smem_u32(&p)));
    return v;
  }
}

// STAGE 1: U^n (buffer cur) -> U* (S).  STAGE 2: U*, U^n -> U^{n+1} (cur^1).
// Block `blk` of the `nblk` blocks that cover one simulation.  PLAIN: no
// forcing, Coriolis or sponge (the common case), compiled without those paths.
// BATCH: `a` lives in shared memory.
template <int C, bool HLLC, int STAGE, bool PLAIN, bool BATCH = false>
__device__ __forceinline__ void sweep_body(const StepArgs32& a, unsigned blk, unsigned nblk) {
  using L = Lay<C>;
  constexpr int SLOT = L::slot(STAGE);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) unsigned long long bars[kWarps][kNbuf];
  __shared__ float rot[2];
  StepCtl* ctl = a.ctl;
  if (!ctl->active) return;
  using GRef = std::conditional_t<BATCH, const Grid&, const Grid>;
  GRef g = a.g;
  const Physics* phys = a.phys;
  const double dtd = ctl->dt;
  const float dt = (float)dtd;
  const int cur = ctl->cur;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (!PLAIN && threadIdx.x == 0) {
    // Coriolis rotation cos/sin(f dt) (rki_kernel_fused.F90:211-214)
    double sn = 0.0, cs = 1.0;
    if (fabs(phys->coriolis_f) > 1.0e-20) cr_sincos(phys->coriolis_f * dtd, sn, cs);
    rot[0] = (float)cs;
    rot[1] = (float)sn;
  }
  if (!PLAIN) __syncthreads();
  const bool has_cor = !PLAIN && fabs(phys->coriolis_f) > 1.0e-20;
  const bool friction = phys->manning_n > 0.0;
  const float gn2dt = (float)(kG * phys->manning_n * phys->manning_n) * dt;
  const bool forcing = !PLAIN && phys->forcing_active != 0;
  const bool sponge_on = !PLAIN && a.bc->sponge_width > 0 && a.bc->sponge_strength > 0.0;
  const float rdx = (float)(1.0 / g.dx), rdy = (float)(1.0 / g.dy);
  const float cosf_ = rot[0], sinf_ = rot[1];

  using FRef = std::conditional_t<BATCH, const FieldSet32&, const FieldSet32>;
  FRef in = STAGE == 2 ? a.S : (cur ? a.U1 : a.U0);
  FRef old = cur ? a.U1 : a.U0;
  FRef out = STAGE == 1 ? a.S : (cur ? a.U0 : a.U1);

  const unsigned nw = nblk * kWarps;
  const unsigned gw = blk * kWarps + warp;
  double part = 0.0, sponge_d = 0.0;
  float wsx = 0.0f, wsy = 0.0f;
  bool bad = false;  // a new surface of this lane is not finite (a NaN in the
                     // momenta reaches the surface through the next fluxes)

  if (gw < (unsigned)(a.nstrips * a.nrowblk)) {  // warp-uniform
    const int strip = (int)(gw % (unsigned)a.nstrips);
    const int rb = (int)(gw / (unsigned)a.nstrips);
    const int x0 = g.ng + strip * L::kStrip;
    const int y0 = g.ng + rb * a.rows;
    const int yend = min(y0 + a.rows, g.nyt - g.ng);
    const int r0 = y0 - 2, rlast = yend + 1;
    const int li = lane == 31 ? -1 : lane;   // column group of this lane in the ring
    const int base = 4 + C * li;             // its first column in the copied segment
    const bool out_lane = lane < 30;
    unsigned char* ring = smem + warp * (kNbuf * SLOT);
    const uint32_t ring_s = smem_u32(ring);
    const uint32_t bar0 = smem_u32(&bars[warp][0]);
    if (lane == 0) {
      for (int s = 0; s < kNbuf; ++s) mbar_init(bar0 + 8 * s, 1);
      fence_mbar_init();
    }
    __syncwarp();

    // Ring bookkeeping without divisions: rows r0, r0+1, ... go to slots 0, 1,
    // ..., kNbuf-1, 0, ...; bit s of `ph` is the parity of the next completion
    // to wait for on slot s.
    auto issue = [&](int r, int s) {  // lane 0
      const uint32_t dst = ring_s + s * SLOT, bar = bar0 + 8 * s;
      const bool with_old = STAGE == 2 && r >= y0 && r < yend;
      mbar_expect_tx(bar, with_old ? L::kSlot2 : L::kSlot1);
      const size_t ro = (size_t)r * (size_t)use_int<BATCH>(g.pitch) + (size_t)(x0 - 4);
      bulk_g2s(dst + L::kOffE, use_ptr<BATCH>(in.eta) + ro, 4 * L::kSeg, bar);
      bulk_g2s(dst + L::kOffU, use_ptr<BATCH>(in.hu) + ro, 4 * L::kSeg, bar);
      bulk_g2s(dst + L::kOffV, use_ptr<BATCH>(in.hv) + ro, 4 * L::kSeg, bar);
      bulk_g2s(dst + L::kOffB, use_ptr<BATCH>(a.b) + ro, 8 * L::kSeg, bar);
      if (with_old) {
        const size_t ro2 = ro + 4;
        bulk_g2s(dst + L::kOffOE, use_ptr<BATCH>(old.eta) + ro2, 4 * L::kStrip, bar);
        bulk_g2s(dst + L::kOffOU, use_ptr<BATCH>(old.hu) + ro2, 4 * L::kStrip, bar);
        bulk_g2s(dst + L::kOffOV, use_ptr<BATCH>(old.hv) + ro2, 4 * L::kStrip, bar);
      }
    };
    auto nxt = [](int s) { return s + 1 == kNbuf ? 0 : s + 1; };
    uint32_t ph = 0;
    int ws = 0;  // slot of the next row to wait for
    // A wait that gives up leaves its slot the next to wait for, so the
    // drain below waits for that row's copies again.
    auto wait_next = [&](long long limit) {
      if (!mbar_wait(bar0 + 8 * ws, (ph >> ws) & 1u, limit)) return -1;
      ph ^= 1u << ws;
      const int s_done = ws;
      ws = nxt(ws);
      return s_done;
    };

    int issued = min(r0 + kNbuf - 1, rlast);
    if (lane == 0)
      for (int r = r0; r <= issued; ++r) issue(r, r - r0);

    // prologue: rows y0-2 .. y0+1, slopes of y0-1 and y0, face y0-1/2
    Row<C> A, B, Cr, D, E;
    bool ok = true;
    int waited = r0 - 1;  // last row whose copies have landed
    auto take = [&](int r, Row<C>& R) {
      if (!ok) return;
      const int sl = wait_next(use_ll<BATCH>(a.wait_cycles));
      ok = sl >= 0;
      if (ok) {
        read_row<C>(ring + sl * SLOT, base, R);
        waited = r;
      }
    };
    take(r0, A);
    take(r0 + 1, B);
    take(y0, Cr);
    take(y0 + 1, D);
    Slope sC[C];
    BotFace bot[C];
    if (ok) {
      Slope sB[C];
      yslopes<C>(A, B, Cr, sB);
      yslopes<C>(B, Cr, D, sC);
      FaceF f[C];
      yfaces<HLLC, C>(B, sB, Cr, sC, f);
#pragma unroll
      for (int k = 0; k < C; ++k) bot[k] = BotFace{f[k].fh, f[k].ft, f[k].en, f[k].dq};
      __syncwarp();
      if (lane == 0) {
        fence_proxy_async();
        for (int r = r0 + kNbuf; r <= min(r0 + kNbuf + 1, rlast); ++r) issue(r, r - r0 - kNbuf);
      }
      issued = min(r0 + kNbuf + 1, rlast);
    }

    const int src_r = (lane + 1) & 31, src_l = (lane + 31) & 31;
    int sj = 2;  // slot of row j
    for (int j = y0; ok && j < yend; ++j) {
      const int sn = wait_next(use_ll<BATCH>(a.wait_cycles));  // row j + 2
      ok = sn >= 0;
      if (!ok) break;
      waited = j + 2;
      read_row<C>(ring + sn * SLOT, base, E);
      Slope sD[C];
      yslopes<C>(Cr, D, E, sD);
      FaceF top[C];
      yfaces<HLLC, C>(Cr, sC, D, sD, top);

      // ---- x direction on row j: neighbour columns by shuffle around the ring ----
      const float pe = __shfl_sync(kFull, Cr.e[0], src_r);
      const float pu = __shfl_sync(kFull, Cr.u[0], src_r);
      const float pv = __shfl_sync(kFull, Cr.v[0], src_r);
      const unsigned pf = __shfl_sync(kFull, Cr.f[0], src_r);
      const float me = __shfl_sync(kFull, Cr.e[C - 1], src_l);
      const float mu = __shfl_sync(kFull, Cr.u[C - 1], src_l);
      const float mv = __shfl_sync(kFull, Cr.v[C - 1], src_l);
      const unsigned mf = __shfl_sync(kFull, Cr.f[C - 1], src_l);
      Slope sx[C];
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const float em = k ? Cr.e[k - 1] : me, um = k ? Cr.u[k - 1] : mu, vm = k ? Cr.v[k - 1] : mv;
        const unsigned fm = k ? Cr.f[k - 1] : mf;
        const float ep = k < C - 1 ? Cr.e[k + 1] : pe, up = k < C - 1 ? Cr.u[k + 1] : pu;
        const float vp = k < C - 1 ? Cr.v[k + 1] : pv;
        const unsigned fp = k < C - 1 ? Cr.f[k + 1] : pf;
        sx[k] = slope(fm, Cr.f[k], fp, em, Cr.e[k], ep, um, Cr.u[k], up, vm, Cr.v[k], vp);
      }
      // left state of this lane's first x-face: the left lane's last column
      const float le = __shfl_sync(kFull, Cr.e[C - 1] + 0.5f * sx[C - 1].e, src_l);
      const float lu = __shfl_sync(kFull, Cr.u[C - 1] + 0.5f * sx[C - 1].u, src_l);
      const float lv = __shfl_sync(kFull, Cr.v[C - 1] + 0.5f * sx[C - 1].v, src_l);
      const float lh = __shfl_sync(kFull, fmaxf(Cr.h[C - 1] + 0.5f * sx[C - 1].e, 0.0f), src_l);
      const double lb = __shfl_sync(kFull, Cr.b[C - 1], src_l);
      FaceF xf[C];
      {
        const float2 half = splat(0.5f), nhalf = splat(-0.5f);
        auto p = [&](float a, float b) { return make_float2(a, b); };
#pragma unroll
        for (int k = 0; k < C; k += 2) {
          // left states: column k - 1 reconstructed right (the left lane's last for k = 0)
          const float eL0 = k ? Cr.e[k - 1] + 0.5f * sx[k - 1].e : le;
          const float uL0 = k ? Cr.u[k - 1] + 0.5f * sx[k - 1].u : lu;
          const float vL0 = k ? Cr.v[k - 1] + 0.5f * sx[k - 1].v : lv;
          const float hL0 = k ? fmaxf(Cr.h[k - 1] + 0.5f * sx[k - 1].e, 0.0f) : lh;
          const double bL0 = k ? Cr.b[k - 1] : lb;
          const FaceF2 o = face2<HLLC>(
              p(eL0, Cr.e[k] + 0.5f * sx[k].e), p(uL0, Cr.u[k] + 0.5f * sx[k].u),
              p(vL0, Cr.v[k] + 0.5f * sx[k].v), p(hL0, fmaxf(Cr.h[k] + 0.5f * sx[k].e, 0.0f)), bL0,
              Cr.b[k], fma2(nhalf, p(sx[k].e, sx[k + 1].e), p(Cr.e[k], Cr.e[k + 1])),
              fma2(nhalf, p(sx[k].u, sx[k + 1].u), p(Cr.u[k], Cr.u[k + 1])),
              fma2(nhalf, p(sx[k].v, sx[k + 1].v), p(Cr.v[k], Cr.v[k + 1])),
              p(fmaxf(Cr.h[k] - 0.5f * sx[k].e, 0.0f), fmaxf(Cr.h[k + 1] - 0.5f * sx[k + 1].e, 0.0f)),
              Cr.b[k], Cr.b[k + 1]);
          xf[k] = FaceF{o.fh.x, o.en.x, o.dq.x, o.ft.x};
          xf[k + 1] = FaceF{o.fh.y, o.en.y, o.dq.y, o.ft.y};
        }
      }
      // right face of the last column = the right lane's first face
      const float rfh = __shfl_sync(kFull, xf[0].fh, src_r);
      const float ren = __shfl_sync(kFull, xf[0].en, src_r);
      const float rft = __shfl_sync(kFull, xf[0].ft, src_r);

      // RK2 save of this row (stage 2), then release the slot of row j
      float oe[C], ou[C], ov[C];
      if (STAGE == 2) {
#pragma unroll
        for (int k = 0; k < C; ++k) { oe[k] = 0.0f; ou[k] = 0.0f; ov[k] = 0.0f; }
        if (out_lane) {
          const unsigned char* pj = ring + sj * SLOT;
          ld_f<C>(pj + L::kOffOE + 4 * C * lane, oe);
          ld_f<C>(pj + L::kOffOU + 4 * C * lane, ou);
          ld_f<C>(pj + L::kOffOV + 4 * C * lane, ov);
        }
      }
      __syncwarp();
      if (j + kNbuf <= rlast) {
        if (lane == 0) {
          fence_proxy_async();
          issue(j + kNbuf, sj);
        }
        issued = j + kNbuf;
      }
      sj = nxt(sj);

      // ---- cell updates of row j ----
      float ne[C], nu[C], nv[C];
      const int ib = x0 + C * li;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        const float Rfh = k < C - 1 ? xf[k + 1].fh : rfh;
        const float Ren = k < C - 1 ? xf[k + 1].en : ren;
        const float Rft = k < C - 1 ? xf[k + 1].ft : rft;
        const float px = cell_pressure(Cr.h[k], sx[k].e), py = cell_pressure(Cr.h[k], sC[k].e);
        const float dE = __fmaf_rn(-__fsub_rn(top[k].fh, bot[k].fh), rdy,
                                   -__fmul_rn(__fsub_rn(Rfh, xf[k].fh), rdx));
        const float dU = __fmaf_rn(
            -__fsub_rn(top[k].ft, bot[k].ft), rdy,
            -__fmul_rn(__fadd_rn(__fadd_rn(__fsub_rn(Ren, xf[k].en), xf[k].dq), px), rdx));
        const float dV = __fmaf_rn(
            -__fadd_rn(__fadd_rn(__fsub_rn(top[k].en, bot[k].en), bot[k].dq), py), rdy,
            -__fmul_rn(__fsub_rn(Rft, xf[k].ft), rdx));
        float e = __fmaf_rn(dt, dE, Cr.e[k]);
        float hu = __fmaf_rn(dt, dU, Cr.u[k]);
        float hv = __fmaf_rn(dt, dV, Cr.v[k]);
        const double bc = Cr.b[k];
        float h;
        const double hd = protect(e, hu, hv, bc, h);
        const int i = ib + k;
        // forcing reads stay in bounds
        const bool valid = out_lane && i < use_int<BATCH>(g.nxt) - use_int<BATCH>(g.ng);
        if (friction) {
          // Manning friction (rki_kernel_fused.F90:121-130): hu / (1 + dt g n^2 |q| h^-7/3)
          const float den = __fmaf_rn(__fmul_rn(gn2dt, sqrt_approx(sq_sum(hu, hv))),
                                      __powf(fmaxf(h, kDryF), -7.0f / 3.0f), 1.0f);
          const float r = hd > kDry ? rcp_approx(den) : 1.0f;
          hu = __fmul_rn(hu, r);
          hv = __fmul_rn(hv, r);
        }
        if ((forcing || has_cor) && hd > kDry) {
          if (forcing && valid) {  // wind, pressure gradient (rki_kernel_fused.F90:131-146)
            const size_t q = (size_t)i + (size_t)j * (size_t)a.fpitch;
            hu = __fmaf_rn(dt, (float)(a.fo.wind_x[q] / kRho), hu);
            hv = __fmaf_rn(dt, (float)(a.fo.wind_y[q] / kRho), hv);
            const float dpdx = (float)((a.fo.atm[q + 1] - a.fo.atm[q - 1]) / (2.0 * g.dx));
            const float dpdy = (float)((a.fo.atm[q + a.fpitch] - a.fo.atm[q - a.fpitch]) / (2.0 * g.dy));
            const float dth = __fmul_rn(dt, h);
            hu = __fmaf_rn(-__fmul_rn(dth, dpdx), (float)(1.0 / kRho), hu);
            hv = __fmaf_rn(-__fmul_rn(dth, dpdy), (float)(1.0 / kRho), hv);
          }
          if (has_cor) {
            const float uo = hu, vo = hv;
            hu = __fmaf_rn(uo, cosf_, __fmul_rn(vo, sinf_));
            hv = __fmaf_rn(vo, cosf_, -__fmul_rn(uo, sinf_));
          }
        }
        if (forcing && valid)
          e = __fmaf_rn(dt, (float)a.fo.precip[(size_t)i + (size_t)j * (size_t)a.fpitch], e);
        double hfin = hd;
        if (STAGE == 2) {  // RK2 average and second clamp (rki_kernel_fused.F90:435-463)
          e = __fmul_rn(0.5f, __fadd_rn(oe[k], e));
          hu = __fmul_rn(0.5f, __fadd_rn(ou[k], hu));
          hv = __fmul_rn(0.5f, __fadd_rn(ov[k], hv));
          hfin = protect(e, hu, hv, bc, h);
        }
        if (sponge_on) {
          const double alpha = sponge_alpha(a.bc, g, i, j);
          if (alpha > 0.0) {
            const float fa = __fmul_rn(dt, (float)alpha);
            const float de = __fmul_rn(-fa, __fadd_rn(fmaxf(h, 0.0f), -(float)a.bc->sponge_h_ref));
            e = __fadd_rn(e, de);
            hu = __fmaf_rn(-fa, hu, hu);
            hv = __fmaf_rn(-fa, hv, hv);
            if (valid) sponge_d += (double)de;
            hfin = (double)e - bc;
            h = fmaxf((float)hfin, 0.0f);
          }
        }
        ne[k] = e;
        nu[k] = hu;
        nv[k] = hv;
        part += valid ? (double)dE : 0.0;
        if (STAGE == 2) {
          const float c = sqrt_approx(__fmul_rn(kGf, h));
          const float h2 = __fmul_rn(h, h);
          const float f =
              __fmul_rn(__fmul_rn(kSqrt2F, h), rsqrt_approx(__fmaf_rn(h2, h2, kEps4F)));
          const bool w = valid && hfin > kDry;
          wsx = fmaxf(wsx, w ? __fmaf_rn(fabsf(hu), f, c) : 0.0f);
          wsy = fmaxf(wsy, w ? __fmaf_rn(fabsf(hv), f, c) : 0.0f);
          bad = bad || (valid && !isfinite(e));
        }
      }
      if (out_lane) {
        const int xend = use_int<BATCH>(g.nxt) - use_int<BATCH>(g.ng);
        const size_t q = (size_t)j * (size_t)use_int<BATCH>(g.pitch) + (size_t)ib;
        if (ib + C - 1 < xend) {
          st_f<C>(use_ptr<BATCH>(out.eta) + q, ne);
          st_f<C>(use_ptr<BATCH>(out.hu) + q, nu);
          st_f<C>(use_ptr<BATCH>(out.hv) + q, nv);
        } else {
#pragma unroll
          for (int k = 0; k < C; ++k)
            if (ib + k < xend) {
              use_ptr<BATCH>(out.eta)[q + k] = ne[k];
              use_ptr<BATCH>(out.hu)[q + k] = nu[k];
              use_ptr<BATCH>(out.hv)[q + k] = nv[k];
            }
        }
      }
      // rotate the row window
      Cr = D;
      D = E;
#pragma unroll
      for (int k = 0; k < C; ++k) {
        sC[k] = sD[k];
        bot[k] = BotFace{top[k].fh, top[k].ft, top[k].en, top[k].dq};
      }
    }
    if (!ok) {
      // a copy did not arrive in time: flag it and let every copy this warp
      // issued land (each wait bounded by the default limit, whatever limit
      // gave up) before the shared memory goes away
      if (lane == 0) atomicExch(&ctl->error, kErrWait);
      for (int r = waited + 1; r <= issued; ++r)
        if (wait_next(kWaitCyclesDefault) < 0) break;
    }
  }

  // per-warp partials (fixed order), CFL maxima, last block closes the step
  part = warp_sum(part);
  sponge_d = warp_sum(sponge_d);
  if (STAGE == 2) {
    wsx = (float)warp_max((double)wsx);
    wsy = (float)warp_max((double)wsy);
    bad = __any_sync(kFull, bad);
  }
  if (lane == 0) {
    double* P = a.partials + (size_t)(STAGE - 1) * 2 * nw;
    P[gw] = part;
    P[nw + gw] = sponge_d;
    if (STAGE == 2) {
      atomic_max_pos(&ctl->msx_next, (double)wsx);
      atomic_max_pos(&ctl->msy_next, (double)wsy);
      if (bad) atomicExch(&ctl->error, kErrNonFinite);
    }
  }
  if (STAGE != 2) return;
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&ctl->done_blocks, 1u) == nblk - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_step(g, ctl, phys, a.partials, nw, dtd, cur);
}

// True when the stage has no forcing, Coriolis or sponge terms.
__device__ __forceinline__ bool plain_physics(const StepArgs32& a) {
  return a.phys->forcing_active == 0 && !(fabs(a.phys->coriolis_f) > 1.0e-20) &&
         !(a.bc->sponge_width > 0 && a.bc->sponge_strength > 0.0);
}

// The host picks the PLAIN build from its copy of the physics; a launch whose
// device-side physics disagree computes nothing and reports kErrPhysics.
__device__ __forceinline__ bool plain_mismatch(const StepArgs32& a) {
  if (plain_physics(a)) return false;
  if (threadIdx.x == 0) atomicExch(&a.ctl->error, kErrPhysics);
  return true;
}

template <int C, bool HLLC, int STAGE, bool PLAIN>
__global__ void __launch_bounds__(kWarps * 32, C == 2 ? 4 : 2) k_sweep(StepArgs32 a) {
  if (PLAIN && plain_mismatch(a)) return;
  sweep_body<C, HLLC, STAGE, PLAIN>(a, blockIdx.x, gridDim.x);
}

// Every simulation of a batch in one launch: map[blockIdx.x] = (simulation,
// block index within that simulation's sweep).
template <int C, bool HLLC, int STAGE, bool PLAIN>
__global__ void __launch_bounds__(kWarps * 32, C == 2 ? 4 : 2)
    k_sweep_batch(const StepArgs32* __restrict__ args, const int2* __restrict__ map) {
  __shared__ StepArgs32 sa;
  const int2 m = map[blockIdx.x];
  if (threadIdx.x == 0) sa = args[m.x];
  __syncthreads();
  const unsigned nblk = (unsigned)((sa.nstrips * sa.nrowblk + kWarps - 1) / kWarps);
  if (PLAIN && plain_mismatch(sa)) return;
  sweep_body<C, HLLC, STAGE, PLAIN, true>(sa, (unsigned)m.y, nblk);
}

// ---------------------------------------------------------------------------
// Boundary conditions in surface form (rki_boundary.F90:40-552)
// ---------------------------------------------------------------------------
// Same edge walk as the FP64 fill; depths are read as max(0, eta - b) in FP64
// and ghost surfaces written as surface_of(h, b).  A wall ghost takes the
// mirrored cell's surface unchanged (its bed is the mirrored bed).
__device__ __forceinline__ void bc32_body(const StepArgs32& a, int stage, int w, int t,
                                          bool writer) {
  const Grid& g = a.g;
  StepCtl* ctl = a.ctl;
  const BcParams* bc = a.bc;
  double dt;
  const bool active = step_begin(ctl, a.phys, g, dt);
  if (writer) {
    ctl->active = active ? 1 : 0;
    ctl->dt = dt;
  }
  if (!active) return;
  const int type = bc->type[w];
  if (type == kNested) return;
  const Edge e = make_edge(w, g);
  if (t >= e.n_tan) return;
  // stage 9: the fill before dt of a narrow grid (see bc_body in the FP64
  // step): time t, the previous dt; stage 1 of a narrow grid also writes the
  // scratch buffer that stage 2 fills next
  const double time = stage == 2 ? ctl->t + dt : ctl->t;
  const double dtb = stage == 9 ? ctl->dt_prev : dt;
  const int cur = ctl->cur;
  const int wide = g.ng > 2 ? g.ng : 2;
  const bool narrow = g.nx_phys() < wide || g.ny_phys() < wide;
  const FieldSet32 F = stage == 2 ? a.S : (cur ? a.U1 : a.U0);
  const FieldSet32 N = stage == 2 ? (cur ? a.U0 : a.U1) : a.S;
  const bool both = stage == 2 || (stage == 1 && narrow);
  double* b = a.b;
  auto depth = [&](size_t q) { return pos((double)F.eta[q] - b[q]); };
  auto put = [&](int ig, int jg, double vh, double vu, double vv) {
    const size_t q = g.at(ig, jg);
    const float ve = surface_of(vh, b[q]);
    const float fu = (float)vu, fv = (float)vv;
    F.eta[q] = ve; F.hu[q] = fu; F.hv[q] = fv;
    if (both) { N.eta[q] = ve; N.hu[q] = fu; N.hv[q] = fv; }
  };
  const int ii = e.ig0 + t * e.dit - e.din;
  const int ji = e.jg0 + t * e.djt - e.djn;

  if (type == kWall || type == kSponge) {
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const size_t m = g.at(ig - (2 * k - 1) * e.din, jg - (2 * k - 1) * e.djn);
      const size_t q = g.at(ig, jg);
      b[q] = b[m];
      const float ve = F.eta[m];
      const float fu = e.normal_u ? -F.hu[m] : F.hu[m];
      const float fv = e.normal_u ? F.hv[m] : -F.hv[m];
      F.eta[q] = ve; F.hu[q] = fu; F.hv[q] = fv;
      if (both) { N.eta[q] = ve; N.hu[q] = fu; N.hv[q] = fv; }
    }
    return;
  }
  const size_t qi = g.at(ii, ji);
  const double hi = depth(qi);
  const double qu = (double)F.hu[qi];
  const double qv = (double)F.hv[qi];
  if (type == kOpen || type == kTidal) {
    const bool prescribe = type == kTidal;
    const double eta_ext = prescribe ? tidal_eta(bc, time) : 0.0;
    const double ei = hi + b[qi];
    const double hmax = dmax(hi, 1.0e-6);
    const double c = sqrt(kG * hmax);
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const double hg = prescribe ? pos(eta_ext - b[g.at(ig, jg)]) : hi;
      const double qn = hg * ((e.normal_u ? qu : qv) / hmax + e.sgn * c * (ei - eta_ext) / hmax);
      if (e.normal_u) put(ig, jg, hg, qn, qv);
      else put(ig, jg, hg, qu, qn);
    }
  } else if (type == kInflow || type == kDischarge) {
    const double in_sgn = -e.sgn;
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const double qn = type == kInflow ? in_sgn * hi * bc->inflow_velocity
                                        : in_sgn * bc->discharge_flux;
      if (e.normal_u) put(ig, jg, hi, qn, qv);
      else put(ig, jg, hi, qu, qn);
    }
  } else if (type == kClamped) {
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      put(ig, jg, pos(bc->clamped_elevation - b[g.at(ig, jg)]), qu, qv);
    }
  } else if (type == kChapman) {
    double* eo = a.eta_old[w];
    const double dd = e.normal_u ? g.dx : g.dy;
    const double ei = hi + b[qi];
    const double eov = stage == 1 ? ei : eo[t];
    const double hmax = dmax(hi, 1.0e-6);
    const double c = sqrt(kG * hmax);
    const int i2 = ii - e.din;
    const int j2 = ji - e.djn;
    double eg;
    if (dtb > 0.0) {
      const double detadt = (ei - eov) / dtb;
      double detadx = 0.0;
      if (i2 >= 0 && i2 < g.nxt && j2 >= 0 && j2 < g.nyt) {
        const size_t q2 = g.at(i2, j2);
        detadx = (depth(q2) + b[q2] - ei) / dd;
      }
      double cp = fabs(detadx) > 1.0e-10 ? -detadt / detadx : 0.0;
      cp = pos(dmin(cp, c));
      eg = eov - cp * dtb / dd * (eov - ei);
    } else {
      eg = ei;
    }
    for (int k = 1; k <= g.ng; ++k) {
      const int ig = e.ig0 + (k - 1) * e.din + t * e.dit;
      const int jg = e.jg0 + (k - 1) * e.djn + t * e.djt;
      const double hg = pos(eg - b[g.at(ig, jg)]);
      const double qn = hg * ((e.normal_u ? qu : qv) / hmax + e.sgn * c * (ei - eg) / hmax);
      if (e.normal_u) put(ig, jg, hg, qn, qv);
      else put(ig, jg, hg, qu, qn);
    }
    eo[t] = ei;
  }
}

__global__ void k_bc32(StepArgs32 a, int stage, int e0, int first_launch) {
  bc32_body(a, stage, e0 + (int)blockIdx.y, (int)(blockIdx.x * blockDim.x + threadIdx.x),
            first_launch && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0);
}

__global__ void k_bc32_batch(const StepArgs32* __restrict__ args, int stage, int e0,
                             int first_launch) {
  __shared__ StepArgs32 sa;
  if (threadIdx.x == 0) sa = args[blockIdx.z];
  __syncthreads();
  bc32_body(sa, stage, e0 + (int)blockIdx.y, (int)(blockIdx.x * blockDim.x + threadIdx.x),
            first_launch && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0);
}

// CFL maxima of the current state (before the first step, or after the host
// changed the state).
__global__ void k_max_speed32(StepArgs32 a) {
  const Grid g = a.g;
  StepCtl* ctl = a.ctl;
  const FieldSet32 F = ctl->cur ? a.U1 : a.U0;
  const int nxp = g.nx_phys(), nyp = g.ny_phys();
  const long long n = (long long)nxp * nyp;
  float mx = 0.0f, my = 0.0f;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const size_t q = g.at(g.ng + (int)(k % nxp), g.ng + (int)(k / nxp));
    const double hd = (double)F.eta[q] - a.b[q];
    float sx, sy;
    wave_speed32(hd, fmaxf((float)hd, 0.0f), F.hu[q], F.hv[q], sx, sy);
    mx = fmaxf(mx, sx);
    my = fmaxf(my, sy);
  }
  const double dmx = warp_max((double)mx), dmy = warp_max((double)my);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&ctl->msx_next, dmx);
    atomic_max_pos(&ctl->msy_next, dmy);
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

// FP64 (h, hu, hv) -> FP32 (eta, hu, hv), every cell incl. ghosts; with
// `bed_out`, also copies the bed into the surface form's layout.
__global__ void k_to_surface(Grid g64, Grid g32, FieldSet src, const double* __restrict__ b64,
                             FieldSet32 dst, double* __restrict__ bed_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g64.nxt) return;
  for (int j = blockIdx.y; j < g64.nyt; j += gridDim.y) {
    const size_t p = g64.at(i, j), q = g32.at(i, j);
    const double b = b64[p];
    if (src.h) dst.eta[q] = surface_of(src.h[p], b);  // a null field is left as it is
    if (src.hu) dst.hu[q] = (float)src.hu[p];
    if (src.hv) dst.hv[q] = (float)src.hv[p];
    if (bed_out) bed_out[q] = b;
  }
}

// FP32 surface form -> FP64 depth form (h = max(0, eta - b)); with
// `bed_out`, also copies the bed back (wall fills mirror it into the ghosts).
__global__ void k_to_depth(Grid g32, Grid g64, FieldSet32 src, const double* __restrict__ b32,
                           FieldSet dst, double* __restrict__ bed_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g32.nxt) return;
  for (int j = blockIdx.y; j < g32.nyt; j += gridDim.y) {
    const size_t q = g32.at(i, j), p = g64.at(i, j);
    const double b = b32[q];
    dst.h[p] = pos((double)src.eta[q] - b);
    dst.hu[p] = (double)src.hu[q];
    dst.hv[p] = (double)src.hv[q];
    if (bed_out) bed_out[p] = b;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

template <int C>
static void shape_t(const Grid& g, int rows, int& nstrips, int& nrowblk) {
  nstrips = (g.nx_phys() + Lay<C>::kStrip - 1) / Lay<C>::kStrip;
  nrowblk = (g.ny_phys() + rows - 1) / rows;
}

void sweep_shape(const Grid& g, int rows, int cpl, int& nstrips, int& nrowblk) {
  if (cpl == 4)
    shape_t<4>(g, rows, nstrips, nrowblk);
  else
    shape_t<2>(g, rows, nstrips, nrowblk);
}

// Columns (from column 0 of a row) the sweep's copies touch.
template <int C>
static size_t extent_t(const Grid& g) {
  int ns, nr;
  shape_t<C>(g, 1, ns, nr);
  return (size_t)g.ng + (size_t)(ns - 1) * Lay<C>::kStrip - 4 + Lay<C>::kSeg;
}

size_t sweep_row_extent(const Grid& g) {
  const size_t a = extent_t<2>(g), b = extent_t<4>(g);
  return a > b ? a : b;
}

size_t partials_doubles32(const Grid& g, int rows) {
  int ns, nr;
  shape_t<2>(g, rows, ns, nr);  // the narrower strips give the most warps
  const size_t blocks = ((size_t)ns * nr + kWarps - 1) / kWarps;
  return 4 * blocks * kWarps;
}

template <int C, bool HLLC, int STAGE>
static cudaError_t set_smem() {
  const int bytes = kWarps * kNbuf * Lay<C>::slot(STAGE);
  cudaError_t e = cudaFuncSetAttribute(k_sweep<C, HLLC, STAGE, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep<C, HLLC, STAGE, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

cudaError_t configure_kernels32() {
  cudaError_t e = set_smem<2, false, 1>();
  if (e == cudaSuccess) e = set_smem<2, false, 2>();
  if (e == cudaSuccess) e = set_smem<2, true, 1>();
  if (e == cudaSuccess) e = set_smem<2, true, 2>();
  if (e == cudaSuccess) e = set_smem<4, false, 1>();
  if (e == cudaSuccess) e = set_smem<4, false, 2>();
  if (e == cudaSuccess) e = set_smem<4, true, 1>();
  if (e == cudaSuccess) e = set_smem<4, true, 2>();
  return e;
}

template <int C>
static int auto_rows_t(const Grid& g) {
  int per_sm = 0, sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<C, false, 2, true>, kWarps * 32,
                                                    kWarps * kNbuf * Lay<C>::kSlot2) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (sms < 1) sms = 148;
  int ns, nr;
  shape_t<C>(g, 1, ns, nr);
  const int warps = per_sm * sms * kWarps;
  int nrb = warps / ns;
  if (nrb < 1) nrb = 1;
  int rows = (g.ny_phys() + nrb - 1) / nrb;
  if (rows < 16) rows = 16;
  return rows;
}

int auto_rows32(const Grid& g, int cpl) { return cpl == 4 ? auto_rows_t<4>(g) : auto_rows_t<2>(g); }

template <int C, int STAGE>
static cudaError_t launch_sweep_t(const StepArgs32& a, cudaStream_t s) {
  const unsigned work = (unsigned)(a.nstrips * a.nrowblk);
  const unsigned blocks = (work + kWarps - 1) / kWarps;
  const size_t bytes = (size_t)kWarps * kNbuf * Lay<C>::slot(STAGE);
  if (a.hllc) {
    if (a.plain)
      k_sweep<C, true, STAGE, true><<<blocks, kWarps * 32, bytes, s>>>(a);
    else
      k_sweep<C, true, STAGE, false><<<blocks, kWarps * 32, bytes, s>>>(a);
  } else {
    if (a.plain)
      k_sweep<C, false, STAGE, true><<<blocks, kWarps * 32, bytes, s>>>(a);
    else
      k_sweep<C, false, STAGE, false><<<blocks, kWarps * 32, bytes, s>>>(a);
  }
  return cudaGetLastError();
}

template <int STAGE>
static cudaError_t launch_sweep(const StepArgs32& a, cudaStream_t s) {
  return a.cpl == 4 ? launch_sweep_t<4, STAGE>(a, s) : launch_sweep_t<2, STAGE>(a, s);
}

static cudaError_t launch_bc32_pass(const StepArgs32& a, int stage, bool first_pass,
                                    cudaStream_t s) {
  const Grid& g = a.g;
  const int tpb = 128;
  const bool pair_x = g.nx_phys() >= (g.ng > 2 ? g.ng : 2);
  const bool pair_y = g.ny_phys() >= (g.ng > 2 ? g.ng : 2);
  int first = first_pass ? 1 : 0;
  auto go = [&](int e0, int count, int n_tan) {
    dim3 grid((unsigned)((n_tan + tpb - 1) / tpb), (unsigned)count);
    k_bc32<<<grid, tpb, 0, s>>>(a, stage, e0, first);
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

static bool narrow32(const Grid& g) {
  const int wide = g.ng > 2 ? g.ng : 2;
  return g.nx_phys() < wide || g.ny_phys() < wide;
}

// The fill of a stage; a narrow grid's step opens with the fill before dt.
cudaError_t launch_bc32(const StepArgs32& a, int stage, cudaStream_t s) {
  if (stage == 1 && narrow32(a.g)) {
    const cudaError_t e = launch_bc32_pass(a, 9, true, s);
    if (e != cudaSuccess) return e;
    return launch_bc32_pass(a, 1, false, s);
  }
  return launch_bc32_pass(a, stage, stage == 1, s);
}

cudaError_t launch_step32(const StepArgs32& a, cudaStream_t s) {
  cudaError_t e = launch_bc32(a, 1, s);
  if (e == cudaSuccess) e = launch_sweep<1>(a, s);
  if (e == cudaSuccess) e = launch_bc32(a, 2, s);
  if (e == cudaSuccess) e = launch_sweep<2>(a, s);
  return e;
}

cudaError_t launch_stage32_only(const StepArgs32& a, int stage, cudaStream_t s) {
  return stage == 1 ? launch_sweep<1>(a, s) : launch_sweep<2>(a, s);
}

int launches_per_step32(const StepArgs32& a) {
  const Grid& g = a.g;
  const int need = g.ng > 2 ? g.ng : 2;
  const int bc = (g.nx_phys() >= need ? 1 : 2) + (g.ny_phys() >= need ? 1 : 2);
  return 2 * bc + 2 + (narrow32(g) ? bc : 0);
}

cudaError_t launch_max_speed32(const StepArgs32& a, cudaStream_t s) {
  const long long n = (long long)a.g.nx_phys() * a.g.ny_phys();
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  if (blocks < 1) blocks = 1;
  k_max_speed32<<<(unsigned)blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_to_surface(const Grid& g64, const Grid& g32, FieldSet src, const double* b64,
                              FieldSet32 dst, double* bed_out, cudaStream_t s) {
  dim3 grid((unsigned)((g64.nxt + 127) / 128), (unsigned)(g64.nyt < 65535 ? g64.nyt : 65535));
  k_to_surface<<<grid, 128, 0, s>>>(g64, g32, src, b64, dst, bed_out);
  return cudaGetLastError();
}

cudaError_t launch_to_depth(const Grid& g32, const Grid& g64, FieldSet32 src, const double* b32,
                            FieldSet dst, double* bed_out, cudaStream_t s) {
  dim3 grid((unsigned)((g32.nxt + 127) / 128), (unsigned)(g32.nyt < 65535 ? g32.nyt : 65535));
  k_to_depth<<<grid, 128, 0, s>>>(g32, g64, src, b32, dst, bed_out);
  return cudaGetLastError();
}

// ---- batches ----------------------------------------------------------------

int batch_sweep_blocks(const StepArgs32& a) { return (a.nstrips * a.nrowblk + kWarps - 1) / kWarps; }

template <int C, bool HLLC, bool PLAIN>
static cudaError_t set_smem_batch_t() {
  cudaError_t e = cudaFuncSetAttribute(k_sweep_batch<C, HLLC, 1, PLAIN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kWarps * kNbuf * Lay<C>::slot(1));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_batch<C, HLLC, 2, PLAIN>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kWarps * kNbuf * Lay<C>::slot(2));
  return e;
}

template <int C, bool HLLC>
static cudaError_t set_smem_batch() {
  cudaError_t e = set_smem_batch_t<C, HLLC, true>();
  return e == cudaSuccess ? set_smem_batch_t<C, HLLC, false>() : e;
}

cudaError_t configure_batch32() {
  cudaError_t e = set_smem_batch<2, false>();
  if (e == cudaSuccess) e = set_smem_batch<2, true>();
  if (e == cudaSuccess) e = set_smem_batch<4, false>();
  if (e == cudaSuccess) e = set_smem_batch<4, true>();
  return e;
}

template <int C, int STAGE>
static cudaError_t launch_sweep_batch_t(const BatchLaunch32& bl, cudaStream_t s) {
  const size_t bytes = (size_t)kWarps * kNbuf * Lay<C>::slot(STAGE);
  const unsigned nb = (unsigned)bl.blocks;
  if (bl.hllc) {
    if (bl.plain)
      k_sweep_batch<C, true, STAGE, true><<<nb, kWarps * 32, bytes, s>>>(bl.args, bl.map);
    else
      k_sweep_batch<C, true, STAGE, false><<<nb, kWarps * 32, bytes, s>>>(bl.args, bl.map);
  } else {
    if (bl.plain)
      k_sweep_batch<C, false, STAGE, true><<<nb, kWarps * 32, bytes, s>>>(bl.args, bl.map);
    else
      k_sweep_batch<C, false, STAGE, false><<<nb, kWarps * 32, bytes, s>>>(bl.args, bl.map);
  }
  return cudaGetLastError();
}

cudaError_t launch_stage32_batch(const BatchLaunch32& bl, int stage, cudaStream_t s) {
  if (stage == 1) return bl.cpl == 4 ? launch_sweep_batch_t<4, 1>(bl, s) : launch_sweep_batch_t<2, 1>(bl, s);
  return bl.cpl == 4 ? launch_sweep_batch_t<4, 2>(bl, s) : launch_sweep_batch_t<2, 2>(bl, s);
}

cudaError_t launch_bc32_batch(const BatchLaunch32& bl, int stage, cudaStream_t s) {
  const int tpb = 128;
  const dim3 gx((unsigned)((bl.max_nyt + tpb - 1) / tpb), 2, (unsigned)bl.n);
  k_bc32_batch<<<gx, tpb, 0, s>>>(bl.args, stage, 0, stage == 1 ? 1 : 0);
  const dim3 gy((unsigned)((bl.max_nxt + tpb - 1) / tpb), 2, (unsigned)bl.n);
  k_bc32_batch<<<gy, tpb, 0, s>>>(bl.args, stage, 2, 0);
  return cudaGetLastError();
}

cudaError_t launch_step32_batch(const BatchLaunch32& bl, cudaStream_t s) {
  cudaError_t e = launch_bc32_batch(bl, 1, s);
  if (e == cudaSuccess) e = launch_stage32_batch(bl, 1, s);
  if (e == cudaSuccess) e = launch_bc32_batch(bl, 2, s);
  if (e == cudaSuccess) e = launch_stage32_batch(bl, 2, s);
  return e;
}

}  // namespace rkb
