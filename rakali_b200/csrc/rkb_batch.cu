// Batches of independent simulations (see rkb_batch.hpp).
#include "rkb_batch.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace rkb {

namespace {

#define RKB_TRY(expr)                      \
  do {                                     \
    cudaError_t e_ = (expr);               \
    if (e_ != cudaSuccess) return -1;      \
  } while (0)

constexpr int kMaxGraphSteps = 256;

}  // namespace

Batch::~Batch() {
  clear_graphs();
  if (dargs_) cudaFree(dargs_);
  if (dmap_) cudaFree(dmap_);
  if (dmaps_) cudaFree(dmaps_);
  if (stream_) cudaStreamDestroy(stream_);
  for (Sim* s : sims_)
    if (s && s->batch == this) s->batch = nullptr;
}

void Batch::clear_graphs() {
  for (auto& ge : graphs_) {
    if (ge.exec) cudaGraphExecDestroy(ge.exec);
    if (ge.graph) cudaGraphDestroy(ge.graph);
  }
  graphs_.clear();
}

void Batch::detach(Sim* s) {
  for (Sim*& m : sims_)
    if (m == s) m = nullptr;
  broken_ = true;
}

int Batch::set_variant(int a, int b) {
  if (prec_ == 64) {
    const bool ok = b == 0 && (a == kTile32x8 || a == kTile32x16 || a == kTile64x4 ||
                               a == kTile16x16 || a == kTile32x8w || a == kTile32x12w ||
                               a == kTile16x15 || a == kTile32x7w || a == kTile16x15t);
    if (!ok) {
      err_ = "FP64 batches take a shared-memory tile (0-3, 6-10) and b = 0";
      return -2;
    }
    if (configure_batch(a, hllc_) != cudaSuccess) return -1;
    tile_ = a;
  } else {
    if ((a != 2 && a != 4) || b < 0) {
      err_ = "FP32 batches take 2 or 4 columns per lane and rows >= 0";
      return -2;
    }
    cpl_ = a;
    rows_ = b;
  }
  clear_graphs();
  return 0;
}

void Batch::variant(int* a, int* b) const {
  if (prec_ == 64) {
    if (a) *a = tile_;
    if (b) *b = 0;
  } else {
    if (a) *a = cpl_;
    if (b) *b = rows_;
  }
}

int Batch::create(const std::vector<Sim*>& sims, int precision, std::string& err) {
  if (sims.empty()) { err = "a batch needs at least one simulation"; return -2; }
  if (precision != 32 && precision != 64) { err = "precision must be 32 or 64"; return -2; }
  hllc_ = sims[0]->phys.use_hllc;
  for (Sim* s : sims) {
    if (!s->is_finalised) { err = "every member must be finalised"; return -1; }
    if (s->batch) { err = "a simulation can belong to one batch only"; return -2; }
    if (s->phys.use_hllc != hllc_) { err = "members must share the Riemann solver (HLL or HLLC)"; return -2; }
    if (s->phys.scheme != 2) { err = "batches run the SSP-RK2 scheme only"; return -2; }
    const int need = s->g.ng > 2 ? s->g.ng : 2;
    if (s->g.nx_phys() < need || s->g.ny_phys() < need) {
      err = "members must be at least max(nghost, 2) cells wide";
      return -2;
    }
  }
  for (size_t a = 0; a < sims.size(); ++a)
    for (size_t b = a + 1; b < sims.size(); ++b)
      if (sims[a] == sims[b]) { err = "a simulation appears twice"; return -2; }
  if (cudaGetDevice(&device_) != cudaSuccess) { err = "no CUDA device"; return -1; }
  if (cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking) != cudaSuccess) {
    err = "stream creation failed";
    return -1;
  }
  prec_ = precision;
  sims_ = sims;
  for (Sim* s : sims_) {
    if (s->set_precision(prec_) != 0) { err = "switching a member's precision failed"; return -1; }
    s->batch = this;
  }
  if (prec_ == 64 ? configure_batch(tile_, hllc_) != cudaSuccess : configure_batch32() != cudaSuccess) {
    err = "kernel configuration failed";
    return -1;
  }
  return 0;
}

// Gather every member's kernel arguments and the block map of one stage
// launch (largest members first, so the tail of a launch is made of small
// work), and upload both.
int Batch::build() {
  const int n = (int)sims_.size();
  std::vector<int> blocks(n), order(n);
  std::vector<StepArgs> a64;
  std::vector<StepArgs32> a32;
  int max_nxt = 0, max_nyt = 0;
  int plain = 1;
  for (int i = 0; i < n; ++i) {
    Sim* s = sims_[i];
    max_nxt = std::max(max_nxt, s->g.nxt);
    max_nyt = std::max(max_nyt, s->g.nyt);
    if (prec_ == 64) {
      StepArgs a = s->device_args();
      a.tile = tile_;
      a.hllc = hllc_;
      plain = plain && a.plain;
      a64.push_back(a);
      blocks[i] = batch_stage_blocks(s->g, tile_);
    } else {
      StepArgs32 a = s->device_args32();
      plain = plain && a.plain;
      a32.push_back(a);
      blocks[i] = batch_sweep_blocks(a);
    }
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return blocks[x] > blocks[y]; });
  std::vector<int2> map;
  for (int i : order)
    for (int k = 0; k < blocks[i]; ++k) map.push_back(make_int2(i, k));
  const size_t args_bytes = prec_ == 64 ? a64.size() * sizeof(StepArgs) : a32.size() * sizeof(StepArgs32);
  bool realloc_ = false;
  if (!dargs_) {
    const size_t cap = (size_t)n * std::max(sizeof(StepArgs), sizeof(StepArgs32));
    RKB_TRY(cudaMalloc(&dargs_, cap));
    realloc_ = true;
  }
  if (map.size() > map_cap_) {
    if (dmap_) cudaFree(dmap_);
    dmap_ = nullptr;
    RKB_TRY(cudaMalloc((void**)&dmap_, map.size() * sizeof(int2)));
    map_cap_ = map.size();
    realloc_ = true;
  }
  RKB_TRY(cudaMemcpyAsync(dargs_, prec_ == 64 ? (const void*)a64.data() : (const void*)a32.data(),
                          args_bytes, cudaMemcpyHostToDevice, stream_));
  RKB_TRY(cudaMemcpyAsync(dmap_, map.data(), map.size() * sizeof(int2), cudaMemcpyHostToDevice,
                          stream_));
  // the TMA-staged tiles need every member's maps (encoded when it was
  // finalised); the maps follow the members' buffers, which never move
  bool maps_ok = prec_ == 64;
  for (Sim* s : sims_) maps_ok = maps_ok && s->tma_status() == 0;
  if (maps_ok && !dmaps_) {
    RKB_TRY(cudaMalloc((void**)&dmaps_, (size_t)n * sizeof(TileMaps)));
    std::vector<TileMaps> hm(n);
    for (int i = 0; i < n; ++i) hm[i] = sims_[i]->tile_maps();
    RKB_TRY(cudaMemcpyAsync(dmaps_, hm.data(), (size_t)n * sizeof(TileMaps),
                            cudaMemcpyHostToDevice, stream_));
  }
  RKB_TRY(cudaStreamSynchronize(stream_));
  const int nblocks = (int)map.size();
  const bool same = prec_ == 64
                        ? (bl_.blocks == nblocks && bl_.max_nxt == max_nxt && bl_.max_nyt == max_nyt &&
                           bl_.tile == tile_ && bl_.plain == plain)
                        : (bl32_.blocks == nblocks && bl32_.max_nxt == max_nxt &&
                           bl32_.max_nyt == max_nyt && bl32_.cpl == cpl_ && bl32_.plain == plain);
  std::vector<int> gsig(n);
  for (int i = 0; i < n; ++i) gsig[i] = sims_[i]->gauge_generation();
  // graphs hold launch shapes and pointers, and the members' gauge recorders
  if (realloc_ || !same || gsig != gauge_sig_) clear_graphs();
  gauge_sig_ = gsig;
  bl_ = BatchLaunch{(const StepArgs*)dargs_, dmap_, n, nblocks, max_nxt, max_nyt, tile_, hllc_,
                    plain, maps_ok ? dmaps_ : nullptr};
  bl32_ = BatchLaunch32{(const StepArgs32*)dargs_, dmap_, n, nblocks, max_nxt, max_nyt,
                        cpl_, hllc_, plain};
  return 0;
}

int Batch::prepare(int mode, double target, int nsteps) {
  if (broken_) {
    err_ = "a member of this batch was destroyed";
    return -1;
  }
  if (cudaSetDevice(device_) != cudaSuccess) return -1;
  for (Sim* s : sims_) {
    if (prec_ == 64) {
      if (s->tile != tile_) s->params_dirty = true;
      s->tile = tile_;
    } else {
      if (s->sweep_cpl != cpl_ || s->sweep_rows != rows_) s->params_dirty = true;
      s->sweep_cpl = cpl_;
      s->sweep_rows = rows_;
    }
    if (s->batch_prepare(mode, target, nsteps) != 0) {
      err_ = "preparing a member failed";
      return -1;
    }
  }
  return build();
}

int Batch::finish() {
  int rc = 0;
  for (Sim* s : sims_)
    if (s->batch_finish() != 0) rc = -1;
  if (rc != 0) err_ = "a member reported a device error";
  return rc;
}

cudaGraphExec_t Batch::graph_for(int steps) {
  for (auto& ge : graphs_)
    if (ge.steps == steps) return ge.exec;
  GraphEntry ge{steps, nullptr, nullptr};
  if (cudaStreamSynchronize(stream_) != cudaSuccess) return nullptr;
  if (cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return nullptr;
  for (int k = 0; k < steps; ++k) {
    if (prec_ == 64)
      launch_step_batch(bl_, stream_);
    else
      launch_step32_batch(bl32_, stream_);
    for (Sim* s : sims_) s->record_gauges(stream_);  // members with gauge stations
  }
  if (cudaStreamEndCapture(stream_, &ge.graph) != cudaSuccess) return nullptr;
  if (cudaGraphInstantiate(&ge.exec, ge.graph, 0) != cudaSuccess) return nullptr;
  graphs_.push_back(ge);
  return ge.exec;
}

int Batch::launch_steps(int left) {
  while (left > 0) {
    int k = 1;
    while (k * 2 <= left && k * 2 <= kMaxGraphSteps) k *= 2;
    cudaGraphExec_t g = graph_for(k);
    if (!g) return -1;
    RKB_TRY(cudaGraphLaunch(g, stream_));
    left -= k;
  }
  return 0;
}

int Batch::step(int n) {
  if (n <= 0) return 0;
  if (prepare(1, 0.0, n) != 0) return -1;
  if (launch_steps(n) != 0) return -1;
  RKB_TRY(cudaStreamSynchronize(stream_));
  return finish();
}

int Batch::advance(double target) {
  if (prepare(0, target, 0) != 0) return -1;
  for (int guard = 0; guard < 1000000; ++guard) {
    // chunk size from the member furthest from the target (dt of its last step)
    double need = 0.0;
    bool any = false;
    for (Sim* s : sims_) {
      if (!(s->time() < target - 1.0e-10)) continue;
      any = true;
      const double est = s->dt() > 0.0 ? std::ceil((target - s->time()) / s->dt() * 1.02) + 1.0 : 1.0;
      need = std::max(need, est);
    }
    if (!any) return 0;
    int k = 1;
    while (k < need && k < kMaxGraphSteps) k *= 2;
    std::vector<double> t0(sims_.size());
    for (size_t i = 0; i < sims_.size(); ++i) t0[i] = sims_[i]->time();
    if (launch_steps(k) != 0) return -1;
    RKB_TRY(cudaStreamSynchronize(stream_));
    if (finish() != 0) return -1;
    bool progress = false;
    for (size_t i = 0; i < sims_.size(); ++i) progress = progress || sims_[i]->time() > t0[i];
    if (!progress) {
      err_ = "no member advanced";
      return -1;
    }
  }
  return -1;
}

int Batch::time_steps(int n, double* ms) {
  if (n <= 0) return -2;
  if (prepare(1, 0.0, n) != 0) return -1;
  for (int k = 1; k <= kMaxGraphSteps && k <= n; k *= 2)  // instantiate outside the timed region
    if (!graph_for(k)) return -1;
  cudaEvent_t e0, e1;
  RKB_TRY(cudaEventCreate(&e0));
  RKB_TRY(cudaEventCreate(&e1));
  RKB_TRY(cudaEventRecord(e0, stream_));
  if (launch_steps(n) != 0) return -1;
  RKB_TRY(cudaEventRecord(e1, stream_));
  RKB_TRY(cudaEventSynchronize(e1));
  float f = 0.0f;
  RKB_TRY(cudaEventElapsedTime(&f, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = f;
  return finish();
}

int Batch::profile_steps(int n, double out[5]) {
  if (n <= 0) return -2;
  if (prepare(1, 0.0, n) != 0) return -1;
  cudaEvent_t ev[5];
  for (auto& e : ev) RKB_TRY(cudaEventCreate(&e));
  double acc[5] = {0, 0, 0, 0, 0};
  for (int k = 0; k < n; ++k) {
    const bool f32 = prec_ == 32;
    RKB_TRY(cudaEventRecord(ev[0], stream_));
    RKB_TRY(f32 ? launch_bc32_batch(bl32_, 1, stream_) : launch_bc_batch(bl_, 1, stream_));
    RKB_TRY(cudaEventRecord(ev[1], stream_));
    RKB_TRY(f32 ? launch_stage32_batch(bl32_, 1, stream_) : launch_stage_batch_only(bl_, 1, stream_));
    RKB_TRY(cudaEventRecord(ev[2], stream_));
    RKB_TRY(f32 ? launch_bc32_batch(bl32_, 2, stream_) : launch_bc_batch(bl_, 2, stream_));
    RKB_TRY(cudaEventRecord(ev[3], stream_));
    RKB_TRY(f32 ? launch_stage32_batch(bl32_, 2, stream_) : launch_stage_batch_only(bl_, 2, stream_));
    RKB_TRY(cudaEventRecord(ev[4], stream_));
    RKB_TRY(cudaEventSynchronize(ev[4]));
    for (int p = 0; p < 4; ++p) {
      float f = 0.0f;
      RKB_TRY(cudaEventElapsedTime(&f, ev[p], ev[p + 1]));
      acc[p] += f;
    }
    float f = 0.0f;
    RKB_TRY(cudaEventElapsedTime(&f, ev[0], ev[4]));
    acc[4] += f;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int p = 0; p < 5; ++p) out[p] = acc[p] / n;
  return finish();
}

// Candidate shapes: FP64 the four shared-memory tiles; FP32 2 or 4 columns
// per lane times rows per warp sweep (0 = one wave of resident warps per member).
int Batch::autotune(int trial_steps, double* best_ms) {
  if (trial_steps <= 0) trial_steps = 3;
  std::vector<std::pair<int, int>> cands;
  if (prec_ == 64) {
    for (int t : {kTile32x16, kTile32x8, kTile64x4, kTile16x16, kTile32x8w, kTile32x12w,
                  kTile16x15, kTile32x7w, kTile16x15t})
      cands.push_back({t, 0});
  } else {
    for (int c : {2, 4})
      for (int r : {0, 16, 32, 64, 128}) cands.push_back({c, r});
  }
  for (Sim* s : sims_)
    if (s->snapshot() != 0) {
      err_ = "snapshot of a member failed";
      return -1;
    }
  const int tile0 = tile_, cpl0 = cpl_, rows0 = rows_;
  double best = -1.0;
  std::pair<int, int> pick{prec_ == 64 ? tile0 : cpl0, prec_ == 64 ? 0 : rows0};
  cudaEvent_t e0, e1;
  RKB_TRY(cudaEventCreate(&e0));
  RKB_TRY(cudaEventCreate(&e1));
  int rc = 0;
  for (const auto& c : cands) {
    if (prec_ == 64) {
      tile_ = c.first;
      if (configure_batch(tile_, hllc_) != cudaSuccess) { rc = -1; break; }
    } else {
      cpl_ = c.first;
      rows_ = c.second;
    }
    if (prepare(1, 0.0, trial_steps + 1) != 0) { rc = -1; break; }
    auto one = [&]() {
      return prec_ == 64 ? launch_step_batch(bl_, stream_) : launch_step32_batch(bl32_, stream_);
    };
    if (one() != cudaSuccess) { rc = -1; break; }  // warm-up step
    if (cudaEventRecord(e0, stream_) != cudaSuccess) { rc = -1; break; }
    for (int k = 0; k < trial_steps; ++k) one();
    if (cudaEventRecord(e1, stream_) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      rc = -1;
      break;
    }
    float f = 0.0f;
    cudaEventElapsedTime(&f, e0, e1);
    if (finish() != 0) { rc = -1; break; }
    const double per = (double)f / trial_steps;
    if (best < 0.0 || per < best) {
      best = per;
      pick = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (Sim* s : sims_)
    if (s->restore() != 0) rc = -1;
  if (prec_ == 64) {
    tile_ = rc == 0 ? pick.first : tile0;
    configure_batch(tile_, hllc_);
  } else {
    cpl_ = rc == 0 ? pick.first : cpl0;
    rows_ = rc == 0 ? pick.second : rows0;
  }
  clear_graphs();
  if (best_ms) *best_ms = best;
  if (rc != 0 && err_.empty()) err_ = "a trial run failed";
  return rc;
}

}  // namespace rkb
