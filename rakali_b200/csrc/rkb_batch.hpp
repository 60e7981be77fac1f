// A batch of independent simulations advanced together: one launch per phase
// covers every member (boundary fills, stage 1, fills, stage 2), chunks of
// steps are captured in CUDA graphs, and each member keeps its own buffers,
// clock, dt and boundary parameters (so tidal phases, sizes and step sizes
// may all differ).
#pragma once

#include <string>
#include <vector>

#include "rkb_sim.hpp"

namespace rkb {

class Batch {
 public:
  Batch() = default;
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Members must be finalised, at least max(nghost, 2) cells wide and share
  // the Riemann solver; `precision` (64 or 32) is applied to all of them.
  int create(const std::vector<Sim*>& sims, int precision, std::string& err);
  int step(int n);                    // n steps of every member
  int advance(double target);         // every member to `target` (own dt)
  int time_steps(int n, double* ms);  // n steps between CUDA events
  // n steps launched phase by phase with events between the phases:
  // out[0..3] = mean ms per step of the stage-1 boundary fills, stage 1, the
  // stage-2 fills and stage 2 (every member in each launch); out[4] = mean ms
  // per step of the whole launch-by-launch sequence (phases plus the gaps
  // between launches).
  int profile_steps(int n, double out[5]);
  // Time each candidate kernel shape for `trial_steps` steps on the live
  // state (restored afterwards), keep the fastest; *best_ms = its time per step.
  int autotune(int trial_steps, double* best_ms);
  // Current kernel shape: FP64 tile, or FP32 columns per lane and rows
  // (0 rows = automatic per member).
  void variant(int* a, int* b) const;
  // Sets the kernel shape (FP64: a = a shared-memory tile, b = 0; FP32: a =
  // 2 or 4 columns per lane, b >= 0 rows per warp sweep); -2 for others.
  int set_variant(int a, int b);
  void detach(Sim* s);  // a member is being destroyed
  const std::string& error() const { return err_; }

 private:
  int build();
  int prepare(int mode, double target, int nsteps);
  int finish();
  int launch_steps(int k);
  cudaGraphExec_t graph_for(int steps);
  void clear_graphs();

  std::vector<Sim*> sims_;
  std::vector<int> gauge_sig_;  // members' gauge generations the graphs were built with
  bool broken_ = false;
  int prec_ = 64;
  int tile_ = kTile32x16;
  int cpl_ = 2, rows_ = 0;
  int hllc_ = 0;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  void* dargs_ = nullptr;
  int2* dmap_ = nullptr;
  TileMaps* dmaps_ = nullptr;  // the members' TMA maps (FP64; null unless all are encoded)
  size_t map_cap_ = 0;
  BatchLaunch bl_{};
  BatchLaunch32 bl32_{};
  std::string err_;
  struct GraphEntry {
    int steps;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
  };
  std::vector<GraphEntry> graphs_;
};

}  // namespace rkb
