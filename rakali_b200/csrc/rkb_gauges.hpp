// Device-recorded gauge time series (rkb_gauges.cu).
#pragma once

#include <vector>

#include "rkb_kernels.h"

namespace rkb {

// Device-resident recorder: stations, the gauge clock and the record buffer.
struct GaugeDev {
  int n, cap;         // stations inside the domain, record capacity
  int count, overflow;
  double interval, next;  // gauge_output_interval (s; <= 0: every step), next gauge time
  const int* ix0;     // per station: 0-based array indices of the stencil's lower-left cell
  const int* iy0;
  const double* wx;   // bilinear weights
  const double* wy;
  double* rec_t;      // [cap] record times
  double* rec;        // [cap][n][3]: eta, u, v
};

// Stations inside the domain with their stencils (host, from x, y in metres).
struct GaugeStencils {
  std::vector<int> station;  // index into the caller's list
  std::vector<int> ix0, iy0;
  std::vector<double> wx, wy;
};

void gauge_stencils(const Grid& g, const double* x, const double* y, int n, GaugeStencils& out);

cudaError_t launch_gauge_record(const Grid& g, const StepCtl* ctl, GaugeDev* gd, int n,
                                const FieldSet& U0, const FieldSet& U1, const double* b,
                                cudaStream_t s);
cudaError_t launch_gauge_record32(const Grid& g, const StepCtl* ctl, GaugeDev* gd, int n,
                                  const FieldSet32& U0, const FieldSet32& U1, const double* b,
                                  cudaStream_t s);

}  // namespace rkb
