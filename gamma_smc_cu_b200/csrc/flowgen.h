// Flow-field generation on the GPU (float64), see flowgen.cu.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace gsmc {

// Piecewise-constant N(t): epoch k starts at t_bounds[k] (scaled time) with
// coalescence rate lam[k] and cumulative rate L_bounds[k] at its start; n = 0
// selects constant Ne.
constexpr int kMaxEpochs = 64;
struct FlowGenEpochs {
  int n;
  double t_bounds[kMaxEpochs];
  double lam[kMaxEpochs];
  double L_bounds[kMaxEpochs];
};

struct FlowGenArgs {
  const double* alpha;  // [mean_n * cv_n] Gamma shape of each cell
  const double* beta;   // [mean_n * cv_n] Gamma rate of each cell
  int mean_n, cv_n;
  int n_steps;          // time grid: 2 n_steps + 1 points
  double t_max_exp;     // -log(1e-3)
  double calibration;   // divisor of the fitted coefficients
  double* u;            // [mean_n * cv_n] outputs
  double* v;
};

size_t flow_field_smem_bytes(int n_steps);
cudaError_t launch_flow_field(const FlowGenArgs& a, const FlowGenEpochs& ep, cudaStream_t stream);

}  // namespace gsmc
