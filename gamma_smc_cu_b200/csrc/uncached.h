// Uncached flow-field forward/backward (gamma_smc_flow_fb), see uncached.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsmc {

struct UncachedArgs {
  const ulonglong2* geno;  // scan genotype layout
  int64_t n_haps;
  const int* seg;          // [n_sites] rounded base pairs entering each site
  const float2* flow;      // [2550] (u, v), 16-byte aligned
  int n_sites;
  const int32_t* pi;
  const int32_t* pj;
  int n_pairs;
  float rho, mu;           // scaled per-bp rates (4 Ne rho, 4 Ne mu)
  float unscale;           // 2 Ne
  float2* fwd;             // [n_sites][n_pairs] forward states
  float* mean;             // [n_sites][ldo]
  float* lower;            // null: no bounds
  float* upper;
  int64_t ldo;
  int* error;              // set to 1 when a CTA's flow-field copy did not land
};

cudaError_t launch_uncached_fb(const UncachedArgs& a, cudaStream_t stream);

}  // namespace gsmc
