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
  long long wait_polls;    // mbarrier polls a CTA waits for that copy before giving up
};

// Polls of the flow-field copy wait when no other budget is set.
constexpr long long kDefaultCopyWaitPolls = 1ll << 24;

// Exact speculative site chunks (as FwdSpec for the forward-only path): chunk
// k of K decodes sites [S k / K, S (k+1) / K) with `burn_in` sites of burn-in
// on its inner sides; the forward and backward states at every chunk boundary
// are checked bitwise and pairs with any mismatch are decoded again whole.
struct UncachedSpec {
  int k_chunks;
  int burn_in;
  float2* rec;          // [k_chunks - 1][4][n_pairs]
  int* repair_list;     // [n_pairs]
  int* repair_count;    // zeroed by the launch
  int* repaired_total;  // incremented by the number repaired
};

cudaError_t launch_uncached_fb(const UncachedArgs& a, cudaStream_t stream);
// Chunked launch (one chunk: the plain kernel): chunks, verify, repair.
cudaError_t launch_uncached_spec(const UncachedArgs& a, const UncachedSpec& sp, cudaStream_t stream);

}  // namespace gsmc
