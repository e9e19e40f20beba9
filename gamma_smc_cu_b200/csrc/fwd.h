// Forward-only (filtered) posterior kernel: FlowContext.run_fwd.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsmc {

// Gap code of the forward-only path at one site: `chunks` lookups in the last
// layer, then one in layer `layer` (-1: none -- site 0 and zero gaps).
struct FwdCode {
  int layer;
  int chunks;
};

struct FwdArgs {
  const ulonglong2* geno;  // scan genotype layout
  int64_t n_haps;
  const FwdCode* code;     // [n_sites]
  const uint4* tab;        // [L][patches] half patches of the hom multi-step table
  int L;
  int n_sites;
  const int32_t* pi;
  const int32_t* pj;
  int n_pairs;
  float two_ne;
  float* mean;             // [n_sites][ldo]
  float* lower;            // null: no bounds
  float* upper;
  int64_t ldo;
};

// Exact speculative site chunks of a forward-only call: chunk k of K covers
// sites [S k / K, S (k+1) / K) after `burn_in` sites from (0, 0); the state
// each chunk reaches at its left boundary is checked bitwise against the left
// chunk's, and pairs with any mismatch are decoded again whole.
struct FwdSpec {
  int k_chunks;
  int burn_in;
  float2* rec;          // [k_chunks - 1][2][n_pairs]
  int* repair_list;     // [n_pairs]
  int* repair_count;    // zeroed by the launch
  int* repaired_total;  // incremented by the number repaired
};

cudaError_t launch_fwd_only(const FwdArgs& a, cudaStream_t stream);
// Chunked launch (one chunk: the plain kernel): chunk kernel, verify, repair.
cudaError_t launch_fwd_spec(const FwdArgs& a, const FwdSpec& sp, cudaStream_t stream);
// CTA size for kernels with one serial chain per pair: spread the warps over
// every SM first (32..max_threads threads).
int chain_cta_threads(int64_t n_pairs, int max_threads);
// n floats -> n halves (round to nearest even) on the device.
cudaError_t launch_to_half(const float* src, void* dst, size_t n, cudaStream_t stream);

}  // namespace gsmc
