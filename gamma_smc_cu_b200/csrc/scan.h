// Device kernels of the Gamma-SMC forward/backward scan and their launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsmc {

constexpr int kScanThreads = 256;     // threads per CTA of the scan
constexpr int kMaxWindows = 32;       // windows one scan launch can carry

// Per-site gap code: the gap of k base pairs entering site s is applied as
// `chunks` lookups in the last hom layer plus one lookup in site layer `layer`,
// with k = chunks * L + layer + 1 (src/kernels/gamma_smc_flow.cu:471-514).
struct SiteCode {
  int layer;
  int chunks;
};

// One padded window: forward over [ps, ce), backward over [pe-1 .. cs],
// outputs for core rows [cs, ce).  Rows of the outputs of this window live at
// out + out_off + (s - out_row0) * ldo + col0 + p.
struct Window {
  int64_t ps, cs, ce, pe;
  int64_t fwd_off;   // element offset of this window's forward-state slot
  int64_t out_off;
  int64_t out_row0;
};

struct ScanArgs {
  const ulonglong2* geno;   // [n_groups][n_haps]: 128 sites per entry, bit b of .x/.y = site 128g+b / 128g+64+b
  int64_t n_haps;
  const SiteCode* code;     // [n_sites]
  const float4* site_tab;   // [4][L][2450][2]
  const float4* chunk_tab;  // [2450][2]
  int L;
  const int32_t* pi;
  const int32_t* pj;
  int64_t n_pairs;          // pairs in this launch (also the forward-state row stride)
  float2* fwd;              // forward states (m, c), slot rows of n_pairs
  float* mean;
  float* lower;
  float* upper;
  float* alpha;
  float* beta;
  int64_t ldo;
  int64_t col0;
  float unscale;            // 2 * Ne
  int n_windows;
  Window win[kMaxWindows];
};

// Launch the fused forward/backward scan over args.n_windows windows.
cudaError_t launch_scan(const ScanArgs& args, bool ci, bool posterior, cudaStream_t stream);

// Pack [n_haps x n_sites] uint8 genotypes.  scan_layout: word-major 128-site
// groups for the scan; otherwise the reference's row-major uint64 words.
cudaError_t launch_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites, void* out,
                           bool scan_layout, cudaStream_t stream);
cudaError_t launch_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites, uint8_t* G,
                          cudaStream_t stream);

}  // namespace gsmc
