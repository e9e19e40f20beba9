// Device kernels of the Gamma-SMC forward/backward scan and their launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsmc {

// Per-site gap code: the gap of k base pairs entering site s is applied as
// `chunks` lookups in the last hom layer plus one lookup in site layer
// j = k - chunks * L - 1 (src/kernels/gamma_smc_flow.cu:471-514).  `layer` is
// j's offset in float4 units (j * kLayerF4) within one direction's tables.
struct SiteCode {
  int layer;
  int chunks;
};
// Zero entries stored before site 0 and after the last site of the code array.
constexpr int kCodePad = 2;

// Output selection of a task.
enum TaskFlags { kTaskCI = 1, kTaskPosterior = 2 };

// One unit of scan work: up to (threads per CTA x pairs per thread) pairs over
// one padded window.  Forward over [ps, ce), backward over [pe-1 .. cs],
// posterior at core rows [cs, ce).  Output element (s, pair j of the task) is
// out[k][out_off + (s - out_row0) * ldo + j] for each selected output k
// (0 mean, 1 lower, 2 upper, 3 alpha, 4 beta).
struct Task {
  int32_t ps, cs, ce, pe;
  int32_t pair_begin;   // first pair (index into pi/pj)
  int32_t pair_count;   // pairs in this task
  int32_t out_row0;
  int32_t flags;        // TaskFlags
  int64_t out_off;
  int64_t ldo;
  float* out[5];
  float unscale;        // 2 * Ne of the task's job
  int32_t pad;
};

struct ScanArgs {
  const ulonglong2* geno;   // [n_groups][n_haps]: 128 sites per entry, bit b of .x/.y = site 128g+b / 128g+64+b
  int64_t n_haps;
  const SiteCode* code;     // [n_sites], with kCodePad zero entries before and after
  const float4* site_tab;   // [2 directions][L][hom, het][2450][2]
  const float4* chunk_tab;  // [2450][2]
  int L;
  const int32_t* pi;
  const int32_t* pj;
  const Task* tasks;
  int n_tasks;
  int* next_task;           // work counter, zero at launch
  float2* fwd;              // per-CTA forward-state slots
  int64_t slot_rows;        // sites per slot (max core length of the tasks)
};

// Threads per CTA of the scan and the pairs one thread carries.
int scan_threads();
int scan_tile_pairs(int pairs_per_thread);

// Resident CTAs of the persistent scan kernel on the current device.
int scan_resident_ctas(int pairs_per_thread);

// Launch the persistent scan over args.n_tasks tasks with `grid` CTAs; each
// CTA owns forward-state slot blockIdx.x of slot_rows x tile pairs float2.
cudaError_t launch_scan(const ScanArgs& args, int grid, int pairs_per_thread,
                        cudaStream_t stream);

// Pack [n_haps x n_sites] uint8 genotypes.  scan_layout: word-major 128-site
// groups for the scan; otherwise the reference's row-major uint64 words.
cudaError_t launch_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites, void* out,
                           bool scan_layout, cudaStream_t stream);
cudaError_t launch_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites, uint8_t* G,
                          cudaStream_t stream);

}  // namespace gsmc
