// Fused Gamma-SMC forward/backward scan for sm_100a.
//
// A persistent kernel: every tile of a CTA (one warp, or the whole CTA) pulls
// tasks -- up to tile width x NP pairs over one padded window -- from a
// device counter.  Each thread walks its pairs
// over the window's sites: forward from the padded start to the core end,
// storing the (m, c) state at core sites in the CTA's slot, then backward from
// the padded end to the core start, combining with the stored forward state
// and writing the posterior at core sites.  Sites are shared by every pair, so
// the gap code (table layer and number of 1000-step chunks) is uniform across
// a task; only hom/het differs per pair.  With NP > 1 a thread's chains are
// independent (instruction-level parallelism) and share the per-site work.
//
// Table lookups read one 32-byte patch (four corners of m and of c) with a
// single 256-bit read-only load; hom and het patches of a layer are adjacent,
// so the het bit selects with one multiply-add.  The arithmetic is the
// reference's cached FB (src/kernels/gamma_smc_flow.cu:112-131, 160-163,
// 408-514, 567-609, 632-669, 678-754, 762-839) with its fused multiply-adds
// written explicitly, so results are bit-identical to it.
#include <cuda_runtime.h>
#include <stdint.h>

#include "scan.h"
#include "scan_device.cuh"
#include "tables.h"

namespace gsmc {
namespace {

// Persistent scan: each CTA takes tasks from a global counter until none are
// left; its forward-state slot is reused task after task.
// Resident CTAs per SM the register budget is fitted to (128 threads each).
// The scan is bound by the latency of its lookup chain and by issue, so warps
// per SM matter.  One pair per thread: 10 CTAs (46-48 registers with a
// one-deep forward-state ring, no spill; 9 CTAs at 56 registers ran level,
// 7-8 slower).
// Two pairs per thread: 8 CTAs (64 registers, no spill) measured 3% faster
// than 7 (69-72 registers).
#ifndef GSMC_MIN_CTAS
#define GSMC_MIN_CTAS 10
#endif
#ifndef GSMC_MIN_CTAS_NP2
#define GSMC_MIN_CTAS_NP2 8
#endif

template <int NP, int WIDTH, bool SUMMARY>
__global__ void __launch_bounds__(kThreads, NP == 1 ? GSMC_MIN_CTAS : GSMC_MIN_CTAS_NP2)
    fb_scan_persistent(const ScanArgs a) {
  // The task descriptor lives in shared memory: its fields are uniform across
  // the tile and read only where used, so they cost no registers.  (Plain
  // loads copy it: the list may be mapped host memory.)
  if constexpr (WIDTH == kThreads) {
    // the whole CTA takes one task at a time
    __shared__ Task task;
    __shared__ int task_id;
    float2* slot = a.fwd + (int64_t)blockIdx.x * a.slot_rows * (kThreads * NP);
    for (;;) {
      __syncthreads();  // everyone is done with the previous task
      if (threadIdx.x == 0) {
        // -1 once the list is exhausted (no task count held in registers)
        const int id = atomicAdd(a.next, 1);
        task_id = id < *a.count ? id : -1;
        if (task_id >= 0) task = a.tasks[task_id];
      }
      __syncthreads();
      if (task_id < 0) break;
      scan_task<NP, kThreads, SUMMARY>(a, task, slot);
    }
  } else {
    // each warp takes its own tasks
    constexpr int kWarps = kThreads / 32;
    __shared__ Task task[kWarps];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* slot = a.fwd + ((int64_t)blockIdx.x * kWarps + w) * a.slot_rows * (32 * NP);
    for (;;) {
      __syncwarp();  // the warp is done with the previous task
      int id = 0;
      if (lane == 0) {
        id = atomicAdd(a.next, 1);
        if (id >= *a.count) id = -1;
      }
      id = __shfl_sync(0xffffffffu, id, 0);
      if (id < 0) break;
      static_assert(sizeof(Task) % 4 == 0, "Task is copied as 32-bit words");
      const int* src = reinterpret_cast<const int*>(a.tasks + id);
      int* dst = reinterpret_cast<int*>(&task[w]);
      for (int i = lane; i < (int)(sizeof(Task) / 4); i += 32) dst[i] = src[i];
      __syncwarp();
      scan_task<NP, 32, SUMMARY>(a, task[w], slot);
    }
  }
}

__device__ __forceinline__ bool same_bits(float2 a, float2 b) {
  return __float_as_int(a.x) == __float_as_int(b.x) && __float_as_int(a.y) == __float_as_int(b.y);
}

// Thread (pair p, window w): all boundaries of w must match for p.
__global__ void spec_verify_kernel(const float2* __restrict__ rec, int64_t n_pairs,
                                   const SpecWindow* __restrict__ win, TaskListHead* head,
                                   Task* __restrict__ repairs, int max_repairs) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const SpecWindow& w = win[blockIdx.y];
  if (p >= n_pairs) return;
  bool ok = true;
  for (int b = 0; b < w.n_bnd && ok; ++b) {
    const float2* r = rec + (int64_t)(w.first_bnd + b) * 4 * n_pairs + p;
    ok = same_bits(r[0], r[n_pairs]) && same_bits(r[2 * n_pairs], r[3 * n_pairs]);
  }
  if (ok) return;
  const int i = atomicAdd(&head->count, 1);
  if (i >= max_repairs) return;  // cannot happen: max_repairs covers every (window, pair)
  Task t = w.repair;
  t.pi += p;
  t.pj += p;
  t.out_off += p;
  t.pair_count = 1;
  repairs[i] = t;
}

__global__ void add_count_kernel(const int* count, int* acc) { *acc += *count; }

// Thread (pair p, checked job blockIdx.y): any boundary whose exact and
// speculative states differ flags the job.
__global__ void exec_verify_kernel(const float2* __restrict__ rec,
                                   const ExecCheck* __restrict__ checks,
                                   int32_t* __restrict__ flags) {
  const ExecCheck& w = checks[blockIdx.y];
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= w.n_pairs) return;
  const int64_t n = w.n_pairs;
  for (int b = 0; b < w.n_bnd; ++b) {
    const float2* r = rec + w.rec_off + (int64_t)b * 4 * n + p;
    if (!same_bits(r[0], r[n]) || !same_bits(r[2 * n], r[3 * n])) {
      flags[w.job] = 1;
      return;
    }
  }
}

// One warp per site row: fold the row's per-warp partials into the site's
// accumulators.  Lane l sums columns l, l + 32, ... in order, then a fixed
// shuffle tree combines the lanes, so the result does not depend on timing.
__global__ void summary_fold_kernel(const float* __restrict__ p_sum,
                                    const float* __restrict__ p_min,
                                    const float* __restrict__ p_max, int64_t rows, int64_t cols,
                                    int64_t ld, double* __restrict__ acc_sum,
                                    float* __restrict__ acc_min,
                                    float* __restrict__ acc_max, bool first) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= rows) return;  // whole warps leave together
  const int64_t base = row * ld;
  double sum = 0.0;
  float mn = __int_as_float(0x7f800000), mx = -__int_as_float(0x7f800000);
  for (int64_t c = lane; c < cols; c += 32) {
    sum += (double)p_sum[base + c];
    mn = fminf(mn, p_min[base + c]);
    mx = fmaxf(mx, p_max[base + c]);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, d);
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, d));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, d));
  }
  if (lane == 0) {
    acc_sum[row] = first ? sum : acc_sum[row] + sum;
    acc_min[row] = first ? mn : fminf(acc_min[row], mn);
    acc_max[row] = first ? mx : fmaxf(acc_max[row], mx);
  }
}

__global__ void summary_finish_kernel(const double* __restrict__ acc_sum, int64_t rows,
                                      double n_pairs, float* __restrict__ site_mean) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < rows) site_mean[s] = (float)(acc_sum[s] / n_pairs);
}

// counts[k] = popcount of the XOR of haplotypes 2k and 2k+1 over all
// 128-site groups (bits past the last site are zero in both).  One CTA per
// diploid; int64 partial sums in a fixed order.
__global__ void het_count_kernel(const ulonglong2* __restrict__ geno, int64_t n_haps,
                                 int64_t n_groups, long long* __restrict__ counts) {
  const int64_t k = blockIdx.x;
  __shared__ long long part[32];
  long long n = 0;
  for (int64_t g = threadIdx.x; g < n_groups; g += blockDim.x) {
    const ulonglong2 a = geno[g * n_haps + 2 * k], b = geno[g * n_haps + 2 * k + 1];
    n += __popcll(a.x ^ b.x) + __popcll(a.y ^ b.y);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) n += __shfl_xor_sync(0xffffffffu, n, d);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
    counts[k] = t;
  }
}

// Pack genotypes: thread (h, word) builds 64 sites of haplotype h.
template <bool SCAN_LAYOUT>
__global__ void bitpack_kernel(const uint8_t* __restrict__ G, int64_t n, int64_t S,
                               int64_t n_words, uint64_t* __restrict__ out) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t h = blockIdx.y;
  if (w >= n_words) return;
  const uint8_t* row = G + h * S;
  const int64_t base = w * 64;
  uint64_t word = 0;
  const int nb = (S - base) < 64 ? (int)(S - base) : 64;
  for (int b = 0; b < nb; ++b) word |= (uint64_t)(row[base + b] & 1u) << b;
  if (SCAN_LAYOUT) {
    // group g = w / 2 holds words 2g, 2g+1 of haplotype h at [g][h]
    out[((w >> 1) * n + h) * 2 + (w & 1)] = word;
  } else {
    out[h * n_words + w] = word;
  }
}

__global__ void unpack_kernel(const uint64_t* __restrict__ packed, int64_t n, int64_t S,
                              int64_t n_words, uint8_t* __restrict__ G) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t h = blockIdx.y;
  if (s >= S) return;
  G[h * S + s] = (uint8_t)((packed[h * n_words + (s >> 6)] >> (s & 63)) & 1ull);
}

}  // namespace

int scan_threads() { return kThreads; }

bool scan_shape_valid(ScanShape shape) {
  return (shape.width == 32 || shape.width == kThreads) &&
         (shape.pairs_per_thread == 1 || shape.pairs_per_thread == 2);
}

int scan_tile_pairs(ScanShape shape) { return shape.width * shape.pairs_per_thread; }

int scan_tiles_per_cta(ScanShape shape) { return kThreads / shape.width; }

namespace {

template <int NP, int WIDTH>
int resident_of() {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fb_scan_persistent<NP, WIDTH, false>,
                                                    kThreads, 0) != cudaSuccess)
    return 0;
  return per_sm;
}

template <bool SUMMARY>
void launch_shape(const ScanArgs& args, int grid, ScanShape shape, cudaStream_t stream) {
  if (shape.width == 32) {
    if (shape.pairs_per_thread == 2)
      fb_scan_persistent<2, 32, SUMMARY><<<grid, kThreads, 0, stream>>>(args);
    else
      fb_scan_persistent<1, 32, SUMMARY><<<grid, kThreads, 0, stream>>>(args);
  } else {
    if (shape.pairs_per_thread == 2)
      fb_scan_persistent<2, kThreads, SUMMARY><<<grid, kThreads, 0, stream>>>(args);
    else
      fb_scan_persistent<1, kThreads, SUMMARY><<<grid, kThreads, 0, stream>>>(args);
  }
}

}  // namespace

int scan_resident_ctas(ScanShape shape) {
  if (!scan_shape_valid(shape)) return 0;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  int per_sm = 0;
  if (shape.width == 32)
    per_sm = shape.pairs_per_thread == 2 ? resident_of<2, 32>() : resident_of<1, 32>();
  else
    per_sm = shape.pairs_per_thread == 2 ? resident_of<2, kThreads>() : resident_of<1, kThreads>();
  return sms * per_sm;
}

cudaError_t launch_scan(const ScanArgs& args, int grid, ScanShape shape, cudaStream_t stream,
                        bool summary) {
  if (grid <= 0) return cudaSuccess;
  if (!scan_shape_valid(shape)) return cudaErrorInvalidValue;
  if (summary)
    launch_shape<true>(args, grid, shape, stream);
  else
    launch_shape<false>(args, grid, shape, stream);
  return cudaGetLastError();
}

cudaError_t launch_spec_verify(const float2* rec, int64_t n_pairs, const SpecWindow* win,
                               int n_win, TaskListHead* head, Task* repairs, int max_repairs,
                               cudaStream_t stream) {
  if (n_pairs <= 0 || n_win <= 0) return cudaSuccess;
  const dim3 grid((unsigned)((n_pairs + 255) / 256), (unsigned)n_win);
  spec_verify_kernel<<<grid, 256, 0, stream>>>(rec, n_pairs, win, head, repairs, max_repairs);
  return cudaGetLastError();
}

cudaError_t launch_exec_verify(const float2* rec, const ExecCheck* checks, int n_checks,
                               int max_pairs, int32_t* flags, cudaStream_t stream) {
  if (n_checks <= 0 || max_pairs <= 0) return cudaSuccess;
  const dim3 grid((unsigned)((max_pairs + 255) / 256), (unsigned)n_checks);
  exec_verify_kernel<<<grid, 256, 0, stream>>>(rec, checks, flags);
  return cudaGetLastError();
}

cudaError_t launch_add_count(const int* count, int* acc, cudaStream_t stream) {
  add_count_kernel<<<1, 1, 0, stream>>>(count, acc);
  return cudaGetLastError();
}

cudaError_t launch_summary_fold(const float* p_sum, const float* p_min, const float* p_max,
                                int64_t rows, int64_t cols, int64_t ld, double* acc_sum,
                                float* acc_min, float* acc_max, bool first, cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return cudaSuccess;
  const int64_t threads = rows * 32;
  summary_fold_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
      p_sum, p_min, p_max, rows, cols, ld, acc_sum, acc_min, acc_max, first);
  return cudaGetLastError();
}

cudaError_t launch_summary_finish(const double* acc_sum, int64_t rows, double n_pairs,
                                  float* site_mean, cudaStream_t stream) {
  if (rows <= 0) return cudaSuccess;
  summary_finish_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(acc_sum, rows, n_pairs,
                                                                           site_mean);
  return cudaGetLastError();
}

cudaError_t launch_het_counts(const ulonglong2* geno, int64_t n_haps, int64_t n_groups,
                              long long* counts, cudaStream_t stream) {
  if (n_haps < 2 || n_groups <= 0) return cudaSuccess;
  het_count_kernel<<<(unsigned)(n_haps / 2), 256, 0, stream>>>(geno, n_haps, n_groups, counts);
  return cudaGetLastError();
}

cudaError_t launch_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites, void* out,
                           bool scan_layout, cudaStream_t stream) {
  if (n_haps <= 0 || n_sites <= 0) return cudaSuccess;
  const int64_t n_words = (n_sites + 63) / 64;
  const dim3 grid((unsigned)((n_words + 127) / 128), (unsigned)n_haps);
  if (scan_layout)
    bitpack_kernel<true><<<grid, 128, 0, stream>>>(G, n_haps, n_sites, n_words,
                                                   static_cast<uint64_t*>(out));
  else
    bitpack_kernel<false><<<grid, 128, 0, stream>>>(G, n_haps, n_sites, n_words,
                                                    static_cast<uint64_t*>(out));
  return cudaGetLastError();
}

cudaError_t launch_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites, uint8_t* G,
                          cudaStream_t stream) {
  if (n_haps <= 0 || n_sites <= 0) return cudaSuccess;
  const int64_t n_words = (n_sites + 63) / 64;
  const dim3 grid((unsigned)((n_sites + 255) / 256), (unsigned)n_haps);
  unpack_kernel<<<grid, 256, 0, stream>>>(packed, n_haps, n_sites, n_words, G);
  return cudaGetLastError();
}

}  // namespace gsmc
