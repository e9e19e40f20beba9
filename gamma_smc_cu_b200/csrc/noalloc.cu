// Allocation-free variant of the device-resident blockwise scan.
//
// Some callers cannot have a library allocate device memory while they call
// it: programs whose framework allocator (a caching allocator, or a pool
// reserved up front) already holds the GPU's memory, so a cudaMalloc would fail
// or fragment it; services that keep tail latency low and cannot take the
// device-wide synchronisation cudaMalloc/cudaFree may cause; and host
// applications that load this library as a plug-in under a device-memory
// budget of their own.  For them this file provides
// gsmc_run_fb_blockwise_device_noalloc: the same computation as
// gsmc_run_fb_blockwise_device, whose only scratch -- the work counter and the
// per-CTA forward-state slots -- lives in one fixed, file-scope device array
// instead of in memory allocated at call time.
//
// Costs and limits:
// * every GPU that loads this library holds kNoAllocScratchBytes (128 MiB) of
//   device memory for the array until the process exits;
// * a window's core must fit one CTA slot: core_block_sites x 128 pairs x
//   8 bytes <= 128 MiB - 256 bytes, i.e. at most 131,071 core sites; the
//   number of CTAs that run at once is bounded by how many slots fit;
// * all calls share the array: calls that overlap on the GPU (different
//   streams, or other host threads) race on it and must be serialised by the
//   caller; the counter is cleared at the start of every call and the slots
//   need no clearing (each task writes its slot rows before reading them);
// * the first call on a device looks the array's address up with
//   cudaGetSymbolAddress (loading this file's device code if needed) and
//   keeps it for the life of the process; make that first call before
//   capturing any stream, and do not call this entry point on a device after
//   a cudaDeviceReset, which would leave the kept address stale.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ctx_view.h"
#include "gsmc_b200.h"
#include "scan.h"
#include "scan_device.cuh"
#include "tables.h"
#include "windows.h"

namespace gsmc {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(128) << 20;
constexpr size_t kCounterBytes = 256;  // work counter, padded to keep slots aligned
constexpr int kMaxDevices = 64;

// The scratch: [counter | per-CTA forward-state slots].  In host code this
// name is only a handle for cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocArgs {
  ScanArgs scan;   // genotypes, gap codes and tables
  const int32_t* pi;  // pair indices
  const int32_t* pj;
  int* counter;    // in the scratch, cleared before the launch
  float2* slots;   // in the scratch
  int64_t slot_rows;
  int64_t n_sites;
  int64_t core;    // clamped to [1, n_sites] on the host
  int64_t flank;   // clamped to [0, n_sites] on the host
  int n_pairs;
  int tiles;       // pair tiles per window
  int n_tasks;     // windows x tiles
  int flags;       // TaskFlags
  float unscale;
  float* out[5];
  int64_t ldo;
  int64_t col0;
};

// Persistent scan over (window, pair tile) tasks numbered window-major; each
// task's descriptor is derived from its number, so no task list is needed.
__global__ void __launch_bounds__(kThreads) fb_scan_noalloc(const NoAllocArgs a) {
  __shared__ Task task;
  __shared__ int id;
  float2* slot = a.slots + (int64_t)blockIdx.x * a.slot_rows * kThreads;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      id = atomicAdd(a.counter, 1);
      if (id < a.n_tasks) {
        const int w = id / a.tiles, tile = id % a.tiles;
        // int64 window arithmetic: every bound lies in [0, n_sites] < 2^31
        const WindowBounds b = window_bounds(w, a.n_sites, a.core, a.flank);
        task.ps = (int32_t)b.ps;
        task.cs = (int32_t)b.cs;
        task.ce = (int32_t)b.ce;
        task.pe = (int32_t)b.pe;
        task.pi = a.pi + (int64_t)tile * kThreads;
        task.pj = a.pj + (int64_t)tile * kThreads;
        task.pair_count = min(kThreads, a.n_pairs - tile * kThreads);
        task.out_row0 = 0;
        task.flags = a.flags;
        task.out_off = a.col0 + (int64_t)tile * kThreads;
        task.ldo = a.ldo;
        for (int k = 0; k < 5; ++k) task.out[k] = a.out[k];
        task.unscale = a.unscale;
        task.bl = task.br = nullptr;  // no speculative chunks here
        task.bstride = 0;
      }
    }
    __syncthreads();
    if (id >= a.n_tasks) break;
    scan_task<1, kThreads>(a.scan, task, slot);
  }
}

// Device address of the scratch array, looked up once per device.
int scratch_address(int device, unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[kMaxDevices] = {};
  if (device < 0 || device >= kMaxDevices)
    return set_error(GSMC_E_INVALID, "device index out of range for the allocation-free path");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      char msg[256];
      std::snprintf(msg, sizeof(msg), "CUDA error: %s (cudaGetSymbolAddress of the scratch array)",
                    cudaGetErrorString(e));
      return set_error(GSMC_E_CUDA, msg);
    }
    addr[device] = static_cast<unsigned char*>(p);
  }
  *out = addr[device];
  return GSMC_OK;
}

}  // namespace
}  // namespace gsmc

using namespace gsmc;

extern "C" int gsmc_run_fb_blockwise_device_noalloc(
    gsmc_ctx* ctx, const int32_t* d_pair_i, const int32_t* d_pair_j, int64_t n_pairs,
    int64_t core_block_sites, int64_t flank_sites, int flags, float* d_mean, float* d_lower,
    float* d_upper, float* d_alpha, float* d_beta, int64_t ld_out, int64_t out_col0,
    void* stream) {
  CtxView v;
  if (!ctx_view(ctx, &v)) return set_error(GSMC_E_INVALID, "null context");
  if (core_block_sites <= 0) return set_error(GSMC_E_INVALID, "core_block_sites must be positive.");
  if (flank_sites < 0) return set_error(GSMC_E_INVALID, "flank_sites must be non-negative.");
  if (n_pairs < 0 || ld_out < 0 || out_col0 < 0 || out_col0 + n_pairs > ld_out)
    return set_error(GSMC_E_INVALID, "bad pair count or output leading dimension");
  if (n_pairs > 0 && (!d_pair_i || !d_pair_j || !d_mean))
    return set_error(GSMC_E_INVALID, "null device pointer");
  if ((flags & GSMC_CI) && n_pairs > 0 && (!d_lower || !d_upper))
    return set_error(GSMC_E_INVALID, "null lower/upper output");
  if ((flags & GSMC_POSTERIOR) && n_pairs > 0 && (!d_alpha || !d_beta))
    return set_error(GSMC_E_INVALID, "null posterior output");
  if (n_pairs > 0x7fffffff - kThreads)
    return set_error(GSMC_E_INVALID, "too many pairs for one call");
  const int64_t S = v.n_sites;
  if (S >= 0x7fffffff) return set_error(GSMC_E_INVALID, "too many sites for one call");
  if (n_pairs == 0 || S == 0) return GSMC_OK;
  // Core and flank clamped to the sequence in int64 before anything is
  // narrowed: a flank of 2^40 means "reach both ends", as in the context path.
  const int64_t core = clamp_core(core_block_sites, S);
  const int64_t flank = clamp_flank(flank_sites, S);
  const size_t slot_bytes = (size_t)core * kThreads * sizeof(float2);
  const int64_t capacity = (int64_t)((kNoAllocScratchBytes - kCounterBytes) / slot_bytes);
  if (capacity < 1) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "core_block_sites=%lld is too large for the allocation-free entry point: it "
                  "needs %zu bytes of scratch per CTA, the fixed scratch holds %zu (at most %zu "
                  "core sites)",
                  (long long)core_block_sites, slot_bytes, kNoAllocScratchBytes - kCounterBytes,
                  (kNoAllocScratchBytes - kCounterBytes) / (kThreads * sizeof(float2)));
    return set_error(GSMC_E_INVALID, msg);
  }
  cudaError_t e = cudaSetDevice(v.device);
  unsigned char* scratch = nullptr;
  if (e == cudaSuccess) {
    const int rc = scratch_address(v.device, &scratch);
    if (rc) return rc;
  }
  const int64_t windows = window_count(S, core);
  const int64_t tiles = (n_pairs + kThreads - 1) / kThreads;
  if (windows * tiles > 0x7fffffff) return set_error(GSMC_E_INVALID, "too many tasks for one call");
  NoAllocArgs a;
  std::memset(&a, 0, sizeof(a));
  a.scan.geno = v.geno;
  a.scan.n_haps = v.n_haps;
  a.scan.code = v.code;
  a.scan.site_tab = v.site_tab;
  a.scan.chunk_tab = v.chunk_tab;
  a.scan.L = v.L;
  a.pi = d_pair_i;
  a.pj = d_pair_j;
  a.counter = reinterpret_cast<int*>(scratch);
  a.slots = reinterpret_cast<float2*>(scratch + kCounterBytes);
  a.slot_rows = core;
  a.n_sites = S;
  a.core = core;
  a.flank = flank;
  a.n_pairs = (int)n_pairs;
  a.tiles = (int)tiles;
  a.n_tasks = (int)(windows * tiles);
  a.flags = ((flags & GSMC_CI) ? kTaskCI : 0) | ((flags & GSMC_POSTERIOR) ? kTaskPosterior : 0);
  a.unscale = 2.0f * v.ne;
  a.out[0] = d_mean;
  a.out[1] = (flags & GSMC_CI) ? d_lower : nullptr;
  a.out[2] = (flags & GSMC_CI) ? d_upper : nullptr;
  a.out[3] = (flags & GSMC_POSTERIOR) ? d_alpha : nullptr;
  a.out[4] = (flags & GSMC_POSTERIOR) ? d_beta : nullptr;
  a.ldo = ld_out;
  a.col0 = out_col0;
  int sms = 0, per_sm = 0;
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.device);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fb_scan_noalloc, kThreads, 0);
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(a.counter, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    const int64_t grid = std::max<int64_t>(
        1, std::min<int64_t>({(int64_t)sms * std::max(per_sm, 1), capacity, (int64_t)a.n_tasks}));
    fb_scan_noalloc<<<(unsigned)grid, kThreads, 0, st>>>(a);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    char msg[256];
    std::snprintf(msg, sizeof(msg), "CUDA error: %s (allocation-free scan)", cudaGetErrorString(e));
    return set_error(GSMC_E_CUDA, msg);
  }
  return GSMC_OK;
}
