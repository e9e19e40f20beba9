// C ABI of the B200 Gamma-SMC scan: contexts, table sets, window planning and
// the host/device entry points declared in include/gsmc_b200.h.
#include <cuda_runtime.h>
#include <sys/mman.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "ctx_view.h"
#include "flowgen.h"
#include "fwd.h"
#include "gsmc_b200.h"
#include "hostcopy.h"
#include "scan.h"
#include "tables.h"
#include "tables_gpu.h"
#include "uncached.h"
#include "planner.h"
#include "windows.h"

using namespace gsmc;

namespace {

thread_local std::string g_last_error;

// Speculative chunking of the calling thread's last gsmc_flow_fb call.
struct FlowFbStats {
  int chunks = 1;
  int64_t repaired = 0;
};
thread_local FlowFbStats g_flow_fb_stats;

// Page-locked result buffers (gsmc_host_alloc): blocks in use, and released
// blocks kept for reuse (up to g_host_cache_cap bytes), oldest first.
struct HostBlk {
  void* p;
  uint64_t bytes;  // usable bytes (a mapped block: the whole mapping)
  bool mapped;     // an anonymous mapping registered with CUDA, else cudaHostAlloc
};
std::mutex g_host_mu;
std::map<void*, HostBlk> g_host_used;
std::vector<HostBlk> g_host_free;
uint64_t g_host_cached = 0;
uint64_t g_host_cache_cap = uint64_t(256) << 30;

// Blocks of at least this many bytes are anonymous mappings advised
// MADV_HUGEPAGE, page-locked with cudaHostRegister: on a B200 host that
// page-locked 16 GB in 2.0 s against 6.5 s for cudaHostAlloc (4 KB pages
// registered: 4.8 s).
constexpr uint64_t kMappedMin = uint64_t(64) << 20;
constexpr uint64_t kHugePage = uint64_t(2) << 20;

// A new page-locked block of at least `bytes`.
cudaError_t new_host_block(uint64_t bytes, HostBlk* out) {
  if (bytes >= kMappedMin) {
    const uint64_t size = (bytes + kHugePage - 1) / kHugePage * kHugePage;
    void* p = mmap(nullptr, size, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (p != MAP_FAILED) {
      madvise(p, size, MADV_HUGEPAGE);  // advice only: ignored where unsupported
      const cudaError_t e = cudaHostRegister(p, size, cudaHostRegisterPortable);
      if (e == cudaSuccess) {
        *out = HostBlk{p, size, true};
        return cudaSuccess;
      }
      munmap(p, size);
      return e;
    }
  }
  void* p = nullptr;
  const cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocPortable);
  if (e == cudaSuccess) *out = HostBlk{p, bytes, false};
  return e;
}

// Take cached blocks out until the cache is within its cap; the caller frees
// them with free_host_blocks after releasing g_host_mu (unpinning a large
// block takes seconds, and other threads' allocations must not wait on it).
std::vector<HostBlk> trim_host_cache_locked() {
  std::vector<HostBlk> out;
  while (g_host_cached > g_host_cache_cap && !g_host_free.empty()) {
    out.push_back(g_host_free.front());
    g_host_cached -= g_host_free.front().bytes;
    g_host_free.erase(g_host_free.begin());
  }
  return out;
}

void free_host_blocks(const std::vector<HostBlk>& blocks) {
  for (const HostBlk& b : blocks) {
    if (b.mapped) {
      cudaHostUnregister(b.p);
      munmap(b.p, b.bytes);
    } else {
      cudaFreeHost(b.p);
    }
  }
}

// mbarrier polls the uncached kernels wait for their flow-field copy.
std::atomic<long long> g_copy_wait_polls{kDefaultCopyWaitPolls};

int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(expr)                                                              \
  do {                                                                              \
    cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(GSMC_E_CUDA, "CUDA error: %s (%s)", cudaGetErrorString(e_), #expr); \
  } while (0)

// ------------------------------------------------------------ table sets --
// One resident set of scan tables per (device, flow field, Ne, mu, rho, L,
// build), shared by every context with those parameters.  (The reference
// keeps a single process-global set and frees it under live contexts when the
// parameters change, src/bindings.cpp:2016-2041.)
//
// A set is built outside the global lock: the first context to ask for a key
// inserts an in-progress entry and builds; others asking for the same key
// wait for it, and other keys proceed meanwhile.  When its last context
// closes, a set is parked: the most recently released set of each device
// stays resident for the next context with the same parameters (as the
// reference's process-wide cache does), and parking a newer set frees the
// older one.  gsmc_free_cached_tables frees parked sets.
struct TableSet {
  int device = 0;
  int L = 0;
  float4* site = nullptr;   // [4][L][2450][2]
  float4* chunk = nullptr;  // [2450][2]
  // the hom multi-step table, kept on the host until the forward-only path
  // first needs its half-precision patch copy (built on the device then)
  std::vector<float> hom_m, hom_c;  // [L][2550]
  uint4* hom_half = nullptr;        // [L][2450] half patches
  std::mutex half_mu;
  int refs = 0;
  bool ready = false;       // build finished (status says how)
  int status = GSMC_OK;
  std::string error;
  double build_seconds = 0.0;  // build + upload
};

// (device, flow field, Ne, mu, rho, layers, float64 GPU build)
using TableKey = std::tuple<int, std::string, float, float, float, int, bool>;
std::mutex g_tables_mu;
std::condition_variable g_tables_cv;
std::map<TableKey, TableSet*> g_tables;
std::map<int, TableSet*> g_parked;  // device -> its released, still resident set

void free_table_set(TableSet* ts) {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ts->device);
  cudaFree(ts->site);
  cudaFree(ts->chunk);
  cudaFree(ts->hom_half);
  cudaSetDevice(prev);
  delete ts;
}

void erase_key_of(TableSet* ts) {
  for (auto it = g_tables.begin(); it != g_tables.end(); ++it)
    if (it->second == ts) {
      g_tables.erase(it);
      return;
    }
}

// Drop one reference (g_tables_mu held).  A built set whose last reference
// goes is parked; the set it displaces, or a set whose build failed, is freed.
void drop_ref_locked(TableSet* ts) {
  if (--ts->refs > 0) return;
  if (ts->status != GSMC_OK) {
    free_table_set(ts);  // already out of the map
    return;
  }
  auto it = g_parked.find(ts->device);
  if (it != g_parked.end() && it->second != ts) {
    TableSet* old = it->second;
    erase_key_of(old);
    free_table_set(old);
  }
  g_parked[ts->device] = ts;
}

// Float64 build on the device (tables_gpu.cu) of one set, into ts.
int build_table_set_f64(const FlowField& ff, double ne, double mu, double rho, int L, TableSet* ts,
                        std::string* err) {
  int prev = 0;
  cudaGetDevice(&prev);
  const size_t site_bytes = (size_t)kScanTables * L * kPatches * 8 * sizeof(float);
  const size_t chunk_bytes = (size_t)kPatches * 8 * sizeof(float);
  cudaError_t e = cudaSetDevice(ts->device);
  if (e == cudaSuccess) e = cudaMalloc(&ts->site, site_bytes);
  if (e == cudaSuccess) e = cudaMalloc(&ts->chunk, chunk_bytes);
  int rc = GSMC_OK;
  if (e != cudaSuccess) {
    cudaGetLastError();
    *err = std::string("CUDA error: ") + cudaGetErrorString(e) + " (scan table allocation)";
    rc = GSMC_E_CUDA;
  } else if (build_tables_gpu_f64(ff, L, 4.0 * ne * rho, 4.0 * ne * mu, ts->site, ts->chunk,
                                  &ts->hom_m, &ts->hom_c, err) != 0) {
    rc = GSMC_E_CUDA;
  }
  cudaSetDevice(prev);
  return rc;
}

// Build and upload of one set (no lock held): the host float32 build that
// matches the reference bit for bit, or the float64 GPU build.
int build_table_set(const char* ff_path, double ne_d, double mu_d, double rho_d, int L, bool f64,
                    TableSet* ts, std::string* err) {
  FlowField ff;
  char buf[512];
  if (load_flow_field(ff_path, &ff, buf, sizeof(buf)) != 0) {
    *err = buf;
    return GSMC_E_IO;
  }
  if (f64) return build_table_set_f64(ff, ne_d, mu_d, rho_d, L, ts, err);
  const float ne = (float)ne_d, mu = (float)mu_d, rho = (float)rho_d;
  float srho, smu;
  scaled_rates(ne, mu, rho, &srho, &smu);
  HostLayers layers;
  build_layers(ff, L, srho, smu, 0, &layers);
  std::vector<float> site, chunk;
  build_scan_layout(layers, &site, &chunk, 0);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaError_t e = cudaSetDevice(ts->device);
  if (e == cudaSuccess) e = cudaMalloc(&ts->site, site.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&ts->chunk, chunk.size() * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemcpy(ts->site, site.data(), site.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(ts->chunk, chunk.data(), chunk.size() * sizeof(float), cudaMemcpyHostToDevice);
  cudaSetDevice(prev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *err = std::string("CUDA error: ") + cudaGetErrorString(e) + " (scan table upload)";
    return GSMC_E_CUDA;
  }
  ts->hom_m = std::move(layers.t[kHomMean]);
  ts->hom_c = std::move(layers.t[kHomCv]);
  return GSMC_OK;
}

// The set for a key, built if needed; *reused is false when this call built
// it.
int acquire_tables(int device, const char* ff_path, double ne, double mu, double rho, int L,
                   bool f64, TableSet** out, bool* reused) {
  const TableKey key{device, std::string(ff_path), (float)ne, (float)mu, (float)rho, L, f64};
  std::unique_lock<std::mutex> lock(g_tables_mu);
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    TableSet* ts = it->second;
    if (ts->refs++ == 0) {
      auto pk = g_parked.find(device);
      if (pk != g_parked.end() && pk->second == ts) g_parked.erase(pk);
    }
    g_tables_cv.wait(lock, [ts] { return ts->ready; });
    if (ts->status != GSMC_OK) {
      const int st = ts->status;
      const std::string msg = ts->error;
      drop_ref_locked(ts);
      return fail(st, "%s", msg.c_str());
    }
    *out = ts;
    *reused = true;
    return GSMC_OK;
  }
  TableSet* ts = new TableSet;
  ts->device = device;
  ts->L = L;
  ts->refs = 1;
  g_tables[key] = ts;
  lock.unlock();
  const auto t0 = std::chrono::steady_clock::now();
  std::string err;
  const int st = build_table_set(ff_path, ne, mu, rho, L, f64, ts, &err);
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  lock.lock();
  ts->build_seconds = secs;
  ts->status = st;
  ts->error = err;
  ts->ready = true;
  g_tables_cv.notify_all();
  if (st != GSMC_OK) {
    erase_key_of(ts);
    drop_ref_locked(ts);
    return fail(st, "%s", err.c_str());
  }
  *out = ts;
  *reused = false;
  return GSMC_OK;
}

void release_tables(TableSet* ts) {
  if (!ts) return;
  std::lock_guard<std::mutex> lock(g_tables_mu);
  drop_ref_locked(ts);
}

// max(1, round-half-even(delta)) (src/kernels/gamma_smc_flow.cu:160-163).
int seg_steps(double delta) {
  const double r = std::nearbyint(delta);
  if (!(r >= 1.0)) return 1;
  if (r > 2147483647.0) return 2147483647;
  return (int)r;
}

struct Block {
  int64_t cs, ce, ps, pe;
};

// Windows core +/- flank clamped to [0, S) (src/bindings.cpp:2517-2534).
std::vector<Block> make_windows(int64_t S, int64_t core, int64_t flank) {
  std::vector<Block> out;
  const int64_t n = window_count(S, core);
  out.reserve((size_t)n);
  for (int64_t w = 0; w < n; ++w) {
    const WindowBounds b = window_bounds(w, S, core, flank);
    out.push_back({b.cs, b.ce, b.ps, b.pe});
  }
  return out;
}

}  // namespace


struct gsmc_ctx {
  int device = 0;
  int64_t n_haps = 0, n_sites = 0, n_groups = 0;
  float ne = 0.0f;
  ulonglong2* geno = nullptr;
  SiteCode* code = nullptr;  // site 0 of the code array (kCodePad entries before it)
  TableSet* tables = nullptr;
  double tables_build_seconds = 0.0;  // this context's table build and upload
  bool tables_reused = false;         // the tables were resident already
  ScanShape shape{128, 1};  // scan launch shape of the current call (pick_shape)
  bool shape_fixed = false; // shape set by the environment, not per call
  cudaStream_t stream = nullptr;
  // scratch, grown on demand and kept for the context's lifetime
  void* pool = nullptr;  // forward-state slots of the persistent CTAs
  size_t pool_bytes = 0;
  int32_t* pairs = nullptr;  // host-path pair indices: [pi | pj]
  int64_t pairs_cap = 0;
  float* stage = nullptr;  // host-path output stage: two halves (or summary partials)
  size_t stage_bytes = 0;
  void* acc = nullptr;     // summary accumulators: double sum, float min, max, mean per site
  size_t acc_bytes = 0;
  // speculative chunks: boundary records, window descriptors, repair list
  float2* spec_rec = nullptr;
  size_t spec_rec_bytes = 0;
  SpecWindow* spec_win = nullptr;
  size_t spec_win_bytes = 0;
  unsigned char* spec_repairs = nullptr;  // [TaskListHead | Task...]
  size_t spec_repairs_bytes = 0;
  void* repair_pool = nullptr;            // forward-state slots of the repair launch
  size_t repair_pool_bytes = 0;
  bool speculate = true;                  // GSMC_SPECULATE=0 turns chunking off
  double pool_fraction = 0.8;             // of free device memory for forward-state slots
  int64_t spec_max_chunk = 16384;         // longest chunk core when a window is cut (0: no cap)
  // Cost of a core site in burn-in sites when chunk cuts are balanced: its
  // forward step also stores the state, its backward step reads it back and
  // combines.  2 measured best of 1-2 (8,192 pairs x 50,000 sites, 12 chunks:
  // 7.25 -> 6.70 ms; all 63,190 pairs, 4 chunks: 31.46 -> 31.17 ms).  The
  // chunk-count model keeps counting plain pair-steps: its wave coefficients
  // were fitted that way, and weighting there moved the slice to 9 chunks
  // (33 ms against 31).
  double core_weight = 2.0;
  int spec_chunks_fixed = 0;              // GSMC_SPEC_CHUNKS: chunks per window, for measurements
  int64_t spec_flank = 2048;              // burn-in sites of a speculative chunk
  int64_t spec_launches = 0;              // launches that ran speculative chunks
  int* spec_repaired = nullptr;           // device: (window, pair)s repaired so far
  // streaming: pinned host halves the sink reads, and the copy stream
  float* pinned = nullptr;
  size_t pinned_bytes = 0;
  cudaStream_t copy_stream = nullptr;
  std::vector<double> positions;  // host copy, for the forward-only gap codes
  FwdCode* fwd_code = nullptr;    // forward-only gap codes, built on first use
  unsigned char* tasks[2] = {nullptr, nullptr};  // task lists of alternating launches
  size_t tasks_cap[2] = {0, 0};                  // bytes
  cudaEvent_t stage_free[2] = {nullptr, nullptr};
  cudaEvent_t launch_done[2] = {nullptr, nullptr};
  // measurement: events around scan launches while timing is on
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  int64_t launches = 0;
  double pair_sites = 0.0;
};

namespace {

template <class T>
int ensure_buffer(T** buf, size_t* cap_bytes, size_t bytes) {
  if (bytes <= *cap_bytes) return GSMC_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap_bytes = 0;
  const cudaError_t e = cudaMalloc(buf, bytes);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    return fail(GSMC_E_NOMEM, "CUDA error: out of memory allocating %zu bytes of scratch", bytes);
  }
  if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (scratch allocation)", cudaGetErrorString(e));
  *cap_bytes = bytes;
  return GSMC_OK;
}

int upload_pairs(gsmc_ctx* ctx, const int32_t* pi, const int32_t* pj, int64_t P) {
  for (int64_t p = 0; p < P; ++p) {
    if (pi[p] < 0 || pi[p] >= ctx->n_haps || pj[p] < 0 || pj[p] >= ctx->n_haps)
      return fail(GSMC_E_INVALID, "pair %lld = (%d, %d) is out of range for %lld haplotypes",
                  (long long)p, pi[p], pj[p], (long long)ctx->n_haps);
  }
  if (P > ctx->pairs_cap) {
    if (ctx->pairs) cudaFree(ctx->pairs);
    ctx->pairs = nullptr;
    ctx->pairs_cap = 0;
    CUDA_TRY(cudaMalloc(&ctx->pairs, 2 * P * sizeof(int32_t)));
    ctx->pairs_cap = P;
  }
  CUDA_TRY(cudaMemcpyAsync(ctx->pairs, pi, P * sizeof(int32_t), cudaMemcpyHostToDevice,
                           ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(ctx->pairs + ctx->pairs_cap, pj, P * sizeof(int32_t),
                           cudaMemcpyHostToDevice, ctx->stream));
  return GSMC_OK;
}

int n_outputs(int flags) {
  return 1 + ((flags & GSMC_CI) ? 2 : 0) + ((flags & GSMC_POSTERIOR) ? 2 : 0);
}

int task_flags(int flags) {
  return ((flags & GSMC_CI) ? kTaskCI : 0) | ((flags & GSMC_POSTERIOR) ? kTaskPosterior : 0);
}

size_t free_device_bytes() {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) return 0;
  return f;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Resident CTAs of the persistent kernel, optionally capped for experiments.
int resident_ctas(ScanShape shape) {
  int r = std::max(1, scan_resident_ctas(shape));
  if (const char* env = std::getenv("GSMC_MAX_CTAS")) r = std::max(1, std::min(r, std::atoi(env)));
  return r;
}

int spec_chunks(const gsmc_ctx* ctx, int64_t tasks, int64_t resident_tiles, int64_t core_len,
                int flags, double row_bytes = 0.0, double slot_budget = 0.0);
plan::ChunkPolicy chunk_policy(const gsmc_ctx* ctx) {
  plan::ChunkPolicy p;
  p.burn_in = ctx->spec_flank;
  p.max_chunk = ctx->spec_max_chunk;
  return p;
}
using plan::chunk_steps;
using plan::launch_cost;
int64_t max_core(const std::vector<Block>& blocks);

// Launch shape of a call over P pairs x `blocks`: two pairs per thread (two
// independent lookup chains per thread; 6-8% faster per pair) when that
// gives every resident CTA two (window, pair tile) tasks; otherwise the shape
// whose best speculative chunking has the lower launch_cost, a two-pair tile
// task taking 1.45 times a one-pair one (twice the pairs per thread, 8
// instead of 10 resident CTAs per SM, 10% faster per pair).
void pick_shape(gsmc_ctx* ctx, int64_t P, const std::vector<Block>& blocks, int flags) {
  if (ctx->shape_fixed) return;
  const ScanShape two{scan_threads(), 2}, one{scan_threads(), 1};
  const int64_t core = max_core(blocks);
  auto cost = [&](ScanShape sh, double per_step) {
    const int64_t tasks = (int64_t)blocks.size() * ceil_div(P, scan_tile_pairs(sh));
    const int64_t tiles = (int64_t)resident_ctas(sh) * scan_tiles_per_cta(sh);
    const int K = spec_chunks(ctx, tasks, tiles, core, flags);
    return per_step * launch_cost(tasks * K, tiles, chunk_steps(core, K, ctx->spec_flank, 1.0));
  };
  const int64_t tasks2 = (int64_t)blocks.size() * ceil_div(P, scan_tile_pairs(two));
  const bool use_two = tasks2 >= 2 * resident_ctas(two) || cost(two, 1.45) <= cost(one, 1.0);
  ctx->shape = use_two ? two : one;
}

// Pair-steps of a task per pair: forward over [ps, ce), backward over [cs, pe).
int64_t task_steps(const Task& t) { return (int64_t)(t.ce - t.ps) + (t.pe - t.cs); }

// Longest tasks first, so the persistent grid's tail is made of short tasks.
void order_longest_first(std::vector<Task>* tasks) {
  std::stable_sort(tasks->begin(), tasks->end(),
                   [](const Task& a, const Task& b) { return task_steps(a) > task_steps(b); });
}

// Host image of a device task list: head (next = 0, count) then the tasks.
void write_task_list(const std::vector<Task>& tasks, unsigned char* dst) {
  TaskListHead head{0, (int)tasks.size()};
  std::memset(dst, 0, kTaskListHead);
  std::memcpy(dst, &head, sizeof(head));
  if (!tasks.empty()) std::memcpy(dst + kTaskListHead, tasks.data(), tasks.size() * sizeof(Task));
}

size_t task_list_bytes(size_t n) { return kTaskListHead + n * sizeof(Task); }

// Where the outputs of one window go: element (s, pair j) at
// out[k][off + (s - row0) * ldo + j].
struct WindowOut {
  float* out[5];
  int64_t off;
  int64_t ldo;
  int64_t row0;
};

// Append the tasks of one window for the n pairs (pi[p], pj[p]), pair tile by
// pair tile; `col` is the output column of pair 0.
void add_window_tasks(const Block& b, const int32_t* pi, const int32_t* pj, int64_t n, int tile,
                      const WindowOut& wo, int64_t col, int flags, float unscale,
                      std::vector<Task>* tasks) {
  for (int64_t j = 0; j < n; j += tile) {
    Task t;
    std::memset(&t, 0, sizeof(t));
    t.ps = (int32_t)b.ps;
    t.cs = (int32_t)b.cs;
    t.ce = (int32_t)b.ce;
    t.pe = (int32_t)b.pe;
    t.pi = pi + j;
    t.pj = pj + j;
    t.pair_count = (int32_t)std::min<int64_t>(tile, n - j);
    t.out_row0 = (int32_t)wo.row0;
    t.flags = flags;
    t.out_off = wo.off + col + j;
    t.ldo = wo.ldo;
    for (int k = 0; k < 5; ++k) t.out[k] = wo.out[k];
    t.unscale = unscale;
    tasks->push_back(t);
  }
}

// Fill the ScanArgs fields that come from the context.
void ctx_scan_args(const gsmc_ctx* ctx, ScanArgs* a) {
  std::memset(a, 0, sizeof(*a));
  a->geno = ctx->geno;
  a->n_haps = ctx->n_haps;
  a->code = ctx->code;
  a->site_tab = ctx->tables->site;
  a->chunk_tab = ctx->tables->chunk;
  a->L = ctx->tables->L;
}

// Upload a task list into buffer `which` and launch the persistent scan with
// up to `grid` CTAs over it; forward-state slots of slot_rows sites.
int launch_tasks(gsmc_ctx* ctx, std::vector<Task>& tasks, int which, int64_t slot_rows, int grid,
                 cudaStream_t stream) {
  if (tasks.empty()) return GSMC_OK;
  order_longest_first(&tasks);
  const size_t bytes = task_list_bytes(tasks.size());
  int rc = ensure_buffer(&ctx->tasks[which], &ctx->tasks_cap[which], bytes);
  if (rc) return rc;
  std::vector<unsigned char> image(bytes);
  write_task_list(tasks, image.data());
  CUDA_TRY(cudaMemcpyAsync(ctx->tasks[which], image.data(), bytes, cudaMemcpyHostToDevice, stream));
  ScanArgs a;
  ctx_scan_args(ctx, &a);
  TaskListHead* head = reinterpret_cast<TaskListHead*>(ctx->tasks[which]);
  a.next = &head->next;
  a.count = &head->count;
  a.tasks = reinterpret_cast<const Task*>(ctx->tasks[which] + kTaskListHead);
  a.fwd = static_cast<float2*>(ctx->pool);
  a.slot_rows = slot_rows;
  const int tiles = scan_tiles_per_cta(ctx->shape);
  grid = (int)std::min<int64_t>(grid, ceil_div((int64_t)tasks.size(), tiles));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ctx->timing) {
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, stream));
  }
  const bool summary = (tasks.front().flags & kTaskSummary) != 0;
  CUDA_TRY(launch_scan(a, grid, ctx->shape, stream, summary));
  ctx->launches++;
  for (const Task& t : tasks) ctx->pair_sites += (double)t.pair_count * (double)(t.ce - t.cs);
  if (ctx->timing) {
    CUDA_TRY(cudaEventRecord(e1, stream));
    ctx->events.emplace_back(e0, e1);
  }
  return GSMC_OK;
}

int64_t max_core(const std::vector<Block>& blocks) {
  int64_t m = 0;
  for (const Block& b : blocks) m = std::max(m, b.ce - b.cs);
  return m;
}

// Bytes of one CTA's forward-state slots for a shape.
size_t cta_slot_bytes(ScanShape shape, int64_t slot_rows) {
  return (size_t)slot_rows * scan_tile_pairs(shape) * scan_tiles_per_cta(shape) * sizeof(float2);
}

// Size the forward-state pool for up to `want` CTAs within `budget` bytes;
// returns the CTA count it can hold (>= 1) or a negative status.
int size_pool(gsmc_ctx* ctx, int64_t slot_rows, int want, size_t budget, int* grid) {
  const size_t slot = cta_slot_bytes(ctx->shape, slot_rows);
  int64_t g = std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)(budget / std::max<size_t>(slot, 1))));
  int rc = ensure_buffer(reinterpret_cast<char**>(&ctx->pool), &ctx->pool_bytes, (size_t)g * slot);
  if (rc) return rc;
  *grid = (int)g;
  return GSMC_OK;
}

// ---------------------------------------------------------- speculation --
// When a launch has fewer (window, pair tile) tasks than the GPU has resident
// tiles, long windows are cut into chunks that run in parallel: chunk k > 0
// starts its forward pass spec_flank (2,048) sites before its core, from
// (0, 0), instead of at the window's start, and chunk k < K-1 starts its
// backward pass spec_flank sites after its core; chunks have at least
// 4 x spec_flank core sites.  Each chunk records its boundary
// states (see Task); a verify kernel compares neighbours bit for bit, and
// every (window, pair) whose speculative trajectories did not join the exact
// ones is decoded again whole by a repair launch on the same stream.  The
// outputs are therefore exactly those of the unchunked window.
constexpr size_t kRepairPoolBytes = size_t(512) << 20;

struct SpecLaunch {
  std::vector<SpecWindow> windows;  // windows cut into more than one chunk
  int64_t n_bnd = 0;                // boundaries over all of them
  int64_t n_pairs = 0;              // pairs of the launch (record stride)
  int64_t max_core = 0;             // longest whole core (repair slot rows)
};

// Cut points of window b's core into K speculative chunks of equal cost
// (chunk_cuts in windows.h).
std::vector<int64_t> chunk_cuts(const Block& b, int K, int64_t flank, double w) {
  std::vector<int64_t> c(std::max(K, 1) + 1);
  gsmc::chunk_cuts(b.ps, b.cs, b.ce, b.pe, std::max(K, 1), flank, w, c.data());
  return c;
}

// Longest chunk core of window b cut into K chunks.
int64_t longest_chunk(const Block& b, int K, int64_t flank, double w) {
  const std::vector<int64_t> c = chunk_cuts(b, K, flank, w);
  int64_t m = 0;
  for (int k = 0; k < K; ++k) m = std::max(m, c[k + 1] - c[k]);
  return m;
}

// Chunks per window for a launch of `tasks` tasks on `resident_tiles` tiles
// (plan::choose_chunks), unless speculation is off, fixed, or a summary.
int spec_chunks(const gsmc_ctx* ctx, int64_t tasks, int64_t resident_tiles, int64_t core_len,
                int flags, double row_bytes, double slot_budget) {
  if (!ctx->speculate || (flags & kTaskSummary) || tasks <= 0) return 1;
  if (ctx->spec_chunks_fixed > 0)
    return (int)std::max<int64_t>(1, std::min<int64_t>(ctx->spec_chunks_fixed, core_len / 64));
  return plan::choose_chunks(chunk_policy(ctx), tasks, resident_tiles, core_len, row_bytes,
                             slot_budget);
}

// Append the tasks of window b for the n pairs at (pi, pj): whole, or in K
// speculative chunks whose boundary records start at record `sl->n_bnd` of
// `rec` (already sized).
void add_spec_window_tasks(const Block& b, int K, int64_t flank, double core_weight, const int32_t* pi,
                           const int32_t* pj, int64_t n, int tile, const WindowOut& wo,
                           int64_t col, int flags, float unscale, float2* rec, SpecLaunch* sl,
                           std::vector<Task>* tasks) {
  if (K <= 1) {
    add_window_tasks(b, pi, pj, n, tile, wo, col, flags, unscale, tasks);
    return;
  }
  const int64_t len = b.ce - b.cs;
  const int64_t bnd0 = sl->n_bnd;
  const std::vector<int64_t> cut = chunk_cuts(b, K, flank, core_weight);
  for (int k = 0; k < K; ++k) {
    const int64_t c0 = cut[k], c1 = cut[k + 1];
    const Block cb{c0, c1, k == 0 ? b.ps : std::max(b.ps, c0 - flank),
                   k == K - 1 ? b.pe : std::min(b.pe, c1 + flank)};
    const size_t first = tasks->size();
    add_window_tasks(cb, pi, pj, n, tile, wo, col, flags, unscale, tasks);
    for (size_t i = first; i < tasks->size(); ++i) {
      Task& t = (*tasks)[i];
      const int64_t j = (int64_t)(i - first) * tile;  // the tile's first pair in the launch
      t.bl = k > 0 ? rec + (bnd0 + k - 1) * 4 * n + j : nullptr;
      t.br = k < K - 1 ? rec + (bnd0 + k) * 4 * n + j : nullptr;
      t.bstride = n;
    }
  }
  SpecWindow w;
  std::memset(&w, 0, sizeof(w));
  w.first_bnd = (int32_t)bnd0;
  w.n_bnd = K - 1;
  std::vector<Task> whole;
  add_window_tasks(b, pi, pj, 1, 1, wo, col, flags, unscale, &whole);
  w.repair = whole[0];
  sl->windows.push_back(w);
  sl->n_bnd += K - 1;
  sl->n_pairs = n;
  sl->max_core = std::max(sl->max_core, len);
}

// Size the record buffer for `n_bnd` boundaries of n pairs.
int spec_reserve(gsmc_ctx* ctx, int64_t n_bnd, int64_t n) {
  if (n_bnd <= 0) return GSMC_OK;
  return ensure_buffer(&ctx->spec_rec, &ctx->spec_rec_bytes,
                       (size_t)n_bnd * 4 * n * sizeof(float2));
}

// After a speculative launch: verify the boundaries, then repair on the
// same stream.  The repair launch always runs (it ends at once when no pair
// needs it), so nothing here waits for the device.
int spec_finish(gsmc_ctx* ctx, const SpecLaunch& sl, cudaStream_t stream) {
  if (sl.windows.empty()) return GSMC_OK;
  const int n_win = (int)sl.windows.size();
  int rc = ensure_buffer(&ctx->spec_win, &ctx->spec_win_bytes, sl.windows.size() * sizeof(SpecWindow));
  if (rc) return rc;
  const int64_t max_rep = (int64_t)n_win * sl.n_pairs;
  rc = ensure_buffer(&ctx->spec_repairs, &ctx->spec_repairs_bytes,
                     kTaskListHead + (size_t)max_rep * sizeof(Task));
  if (rc) return rc;
  const ScanShape rshape{32, 1};
  const size_t warp_slot = (size_t)sl.max_core * 32 * sizeof(float2);
  const int64_t rctas = std::max<int64_t>(1, std::min<int64_t>(
      16, (int64_t)(kRepairPoolBytes / (warp_slot * scan_tiles_per_cta(rshape)))));
  rc = ensure_buffer(reinterpret_cast<char**>(&ctx->repair_pool), &ctx->repair_pool_bytes,
                     (size_t)rctas * scan_tiles_per_cta(rshape) * warp_slot);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(ctx->spec_win, sl.windows.data(), sl.windows.size() * sizeof(SpecWindow),
                           cudaMemcpyHostToDevice, stream));
  TaskListHead* head = reinterpret_cast<TaskListHead*>(ctx->spec_repairs);
  Task* repairs = reinterpret_cast<Task*>(ctx->spec_repairs + kTaskListHead);
  CUDA_TRY(cudaMemsetAsync(head, 0, sizeof(TaskListHead), stream));
  CUDA_TRY(launch_spec_verify(ctx->spec_rec, sl.n_pairs, ctx->spec_win, n_win, head, repairs,
                              (int)std::min<int64_t>(max_rep, 0x7fffffff), stream));
  if (!ctx->spec_repaired) {
    CUDA_TRY(cudaMalloc(&ctx->spec_repaired, sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(ctx->spec_repaired, 0, sizeof(int), stream));
  }
  CUDA_TRY(launch_add_count(&head->count, ctx->spec_repaired, stream));
  ScanArgs a;
  ctx_scan_args(ctx, &a);
  a.next = &head->next;
  a.count = &head->count;
  a.tasks = repairs;
  a.fwd = static_cast<float2*>(ctx->repair_pool);
  a.slot_rows = sl.max_core;
  CUDA_TRY(launch_scan(a, (int)rctas, rshape, stream, false));
  ctx->spec_launches++;
  ctx->launches += 3;  // verify, count fold, repair scan
  return GSMC_OK;
}

// All windows x all pairs in one persistent launch, outputs written straight
// into the caller's device arrays.
int run_direct(gsmc_ctx* ctx, const int32_t* d_pi, const int32_t* d_pj, int64_t P,
               const std::vector<Block>& blocks, int flags, float* const out[5], int64_t ld,
               int64_t col0, cudaStream_t stream) {
  if (P == 0 || blocks.empty()) return GSMC_OK;
  pick_shape(ctx, P, blocks, flags);
  const int tile = scan_tile_pairs(ctx->shape);
  const int64_t resident_tiles = (int64_t)resident_ctas(ctx->shape) * scan_tiles_per_cta(ctx->shape);
  const int64_t plain_tasks = (int64_t)blocks.size() * ceil_div(P, tile);
  const size_t budget = (size_t)(ctx->pool_fraction * (double)free_device_bytes()) + ctx->pool_bytes;
  std::vector<int> K(blocks.size());
  int64_t n_bnd = 0;
  for (size_t i = 0; i < blocks.size(); ++i)
    K[i] = spec_chunks(ctx, plain_tasks, resident_tiles, blocks[i].ce - blocks[i].cs, flags,
                       (double)tile * sizeof(float2), (double)budget);
  if (ctx->speculate && ctx->spec_chunks_fixed == 0 && !(flags & kTaskSummary)) {
    std::vector<int64_t> core(blocks.size());
    for (size_t i = 0; i < blocks.size(); ++i) core[i] = blocks[i].ce - blocks[i].cs;
    plan::split_tail(chunk_policy(ctx), ceil_div(P, tile), resident_tiles, core, &K);
  }
  for (size_t i = 0; i < blocks.size(); ++i) n_bnd += K[i] - 1;
  int rc = spec_reserve(ctx, n_bnd, P);
  if (rc) return rc;
  std::vector<Task> tasks;
  SpecLaunch sl;
  WindowOut wo{{out[0], out[1], out[2], out[3], out[4]}, 0, ld, 0};
  for (size_t i = 0; i < blocks.size(); ++i)
    add_spec_window_tasks(blocks[i], K[i], ctx->spec_flank, ctx->core_weight, d_pi, d_pj, P, tile, wo, col0,
                          task_flags(flags),
                          2.0f * ctx->ne, ctx->spec_rec, &sl, &tasks);
  int64_t slot_rows = 0;
  for (const Task& t : tasks) slot_rows = std::max<int64_t>(slot_rows, t.ce - t.cs);
  const int want = (int)std::min<int64_t>(resident_ctas(ctx->shape),
                                          ceil_div((int64_t)tasks.size(), scan_tiles_per_cta(ctx->shape)));
  int grid = 0;
  rc = size_pool(ctx, slot_rows, want, budget, &grid);
  if (rc) return rc;
  rc = launch_tasks(ctx, tasks, 0, slot_rows, grid, stream);
  if (rc) return rc;
  return spec_finish(ctx, sl, stream);
}

// Site chunks of a forward-only call over n pairs x S sites: enough (pair,
// chunk) threads to fill every SM (2,048 threads each), each chunk at least
// four burn-ins long.
int fwd_chunks(const gsmc_ctx* ctx, int64_t n, int64_t S) {
  if (!ctx->speculate || n <= 0) return 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
  const int64_t want = ceil_div((int64_t)sms * 2048, n);
  return (int)std::max<int64_t>(1, std::min<int64_t>(want, S / (4 * ctx->spec_flank)));
}

// Whether a summary over P pairs x `blocks` should go through per-pair means
// in speculative chunks: its plain tasks (one-pair-per-thread 128-pair tiles)
// leave resident tiles idle and its longest window can be cut.
bool summary_by_pairs(const gsmc_ctx* ctx, int64_t P, const std::vector<Block>& blocks) {
  const ScanShape one{scan_threads(), 1};
  const int64_t tasks = (int64_t)blocks.size() * ceil_div(P, scan_tile_pairs(one));
  const int64_t resident_tiles = (int64_t)resident_ctas(one) * scan_tiles_per_cta(one);
  if (tasks >= 2 * resident_tiles) return false;  // the plain tasks fill the GPU
  return spec_chunks(ctx, tasks, resident_tiles, max_core(blocks), 0) > 1;
}

// Windows x pairs into HOST arrays.  Windows go in groups; each group's
// launch writes its core rows into one half of a device stage while the
// copier streams the previous group's half to the host.
int run_to_host(gsmc_ctx* ctx, int64_t P, const std::vector<Block>& blocks, int64_t pair_cap,
                int flags, float* const host[5], int64_t row0) {
  if (P == 0 || blocks.empty()) return GSMC_OK;
  pick_shape(ctx, std::min(P, pair_cap), blocks, flags);
  HostCopier* copier = HostCopier::for_current_device();
  if (!copier) return fail(GSMC_E_CUDA, "CUDA error: no device for the host copier");
  const int nout = n_outputs(flags);
  const int tile = scan_tile_pairs(ctx->shape) * scan_tiles_per_cta(ctx->shape);  // pairs per CTA
  const int64_t core = max_core(blocks);
  const int64_t nb = (int64_t)blocks.size();
  const int resident = resident_ctas(ctx->shape);
  const size_t budget = (size_t)(0.75 * (double)free_device_bytes()) + ctx->pool_bytes +
                        ctx->stage_bytes;
  const size_t slot = cta_slot_bytes(ctx->shape, core);
  // pair chunk and windows per group: enough tasks per launch to fill the GPU
  // twice, within the budget for pool + two stage halves
  int64_t chunk = std::min<int64_t>(P, pair_cap > 0 ? pair_cap : P);
  int64_t group = 1;
  for (;;) {
    group = std::min<int64_t>(nb, std::max<int64_t>(1, ceil_div(2 * resident, ceil_div(chunk, tile))));
    for (;;) {
      const int64_t want = std::min<int64_t>(resident, group * ceil_div(chunk, tile));
      const size_t need = (size_t)want * slot + 2 * (size_t)group * core * chunk * nout * sizeof(float);
      if (need <= budget || group == 1) break;
      --group;
    }
    const int64_t want = std::min<int64_t>(resident, group * ceil_div(chunk, tile));
    const size_t need = (size_t)want * slot + 2 * (size_t)group * core * chunk * nout * sizeof(float);
    if (need <= budget || chunk <= tile) break;
    chunk = std::max<int64_t>(tile, chunk / 2);
  }
  chunk = plan::even_part(P, chunk);  // equal pair chunks, no small last one
  const size_t half = (size_t)group * core * chunk * nout;  // floats per stage half
  int rc = ensure_buffer(&ctx->stage, &ctx->stage_bytes, 2 * half * sizeof(float));
  if (rc) return rc;
  const size_t pool_budget = budget > 2 * half * sizeof(float) ? budget - 2 * half * sizeof(float) : slot;
  // speculative chunks per window (the same for every launch): a full
  // group's plain tasks decide; slots need only the longest chunk core
  const int ptile = scan_tile_pairs(ctx->shape);
  const int64_t resident_tiles = (int64_t)resident * scan_tiles_per_cta(ctx->shape);
  std::vector<int> K(blocks.size());
  int64_t slot_rows = 0, max_k = 1;
  for (size_t i = 0; i < blocks.size(); ++i) {
    const int64_t len = blocks[i].ce - blocks[i].cs;
    K[i] = spec_chunks(ctx, group * ceil_div(chunk, ptile), resident_tiles, len, flags,
                       (double)ptile * sizeof(float2), (double)pool_budget);
    slot_rows = std::max(slot_rows, K[i] > 1 ? longest_chunk(blocks[i], K[i], ctx->spec_flank, ctx->core_weight) : len);
    max_k = std::max<int64_t>(max_k, K[i]);
  }
  // CTAs one launch can keep busy: its (chunk, pair tile) tasks, at most
  const int busy = (int)std::min<int64_t>(resident, group * max_k * ceil_div(chunk, tile));
  int grid = 0;
  rc = size_pool(ctx, slot_rows, busy, pool_budget, &grid);
  if (rc) return rc;
  for (int i = 0; i < 2; ++i) {
    if (!ctx->stage_free[i]) CUDA_TRY(cudaEventCreateWithFlags(&ctx->stage_free[i], cudaEventDisableTiming));
    if (!ctx->launch_done[i]) CUDA_TRY(cudaEventCreateWithFlags(&ctx->launch_done[i], cudaEventDisableTiming));
  }
  const int32_t* d_pi = ctx->pairs;
  const int32_t* d_pj = ctx->pairs + ctx->pairs_cap;
  const int selected[5] = {1, (flags & GSMC_CI) ? 1 : 0, (flags & GSMC_CI) ? 1 : 0,
                           (flags & GSMC_POSTERIOR) ? 1 : 0, (flags & GSMC_POSTERIOR) ? 1 : 0};
  int64_t launch = 0;
  int first_err = GSMC_OK;
  for (int64_t off = 0; off < P && !first_err; off += chunk) {
    const int64_t n = std::min(chunk, P - off);
    for (int64_t g0 = 0; g0 < nb && !first_err; g0 += group, ++launch) {
      const int h = (int)(launch & 1);
      const int64_t ng = std::min(group, nb - g0);
      float* base = ctx->stage + (size_t)h * half;
      if (launch >= 2) CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->stage_free[h], 0));
      // stage layout of this half: [output k][window i][core rows][n pairs]
      std::vector<Task> tasks;
      int64_t n_bnd = 0;
      for (int64_t i = 0; i < ng; ++i) n_bnd += K[g0 + i] - 1;
      rc = spec_reserve(ctx, n_bnd, n);
      if (rc) return rc;
      SpecLaunch sl;
      for (int64_t i = 0; i < ng; ++i) {
        const Block& b = blocks[g0 + i];
        WindowOut wo;
        int used = 0;
        for (int k = 0; k < 5; ++k)
          wo.out[k] = selected[k] ? base + (size_t)(used++) * group * core * n : nullptr;
        wo.off = i * core * n;
        wo.ldo = n;
        wo.row0 = b.cs;
        add_spec_window_tasks(b, K[g0 + i], ctx->spec_flank, ctx->core_weight, d_pi + off, d_pj + off, n, ptile, wo, 0,
                              task_flags(flags), 2.0f * ctx->ne, ctx->spec_rec, &sl, &tasks);
      }
      rc = launch_tasks(ctx, tasks, h, slot_rows, grid, ctx->stream);
      if (rc) return rc;
      rc = spec_finish(ctx, sl, ctx->stream);
      if (rc) return rc;
      CUDA_TRY(cudaEventRecord(ctx->launch_done[h], ctx->stream));
      for (int64_t i = 0; i < ng; ++i) {
        const Block& b = blocks[g0 + i];
        int used = 0;
        for (int k = 0; k < 5; ++k) {
          if (!selected[k]) continue;
          const float* src = base + (size_t)(used++) * group * core * n + (size_t)i * core * n;
          const int e = copier->enqueue(host[k] + (size_t)(b.cs - row0) * P + off, (size_t)P * sizeof(float),
                                        src, (size_t)n * sizeof(float), (size_t)n * sizeof(float),
                                        (size_t)(b.ce - b.cs), ctx->launch_done[h]);
          if (e != cudaSuccess && !first_err)
            first_err = fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)",
                             cudaGetErrorString((cudaError_t)e));
        }
      }
      const int e = copier->record_reads_done(ctx->stage_free[h]);
      if (e != cudaSuccess && !first_err)
        first_err = fail(GSMC_E_CUDA, "CUDA error: %s (copy event)", cudaGetErrorString((cudaError_t)e));
    }
  }
  const int e = copier->drain();
  if (first_err) return first_err;
  if (e != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)", cudaGetErrorString((cudaError_t)e));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return GSMC_OK;
}

int check_ctx(const gsmc_ctx* ctx) {
  if (!ctx) return fail(GSMC_E_INVALID, "null context");
  return GSMC_OK;
}

}  // namespace

extern "C" {

const char* gsmc_last_error(void) { return g_last_error.c_str(); }

const char* gsmc_version(void) { return "gamma_smc_cu_b200 0.1.0 (sm_100a)"; }

int gsmc_mem_info(uint64_t* free_bytes, uint64_t* total_bytes) {
  size_t f = 0, t = 0;
  CUDA_TRY(cudaMemGetInfo(&f, &t));
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return GSMC_OK;
}

int gsmc_get_device_count(int* count) {
  CUDA_TRY(cudaGetDeviceCount(count));
  return GSMC_OK;
}

int gsmc_set_device(int device) {
  CUDA_TRY(cudaSetDevice(device));
  return GSMC_OK;
}

int gsmc_get_device(int* device) {
  CUDA_TRY(cudaGetDevice(device));
  return GSMC_OK;
}

int gsmc_ctx_create(const uint8_t* G, int64_t n_haps, int64_t n_sites, const double* positions,
                    double Ne, double mu, double rho, const char* flow_field_path,
                    int cache_steps, gsmc_ctx** out) {
  return gsmc_ctx_create_ex(G, n_haps, n_sites, positions, Ne, mu, rho, flow_field_path,
                            cache_steps, 0, out);
}

int gsmc_ctx_create_ex(const uint8_t* G, int64_t n_haps, int64_t n_sites, const double* positions,
                       double Ne, double mu, double rho, const char* flow_field_path,
                       int cache_steps, int flags, gsmc_ctx** out) {
  if (!out) return fail(GSMC_E_INVALID, "null output handle");
  *out = nullptr;
  if (n_haps < 0 || n_sites < 0) return fail(GSMC_E_INVALID, "negative genotype shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  if ((n_haps * n_sites > 0 && !G) || (n_sites > 0 && !positions))
    return fail(GSMC_E_INVALID, "null genotype or position array");
  if (!flow_field_path) return fail(GSMC_E_INVALID, "null flow field path");
  const int L = cache_steps <= 0 ? 1000 : cache_steps;  // src/bindings.cpp:2569-2572
  if (L > kMaxCacheSteps)
    return fail(GSMC_E_INVALID, "cache_steps must be at most %d", kMaxCacheSteps);
  auto ctx = std::make_unique<gsmc_ctx>();
  CUDA_TRY(cudaGetDevice(&ctx->device));
  ctx->n_haps = n_haps;
  ctx->n_sites = n_sites;
  ctx->ne = (float)Ne;
  ctx->n_groups = (n_sites + 127) / 128;
  if (const char* env = std::getenv("GSMC_PAIRS_PER_THREAD")) {
    const int v = std::atoi(env);
    if (v == 1 || v == 2) ctx->shape.pairs_per_thread = v;
    ctx->shape_fixed = true;
  }
  if (const char* env = std::getenv("GSMC_SPECULATE")) ctx->speculate = std::atoi(env) != 0;
  if (const char* env = std::getenv("GSMC_SPEC_FLANK"))
    ctx->spec_flank = std::max<int64_t>(1, std::atoll(env));
  if (const char* env = std::getenv("GSMC_SPEC_CHUNKS"))
    ctx->spec_chunks_fixed = std::max(0, std::atoi(env));
  if (const char* env = std::getenv("GSMC_CORE_WEIGHT"))
    ctx->core_weight = std::min(8.0, std::max(0.25, std::atof(env)));
  if (const char* env = std::getenv("GSMC_SPEC_MAX_CHUNK"))
    ctx->spec_max_chunk = std::max<int64_t>(0, std::atoll(env));
  if (const char* env = std::getenv("GSMC_POOL_FRACTION"))
    ctx->pool_fraction = std::min(0.97, std::max(0.1, std::atof(env)));
  if (const char* env = std::getenv("GSMC_SCAN_WIDTH")) {
    const int v = std::atoi(env);
    if (v == 32 || v == 128) ctx->shape.width = v;
    ctx->shape_fixed = true;
  }
  bool reused = false;
  int rc = acquire_tables(ctx->device, flow_field_path, Ne, mu, rho, L,
                          (flags & GSMC_TABLES_GPU_F64) != 0, &ctx->tables, &reused);
  if (rc == GSMC_OK) {
    ctx->tables_reused = reused;
    ctx->tables_build_seconds = reused ? 0.0 : ctx->tables->build_seconds;
  }
  if (rc) return rc;
  struct Guard {
    std::unique_ptr<gsmc_ctx>* p;
    ~Guard() {
      if (*p) gsmc_ctx_destroy(p->release());
    }
  } guard{&ctx};
  CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  const size_t geno_bytes = (size_t)std::max<int64_t>(ctx->n_groups, 1) * std::max<int64_t>(n_haps, 1) * sizeof(ulonglong2);
  CUDA_TRY(cudaMalloc(&ctx->geno, geno_bytes));
  CUDA_TRY(cudaMemsetAsync(ctx->geno, 0, geno_bytes, ctx->stream));
  if (n_haps > 0 && n_sites > 0) {
    uint8_t* dG = nullptr;
    CUDA_TRY(cudaMalloc(&dG, (size_t)n_haps * n_sites));
    cudaError_t e = cudaMemcpyAsync(dG, G, (size_t)n_haps * n_sites, cudaMemcpyHostToDevice,
                                    ctx->stream);
    if (e == cudaSuccess) e = launch_bitpack(dG, n_haps, n_sites, ctx->geno, true, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dG);
    if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (bitpack)", cudaGetErrorString(e));
  }
  // Gap codes with two zero entries before site 0 and after the last site, so
  // the kernel can prefetch the codes two sites ahead without a bound check.
  std::vector<SiteCode> codes((size_t)n_sites + 2 * kCodePad, SiteCode{0, 0});
  for (int64_t s = 0; s < n_sites; ++s) {
    const int k = seg_steps(s == 0 ? positions[0] + 1.0 : positions[s] - positions[s - 1]);
    const int chunks = (k - 1) / L;
    codes[s + kCodePad] = SiteCode{(k - chunks * L - 1) * kLayerF4, chunks};
  }
  ctx->positions.assign(positions, positions + n_sites);
  SiteCode* code_base = nullptr;
  CUDA_TRY(cudaMalloc(&code_base, codes.size() * sizeof(SiteCode)));
  ctx->code = code_base + kCodePad;
  CUDA_TRY(cudaMemcpy(code_base, codes.data(), codes.size() * sizeof(SiteCode),
                      cudaMemcpyHostToDevice));
  *out = ctx.release();
  return GSMC_OK;
}

int gsmc_ctx_destroy(gsmc_ctx* ctx) {
  if (!ctx) return GSMC_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& ev : ctx->events) {
    cudaEventSynchronize(ev.second);
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  cudaFree(ctx->geno);
  if (ctx->code) cudaFree(ctx->code - kCodePad);
  cudaFree(ctx->pool);
  cudaFree(ctx->pairs);
  cudaFree(ctx->stage);
  cudaFree(ctx->acc);
  cudaFree(ctx->spec_rec);
  cudaFree(ctx->spec_win);
  cudaFree(ctx->spec_repairs);
  cudaFree(ctx->repair_pool);
  cudaFree(ctx->spec_repaired);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->copy_stream) {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamDestroy(ctx->copy_stream);
  }
  cudaFree(ctx->fwd_code);
  for (int i = 0; i < 2; ++i) {
    cudaFree(ctx->tasks[i]);
    if (ctx->stage_free[i]) cudaEventDestroy(ctx->stage_free[i]);
    if (ctx->launch_done[i]) cudaEventDestroy(ctx->launch_done[i]);
  }
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  cudaSetDevice(prev);
  release_tables(ctx->tables);
  delete ctx;
  return GSMC_OK;
}

int gsmc_ctx_release_scratch(gsmc_ctx* ctx) {
  if (int rc = check_ctx(ctx)) return rc;
  CUDA_TRY(cudaSetDevice(ctx->device));
  if (ctx->stream) CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (ctx->copy_stream) CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
  auto drop = [](auto** buf, size_t* bytes) {
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    *bytes = 0;
  };
  drop(&ctx->pool, &ctx->pool_bytes);
  drop(&ctx->stage, &ctx->stage_bytes);
  drop(&ctx->acc, &ctx->acc_bytes);
  drop(&ctx->spec_rec, &ctx->spec_rec_bytes);
  drop(&ctx->spec_win, &ctx->spec_win_bytes);
  drop(&ctx->spec_repairs, &ctx->spec_repairs_bytes);
  drop(&ctx->repair_pool, &ctx->repair_pool_bytes);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  ctx->pinned = nullptr;
  ctx->pinned_bytes = 0;
  return GSMC_OK;
}

int gsmc_ctx_info(const gsmc_ctx* ctx, int* device, int64_t* n_haps, int64_t* n_sites) {
  if (int rc = check_ctx(ctx)) return rc;
  if (device) *device = ctx->device;
  if (n_haps) *n_haps = ctx->n_haps;
  if (n_sites) *n_sites = ctx->n_sites;
  return GSMC_OK;
}

int gsmc_ctx_scratch_bytes(const gsmc_ctx* ctx, uint64_t* bytes) {
  if (int rc = check_ctx(ctx)) return rc;
  *bytes = ctx->pool_bytes + ctx->stage_bytes + ctx->pairs_cap * 2 * sizeof(int32_t);
  return GSMC_OK;
}

int gsmc_flow_fb_stats(int* chunks, int64_t* repaired) {
  if (chunks) *chunks = g_flow_fb_stats.chunks;
  if (repaired) *repaired = g_flow_fb_stats.repaired;
  return GSMC_OK;
}

int gsmc_ctx_scan_shape(const gsmc_ctx* ctx, int* width, int* pairs_per_thread) {
  if (int rc = check_ctx(ctx)) return rc;
  if (width) *width = ctx->shape.width;
  if (pairs_per_thread) *pairs_per_thread = ctx->shape.pairs_per_thread;
  return GSMC_OK;
}

int gsmc_ctx_spec_stats(gsmc_ctx* ctx, int64_t* launches, int64_t* repaired) {
  if (int rc = check_ctx(ctx)) return rc;
  int r = 0;
  if (ctx->spec_repaired) {
    CUDA_TRY(cudaSetDevice(ctx->device));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(cudaMemcpy(&r, ctx->spec_repaired, sizeof(int), cudaMemcpyDeviceToHost));
  }
  if (launches) *launches = ctx->spec_launches;
  if (repaired) *repaired = r;
  return GSMC_OK;
}

int gsmc_ctx_timing(gsmc_ctx* ctx, int enable) {
  if (int rc = check_ctx(ctx)) return rc;
  ctx->timing = enable != 0;
  return GSMC_OK;
}

int gsmc_ctx_timing_read(gsmc_ctx* ctx, double* kernel_ms, int64_t* launches,
                         double* pair_sites) {
  if (int rc = check_ctx(ctx)) return rc;
  double total = 0.0;
  cudaError_t err = cudaSuccess;
  for (auto& ev : ctx->events) {
    float ms = 0.0f;
    cudaError_t e = cudaEventSynchronize(ev.second);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.first, ev.second);
    if (e != cudaSuccess && err == cudaSuccess) err = e;
    total += ms;
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  ctx->events.clear();
  if (kernel_ms) *kernel_ms = total;
  if (launches) *launches = ctx->launches;
  if (pair_sites) *pair_sites = ctx->pair_sites;
  ctx->launches = 0;
  ctx->pair_sites = 0.0;
  if (err != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (timing events)", cudaGetErrorString(err));
  return GSMC_OK;
}

int gsmc_block_count(int64_t n_sites, int64_t core, int64_t* n_blocks) {
  if (core <= 0) return fail(GSMC_E_INVALID, "core_block_sites must be positive.");
  *n_blocks = n_sites <= 0 ? 0 : (n_sites + core - 1) / core;
  return GSMC_OK;
}


static int run_host_common(gsmc_ctx* ctx, const int32_t* pi, const int32_t* pj, int64_t P,
                           const std::vector<Block>& blocks, int64_t pair_cap, int flags,
                           float* mean, float* lower, float* upper, float* alpha,
                           float* beta) {
  if (P < 0) return fail(GSMC_E_INVALID, "negative pair count");
  if (P > 0 && (!pi || !pj)) return fail(GSMC_E_INVALID, "null pair arrays");
  if (P > 0 && ctx->n_sites > 0 && !mean) return fail(GSMC_E_INVALID, "null mean output");
  if ((flags & GSMC_CI) && P > 0 && ctx->n_sites > 0 && (!lower || !upper))
    return fail(GSMC_E_INVALID, "null lower/upper output");
  if ((flags & GSMC_POSTERIOR) && P > 0 && ctx->n_sites > 0 && (!alpha || !beta))
    return fail(GSMC_E_INVALID, "null posterior output");
  if (P == 0 || ctx->n_sites == 0) return GSMC_OK;
  CUDA_TRY(cudaSetDevice(ctx->device));
  int rc = upload_pairs(ctx, pi, pj, P);
  if (rc) return rc;
  float* host[5] = {mean, (flags & GSMC_CI) ? lower : nullptr, (flags & GSMC_CI) ? upper : nullptr,
                    (flags & GSMC_POSTERIOR) ? alpha : nullptr,
                    (flags & GSMC_POSTERIOR) ? beta : nullptr};
  return run_to_host(ctx, P, blocks, pair_cap, flags, host, blocks.empty() ? 0 : blocks[0].cs);
}

int gsmc_run_fb(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs,
                int flags, float* mean, float* lower, float* upper, float* alpha, float* beta) {
  if (int rc = check_ctx(ctx)) return rc;
  std::vector<Block> one;
  if (ctx->n_sites > 0) one.push_back({0, ctx->n_sites, 0, ctx->n_sites});
  return run_host_common(ctx, pair_i, pair_j, n_pairs, one, -1, flags, mean, lower, upper,
                         alpha, beta);
}

int gsmc_run_fb_summary(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                        int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                        int64_t pair_batch_size, float* site_mean, float* site_min,
                        float* site_max) {
  if (int rc = check_ctx(ctx)) return rc;
  if (n_pairs < 0) return fail(GSMC_E_INVALID, "negative pair count");
  if (flank_sites < 0) return fail(GSMC_E_INVALID, "flank_sites must be non-negative.");
  if (pair_batch_size == 0 || pair_batch_size < -1)
    return fail(GSMC_E_INVALID, "pair_batch_size must be positive or -1 for auto.");
  const int64_t S = ctx->n_sites;
  if (n_pairs == 0 || S == 0) return GSMC_OK;
  if (!pair_i || !pair_j) return fail(GSMC_E_INVALID, "null pair arrays");
  if (!site_mean || !site_min || !site_max) return fail(GSMC_E_INVALID, "null summary output");
  CUDA_TRY(cudaSetDevice(ctx->device));
  int rc = upload_pairs(ctx, pair_i, pair_j, n_pairs);
  if (rc) return rc;
  std::vector<Block> blocks;
  if (core_block_sites <= 0 || core_block_sites >= S)
    blocks.push_back({0, S, 0, S});
  else
    blocks = make_windows(S, core_block_sites, flank_sites);
  const int64_t core = max_core(blocks);
  // accumulators: double sum, float min, max, mean per site
  rc = ensure_buffer(reinterpret_cast<char**>(&ctx->acc), &ctx->acc_bytes, (size_t)S * 20);
  if (rc) return rc;
  double* acc_sum = static_cast<double*>(ctx->acc);
  float* acc_min = reinterpret_cast<float*>(acc_sum + S);
  float* acc_max = acc_min + S;
  float* d_mean = acc_max + S;
  const int32_t* d_pi = ctx->pairs;
  const int32_t* d_pj = ctx->pairs + ctx->pairs_cap;
  if (summary_by_pairs(ctx, n_pairs, blocks)) {
    // Too few (window, pair tile) tasks to fill the GPU, and a warp's partial
    // sums cannot be cut into speculative chunks (a repaired pair could not be
    // taken back out of them): decode per-pair means in exact speculative
    // chunks into a [sites x pair batch] matrix and fold it per site.
    const size_t budget = (size_t)(0.7 * (double)free_device_bytes()) + ctx->pool_bytes +
                          ctx->stage_bytes;
    int64_t batch = std::max<int64_t>(1, (int64_t)(0.3 * (double)budget / (double)(S * 4)));
    batch = std::min(batch, n_pairs);
    if (pair_batch_size > 0) batch = std::min(batch, pair_batch_size);
    // equal batches: a small last one would run its long windows on a mostly
    // idle GPU (63,190 pairs in batches of 28,775 left 5,640 for the last)
    batch = plan::even_part(n_pairs, batch);
    rc = ensure_buffer(&ctx->stage, &ctx->stage_bytes, (size_t)S * batch * sizeof(float));
    if (rc) return rc;
    for (int64_t off = 0; off < n_pairs; off += batch) {
      const int64_t n = std::min(batch, n_pairs - off);
      float* const out[5] = {ctx->stage, nullptr, nullptr, nullptr, nullptr};
      rc = run_direct(ctx, d_pi + off, d_pj + off, n, blocks, 0, out, n, 0, ctx->stream);
      if (rc) return rc;
      CUDA_TRY(launch_summary_fold(ctx->stage, ctx->stage, ctx->stage, S, n, n, acc_sum, acc_min,
                                   acc_max, off == 0, ctx->stream));
    }
    CUDA_TRY(launch_summary_finish(acc_sum, S, (double)n_pairs, d_mean, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(site_mean, d_mean, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(site_min, acc_min, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(site_max, acc_max, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return GSMC_OK;
  }
  pick_shape(ctx, n_pairs, blocks, kTaskSummary);  // summaries are never chunked
  const int tile = scan_tile_pairs(ctx->shape);
  const int warps = ctx->shape.width / 32;  // partial columns per pair tile
  const int resident = resident_ctas(ctx->shape);
  const int tiles_per_cta = scan_tiles_per_cta(ctx->shape);
  // pair chunk: partials (3 x S x columns floats) within ~40% of the budget
  const size_t budget = (size_t)(0.7 * (double)free_device_bytes()) + ctx->pool_bytes +
                        ctx->stage_bytes;
  const size_t per_tile = (size_t)3 * S * warps * sizeof(float);
  int64_t chunk_tiles = std::max<int64_t>(1, (int64_t)(0.4 * (double)budget / (double)per_tile));
  chunk_tiles = std::min<int64_t>(chunk_tiles, ceil_div(n_pairs, tile));
  if (pair_batch_size > 0)
    chunk_tiles = std::min<int64_t>(chunk_tiles, std::max<int64_t>(1, pair_batch_size / tile));
  {  // equal pair chunks (no small last one)
    const int64_t all_tiles = ceil_div(n_pairs, tile);
    chunk_tiles = plan::even_part(all_tiles, chunk_tiles);
  }
  const int64_t chunk = chunk_tiles * tile;
  const int64_t cols = chunk_tiles * warps;
  rc = ensure_buffer(&ctx->stage, &ctx->stage_bytes, (size_t)3 * S * cols * sizeof(float));
  if (rc) return rc;
  float* p_sum = ctx->stage;
  float* p_min = p_sum + (size_t)S * cols;
  float* p_max = p_min + (size_t)S * cols;
  const int busy = (int)std::min<int64_t>(
      resident, ceil_div((int64_t)blocks.size() * chunk_tiles, tiles_per_cta));
  const size_t slot = cta_slot_bytes(ctx->shape, core);
  const size_t pool_budget = budget > (size_t)3 * S * cols * 4 ? budget - (size_t)3 * S * cols * 4 : slot;
  int grid = 0;
  rc = size_pool(ctx, core, busy, pool_budget, &grid);
  if (rc) return rc;
  int which = 0;
  for (int64_t off = 0; off < n_pairs; off += chunk, which ^= 1) {
    const int64_t n = std::min(chunk, n_pairs - off);
    std::vector<Task> tasks;
    for (const Block& b : blocks) {
      WindowOut wo{{p_sum, p_min, p_max, nullptr, nullptr}, 0, cols, 0};
      const size_t first = tasks.size();
      add_window_tasks(b, d_pi + off, d_pj + off, n, tile, wo, 0, kTaskSummary, 2.0f * ctx->ne,
                       &tasks);
      // a tile's partials go to its own columns: warps x tile index
      for (size_t i = first; i < tasks.size(); ++i) tasks[i].out_off = (int64_t)(i - first) * warps;
    }
    rc = launch_tasks(ctx, tasks, which, core, grid, ctx->stream);
    if (rc) return rc;
    // columns written: every warp of a full tile, and of the last tile the
    // warps that hold a pair (warp w of a tile starts at pair 32 w; warps
    // past the last pair leave without writing)
    const int64_t rem = n % tile;
    const int64_t used_cols = (n / tile) * warps +
                              (rem ? ceil_div(std::min<int64_t>(rem, ctx->shape.width), 32) : 0);
    CUDA_TRY(launch_summary_fold(p_sum, p_min, p_max, S, used_cols, cols, acc_sum, acc_min,
                                 acc_max, off == 0, ctx->stream));
  }
  CUDA_TRY(launch_summary_finish(acc_sum, S, (double)n_pairs, d_mean, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(site_mean, d_mean, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(site_min, acc_min, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaMemcpyAsync(site_max, acc_max, S * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return GSMC_OK;
}

int gsmc_run_fwd(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs,
                 int flags, float* mean, float* lower, float* upper) {
  if (int rc = check_ctx(ctx)) return rc;
  if (n_pairs < 0) return fail(GSMC_E_INVALID, "negative pair count");
  const int64_t S = ctx->n_sites;
  const bool ci = (flags & GSMC_CI) != 0;
  if (n_pairs == 0 || S == 0) return GSMC_OK;
  if (!pair_i || !pair_j || !mean || (ci && (!lower || !upper)))
    return fail(GSMC_E_INVALID, "null pair or output array");
  if (S > 0x7fffffff) return fail(GSMC_E_INVALID, "too many sites");
  CUDA_TRY(cudaSetDevice(ctx->device));
  int rc = upload_pairs(ctx, pair_i, pair_j, n_pairs);
  if (rc) return rc;
  TableSet* ts = ctx->tables;
  const int L = ts->L;
  {
    // half patches of the hom table, once per table set
    std::lock_guard<std::mutex> lock(ts->half_mu);
    if (!ts->hom_half) {
      std::vector<float> patches((size_t)L * kPatches * 8);
      for (int k = 0; k < L; ++k)
        pack_patches(ts->hom_m.data() + (size_t)k * kCells, ts->hom_c.data() + (size_t)k * kCells,
                     patches.data() + (size_t)k * kPatches * 8);
      float* tmp = nullptr;
      CUDA_TRY(cudaMalloc(&tmp, patches.size() * sizeof(float)));
      cudaError_t e = cudaMemcpy(tmp, patches.data(), patches.size() * sizeof(float),
                                 cudaMemcpyHostToDevice);
      uint4* half = nullptr;
      if (e == cudaSuccess) e = cudaMalloc(&half, patches.size() * 2);
      if (e == cudaSuccess) e = launch_to_half(tmp, half, patches.size(), ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      cudaFree(tmp);
      if (e != cudaSuccess) {
        cudaFree(half);
        return fail(GSMC_E_CUDA, "CUDA error: %s (half table)", cudaGetErrorString(e));
      }
      ts->hom_half = half;
    }
  }
  if (!ctx->fwd_code) {
    // gap k = trunc(pos[s] - pos[s-1] + 0.5): `chunks` lookups in layer L-1,
    // then layer k - chunks * L - 1; nothing at site 0 or for k <= 0
    // (src/kernels/gamma_smc_flow.cu:1176-1188, 1225-1231)
    std::vector<FwdCode> codes((size_t)S, FwdCode{-1, 0});
    double prev = 0.0;
    for (int64_t s2 = 0; s2 < S; ++s2) {
      const double g = ctx->positions[s2] - prev + 0.5;
      prev = ctx->positions[s2];
      const int k = g >= 2147483647.0 ? 2147483647 : (int)g;
      if (s2 == 0 || k <= 0) continue;
      const int chunks = (k - 1) / L;
      codes[s2] = FwdCode{k - chunks * L - 1, chunks};
    }
    CUDA_TRY(cudaMalloc(&ctx->fwd_code, codes.size() * sizeof(FwdCode)));
    CUDA_TRY(cudaMemcpy(ctx->fwd_code, codes.data(), codes.size() * sizeof(FwdCode),
                        cudaMemcpyHostToDevice));
  }
  // pair chunks whose outputs fit the stage; rows copied to the host arrays
  const int nout = ci ? 3 : 1;
  const size_t budget = (size_t)(0.5 * (double)free_device_bytes()) + ctx->stage_bytes;
  int64_t chunk = std::max<int64_t>(1, (int64_t)(budget / ((size_t)S * nout * sizeof(float))));
  chunk = std::min<int64_t>(chunk, n_pairs);
  if (chunk < n_pairs) chunk = std::max<int64_t>(128, chunk / 128 * 128);
  rc = ensure_buffer(&ctx->stage, &ctx->stage_bytes, (size_t)S * chunk * nout * sizeof(float));
  if (rc) return rc;
  HostCopier* copier = HostCopier::for_current_device();
  if (!copier) return fail(GSMC_E_CUDA, "CUDA error: no device for the host copier");
  cudaEvent_t done = nullptr;
  CUDA_TRY(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
  int first = GSMC_OK;
  float* host[3] = {mean, lower, upper};
  for (int64_t off = 0; off < n_pairs && first == GSMC_OK; off += chunk) {
    const int64_t n = std::min(chunk, n_pairs - off);
    // the stage is rewritten only after the previous chunk's copies read it
    int e = copier->drain();
    FwdArgs a;
    std::memset(&a, 0, sizeof(a));
    a.geno = ctx->geno;
    a.n_haps = ctx->n_haps;
    a.code = ctx->fwd_code;
    a.tab = ts->hom_half;
    a.L = L;
    a.n_sites = (int)S;
    a.pi = ctx->pairs + off;
    a.pj = ctx->pairs + ctx->pairs_cap + off;
    a.n_pairs = (int)n;
    a.two_ne = 2.0f * ctx->ne;
    a.mean = ctx->stage;
    a.lower = ci ? ctx->stage + (size_t)S * n : nullptr;
    a.upper = ci ? ctx->stage + (size_t)2 * S * n : nullptr;
    a.ldo = n;
    FwdSpec sp;
    std::memset(&sp, 0, sizeof(sp));
    sp.k_chunks = fwd_chunks(ctx, n, S);
    if (sp.k_chunks > 1) {
      rc = ensure_buffer(&ctx->spec_rec, &ctx->spec_rec_bytes,
                         (size_t)(sp.k_chunks - 1) * 2 * n * sizeof(float2));
      if (!rc)
        rc = ensure_buffer(&ctx->spec_repairs, &ctx->spec_repairs_bytes, (size_t)(n + 1) * sizeof(int));
      if (!rc && !ctx->spec_repaired) {
        CUDA_TRY(cudaMalloc(&ctx->spec_repaired, sizeof(int)));
        CUDA_TRY(cudaMemsetAsync(ctx->spec_repaired, 0, sizeof(int), ctx->stream));
      }
      if (rc) {
        copier->drain();
        cudaEventDestroy(done);
        return rc;
      }
      sp.burn_in = (int)std::min<int64_t>(ctx->spec_flank, S);
      sp.rec = ctx->spec_rec;
      sp.repair_count = reinterpret_cast<int*>(ctx->spec_repairs);
      sp.repair_list = sp.repair_count + 1;
      sp.repaired_total = ctx->spec_repaired;
      ctx->spec_launches++;
    }
    if (e == cudaSuccess) e = launch_fwd_spec(a, sp, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(done, ctx->stream);
    for (int k = 0; k < nout && e == cudaSuccess; ++k)
      e = copier->enqueue(host[k] + off, (size_t)n_pairs * sizeof(float),
                          ctx->stage + (size_t)k * S * n, (size_t)n * sizeof(float),
                          (size_t)n * sizeof(float), (size_t)S, done);
    if (e != cudaSuccess)
      first = fail(GSMC_E_CUDA, "CUDA error: %s (forward-only)", cudaGetErrorString((cudaError_t)e));
  }
  const int e = copier->drain();
  cudaEventDestroy(done);
  if (first) return first;
  if (e != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)", cudaGetErrorString((cudaError_t)e));
  return GSMC_OK;
}

int gsmc_run_fb_blockwise_stream(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                                 int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                                 int64_t pair_batch_size, int flags, gsmc_sink_fn sink,
                                 void* user, uint64_t max_chunk_bytes) {
  if (int rc = check_ctx(ctx)) return rc;
  if (core_block_sites <= 0) return fail(GSMC_E_INVALID, "core_block_sites must be positive.");
  if (flank_sites < 0) return fail(GSMC_E_INVALID, "flank_sites must be non-negative.");
  if (pair_batch_size == 0 || pair_batch_size < -1)
    return fail(GSMC_E_INVALID, "pair_batch_size must be positive or -1 for auto.");
  if (n_pairs < 0) return fail(GSMC_E_INVALID, "negative pair count");
  if (!sink) return fail(GSMC_E_INVALID, "null sink");
  const int64_t S = ctx->n_sites;
  if (n_pairs == 0 || S == 0) return GSMC_OK;
  if (!pair_i || !pair_j) return fail(GSMC_E_INVALID, "null pair arrays");
  CUDA_TRY(cudaSetDevice(ctx->device));
  int rc = upload_pairs(ctx, pair_i, pair_j, n_pairs);
  if (rc) return rc;
  const std::vector<Block> blocks = make_windows(S, core_block_sites, flank_sites);
  const int64_t core = max_core(blocks);
  const int nout = n_outputs(flags);
  pick_shape(ctx, n_pairs, blocks, kTaskSummary);  // this path does not chunk speculatively
  const int tile = scan_tile_pairs(ctx->shape);
  const int tiles_per_cta = scan_tiles_per_cta(ctx->shape);
  // a unit is one window x one pair chunk; its outputs fill one stage half
  const uint64_t unit_cap = max_chunk_bytes ? max_chunk_bytes : (uint64_t)1 << 30;
  int64_t chunk = std::max<int64_t>(
      tile, (int64_t)(unit_cap / ((uint64_t)core * nout * sizeof(float))) / tile * tile);
  if (pair_batch_size > 0) chunk = std::max<int64_t>(1, std::min(chunk, pair_batch_size));
  chunk = std::min(chunk, n_pairs);
  const size_t half = (size_t)core * chunk * nout;  // floats
  rc = ensure_buffer(&ctx->stage, &ctx->stage_bytes, 2 * half * sizeof(float));
  if (rc) return rc;
  if (ctx->pinned_bytes < 2 * half * sizeof(float)) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    if (cudaHostAlloc(&ctx->pinned, 2 * half * sizeof(float), cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      return fail(GSMC_E_NOMEM, "cudaHostAlloc of %zu bytes of pinned staging failed",
                  2 * half * sizeof(float));
    }
    ctx->pinned_bytes = 2 * half * sizeof(float);
  }
  if (!ctx->copy_stream) CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  const int busy = (int)std::min<int64_t>(resident_ctas(ctx->shape),
                                          ceil_div(ceil_div(chunk, tile), tiles_per_cta));
  const size_t budget = (size_t)(0.8 * (double)free_device_bytes()) + ctx->pool_bytes;
  int grid = 0;
  rc = size_pool(ctx, core, busy, budget, &grid);
  if (rc) return rc;
  struct Events {
    cudaEvent_t computed[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    ~Events() {
      for (int i = 0; i < 2; ++i) {
        if (computed[i]) cudaEventDestroy(computed[i]);
        if (copied[i]) cudaEventDestroy(copied[i]);
      }
    }
  } ev;
  for (int i = 0; i < 2; ++i) {
    CUDA_TRY(cudaEventCreateWithFlags(&ev.computed[i], cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&ev.copied[i], cudaEventDisableTiming));
  }
  const int32_t* d_pi = ctx->pairs;
  const int32_t* d_pj = ctx->pairs + ctx->pairs_cap;
  const int selected[5] = {1, (flags & GSMC_CI) ? 1 : 0, (flags & GSMC_CI) ? 1 : 0,
                           (flags & GSMC_POSTERIOR) ? 1 : 0, (flags & GSMC_POSTERIOR) ? 1 : 0};
  struct Unit {
    int64_t b, off, n;
  };
  std::vector<Unit> units;
  for (size_t b = 0; b < blocks.size(); ++b)
    for (int64_t off = 0; off < n_pairs; off += chunk)
      units.push_back({(int64_t)b, off, std::min(chunk, n_pairs - off)});
  // hand unit u (already copied into pinned half u & 1) to the sink
  auto deliver = [&](size_t u) -> int {
    const Unit& un = units[u];
    const Block& blk = blocks[un.b];
    CUDA_TRY(cudaEventSynchronize(ev.copied[u & 1]));
    const float* base = ctx->pinned + (u & 1) * half;
    const float* outs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int used = 0;
    for (int k = 0; k < 5; ++k)
      if (selected[k]) outs[k] = base + (size_t)(used++) * (blk.ce - blk.cs) * un.n;
    if (sink(user, blk.cs, blk.ce, un.off, un.off + un.n, outs, un.n) != 0)
      return fail(GSMC_E_INVALID, "the sink stopped the stream");
    return GSMC_OK;
  };
  for (size_t u = 0; u < units.size(); ++u) {
    const Unit& un = units[u];
    const Block& blk = blocks[un.b];
    const int h = (int)(u & 1);
    float* st = ctx->stage + (size_t)h * half;
    const int64_t rows = blk.ce - blk.cs;
    // the stage half is rewritten only after unit u-2's copy has read it
    if (u >= 2) CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ev.copied[h], 0));
    std::vector<Task> tasks;
    WindowOut wo;
    int used = 0;
    for (int k = 0; k < 5; ++k) wo.out[k] = selected[k] ? st + (size_t)(used++) * rows * un.n : nullptr;
    wo.off = 0;
    wo.ldo = un.n;
    wo.row0 = blk.cs;
    add_window_tasks(blk, d_pi + un.off, d_pj + un.off, un.n, tile, wo, 0, task_flags(flags),
                     2.0f * ctx->ne, &tasks);
    rc = launch_tasks(ctx, tasks, h, core, grid, ctx->stream);
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(ev.computed[h], ctx->stream));
    CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ev.computed[h], 0));
    CUDA_TRY(cudaMemcpyAsync(ctx->pinned + (size_t)h * half, st,
                             (size_t)rows * un.n * nout * sizeof(float), cudaMemcpyDeviceToHost,
                             ctx->copy_stream));
    CUDA_TRY(cudaEventRecord(ev.copied[h], ctx->copy_stream));
    // while the GPU computes unit u, the host hands unit u-1 to the sink
    if (u >= 1) {
      rc = deliver(u - 1);
      if (rc) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamSynchronize(ctx->copy_stream);
        return rc;
      }
    }
  }
  rc = deliver(units.size() - 1);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return rc;
}

int gsmc_run_fb_window(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                       int64_t n_pairs, int64_t site_begin, int64_t site_end, int flags,
                       float* mean, float* lower, float* upper, float* alpha, float* beta) {
  if (int rc = check_ctx(ctx)) return rc;
  if (site_begin < 0 || site_end > ctx->n_sites || site_begin > site_end)
    return fail(GSMC_E_INVALID, "site window [%lld, %lld) is out of range for %lld sites",
                (long long)site_begin, (long long)site_end, (long long)ctx->n_sites);
  std::vector<Block> one;
  if (site_end > site_begin) one.push_back({site_begin, site_end, site_begin, site_end});
  return run_host_common(ctx, pair_i, pair_j, n_pairs, one, -1, flags, mean, lower, upper,
                         alpha, beta);
}

int gsmc_run_fb_blockwise(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                          int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                          int64_t pair_batch_size, int max_streams, int flags,
                          int32_t* blocks_out, float* mean, float* lower, float* upper,
                          float* alpha, float* beta) {
  if (int rc = check_ctx(ctx)) return rc;
  // Argument checks and messages of src/bindings.cpp:3000-3016.
  if (core_block_sites <= 0) return fail(GSMC_E_INVALID, "core_block_sites must be positive.");
  if (flank_sites < 0) return fail(GSMC_E_INVALID, "flank_sites must be non-negative.");
  if (pair_batch_size == 0 || pair_batch_size < -1)
    return fail(GSMC_E_INVALID, "pair_batch_size must be positive or -1 for auto.");
  if (max_streams <= 0) return fail(GSMC_E_INVALID, "max_streams must be positive.");
  if ((flags & GSMC_POSTERIOR) && max_streams > 1)
    return fail(GSMC_E_INVALID,
                "return_posterior=True is currently only supported with max_streams=1. "
                "Run blockwise posterior decoding in single-stream mode.");
  const std::vector<Block> blocks = make_windows(ctx->n_sites, core_block_sites, flank_sites);
  if (blocks_out)
    for (size_t b = 0; b < blocks.size(); ++b) {
      blocks_out[4 * b + 0] = (int32_t)blocks[b].cs;
      blocks_out[4 * b + 1] = (int32_t)blocks[b].ce;
      blocks_out[4 * b + 2] = (int32_t)blocks[b].ps;
      blocks_out[4 * b + 3] = (int32_t)blocks[b].pe;
    }
  // Every window of every pair chunk runs on the persistent kernel regardless
  // of max_streams: the copy engine already overlaps transfers with compute.
  return run_host_common(ctx, pair_i, pair_j, n_pairs, blocks, pair_batch_size, flags, mean,
                         lower, upper, alpha, beta);
}

int gsmc_run_fb_blockwise_device(gsmc_ctx* ctx, const int32_t* d_pair_i, const int32_t* d_pair_j,
                                 int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                                 int flags, float* d_mean, float* d_lower, float* d_upper,
                                 float* d_alpha, float* d_beta, int64_t ld_out, int64_t out_col0,
                                 void* stream) {
  if (int rc = check_ctx(ctx)) return rc;
  if (core_block_sites <= 0) return fail(GSMC_E_INVALID, "core_block_sites must be positive.");
  if (flank_sites < 0) return fail(GSMC_E_INVALID, "flank_sites must be non-negative.");
  if (n_pairs < 0 || ld_out < 0 || out_col0 < 0 || out_col0 + n_pairs > ld_out)
    return fail(GSMC_E_INVALID, "bad pair count or output leading dimension");
  if (n_pairs > 0 && (!d_pair_i || !d_pair_j || !d_mean))
    return fail(GSMC_E_INVALID, "null device pointer");
  if ((flags & GSMC_CI) && n_pairs > 0 && (!d_lower || !d_upper))
    return fail(GSMC_E_INVALID, "null lower/upper output");
  if ((flags & GSMC_POSTERIOR) && n_pairs > 0 && (!d_alpha || !d_beta))
    return fail(GSMC_E_INVALID, "null posterior output");
  CUDA_TRY(cudaSetDevice(ctx->device));
  const std::vector<Block> blocks = make_windows(ctx->n_sites, core_block_sites, flank_sites);
  float* const out[5] = {d_mean, (flags & GSMC_CI) ? d_lower : nullptr,
                         (flags & GSMC_CI) ? d_upper : nullptr,
                         (flags & GSMC_POSTERIOR) ? d_alpha : nullptr,
                         (flags & GSMC_POSTERIOR) ? d_beta : nullptr};
  return run_direct(ctx, d_pair_i, d_pair_j, n_pairs, blocks, flags, out, ld_out, out_col0,
                    static_cast<cudaStream_t>(stream));
}

int gsmc_copy_to_host(int64_t n, void* const* dst, const void* const* src, const uint64_t* bytes,
                      void* stream) {
  if (n < 0 || (n > 0 && (!dst || !src || !bytes))) return fail(GSMC_E_INVALID, "bad copy list");
  if (n == 0) return GSMC_OK;
  HostCopier* copier = HostCopier::for_current_device();
  if (!copier) return fail(GSMC_E_CUDA, "CUDA error: no device for the host copier");
  cudaEvent_t ready = nullptr;
  CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ready, static_cast<cudaStream_t>(stream));
  int first = (int)e;
  for (int64_t i = 0; i < n && first == cudaSuccess; ++i) {
    if (bytes[i] == 0) continue;
    if (!dst[i] || !src[i]) {
      first = -1;
      break;
    }
    first = copier->enqueue(dst[i], (size_t)bytes[i], src[i], (size_t)bytes[i], (size_t)bytes[i], 1,
                            ready);
  }
  const int drained = copier->drain();
  cudaEventDestroy(ready);
  if (first == -1) return fail(GSMC_E_INVALID, "null pointer in the copy list");
  if (first != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)", cudaGetErrorString((cudaError_t)first));
  if (drained != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)", cudaGetErrorString((cudaError_t)drained));
  return GSMC_OK;
}

int gsmc_generate_flow_field(const double* alpha, const double* beta, int mean_n, int cv_n,
                             int n_steps, int n_epochs, const double* epoch_start,
                             const double* epoch_rate, const double* epoch_cum,
                             double calibration, double* u, double* v) {
  if (mean_n <= 0 || cv_n <= 0 || !alpha || !beta || !u || !v)
    return fail(GSMC_E_INVALID, "bad flow-field grid");
  if (n_steps < 2 || flow_field_smem_bytes(n_steps) > 200 * 1024)
    return fail(GSMC_E_INVALID, "n_steps must be in [2, 2559]");
  if (n_epochs < 0 || n_epochs > kMaxEpochs)
    return fail(GSMC_E_INVALID, "at most %d epochs are supported", kMaxEpochs);
  if (n_epochs > 0 && (!epoch_start || !epoch_rate || !epoch_cum))
    return fail(GSMC_E_INVALID, "null epoch arrays");
  FlowGenEpochs ep;
  std::memset(&ep, 0, sizeof(ep));
  ep.n = n_epochs;
  for (int k = 0; k < n_epochs; ++k) {
    ep.t_bounds[k] = epoch_start[k];
    ep.lam[k] = epoch_rate[k];
    ep.L_bounds[k] = epoch_cum[k];
  }
  const size_t cells = (size_t)mean_n * cv_n;
  double* d = nullptr;
  CUDA_TRY(cudaMalloc(&d, 4 * cells * sizeof(double)));
  FlowGenArgs a;
  a.alpha = d;
  a.beta = d + cells;
  a.u = d + 2 * cells;
  a.v = d + 3 * cells;
  a.mean_n = mean_n;
  a.cv_n = cv_n;
  a.n_steps = n_steps;
  a.t_max_exp = -std::log(1e-3);
  a.calibration = calibration;
  cudaError_t e = cudaMemcpy(d, alpha, cells * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + cells, beta, cells * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_flow_field(a, ep, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(u, a.u, cells * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(v, a.v, cells * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (flow field)", cudaGetErrorString(e));
  return GSMC_OK;
}

int gsmc_flow_fb(const uint8_t* G, int64_t n_haps, int64_t n_sites, const double* positions,
                 const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs, double Ne,
                 double mu, double rho, const char* flow_field_path, int flags, float* mean,
                 float* lower, float* upper) {
  if (n_haps < 0 || n_sites < 0 || n_pairs < 0) return fail(GSMC_E_INVALID, "negative shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  if (n_sites > 0x7fffffff) return fail(GSMC_E_INVALID, "too many sites");
  const bool ci = (flags & GSMC_CI) != 0;
  if (!flow_field_path) return fail(GSMC_E_INVALID, "null flow field path");
  if (n_pairs == 0 || n_sites == 0) return GSMC_OK;
  if (!G || !positions || !pair_i || !pair_j || !mean || (ci && (!lower || !upper)))
    return fail(GSMC_E_INVALID, "null input or output array");
  for (int64_t p = 0; p < n_pairs; ++p)
    if (pair_i[p] < 0 || pair_i[p] >= n_haps || pair_j[p] < 0 || pair_j[p] >= n_haps)
      return fail(GSMC_E_INVALID, "pair %lld = (%d, %d) is out of range for %lld haplotypes",
                  (long long)p, pair_i[p], pair_j[p], (long long)n_haps);
  FlowField ff;
  char err[512];
  if (load_flow_field(flow_field_path, &ff, err, sizeof(err)) != 0)
    return fail(GSMC_E_IO, "%s", err);
  // rates as the reference's launcher forms them in float
  // (src/kernels/gamma_smc_flow.cu:342-344)
  const float ne = (float)Ne, fmu = (float)mu, frho = (float)rho;
  const float lambda = 1.0f / (2.0f * ne);
  const float srho = 4.0f * ne * frho;
  const float smu = 2.0f * fmu / lambda;
  std::vector<float2> flow(kCells);
  for (int i = 0; i < kCells; ++i) flow[i] = make_float2(ff.u[i], ff.v[i]);
  std::vector<int> seg((size_t)n_sites);
  for (int64_t s2 = 0; s2 < n_sites; ++s2)
    seg[s2] = seg_steps(s2 == 0 ? positions[0] + 1.0 : positions[s2] - positions[s2 - 1]);
  const int64_t groups = (n_sites + 127) / 128;
  // pair chunk: forward states (8 B) + outputs per pair-site within the budget
  const int nout = ci ? 3 : 1;
  const size_t per_pair = (size_t)n_sites * (8 + 4 * nout);
  const size_t budget = (size_t)(0.6 * (double)free_device_bytes());
  int64_t chunk = std::min<int64_t>(n_pairs, std::max<int64_t>(1, (int64_t)(budget / per_pair)));
  if (chunk < n_pairs) {
    chunk = std::max<int64_t>(256, chunk / 256 * 256);
    // equal chunks (multiples of 256, none larger than the budget's)
    chunk = plan::even_part(n_pairs, chunk, 256);
  }
  struct Bufs {
    uint8_t* G = nullptr;
    ulonglong2* geno = nullptr;
    int* seg = nullptr;
    float2* flow = nullptr;
    int32_t* pairs = nullptr;
    float2* fwd = nullptr;
    float* out = nullptr;
    int* error = nullptr;
    float2* rec = nullptr;  // speculative chunks: boundary records
    int* rep = nullptr;     // [repaired total | repair count | repair list]
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    ~Bufs() {
      if (st) cudaStreamSynchronize(st);
      cudaFree(G);
      cudaFree(geno);
      cudaFree(seg);
      cudaFree(flow);
      cudaFree(pairs);
      cudaFree(fwd);
      cudaFree(out);
      cudaFree(error);
      cudaFree(rec);
      cudaFree(rep);
      if (done) cudaEventDestroy(done);
      if (st) cudaStreamDestroy(st);
    }
  } b;
  CUDA_TRY(cudaStreamCreateWithFlags(&b.st, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
  CUDA_TRY(cudaMalloc(&b.G, (size_t)n_haps * n_sites));
  CUDA_TRY(cudaMalloc(&b.geno, (size_t)groups * n_haps * sizeof(ulonglong2)));
  CUDA_TRY(cudaMalloc(&b.seg, seg.size() * sizeof(int)));
  CUDA_TRY(cudaMalloc(&b.flow, flow.size() * sizeof(float2)));
  CUDA_TRY(cudaMalloc(&b.pairs, 2 * (size_t)n_pairs * sizeof(int32_t)));
  CUDA_TRY(cudaMalloc(&b.error, sizeof(int)));
  if (cudaMalloc(&b.fwd, (size_t)n_sites * chunk * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&b.out, (size_t)n_sites * chunk * nout * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return fail(GSMC_E_NOMEM, "CUDA error: out of memory for %lld pairs x %lld sites",
                (long long)chunk, (long long)n_sites);
  }
  CUDA_TRY(cudaMemsetAsync(b.geno, 0, (size_t)groups * n_haps * sizeof(ulonglong2), b.st));
  CUDA_TRY(cudaMemsetAsync(b.error, 0, sizeof(int), b.st));
  CUDA_TRY(cudaMemcpyAsync(b.G, G, (size_t)n_haps * n_sites, cudaMemcpyHostToDevice, b.st));
  CUDA_TRY(launch_bitpack(b.G, n_haps, n_sites, b.geno, true, b.st));
  CUDA_TRY(cudaMemcpyAsync(b.seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice, b.st));
  CUDA_TRY(cudaMemcpyAsync(b.flow, flow.data(), flow.size() * sizeof(float2), cudaMemcpyHostToDevice,
                           b.st));
  CUDA_TRY(cudaMemcpyAsync(b.pairs, pair_i, n_pairs * sizeof(int32_t), cudaMemcpyHostToDevice, b.st));
  CUDA_TRY(cudaMemcpyAsync(b.pairs + n_pairs, pair_j, n_pairs * sizeof(int32_t),
                           cudaMemcpyHostToDevice, b.st));
  // exact speculative site chunks when the pairs of a chunk cannot fill every
  // SM (2,048 threads each); chunks of at least four burn-ins
  bool speculate = true;
  int64_t burn = 2048;
  if (const char* env = std::getenv("GSMC_SPECULATE")) speculate = std::atoi(env) != 0;
  if (const char* env = std::getenv("GSMC_SPEC_FLANK")) burn = std::max<int64_t>(1, std::atoll(env));
  int sms = 148;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto chunks_for = [&](int64_t n) {
    if (!speculate) return 1;
    return (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div((int64_t)sms * 2048, n),
                                                       n_sites / (4 * burn)));
  };
  const int k_max = chunks_for(std::min(chunk, n_pairs));
  g_flow_fb_stats = FlowFbStats{};
  if (k_max > 1) {
    CUDA_TRY(cudaMalloc(&b.rec, (size_t)(k_max - 1) * 4 * chunk * sizeof(float2)));
    CUDA_TRY(cudaMalloc(&b.rep, (size_t)(chunk + 2) * sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(b.rep, 0, sizeof(int), b.st));
  }
  CUDA_TRY(cudaStreamSynchronize(b.st));  // host sources may go away after this call
  HostCopier* copier = HostCopier::for_current_device();
  if (!copier) return fail(GSMC_E_CUDA, "CUDA error: no device for the host copier");
  float* host[3] = {mean, lower, upper};
  int first = GSMC_OK;
  for (int64_t off = 0; off < n_pairs && first == GSMC_OK; off += chunk) {
    const int64_t n = std::min(chunk, n_pairs - off);
    int e = copier->drain();  // the previous chunk's copies have read the outputs
    UncachedArgs a;
    std::memset(&a, 0, sizeof(a));
    a.geno = b.geno;
    a.n_haps = n_haps;
    a.seg = b.seg;
    a.flow = b.flow;
    a.n_sites = (int)n_sites;
    a.pi = b.pairs + off;
    a.pj = b.pairs + n_pairs + off;
    a.n_pairs = (int)n;
    a.rho = srho;
    a.mu = smu;
    a.unscale = 2.0f * ne;
    a.fwd = b.fwd;
    a.mean = b.out;
    a.lower = ci ? b.out + (size_t)n_sites * n : nullptr;
    a.upper = ci ? b.out + (size_t)2 * n_sites * n : nullptr;
    a.ldo = n;
    a.error = b.error;
    a.wait_polls = g_copy_wait_polls.load();
    UncachedSpec sp;
    std::memset(&sp, 0, sizeof(sp));
    sp.k_chunks = std::min(k_max, chunks_for(n));
    if (sp.k_chunks > 1) {
      sp.burn_in = (int)std::min<int64_t>(burn, n_sites);
      sp.rec = b.rec;
      sp.repaired_total = b.rep;
      sp.repair_count = b.rep + 1;
      sp.repair_list = b.rep + 2;
      g_flow_fb_stats.chunks = std::max(g_flow_fb_stats.chunks, sp.k_chunks);
    }
    if (e == cudaSuccess) e = launch_uncached_spec(a, sp, b.st);
    if (e == cudaSuccess) e = cudaEventRecord(b.done, b.st);
    for (int k = 0; k < nout && e == cudaSuccess; ++k)
      e = copier->enqueue(host[k] + off, (size_t)n_pairs * sizeof(float),
                          b.out + (size_t)k * n_sites * n, (size_t)n * sizeof(float),
                          (size_t)n * sizeof(float), (size_t)n_sites, b.done);
    if (e != cudaSuccess)
      first = fail(GSMC_E_CUDA, "CUDA error: %s (flow FB)", cudaGetErrorString((cudaError_t)e));
  }
  const int e = copier->drain();
  if (first) return first;
  if (e != cudaSuccess)
    return fail(GSMC_E_CUDA, "CUDA error: %s (device to host copy)", cudaGetErrorString((cudaError_t)e));
  int flag = 0;
  CUDA_TRY(cudaMemcpy(&flag, b.error, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) return fail(GSMC_E_TIMEOUT, "the flow field copy into shared memory did not complete");
  if (b.rep) {
    int repaired = 0;
    CUDA_TRY(cudaMemcpy(&repaired, b.rep, sizeof(int), cudaMemcpyDeviceToHost));
    g_flow_fb_stats.repaired = repaired;
  }
  return GSMC_OK;
}

int gsmc_host_alloc(uint64_t bytes, void** ptr) {
  if (!ptr) return fail(GSMC_E_INVALID, "null output pointer");
  *ptr = nullptr;
  if (bytes == 0) bytes = 1;
  {
    std::lock_guard<std::mutex> lock(g_host_mu);
    // the smallest cached block that fits without wasting more than half of it
    auto best = g_host_free.end();
    for (auto it = g_host_free.begin(); it != g_host_free.end(); ++it)
      if (it->bytes >= bytes && it->bytes / 2 <= bytes &&
          (best == g_host_free.end() || it->bytes < best->bytes))
        best = it;
    if (best != g_host_free.end()) {
      *ptr = best->p;
      g_host_used[best->p] = *best;
      g_host_cached -= best->bytes;
      g_host_free.erase(best);
      return GSMC_OK;
    }
  }
  // Page-locking runs outside the lock: it takes seconds for tens of GB.
  HostBlk blk{};
  cudaError_t e = new_host_block(bytes, &blk);
  if (e != cudaSuccess) {
    // release the cache and try once more
    cudaGetLastError();
    std::vector<HostBlk> drop;
    {
      std::lock_guard<std::mutex> lock(g_host_mu);
      drop.swap(g_host_free);
      g_host_cached = 0;
    }
    if (!drop.empty()) {
      free_host_blocks(drop);
      e = new_host_block(bytes, &blk);
    }
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(GSMC_E_NOMEM, "CUDA error: %s (page-locked host buffer of %llu bytes)",
                cudaGetErrorString(e), (unsigned long long)bytes);
  }
  {
    std::lock_guard<std::mutex> lock(g_host_mu);
    g_host_used[blk.p] = blk;
  }
  *ptr = blk.p;
  return GSMC_OK;
}

int gsmc_host_free(void* ptr) {
  if (!ptr) return GSMC_OK;
  std::vector<HostBlk> drop;
  {
    std::lock_guard<std::mutex> lock(g_host_mu);
    auto it = g_host_used.find(ptr);
    if (it == g_host_used.end()) return fail(GSMC_E_INVALID, "not a gsmc_host_alloc buffer");
    g_host_free.push_back(it->second);
    g_host_cached += it->second.bytes;
    g_host_used.erase(it);
    drop = trim_host_cache_locked();
  }
  free_host_blocks(drop);
  return GSMC_OK;
}

int gsmc_host_cache_limit(uint64_t max_cached_bytes) {
  std::vector<HostBlk> drop;
  {
    std::lock_guard<std::mutex> lock(g_host_mu);
    g_host_cache_cap = max_cached_bytes;
    drop = trim_host_cache_locked();
  }
  free_host_blocks(drop);
  return GSMC_OK;
}

int gsmc_ctx_tables_info(const gsmc_ctx* ctx, double* build_seconds, int* reused) {
  if (int rc = check_ctx(ctx)) return rc;
  if (build_seconds) *build_seconds = ctx->tables_build_seconds;
  if (reused) *reused = ctx->tables_reused ? 1 : 0;
  return GSMC_OK;
}

int gsmc_free_cached_tables(void) {
  std::lock_guard<std::mutex> lock(g_tables_mu);
  for (auto& kv : g_parked) {
    erase_key_of(kv.second);
    free_table_set(kv.second);
  }
  g_parked.clear();
  return GSMC_OK;
}

int gsmc_set_copy_wait_polls(int64_t polls, int64_t* previous) {
  if (polls < 0) return fail(GSMC_E_INVALID, "the poll budget must be non-negative");
  const long long prev = g_copy_wait_polls.exchange(polls);
  if (previous) *previous = prev;
  return GSMC_OK;
}

int gsmc_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites, uint64_t* packed) {
  if (n_haps < 0 || n_sites < 0) return fail(GSMC_E_INVALID, "negative shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  if (n_haps == 0 || n_sites == 0) return GSMC_OK;
  const int64_t nw = (n_sites + 63) / 64;
  uint8_t* dG = nullptr;
  uint64_t* dP = nullptr;
  CUDA_TRY(cudaMalloc(&dG, (size_t)n_haps * n_sites));
  cudaError_t e = cudaMalloc(&dP, (size_t)n_haps * nw * 8);
  if (e == cudaSuccess) e = cudaMemcpy(dG, G, (size_t)n_haps * n_sites, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_bitpack(dG, n_haps, n_sites, dP, false, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(packed, dP, (size_t)n_haps * nw * 8, cudaMemcpyDeviceToHost);
  cudaFree(dG);
  cudaFree(dP);
  if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (bitpack)", cudaGetErrorString(e));
  return GSMC_OK;
}

int gsmc_diploid_het_counts(const uint8_t* G, int64_t n_haps, int64_t n_sites, int64_t* counts) {
  if (n_haps < 0 || n_sites < 0) return fail(GSMC_E_INVALID, "negative shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  const int64_t nd = n_haps / 2;
  if (nd == 0) return GSMC_OK;
  if (!counts || (n_sites > 0 && !G)) return fail(GSMC_E_INVALID, "null array");
  if (n_sites == 0) {
    std::fill(counts, counts + nd, (int64_t)0);
    return GSMC_OK;
  }
  const int64_t groups = (n_sites + 127) / 128;
  uint8_t* dG = nullptr;
  ulonglong2* dP = nullptr;
  long long* dC = nullptr;
  CUDA_TRY(cudaMalloc(&dG, (size_t)n_haps * n_sites));
  cudaError_t e = cudaMalloc(&dP, (size_t)groups * n_haps * sizeof(ulonglong2));
  if (e == cudaSuccess) e = cudaMalloc(&dC, (size_t)nd * sizeof(long long));
  if (e == cudaSuccess) e = cudaMemset(dP, 0, (size_t)groups * n_haps * sizeof(ulonglong2));
  if (e == cudaSuccess) e = cudaMemcpy(dG, G, (size_t)n_haps * n_sites, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_bitpack(dG, n_haps, n_sites, dP, true, nullptr);
  if (e == cudaSuccess) e = launch_het_counts(dP, n_haps, groups, dC, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(counts, dC, (size_t)nd * sizeof(long long), cudaMemcpyDeviceToHost);
  cudaFree(dG);
  cudaFree(dP);
  cudaFree(dC);
  if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (het counts)", cudaGetErrorString(e));
  return GSMC_OK;
}

int gsmc_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites, uint8_t* G) {
  if (n_haps < 0 || n_sites < 0) return fail(GSMC_E_INVALID, "negative shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  if (n_haps == 0 || n_sites == 0) return GSMC_OK;
  const int64_t nw = (n_sites + 63) / 64;
  uint8_t* dG = nullptr;
  uint64_t* dP = nullptr;
  CUDA_TRY(cudaMalloc(&dG, (size_t)n_haps * n_sites));
  cudaError_t e = cudaMalloc(&dP, (size_t)n_haps * nw * 8);
  if (e == cudaSuccess) e = cudaMemcpy(dP, packed, (size_t)n_haps * nw * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_unpack(dP, n_haps, n_sites, dG, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(G, dG, (size_t)n_haps * n_sites, cudaMemcpyDeviceToHost);
  cudaFree(dG);
  cudaFree(dP);
  if (e != cudaSuccess) return fail(GSMC_E_CUDA, "CUDA error: %s (unpack)", cudaGetErrorString(e));
  return GSMC_OK;
}

int gsmc_ctx_table_layer(const gsmc_ctx* ctx, int table, int layer, float* out) {
  if (int rc = check_ctx(ctx)) return rc;
  if (table < 0 || table > 4) return fail(GSMC_E_INVALID, "table must be in [0, 4]");
  const int L = ctx->tables->L;
  if (table < 4 && (layer < 0 || layer >= L)) return fail(GSMC_E_INVALID, "layer out of range");
  std::vector<float> patches((size_t)kPatches * 8);
  const float4* src = table == 4 ? ctx->tables->chunk
                                 : ctx->tables->site + scan_layer_offset(table, layer, L);
  CUDA_TRY(cudaSetDevice(ctx->device));
  CUDA_TRY(cudaMemcpy(patches.data(), src, patches.size() * sizeof(float), cudaMemcpyDeviceToHost));
  // Rebuild the 51 x 50 grids from the patches' corners.
  for (int r = 0; r < kRows; ++r)
    for (int q = 0; q < kCols; ++q) {
      const int pr = std::min(r, kPatchRows - 1), pq = std::min(q, kPatchCols - 1);
      const int corner = (r - pr) * 2 + (q - pq);
      const float* p = patches.data() + (size_t)(pr * kPatchCols + pq) * 8;
      out[r * kCols + q] = p[corner];
      out[kCells + r * kCols + q] = p[4 + corner];
    }
  return GSMC_OK;
}

}  // extern "C"

namespace gsmc {

bool ctx_view(const gsmc_ctx* ctx, CtxView* out) {
  if (!ctx || !out) return false;
  out->device = ctx->device;
  out->n_haps = ctx->n_haps;
  out->n_sites = ctx->n_sites;
  out->geno = ctx->geno;
  out->code = ctx->code;
  out->site_tab = ctx->tables->site;
  out->chunk_tab = ctx->tables->chunk;
  out->L = ctx->tables->L;
  out->ne = ctx->ne;
  return true;
}

int set_error(int code, const char* msg) { return fail(code, "%s", msg); }

}  // namespace gsmc
