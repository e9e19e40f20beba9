// Batched execution of many scan jobs in one persistent launch.
//
// A job is a set of pairs over a window [site_begin, site_end) of the
// context's sites, with its own output selection and output arrays.  Its
// window is decoded the way the reference's block kernels decode a padded
// window (src/kernels/gamma_smc_flow.cu:632-669, 762-839): the scan restarts
// at (m, c) = (0, 0), and a window that does not start at site 0 enters its
// first site by one base pair.  An executor may cut a long window into chunks
// of core_block_sites with flank_sites of burn-in on each side, as
// run_fb_blockwise does for a whole chromosome (src/bindings.cpp:2517-2534);
// with a flank of 1024 sites or more the chunked result equals the unchunked
// one to float32 precision on realistic data.
//
// Every (chunk, pair tile) of every job becomes one task of a single device
// task list; the persistent kernel's tiles pull tasks longest-first, so jobs
// of very different sizes share the GPU without per-job launches.  An
// executor owns all scratch of one in-flight launch (forward-state pool,
// task list, pinned upload images), so runs allocate nothing; several
// executors of one context may run concurrently on different streams.  The
// task list is written into mapped pinned memory that the kernel reads
// directly (a task descriptor is read once per task), so a run is "reset the
// task counter, launch the kernel"; with use_graph those two steps are
// replayed as one CUDA graph.  Two list images alternate, so the host can
// prepare run k+1 while run k is on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <utility>
#include <vector>

#include "ctx_view.h"
#include "gsmc_b200.h"
#include "scan.h"

using namespace gsmc;

struct gsmc_exec {
  CtxView v;
  ScanShape shape{32, 1};
  int64_t core = 0;       // sites per chunk; <= 0: whole windows
  int64_t flank = 2048;
  int64_t slot_rows = 0;  // longest core a task may have
  int64_t max_tasks = 0;
  int grid = 0;           // CTAs whose slots the pool holds
  void* pool = nullptr;
  size_t pool_bytes = 0;
  int* d_next = nullptr;                          // task counter (device)
  unsigned char* h_list[2] = {nullptr, nullptr};  // mapped pinned task lists, alternating
  unsigned char* m_list[2] = {nullptr, nullptr};  // their device addresses
  cudaEvent_t done[2] = {nullptr, nullptr};       // the last run reading the image is done
  bool used[2] = {false, false};
  int next_image = 0;
  bool use_graph = false;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // reset + scan over image 0 / 1
  // checked runs (chunking executors): boundary records of the chunked jobs
  // and, per image, the mapped descriptors the verify kernel reads
  float2* rec = nullptr;
  int64_t rec_cap = 0;  // float2
  ExecCheck* h_check[2] = {nullptr, nullptr};
  ExecCheck* m_check[2] = {nullptr, nullptr};
  // measurement
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  int64_t launches = 0;
  double pair_sites = 0.0;
};

namespace {

int fail_cuda(cudaError_t e, const char* what) {
  char msg[256];
  std::snprintf(msg, sizeof(msg), "CUDA error: %s (%s)", cudaGetErrorString(e), what);
  return set_error(GSMC_E_CUDA, msg);
}

int fail_invalid(const char* fmt, long long a = 0, long long b = 0) {
  char msg[256];
  std::snprintf(msg, sizeof(msg), fmt, a, b);
  return set_error(GSMC_E_INVALID, msg);
}

#define EXEC_TRY(expr, what)                    \
  do {                                          \
    cudaError_t e_ = (expr);                    \
    if (e_ != cudaSuccess) return fail_cuda(e_, what); \
  } while (0)

size_t list_bytes(int64_t n) { return kTaskListHead + (size_t)n * sizeof(Task); }

void release(gsmc_exec* x) {
  if (!x) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(x->v.device);
  for (int i = 0; i < 2; ++i)
    if (x->done[i]) {
      cudaEventSynchronize(x->done[i]);
      cudaEventDestroy(x->done[i]);
    }
  for (auto& ev : x->events) {
    cudaEventSynchronize(ev.second);
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  for (int i = 0; i < 2; ++i)
    if (x->gexec[i]) cudaGraphExecDestroy(x->gexec[i]);
  cudaFree(x->pool);
  cudaFree(x->d_next);
  cudaFree(x->rec);
  for (int i = 0; i < 2; ++i) {
    cudaFreeHost(x->h_list[i]);
    if (x->h_check[i]) cudaFreeHost(x->h_check[i]);
  }
  cudaSetDevice(prev);
  delete x;
}

void scan_args(const gsmc_exec* x, int img, ScanArgs* a) {
  std::memset(a, 0, sizeof(*a));
  a->geno = x->v.geno;
  a->n_haps = x->v.n_haps;
  a->code = x->v.code;
  a->site_tab = x->v.site_tab;
  a->chunk_tab = x->v.chunk_tab;
  a->L = x->v.L;
  a->next = x->d_next;
  a->count = &reinterpret_cast<const TaskListHead*>(x->m_list[img])->count;
  a->tasks = reinterpret_cast<const Task*>(x->m_list[img] + kTaskListHead);
  a->fwd = static_cast<float2*>(x->pool);
  a->slot_rows = x->slot_rows;
}

// Enqueue "reset the task counter, run the scan over image img" on a stream.
cudaError_t enqueue_run(const gsmc_exec* x, int img, int grid, cudaStream_t st) {
  ScanArgs a;
  scan_args(x, img, &a);
  cudaError_t e = cudaMemsetAsync(x->d_next, 0, sizeof(int), st);
  if (e == cudaSuccess) e = launch_scan(a, grid, x->shape, st);
  return e;
}

// Capture one graph per list image; a run then is one graph launch.
int build_graphs(gsmc_exec* x) {
  cudaStream_t cap = nullptr;
  EXEC_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "graph capture stream");
  cudaError_t e = cudaSuccess;
  for (int img = 0; img < 2 && e == cudaSuccess; ++img) {
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) break;
    const cudaError_t e1 = enqueue_run(x, img, x->grid, cap);
    e = cudaStreamEndCapture(cap, &g);
    if (e == cudaSuccess) e = e1;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x->gexec[img], g, 0);
    if (g) cudaGraphDestroy(g);
  }
  cudaStreamDestroy(cap);
  if (e != cudaSuccess) return fail_cuda(e, "building the scan graphs");
  return GSMC_OK;
}

// Tasks of one job: its window cut into chunks, each chunk into pair tiles.
// With `checks` (a checked run) a chunked job's tasks also write their
// boundary records into x->rec from float2 *rec_used on, and the job gets a
// descriptor for the verify kernel.
int job_tasks(const gsmc_exec* x, const gsmc_job& j, int64_t index, std::vector<Task>* out,
              int64_t* rec_used = nullptr, std::vector<ExecCheck>* checks = nullptr) {
  const int64_t S = x->v.n_sites;
  if (j.n_pairs < 0) return fail_invalid("job %lld: negative pair count", index);
  if (j.site_begin < 0 || j.site_end > S || j.site_begin > j.site_end)
    return fail_invalid("job %lld: site window out of range [0, %lld]", index, S);
  if (j.n_pairs == 0 || j.site_begin == j.site_end) return GSMC_OK;
  if (!j.pair_i || !j.pair_j || !j.out[0]) return fail_invalid("job %lld: null device pointer", index);
  if ((j.flags & GSMC_CI) && (!j.out[1] || !j.out[2]))
    return fail_invalid("job %lld: null lower/upper output", index);
  if ((j.flags & GSMC_POSTERIOR) && (!j.out[3] || !j.out[4]))
    return fail_invalid("job %lld: null posterior output", index);
  if (j.out_col0 < 0 || j.ld_out < j.out_col0 + j.n_pairs)
    return fail_invalid("job %lld: ld_out is smaller than out_col0 + n_pairs", index);
  const int64_t s0 = j.site_begin, s1 = j.site_end;
  const int64_t core = (x->core <= 0 || s1 - s0 <= x->core) ? s1 - s0 : x->core;
  if (core > x->slot_rows)
    return fail_invalid("job %lld: window of %lld sites exceeds the executor's max_window_sites",
                        index, s1 - s0);
  const int tile = scan_tile_pairs(x->shape);
  const int tf = ((j.flags & GSMC_CI) ? kTaskCI : 0) | ((j.flags & GSMC_POSTERIOR) ? kTaskPosterior : 0);
  const int64_t n_chunks = (s1 - s0 + core - 1) / core;
  float2* rec = nullptr;
  if (checks && n_chunks > 1) {
    const int64_t need = (n_chunks - 1) * 4 * j.n_pairs;
    if (*rec_used + need > x->rec_cap)
      return fail_invalid("job %lld: the run needs more boundary records than the executor "
                          "holds (%lld float2)", index, x->rec_cap);
    rec = x->rec + *rec_used;
    checks->push_back(ExecCheck{*rec_used, (int32_t)(n_chunks - 1), (int32_t)j.n_pairs,
                                (int32_t)index, 0});
    *rec_used += need;
  }
  for (int64_t cs = s0; cs < s1; cs += core) {
    const int64_t k = (cs - s0) / core;
    const int64_t ce = std::min(s1, cs + core);
    const int64_t ps = std::max(s0, cs - x->flank), pe = std::min(s1, ce + x->flank);
    for (int64_t p = 0; p < j.n_pairs; p += tile) {
      Task t;
      std::memset(&t, 0, sizeof(t));
      t.ps = (int32_t)ps;
      t.cs = (int32_t)cs;
      t.ce = (int32_t)ce;
      t.pe = (int32_t)pe;
      t.pi = j.pair_i + p;
      t.pj = j.pair_j + p;
      t.pair_count = (int32_t)std::min<int64_t>(tile, j.n_pairs - p);
      t.out_row0 = (int32_t)s0;
      t.flags = tf;
      t.unscale = 2.0f * x->v.ne;
      t.out_off = j.out_col0 + p;
      t.ldo = j.ld_out;
      for (int o = 0; o < 5; ++o) {
        const bool sel = o == 0 || (o < 3 ? (j.flags & GSMC_CI) : (j.flags & GSMC_POSTERIOR));
        t.out[o] = sel ? j.out[o] : nullptr;
      }
      if (rec) {
        t.bl = k > 0 ? rec + (k - 1) * 4 * j.n_pairs + p : nullptr;
        t.br = k < n_chunks - 1 ? rec + k * 4 * j.n_pairs + p : nullptr;
        t.bstride = j.n_pairs;
      }
      out->push_back(t);
    }
  }
  return GSMC_OK;
}

// One run; with `flags` (device, n_jobs) the chunked jobs are checked.
int exec_run(gsmc_exec* x, const gsmc_job* jobs, int64_t n_jobs, void* stream, int32_t* flags) {
  if (!x) return set_error(GSMC_E_INVALID, "null executor");
  if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return set_error(GSMC_E_INVALID, "bad job list");
  std::vector<Task> tasks;
  std::vector<ExecCheck> checks;
  int64_t rec_used = 0;
  const bool check = flags && x->rec;
  for (int64_t i = 0; i < n_jobs; ++i) {
    const int rc = job_tasks(x, jobs[i], i, &tasks, check ? &rec_used : nullptr,
                             check ? &checks : nullptr);
    if (rc) return rc;
    if ((int64_t)tasks.size() > x->max_tasks)
      return fail_invalid("the jobs need more than max_tasks = %lld tasks", x->max_tasks);
  }
  if (flags && n_jobs > 0) {
    EXEC_TRY(cudaSetDevice(x->v.device), "cudaSetDevice");
    EXEC_TRY(cudaMemsetAsync(flags, 0, (size_t)n_jobs * sizeof(int32_t),
                             static_cast<cudaStream_t>(stream)), "clearing the job flags");
  }
  if (tasks.empty()) return GSMC_OK;
  // longest first: the grid's tail is made of the shortest tasks
  std::stable_sort(tasks.begin(), tasks.end(), [](const Task& a, const Task& b) {
    return (a.ce - a.ps) + (a.pe - a.cs) > (b.ce - b.ps) + (b.pe - b.cs);
  });
  EXEC_TRY(cudaSetDevice(x->v.device), "cudaSetDevice");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int img = x->next_image;
  x->next_image ^= 1;
  // the last run that read this image must be done before it is rewritten
  if (x->used[img]) EXEC_TRY(cudaEventSynchronize(x->done[img]), "previous run");
  unsigned char* h = x->h_list[img];
  const TaskListHead head{0, (int)tasks.size()};
  std::memcpy(h, &head, sizeof(head));
  std::memcpy(h + kTaskListHead, tasks.data(), tasks.size() * sizeof(Task));
  if (!checks.empty()) std::memcpy(x->h_check[img], checks.data(), checks.size() * sizeof(ExecCheck));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (x->timing) {
    EXEC_TRY(cudaEventCreate(&e0), "cudaEventCreate");
    EXEC_TRY(cudaEventCreate(&e1), "cudaEventCreate");
    EXEC_TRY(cudaEventRecord(e0, st), "cudaEventRecord");
  }
  if (x->use_graph) {
    EXEC_TRY(cudaGraphLaunch(x->gexec[img], st), "cudaGraphLaunch");
  } else {
    const int tiles = scan_tiles_per_cta(x->shape);
    const int grid = (int)std::min<int64_t>(x->grid, ((int64_t)tasks.size() + tiles - 1) / tiles);
    EXEC_TRY(enqueue_run(x, img, grid, st), "scan launch");
  }
  if (!checks.empty()) {
    int max_pairs = 0;
    for (const ExecCheck& c : checks) max_pairs = std::max(max_pairs, c.n_pairs);
    EXEC_TRY(launch_exec_verify(x->rec, x->m_check[img], (int)checks.size(), max_pairs, flags, st),
             "boundary check");
    x->launches++;
  }
  EXEC_TRY(cudaEventRecord(x->done[img], st), "cudaEventRecord");
  x->used[img] = true;
  if (x->timing) {
    EXEC_TRY(cudaEventRecord(e1, st), "cudaEventRecord");
    x->events.emplace_back(e0, e1);
  }
  x->launches++;
  for (const Task& t : tasks) x->pair_sites += (double)t.pair_count * (double)(t.ce - t.cs);
  return GSMC_OK;
}

}  // namespace

extern "C" {

int gsmc_exec_create(gsmc_ctx* ctx, const gsmc_exec_config* cfg, gsmc_exec** out) {
  if (!out) return set_error(GSMC_E_INVALID, "null output handle");
  *out = nullptr;
  std::unique_ptr<gsmc_exec, void (*)(gsmc_exec*)> x(new gsmc_exec, release);
  if (!ctx_view(ctx, &x->v)) return set_error(GSMC_E_INVALID, "null context");
  gsmc_exec_config c;
  std::memset(&c, 0, sizeof(c));
  c.flank_sites = -1;
  if (cfg) c = *cfg;
  x->shape.width = c.tile_width == 0 ? 32 : c.tile_width;
  x->shape.pairs_per_thread = c.pairs_per_thread == 0 ? 1 : c.pairs_per_thread;
  if (!scan_shape_valid(x->shape))
    return set_error(GSMC_E_INVALID, "tile_width must be 32 or 128 and pairs_per_thread 1 or 2");
  x->core = c.core_block_sites;
  x->flank = c.flank_sites < 0 ? 2048 : c.flank_sites;
  const int64_t S = std::max<int64_t>(x->v.n_sites, 1);
  const int64_t wmax = c.max_window_sites > 0 ? std::min(c.max_window_sites, S) : S;
  x->slot_rows = x->core > 0 ? std::min(x->core, wmax) : wmax;
  x->max_tasks = c.max_tasks > 0 ? c.max_tasks : (int64_t)1 << 16;
  if (x->max_tasks > 0x7fffffff) return set_error(GSMC_E_INVALID, "max_tasks is too large");
  x->use_graph = c.use_graph != 0;
  EXEC_TRY(cudaSetDevice(x->v.device), "cudaSetDevice");
  // forward-state pool: one slot per tile of every CTA, within the budget
  const size_t cta_bytes = (size_t)x->slot_rows * scan_tile_pairs(x->shape) *
                           scan_tiles_per_cta(x->shape) * sizeof(float2);
  size_t budget = c.max_pool_bytes;
  if (budget == 0) {
    size_t f = 0, t = 0;
    EXEC_TRY(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
    budget = f / 2;
  }
  int64_t grid = std::max(1, scan_resident_ctas(x->shape));
  if (c.max_ctas > 0) grid = std::min<int64_t>(grid, c.max_ctas);
  grid = std::min<int64_t>(grid, (int64_t)(budget / std::max<size_t>(cta_bytes, 1)));
  if (grid < 1) {
    char msg[256];
    std::snprintf(msg, sizeof(msg),
                  "the forward-state pool budget (%zu bytes) does not hold one CTA's slots "
                  "(%zu bytes); lower core_block_sites or max_window_sites",
                  budget, cta_bytes);
    return set_error(GSMC_E_NOMEM, msg);
  }
  x->grid = (int)grid;
  x->pool_bytes = (size_t)grid * cta_bytes;
  if (cudaMalloc(&x->pool, x->pool_bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_error(GSMC_E_NOMEM, "cudaMalloc of the forward-state pool failed");
  }
  EXEC_TRY(cudaMalloc(&x->d_next, 256), "cudaMalloc of the task counter");
  if (x->core > 0) {
    // records of a checked run: (chunks - 1) x 4 per pair of a chunked job,
    // at most 4 per pair slot of a task
    x->rec_cap = 4 * x->max_tasks * scan_tile_pairs(x->shape);
    if (cudaMalloc(&x->rec, (size_t)x->rec_cap * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return set_error(GSMC_E_NOMEM, "cudaMalloc of the boundary records failed");
    }
    for (int i = 0; i < 2; ++i) {
      EXEC_TRY(cudaHostAlloc(&x->h_check[i], (size_t)x->max_tasks * sizeof(ExecCheck),
                             cudaHostAllocMapped), "cudaHostAlloc");
      void* dp = nullptr;
      EXEC_TRY(cudaHostGetDevicePointer(&dp, x->h_check[i], 0), "cudaHostGetDevicePointer");
      x->m_check[i] = static_cast<ExecCheck*>(dp);
    }
  }
  const size_t lb = list_bytes(x->max_tasks);
  for (int i = 0; i < 2; ++i) {
    EXEC_TRY(cudaHostAlloc(&x->h_list[i], lb, cudaHostAllocMapped), "cudaHostAlloc");
    std::memset(x->h_list[i], 0, kTaskListHead);
    void* dp = nullptr;
    EXEC_TRY(cudaHostGetDevicePointer(&dp, x->h_list[i], 0), "cudaHostGetDevicePointer");
    x->m_list[i] = static_cast<unsigned char*>(dp);
    EXEC_TRY(cudaEventCreateWithFlags(&x->done[i], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (x->use_graph) {
    const int rc = build_graphs(x.get());
    if (rc) return rc;
  }
  *out = x.release();
  return GSMC_OK;
}

int gsmc_exec_destroy(gsmc_exec* x) {
  release(x);
  return GSMC_OK;
}

int gsmc_exec_info(const gsmc_exec* x, int* grid, uint64_t* pool_bytes, int64_t* slot_rows,
                   int64_t* max_tasks) {
  if (!x) return set_error(GSMC_E_INVALID, "null executor");
  if (grid) *grid = x->grid;
  if (pool_bytes) *pool_bytes = x->pool_bytes;
  if (slot_rows) *slot_rows = x->slot_rows;
  if (max_tasks) *max_tasks = x->max_tasks;
  return GSMC_OK;
}

int gsmc_exec_run(gsmc_exec* x, const gsmc_job* jobs, int64_t n_jobs, void* stream) {
  return exec_run(x, jobs, n_jobs, stream, nullptr);
}

int gsmc_exec_run_checked(gsmc_exec* x, const gsmc_job* jobs, int64_t n_jobs, void* stream,
                          int32_t* job_flags) {
  if (n_jobs > 0 && !job_flags) return set_error(GSMC_E_INVALID, "null job flags");
  return exec_run(x, jobs, n_jobs, stream, job_flags);
}

int gsmc_exec_timing(gsmc_exec* x, int enable) {
  if (!x) return set_error(GSMC_E_INVALID, "null executor");
  x->timing = enable != 0;
  return GSMC_OK;
}

int gsmc_exec_timing_read(gsmc_exec* x, double* kernel_ms, int64_t* launches, double* pair_sites) {
  if (!x) return set_error(GSMC_E_INVALID, "null executor");
  double total = 0.0;
  cudaError_t err = cudaSuccess;
  for (auto& ev : x->events) {
    float ms = 0.0f;
    cudaError_t e = cudaEventSynchronize(ev.second);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev.first, ev.second);
    if (e != cudaSuccess && err == cudaSuccess) err = e;
    total += ms;
    cudaEventDestroy(ev.first);
    cudaEventDestroy(ev.second);
  }
  x->events.clear();
  if (kernel_ms) *kernel_ms = total;
  if (launches) *launches = x->launches;
  if (pair_sites) *pair_sites = x->pair_sites;
  x->launches = 0;
  x->pair_sites = 0.0;
  if (err != cudaSuccess) return fail_cuda(err, "timing events");
  return GSMC_OK;
}

}  // extern "C"
