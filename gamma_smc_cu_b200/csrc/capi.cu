// C ABI of the B200 Gamma-SMC scan: contexts, table sets, window planning and
// the host/device entry points declared in include/gsmc_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "gsmc_b200.h"
#include "scan.h"
#include "tables.h"

using namespace gsmc;

namespace {

thread_local std::string g_last_error;

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
// One resident set of scan tables per (device, flow field, Ne, mu, rho, L),
// shared by every context with those parameters and freed with the last one.
// (The reference keeps a single process-global set and frees it under live
// contexts when the parameters change, src/bindings.cpp:2016-2041.)
struct TableSet {
  int device = 0;
  int L = 0;
  float4* site = nullptr;   // [4][L][2450][2]
  float4* chunk = nullptr;  // [2450][2]
  int refs = 0;
};

using TableKey = std::tuple<int, std::string, float, float, float, int>;
std::mutex g_tables_mu;
std::map<TableKey, TableSet*> g_tables;

int acquire_tables(int device, const char* ff_path, float ne, float mu, float rho, int L,
                   TableSet** out) {
  std::lock_guard<std::mutex> lock(g_tables_mu);
  TableKey key{device, std::string(ff_path), ne, mu, rho, L};
  auto it = g_tables.find(key);
  if (it != g_tables.end()) {
    it->second->refs++;
    *out = it->second;
    return GSMC_OK;
  }
  FlowField ff;
  char err[512];
  if (load_flow_field(ff_path, &ff, err, sizeof(err)) != 0) return fail(GSMC_E_IO, "%s", err);
  float srho, smu;
  scaled_rates(ne, mu, rho, &srho, &smu);
  HostLayers layers;
  build_layers(ff, L, srho, smu, 0, &layers);
  std::vector<float> site, chunk;
  build_scan_layout(layers, &site, &chunk, 0);
  auto ts = std::make_unique<TableSet>();
  ts->device = device;
  ts->L = L;
  CUDA_TRY(cudaMalloc(&ts->site, site.size() * sizeof(float)));
  if (cudaMalloc(&ts->chunk, chunk.size() * sizeof(float)) != cudaSuccess) {
    cudaFree(ts->site);
    return fail(GSMC_E_CUDA, "CUDA error: cudaMalloc of the chunk table failed");
  }
  CUDA_TRY(cudaMemcpy(ts->site, site.data(), site.size() * sizeof(float), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(ts->chunk, chunk.data(), chunk.size() * sizeof(float),
                      cudaMemcpyHostToDevice));
  ts->refs = 1;
  *out = ts.get();
  g_tables[key] = ts.release();
  return GSMC_OK;
}

void release_tables(TableSet* ts) {
  if (!ts) return;
  std::lock_guard<std::mutex> lock(g_tables_mu);
  if (--ts->refs > 0) return;
  for (auto it = g_tables.begin(); it != g_tables.end(); ++it)
    if (it->second == ts) {
      g_tables.erase(it);
      break;
    }
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ts->device);
  cudaFree(ts->site);
  cudaFree(ts->chunk);
  cudaSetDevice(prev);
  delete ts;
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
  for (int64_t cs = 0; cs < S; cs += core) {
    const int64_t ce = std::min(S, cs + core);
    out.push_back({cs, ce, std::max<int64_t>(0, cs - flank), std::min(S, ce + flank)});
  }
  return out;
}

}  // namespace

struct gsmc_ctx {
  int device = 0;
  int64_t n_haps = 0, n_sites = 0, n_groups = 0;
  float ne = 0.0f;
  ulonglong2* geno = nullptr;
  SiteCode* code = nullptr;
  TableSet* tables = nullptr;
  // forward-state pool and pair-index buffer, grown on demand
  void* pool = nullptr;
  size_t pool_bytes = 0;
  int32_t* pairs = nullptr;
  int64_t pairs_cap = 0;
  float* stage = nullptr;  // device staging of host-bound outputs
  size_t stage_bytes = 0;
  cudaStream_t stream = nullptr;
  // measurement: events around scan launches while timing is on
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
  int64_t launches = 0;
  double pair_sites = 0.0;
};

namespace {

// Launch the scan, bracketed by events on `stream` when timing is enabled.
cudaError_t launch_counted(gsmc_ctx* ctx, const ScanArgs& a, bool ci, bool post,
                           cudaStream_t stream) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ctx->timing) {
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = launch_scan(a, ci, post, stream);
  if (e != cudaSuccess) return e;
  ctx->launches++;
  for (int i = 0; i < a.n_windows; ++i)
    ctx->pair_sites += (double)a.n_pairs * (double)(a.win[i].ce - a.win[i].cs);
  if (ctx->timing) {
    e = cudaEventRecord(e1, stream);
    if (e != cudaSuccess) return e;
    ctx->events.emplace_back(e0, e1);
  }
  return cudaSuccess;
}

int ensure_pool(gsmc_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->pool_bytes) return GSMC_OK;
  if (ctx->pool) cudaFree(ctx->pool);
  ctx->pool = nullptr;
  ctx->pool_bytes = 0;
  CUDA_TRY(cudaMalloc(&ctx->pool, bytes));
  ctx->pool_bytes = bytes;
  return GSMC_OK;
}

int ensure_stage(gsmc_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->stage_bytes) return GSMC_OK;
  if (ctx->stage) cudaFree(ctx->stage);
  ctx->stage = nullptr;
  ctx->stage_bytes = 0;
  CUDA_TRY(cudaMalloc(&ctx->stage, bytes));
  ctx->stage_bytes = bytes;
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

ScanArgs base_args(const gsmc_ctx* ctx) {
  ScanArgs a;
  std::memset(&a, 0, sizeof(a));
  a.geno = ctx->geno;
  a.n_haps = ctx->n_haps;
  a.code = ctx->code;
  a.site_tab = ctx->tables->site;
  a.chunk_tab = ctx->tables->chunk;
  a.L = ctx->tables->L;
  a.unscale = 2.0f * ctx->ne;
  return a;
}

int n_outputs(int flags) {
  return 1 + ((flags & GSMC_CI) ? 2 : 0) + ((flags & GSMC_POSTERIOR) ? 2 : 0);
}

size_t free_device_bytes() {
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) return 0;
  return f;
}

// Plan pair chunk and windows per launch so that `per_pair_site` bytes of
// scratch per (pair, core site) fit the budget.
void plan(int64_t P, int64_t core_max, size_t per_pair_site, size_t budget, int64_t n_blocks,
          int64_t pair_cap, int64_t* chunk, int64_t* wins) {
  const size_t per_pair_window = std::max<size_t>(1, per_pair_site * (size_t)std::max<int64_t>(core_max, 1));
  int64_t c = std::min<int64_t>(P, pair_cap > 0 ? pair_cap : P);
  while (c > 1 && per_pair_window * (size_t)c > budget) c = (c + 1) / 2;
  c = std::max<int64_t>(c, 1);
  int64_t w = (int64_t)(budget / (per_pair_window * (size_t)c));
  w = std::max<int64_t>(1, std::min<int64_t>({w, n_blocks, (int64_t)kMaxWindows}));
  *chunk = c;
  *wins = w;
}

// Device outputs of one call: pointers to [n_sites x ld] arrays.
struct DeviceOut {
  float* o[5];
  int64_t ld;
  int64_t col0;
};

// Run windows for all pairs writing device outputs directly.
int run_direct(gsmc_ctx* ctx, const int32_t* d_pi, const int32_t* d_pj, int64_t P,
               const std::vector<Block>& blocks, int flags, const DeviceOut& out,
               cudaStream_t stream) {
  if (P == 0 || blocks.empty()) return GSMC_OK;
  int64_t core_max = 0;
  for (const Block& b : blocks) core_max = std::max(core_max, b.ce - b.cs);
  const size_t budget = (size_t)(0.45 * (double)free_device_bytes()) + ctx->pool_bytes;
  int64_t chunk, wins;
  plan(P, core_max, sizeof(float2), budget, (int64_t)blocks.size(), -1, &chunk, &wins);
  int rc = ensure_pool(ctx, (size_t)chunk * core_max * wins * sizeof(float2));
  if (rc) return rc;
  ScanArgs a = base_args(ctx);
  a.fwd = static_cast<float2*>(ctx->pool);
  a.mean = out.o[0];
  a.lower = out.o[1];
  a.upper = out.o[2];
  a.alpha = out.o[3];
  a.beta = out.o[4];
  a.ldo = out.ld;
  const bool ci = flags & GSMC_CI, post = flags & GSMC_POSTERIOR;
  for (int64_t off = 0; off < P; off += chunk) {
    const int64_t n = std::min(chunk, P - off);
    a.pi = d_pi + off;
    a.pj = d_pj + off;
    a.n_pairs = n;
    a.col0 = out.col0 + off;
    for (size_t b0 = 0; b0 < blocks.size(); b0 += wins) {
      const int nw = (int)std::min<int64_t>(wins, (int64_t)blocks.size() - (int64_t)b0);
      a.n_windows = nw;
      for (int i = 0; i < nw; ++i) {
        const Block& b = blocks[b0 + i];
        a.win[i] = Window{b.ps, b.cs, b.ce, b.pe, (int64_t)i * core_max * n, 0, 0};
      }
      CUDA_TRY(launch_counted(ctx, a, ci, post, stream));
    }
  }
  return GSMC_OK;
}

// Run windows writing HOST outputs: each launch writes window cores into a
// device stage, copied out with one 2-D copy per output and window.
int run_to_host(gsmc_ctx* ctx, int64_t P, const std::vector<Block>& blocks, int64_t pair_cap,
                int flags, float* const host[5]) {
  if (P == 0 || blocks.empty()) return GSMC_OK;
  const int nout = n_outputs(flags);
  int64_t core_max = 0;
  for (const Block& b : blocks) core_max = std::max(core_max, b.ce - b.cs);
  const size_t budget =
      (size_t)(0.8 * (double)free_device_bytes()) + ctx->pool_bytes + ctx->stage_bytes;
  int64_t chunk, wins;
  plan(P, core_max, sizeof(float2) + nout * sizeof(float), budget, (int64_t)blocks.size(),
       pair_cap, &chunk, &wins);
  int rc = ensure_pool(ctx, (size_t)chunk * core_max * wins * sizeof(float2));
  if (rc) return rc;
  const size_t slot = (size_t)chunk * core_max;
  rc = ensure_stage(ctx, slot * wins * nout * sizeof(float));
  if (rc) return rc;
  ScanArgs a = base_args(ctx);
  a.fwd = static_cast<float2*>(ctx->pool);
  float* dev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  const int which[5] = {1, (flags & GSMC_CI) ? 1 : 0, (flags & GSMC_CI) ? 1 : 0,
                        (flags & GSMC_POSTERIOR) ? 1 : 0, (flags & GSMC_POSTERIOR) ? 1 : 0};
  int used = 0;
  for (int k = 0; k < 5; ++k)
    if (which[k]) dev[k] = ctx->stage + (size_t)(used++) * slot * wins;
  a.mean = dev[0];
  a.lower = dev[1];
  a.upper = dev[2];
  a.alpha = dev[3];
  a.beta = dev[4];
  const bool ci = flags & GSMC_CI, post = flags & GSMC_POSTERIOR;
  for (int64_t off = 0; off < P; off += chunk) {
    const int64_t n = std::min(chunk, P - off);
    a.pi = ctx->pairs + off;
    a.pj = ctx->pairs + ctx->pairs_cap + off;
    a.n_pairs = n;
    a.ldo = n;
    a.col0 = 0;
    for (size_t b0 = 0; b0 < blocks.size(); b0 += wins) {
      const int nw = (int)std::min<int64_t>(wins, (int64_t)blocks.size() - (int64_t)b0);
      a.n_windows = nw;
      for (int i = 0; i < nw; ++i) {
        const Block& b = blocks[b0 + i];
        a.win[i] = Window{b.ps, b.cs, b.ce, b.pe, (int64_t)i * core_max * n,
                          (int64_t)(i * slot), b.cs};
      }
      CUDA_TRY(launch_counted(ctx, a, ci, post, ctx->stream));
      for (int i = 0; i < nw; ++i) {
        const Block& b = blocks[b0 + i];
        for (int k = 0; k < 5; ++k) {
          if (!dev[k]) continue;
          CUDA_TRY(cudaMemcpy2DAsync(host[k] + (size_t)b.cs * P + off, (size_t)P * sizeof(float),
                                     dev[k] + (size_t)i * slot, (size_t)n * sizeof(float),
                                     (size_t)n * sizeof(float), (size_t)(b.ce - b.cs),
                                     cudaMemcpyDeviceToHost, ctx->stream));
        }
      }
      CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
  }
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
  if (!out) return fail(GSMC_E_INVALID, "null output handle");
  *out = nullptr;
  if (n_haps < 0 || n_sites < 0) return fail(GSMC_E_INVALID, "negative genotype shape");
  if (n_haps > 65535) return fail(GSMC_E_INVALID, "at most 65535 haplotypes are supported");
  if ((n_haps * n_sites > 0 && !G) || (n_sites > 0 && !positions))
    return fail(GSMC_E_INVALID, "null genotype or position array");
  if (!flow_field_path) return fail(GSMC_E_INVALID, "null flow field path");
  const int L = cache_steps <= 0 ? 1000 : cache_steps;  // src/bindings.cpp:2569-2572
  auto ctx = std::make_unique<gsmc_ctx>();
  CUDA_TRY(cudaGetDevice(&ctx->device));
  ctx->n_haps = n_haps;
  ctx->n_sites = n_sites;
  ctx->ne = (float)Ne;
  ctx->n_groups = (n_sites + 127) / 128;
  int rc = acquire_tables(ctx->device, flow_field_path, (float)Ne, (float)mu, (float)rho, L,
                          &ctx->tables);
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
  std::vector<SiteCode> codes((size_t)n_sites);
  for (int64_t s = 0; s < n_sites; ++s) {
    const int k = seg_steps(s == 0 ? positions[0] + 1.0 : positions[s] - positions[s - 1]);
    const int chunks = (k - 1) / L;
    codes[s] = SiteCode{k - chunks * L - 1, chunks};
  }
  CUDA_TRY(cudaMalloc(&ctx->code, std::max<size_t>(1, codes.size()) * sizeof(SiteCode)));
  if (n_sites > 0)
    CUDA_TRY(cudaMemcpy(ctx->code, codes.data(), codes.size() * sizeof(SiteCode),
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
  cudaFree(ctx->code);
  cudaFree(ctx->pool);
  cudaFree(ctx->pairs);
  cudaFree(ctx->stage);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  cudaSetDevice(prev);
  release_tables(ctx->tables);
  delete ctx;
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
  return run_to_host(ctx, P, blocks, pair_cap, flags, host);
}

int gsmc_run_fb(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs,
                int flags, float* mean, float* lower, float* upper, float* alpha, float* beta) {
  if (int rc = check_ctx(ctx)) return rc;
  std::vector<Block> one;
  if (ctx->n_sites > 0) one.push_back({0, ctx->n_sites, 0, ctx->n_sites});
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
  DeviceOut out{{d_mean, (flags & GSMC_CI) ? d_lower : nullptr, (flags & GSMC_CI) ? d_upper : nullptr,
                 (flags & GSMC_POSTERIOR) ? d_alpha : nullptr,
                 (flags & GSMC_POSTERIOR) ? d_beta : nullptr},
                ld_out, out_col0};
  return run_direct(ctx, d_pair_i, d_pair_j, n_pairs, blocks, flags, out,
                    static_cast<cudaStream_t>(stream));
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
                                 : ctx->tables->site + ((size_t)table * L + layer) * kPatches * 2;
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
