/*
 * gsmc_b200.h - C ABI of the B200-native Gamma-SMC forward/backward scan.
 *
 * Plain C types only (no torch, no pybind11).  Every function returns a
 * status: GSMC_OK (0) or a negative GSMC_E* code; gsmc_last_error() gives the
 * message of the last failure on the calling thread.  Host pointers are
 * ordinary pageable or pinned memory; "_device" entry points take device
 * pointers and a cudaStream_t passed as void*.
 *
 * Output arrays are site-major: element (s, p) of an [n_sites x n_pairs]
 * result is out[s * n_pairs + p], as in the reference (float32).
 *
 * Each entry point names the reference interface it replaces (paths are
 * relative to the gamma_smc_cu source tree).
 */
#ifndef GSMC_B200_H
#define GSMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  GSMC_OK = 0,
  GSMC_E_INVALID = -1,   /* bad argument: the reference raised ValueError   */
  GSMC_E_CUDA = -2,      /* CUDA runtime error: reference RuntimeError       */
  GSMC_E_IO = -3,        /* flow field could not be loaded                   */
  GSMC_E_NOMEM = -4,     /* host or device allocation failed                 */
  GSMC_E_TIMEOUT = -5    /* a bounded device wait gave up                    */
};

/* Output selection flags for the run_* calls. */
enum {
  GSMC_CI = 1,         /* write lower/upper Wilson-Hilferty 95% bounds (mean_only=False) */
  GSMC_POSTERIOR = 2   /* write posterior_alpha/posterior_beta (return_posterior=True) */
};

typedef struct gsmc_ctx gsmc_ctx;

/* Message of the last failed call on this thread ("" if none). */
const char* gsmc_last_error(void);

/* Library version string. */
const char* gsmc_version(void);

/* cudaMemGetInfo on the current device.
 * Replaces _core.cuda_mem_info (src/bindings.cpp:3646-3652). */
int gsmc_mem_info(uint64_t* free_bytes, uint64_t* total_bytes);

/* Replace _core.get_device_count / set_device / get_device
 * (src/bindings.cpp:3630-3644). */
int gsmc_get_device_count(int* count);
int gsmc_set_device(int device);
int gsmc_get_device(int* device);

/*
 * Create a context on the current device: loads the flow field, builds or
 * reuses the multi-step tables for (Ne, mu, rho, cache_steps), uploads and
 * bit-packs the genotypes, uploads the positions.
 *   G          [n_haps x n_sites] uint8, row-major (bit 0 of each byte is used)
 *   positions  [n_sites] float64 site coordinates
 *   cache_steps <= 0 selects 1000.
 * Replaces FlowContext::FlowContext (src/bindings.cpp:2552-2670) together with
 * ensure_flow_field / ensure_cache (src/bindings.cpp:2002-2157) and
 * bitpack_genotypes_gpu (src/kernels/bitpack.cu:32-38).  Tables are owned per
 * parameter set and reference-counted, never freed under a live context.
 * A context serves one call at a time (its scratch, stream and launch shape
 * belong to the running call); threads that decode concurrently use one
 * context each, or executors (gsmc_exec_*) of a shared context.
 */
int gsmc_ctx_create(const uint8_t* G, int64_t n_haps, int64_t n_sites,
                    const double* positions, double Ne, double mu, double rho,
                    const char* flow_field_path, int cache_steps,
                    gsmc_ctx** out);

/* Flags of gsmc_ctx_create_ex. */
enum {
  /* Build the scan tables on the GPU in float64 (every cell's chain carried
   * in float64, rounded to float32 only when stored) instead of the host
   * float32 build that reproduces the reference's tables bit for bit. */
  GSMC_TABLES_GPU_F64 = 1
};

/*
 * gsmc_ctx_create with flags (GSMC_TABLES_GPU_F64).  The float64 tables are a
 * separate resident set from the float32 ones of the same parameters; results
 * through them differ from the reference's in the last bits of the tables
 * (the deviation of the posterior means is measured by the tests and the
 * benchmark).  Replaces the same reference code as gsmc_ctx_create, plus the
 * table build the reference does on the host (src/flow_field.cpp:205-388).
 */
int gsmc_ctx_create_ex(const uint8_t* G, int64_t n_haps, int64_t n_sites,
                       const double* positions, double Ne, double mu, double rho,
                       const char* flow_field_path, int cache_steps, int flags,
                       gsmc_ctx** out);

/* Release a context (FlowContext::~FlowContext, src/bindings.cpp:2672-2677). */
int gsmc_ctx_destroy(gsmc_ctx* ctx);

/* Properties device_id / n_haps / n_sites (src/bindings.cpp:3727-3730). */
int gsmc_ctx_info(const gsmc_ctx* ctx, int* device, int64_t* n_haps,
                  int64_t* n_sites);

/*
 * Full-sequence forward/backward for n_pairs pairs (pair_i[p], pair_j[p]) into
 * HOST arrays of [n_sites x n_pairs] float32.  mean is required; lower/upper
 * are written when flags has GSMC_CI, alpha/beta when flags has
 * GSMC_POSTERIOR (others may be NULL).  Pair indices outside [0, n_haps) are
 * rejected with GSMC_E_INVALID.
 * Replaces FlowContext::run_fb (src/bindings.cpp:2897-2989) and
 * gamma_smc_flow_cached_fb_gpu (src/kernels/gamma_smc_flow.cu:844-903).
 */
int gsmc_run_fb(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                int64_t n_pairs, int flags, float* mean, float* lower,
                float* upper, float* alpha, float* beta);

/*
 * Forward/backward over one window [site_begin, site_end) of the context's
 * sites into HOST arrays of [site_end - site_begin x n_pairs] float32.  The
 * window is decoded as the reference's block kernels decode a padded window:
 * the scan restarts at (m, c) = (0, 0) and a window that does not start at
 * site 0 enters its first site by one base pair.  [0, n_sites) is run_fb.
 * Replaces one window of gamma_smc_flow_cached_fb_block_gpu
 * (src/kernels/gamma_smc_flow.cu:632-669, 762-839, 970-997) driven like
 * FlowContext::run_fb (src/bindings.cpp:2897-2989); a per-request query.
 */
int gsmc_run_fb_window(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                       int64_t n_pairs, int64_t site_begin, int64_t site_end, int flags,
                       float* mean, float* lower, float* upper, float* alpha, float* beta);

/*
 * Per-site summary over pairs without materialising [n_sites x n_pairs]:
 * site_mean[s] = mean over the pairs of the posterior mean at site s, and
 * site_min / site_max its extremes, into HOST arrays of n_sites float32.
 * The scan reduces each warp's pairs in registers; partials are folded in a
 * fixed order with a float64 sum, so results are deterministic.
 * core_block_sites <= 0 decodes the full sequence (the reference's
 * run_fb_summary); > 0 decodes blockwise with flank_sites.  pair_batch_size
 * (-1 = auto) caps the pairs folded per pass.
 * Replaces FlowContext::run_fb_summary (src/bindings.cpp:2695-2788) and
 * gamma_smc_flow_cached_fb_reduce_gpu (src/kernels/gamma_smc_flow.cu:
 * 1574-1683), whose float atomics are order-dependent and whose min/max
 * outputs are never written.
 */
int gsmc_run_fb_summary(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                        int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                        int64_t pair_batch_size, float* site_mean, float* site_min,
                        float* site_max);

/*
 * Forward-only (filtered) posterior for n_pairs pairs into HOST arrays of
 * [n_sites x n_pairs] float32: mean, and lower/upper when flags has GSMC_CI.
 * Decoded as the reference's run_fwd: the hom multi-step table rounded to
 * float16, a closed-form het emission, no backward pass.
 * Replaces FlowContext::run_fwd (src/bindings.cpp:2794-2849) and
 * gamma_smc_flow_h2_fwd_gpu (src/kernels/gamma_smc_flow.cu:1136-1295).
 */
int gsmc_run_fwd(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs,
                 int flags, float* mean, float* lower, float* upper);

/*
 * Sink of a streamed blockwise run: called once per (window, pair chunk) with
 * the core rows [site_begin, site_end) of pairs [pair_begin, pair_end) in
 * pinned host memory -- outputs[k] (mean, lower, upper, alpha, beta; NULL
 * where not selected) holds element (s, p) at
 * outputs[k][(s - site_begin) * ld + (p - pair_begin)] and stays valid only
 * until the sink returns.  Return 0 to continue, anything else to stop.
 */
typedef int (*gsmc_sink_fn)(void* user, int64_t site_begin, int64_t site_end, int64_t pair_begin,
                            int64_t pair_end, const float* const* outputs, int64_t ld);

/*
 * Blockwise forward/backward streamed to a host sink instead of one
 * [n_sites x n_pairs] array, for results larger than host memory: each
 * (window, pair chunk) unit is computed into a device stage, copied to a
 * pinned host buffer on a second stream and handed to `sink` on the calling
 * thread, while the GPU already computes the next unit (double-buffered).
 * max_chunk_bytes (0 = 1 GiB) bounds one unit's outputs; pair_batch_size
 * (-1 = auto) caps its pairs.  Values are those of gsmc_run_fb_blockwise.
 * The sink form of FlowContext::run_fb_blockwise (src/bindings.cpp:
 * 2991-3345), which fills one pinned host array.
 */
int gsmc_run_fb_blockwise_stream(gsmc_ctx* ctx, const int32_t* pair_i, const int32_t* pair_j,
                                 int64_t n_pairs, int64_t core_block_sites, int64_t flank_sites,
                                 int64_t pair_batch_size, int flags, gsmc_sink_fn sink,
                                 void* user, uint64_t max_chunk_bytes);

/* Number of windows make_block_windows yields for (n_sites, core_block_sites). */
int gsmc_block_count(int64_t n_sites, int64_t core_block_sites, int64_t* n_blocks);

/*
 * Blockwise forward/backward into HOST arrays of [n_sites x n_pairs] float32.
 * Windows are (core_start, core_stop, padded_start, padded_stop) with padded =
 * core +/- flank_sites clamped to [0, n_sites); each padded window restarts the
 * scan and only its core rows are kept.  blocks_out receives n_blocks x 4 int32
 * rows (size it with gsmc_block_count).  pair_batch_size (-1 = auto) caps the
 * pairs per launch; max_streams > 1 overlaps windows; neither changes values.
 * Replaces FlowContext::run_fb_blockwise (src/bindings.cpp:2991-3345) and the
 * block kernels it launches (src/kernels/gamma_smc_flow.cu:618-669, 762-997).
 */
int gsmc_run_fb_blockwise(gsmc_ctx* ctx, const int32_t* pair_i,
                          const int32_t* pair_j, int64_t n_pairs,
                          int64_t core_block_sites, int64_t flank_sites,
                          int64_t pair_batch_size, int max_streams, int flags,
                          int32_t* blocks_out, float* mean, float* lower,
                          float* upper, float* alpha, float* beta);

/*
 * Device-resident blockwise forward/backward: pair_i/pair_j and all outputs
 * are DEVICE pointers; outputs are [n_sites x ld_out] float32 with pair p of
 * this call written at column out_col0 + p.  core_block_sites >= n_sites with
 * flank_sites = 0 is the full-sequence run_fb.  Work is enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream); scratch comes from the
 * context's pool.  Returns after enqueueing; the caller synchronises.
 * Same semantics as gsmc_run_fb_blockwise; no reference counterpart (the
 * reference only offers host outputs).
 */
int gsmc_run_fb_blockwise_device(gsmc_ctx* ctx, const int32_t* d_pair_i,
                                 const int32_t* d_pair_j, int64_t n_pairs,
                                 int64_t core_block_sites, int64_t flank_sites,
                                 int flags, float* d_mean, float* d_lower,
                                 float* d_upper, float* d_alpha, float* d_beta,
                                 int64_t ld_out, int64_t out_col0, void* stream);

/*
 * Same as gsmc_run_fb_blockwise_device, but the call allocates no device
 * memory: for callers that cannot have it allocate (a framework allocator
 * that already holds the GPU's memory, a service that cannot take the
 * device-wide synchronisation cudaMalloc/cudaFree may cause, a host
 * application with its own device-memory budget for plug-ins).
 * Its scratch is a fixed 128 MiB device array held by every GPU that loads
 * the library until exit; core_block_sites above 131,071 (one CTA slot no
 * longer fits) is rejected with GSMC_E_INVALID.  All calls share that array:
 * calls that overlap on the GPU race and must be serialised by the caller.
 * The first call on each device looks the array's address up and keeps it
 * for the life of the process; make it before any stream capture, and do not
 * use this entry point on a device after cudaDeviceReset (the kept address
 * would then be stale).  core_block_sites and flank_sites are clamped to the
 * sequence length in int64, as the context path does.  No counterpart in the
 * reference.
 */
int gsmc_run_fb_blockwise_device_noalloc(gsmc_ctx* ctx, const int32_t* d_pair_i,
                                         const int32_t* d_pair_j, int64_t n_pairs,
                                         int64_t core_block_sites, int64_t flank_sites,
                                         int flags, float* d_mean, float* d_lower,
                                         float* d_upper, float* d_alpha, float* d_beta,
                                         int64_t ld_out, int64_t out_col0, void* stream);

/* ------------------------------------------------------------ batching --
 * Many jobs -- each a pair set over a site window with its own outputs -- in
 * one persistent launch.  No reference counterpart: the reference launches
 * one kernel pair per call and per block (src/bindings.cpp:3094-3201).
 */
typedef struct gsmc_exec gsmc_exec;

typedef struct gsmc_exec_config {
  int32_t tile_width;        /* threads sharing a pair tile: 32 (a warp) or 128 (a CTA); 0 = 32 */
  int32_t pairs_per_thread;  /* independent pair chains per thread: 1 or 2; 0 = 1 */
  int64_t core_block_sites;  /* sites per chunk of a job window; <= 0 = whole windows */
  int64_t flank_sites;       /* burn-in sites on each side of a chunk; < 0 = 2048 */
  int64_t max_window_sites;  /* longest window with core_block_sites <= 0; 0 = n_sites */
  int64_t max_tasks;         /* (chunk, pair tile) tasks per run; 0 = 65536 */
  uint64_t max_pool_bytes;   /* forward-state pool cap; 0 = half of the free device memory */
  int32_t max_ctas;          /* cap on the persistent grid; 0 = every resident CTA */
  int32_t use_graph;         /* 1 = replay upload + launch as one CUDA graph */
} gsmc_exec_config;

typedef struct gsmc_job {
  const int32_t* pair_i;     /* DEVICE [n_pairs] haplotype indices */
  const int32_t* pair_j;
  int64_t n_pairs;
  int64_t site_begin;        /* window [site_begin, site_end) of the context's sites */
  int64_t site_end;
  int32_t flags;             /* GSMC_CI | GSMC_POSTERIOR */
  int32_t reserved;
  float* out[5];             /* DEVICE mean, lower, upper, alpha, beta: element (s, p) at
                                out[k][(s - site_begin) * ld_out + out_col0 + p] */
  int64_t ld_out;
  int64_t out_col0;
} gsmc_job;

/*
 * Create an executor: the forward-state pool, device task list and pinned
 * upload buffers of one in-flight launch (all scratch, allocated here once).
 * cfg may be NULL for defaults.  Several executors of one context may run
 * concurrently on different streams; one executor's runs must be ordered on
 * one stream.
 */
int gsmc_exec_create(gsmc_ctx* ctx, const gsmc_exec_config* cfg, gsmc_exec** out);
int gsmc_exec_destroy(gsmc_exec* exec);
int gsmc_exec_info(const gsmc_exec* exec, int* grid, uint64_t* pool_bytes, int64_t* slot_rows,
                   int64_t* max_tasks);

/*
 * Enqueue all jobs as one persistent launch on `stream` and return.  Each
 * job's window is decoded as by gsmc_run_fb_window, cut into chunks of
 * core_block_sites with flank_sites of burn-in when the executor chunks.
 * Device pair indices are not validated on the host: out-of-range pairs are
 * skipped on the device and their output columns left unwritten.
 */
int gsmc_exec_run(gsmc_exec* exec, const gsmc_job* jobs, int64_t n_jobs, void* stream);

/*
 * gsmc_exec_run that also checks the chunked jobs: job_flags (device memory,
 * n_jobs int32, cleared by the call on `stream`) gets 1 for every job whose
 * window was cut into chunks and whose chunks' boundary states (the forward
 * and backward states each chunk reached from its burn-in against the exact
 * ones of its neighbours) differ somewhere, bit for bit.  Unflagged jobs'
 * outputs equal their whole-window decode (gsmc_run_fb_window) exactly; a
 * flagged job should be decoded again whole (the Python layer does).  No
 * reference counterpart.
 */
int gsmc_exec_run_checked(gsmc_exec* exec, const gsmc_job* jobs, int64_t n_jobs, void* stream,
                          int32_t* job_flags);

/* Kernel timing of an executor's launches (as gsmc_ctx_timing). */
int gsmc_exec_timing(gsmc_exec* exec, int enable);
int gsmc_exec_timing_read(gsmc_exec* exec, double* kernel_ms, int64_t* launches,
                          double* pair_sites);

/*
 * Copy n device regions (src[i], bytes[i]) into host memory dst[i] -- pageable
 * or pinned -- once the work already enqueued on `stream` has finished;
 * returns when every byte has landed.  Data moves through the library's
 * pinned ring with parallel host threads, so large pageable results need no
 * pinning.  For collecting the outputs of gsmc_exec_run; no reference
 * counterpart (the reference copied with blocking cudaMemcpy,
 * src/bindings.cpp:2965-2975).
 */
int gsmc_copy_to_host(int64_t n, void* const* dst, const void* const* src,
                      const uint64_t* bytes, void* stream);

/*
 * Frees the context's device scratch (forward-state slots, output stages,
 * summary accumulators, speculation buffers) and its pinned staging, after
 * waiting for its streams.  The next call allocates again; genotypes and
 * tables stay resident.  For callers that share the device with other
 * allocations between calls.  No reference counterpart.
 */
int gsmc_ctx_release_scratch(gsmc_ctx* ctx);

/* Bytes of device scratch the context currently holds (forward-state pool). */
int gsmc_ctx_scratch_bytes(const gsmc_ctx* ctx, uint64_t* bytes);

/*
 * Speculative chunking statistics of a context: launches that cut windows
 * into parallel chunks (when a call has too few pair tiles to fill the GPU)
 * and the (window, pair)s whose chunks failed the bitwise boundary check and
 * were decoded again whole.  Waits for the context's stream.  No reference
 * counterpart.
 */
int gsmc_ctx_spec_stats(gsmc_ctx* ctx, int64_t* launches, int64_t* repaired);

/*
 * Launch shape of the context's most recent scan: threads sharing a task (128
 * = the CTA, 32 = a warp) and pairs per thread (1 or 2).  Calls with enough
 * pair tiles to give every resident CTA two tasks run two pairs per thread.
 * No reference counterpart.
 */
int gsmc_ctx_scan_shape(const gsmc_ctx* ctx, int* width, int* pairs_per_thread);

/*
 * Speculative chunking of the calling thread's last gsmc_flow_fb call: site
 * chunks per pair (1 = none; a call whose pairs cannot fill every SM cuts the
 * sites into chunks with burn-ins, checked bitwise at every boundary) and the
 * pairs whose check failed and were decoded again whole.  No reference
 * counterpart.
 */
int gsmc_flow_fb_stats(int* chunks, int64_t* repaired);

/*
 * Kernel timing for measurement: while enabled, every scan launch of this
 * context is bracketed by CUDA events on the stream it is launched on.
 * gsmc_ctx_timing_read synchronises those events and returns the summed
 * kernel milliseconds, the number of launches and the pair-sites (pairs x
 * core sites) they produced since the last read, then resets the counters.
 * No reference counterpart.
 */
int gsmc_ctx_timing(gsmc_ctx* ctx, int enable);
int gsmc_ctx_timing_read(gsmc_ctx* ctx, double* kernel_ms, int64_t* launches,
                         double* pair_sites);

/*
 * Per-diploid heterozygous site counts on the device: counts[k] = number of
 * sites where haplotypes 2k and 2k+1 differ, k < n_haps / 2 (int64, exact),
 * from bit-packed genotypes (XOR + popcount).  The chromosome-wide sums of
 * the theta/rho auto-calibration, _estimate_scaled_params
 * (python/gamma_smc_cu/infer.py:44-99), which counts with numpy.
 */
int gsmc_diploid_het_counts(const uint8_t* G, int64_t n_haps, int64_t n_sites, int64_t* counts);

/*
 * Flow field on the GPU in float64: for every cell of a mean_n x cv_n grid
 * with Gamma(alpha[c], beta[c]), the least-squares drift (u[c], v[c]) of
 * (log10 mean, log10 CV) per unit of scaled time, divided by `calibration`
 * (the reference uses 5.302).  n_epochs = 0 is constant Ne; otherwise epoch
 * k of a piecewise-constant N(t) starts at scaled time epoch_start[k] with
 * coalescence rate epoch_rate[k] (Ne_ref / N_k) and cumulative rate
 * epoch_cum[k].  Time grid of 2 n_steps + 1 points.  Cells the reference
 * skips or cannot fit are 0.
 * Replaces generate_flow_field (python/gamma_smc_cu/demographic.py:146-208)
 * and its distribution-difference helpers (:17-143), which run on the CPU.
 */
int gsmc_generate_flow_field(const double* alpha, const double* beta, int mean_n, int cv_n,
                             int n_steps, int n_epochs, const double* epoch_start,
                             const double* epoch_rate, const double* epoch_cum,
                             double calibration, double* u, double* v);

/*
 * Uncached flow-field forward/backward for n_pairs pairs of G into HOST arrays
 * of [n_sites x n_pairs] float32 (mean; lower/upper with GSMC_CI): every gap
 * is integrated on the 51 x 50 flow field staged in shared memory (one
 * per-bp recombination step, then sub-steps of at most 0.1 scaled
 * recombination with hom emissions), no multi-step tables; rates are the raw
 * (mu, rho) scaled by 4 Ne.  No context: G and positions are uploaded per
 * call.  GSMC_E_TIMEOUT if the shared-memory staging did not complete.
 * Replaces gamma_smc_flow_fb (src/bindings.cpp:2159-2300) and
 * gamma_smc_flow_fb_gpu (src/kernels/gamma_smc_flow.cu:168-398).
 */
int gsmc_flow_fb(const uint8_t* G, int64_t n_haps, int64_t n_sites, const double* positions,
                 const int32_t* pair_i, const int32_t* pair_j, int64_t n_pairs, double Ne,
                 double mu, double rho, const char* flow_field_path, int flags, float* mean,
                 float* lower, float* upper);

/*
 * Table build of a context: *build_seconds = build + upload of its scan
 * tables by this context (0 when it reused a resident set), *reused = 1 when
 * a set with the same (device, flow field, Ne, mu, rho, cache_steps, build)
 * was resident already (held by another context, or parked: the most
 * recently released set of each device stays resident, as the reference's
 * process-wide table cache does, src/bindings.cpp:1884-2157).  Either
 * pointer may be NULL.
 */
int gsmc_ctx_tables_info(const gsmc_ctx* ctx, double* build_seconds, int* reused);

/*
 * Free the parked table sets (those no live context holds); sets in use stay.
 * No reference counterpart.
 */
int gsmc_free_cached_tables(void);

/*
 * Page-locked host buffers for results, cached for reuse.  A host output
 * array that is page-locked is written by the device-to-host DMA directly
 * (no staging ring, no host thread touching the data), which is what repeated
 * large calls want; page-locking is slow (seconds per 10 GB), so released
 * buffers are kept and handed out again to requests they fit (at most twice
 * the request).  Buffers of 64 MB or more are anonymous mappings of whole
 * 2 MB pages advised MADV_HUGEPAGE and registered with cudaHostRegister
 * (about three times faster to page-lock than cudaHostAlloc's memory);
 * smaller ones come from cudaHostAlloc.  gsmc_host_free returns a buffer to the cache;
 * gsmc_host_cache_limit bounds the bytes kept cached (default 256 GiB;
 * 0 frees every cached buffer).  No reference counterpart (the reference
 * pins its fresh output arrays with cudaHostRegister on every call,
 * src/bindings.cpp:3086-3092).
 */
int gsmc_host_alloc(uint64_t bytes, void** ptr);
int gsmc_host_free(void* ptr);
int gsmc_host_cache_limit(uint64_t max_cached_bytes);

/*
 * Poll budget of the uncached kernels' wait for their shared-memory copy of
 * the flow field (default 2^24 mbarrier polls, process-wide, read at each
 * gsmc_flow_fb call).  A CTA whose copy has not landed within the budget
 * sets an error flag, waits (bounded) for the copy to finish and skips its
 * pairs; the call then returns GSMC_E_TIMEOUT and the next call runs
 * normally.  A budget of 0 gives up at once, which tests use to exercise that
 * path.  *previous (if not NULL) receives the old budget.  No reference
 * counterpart (the reference waits without a limit and prints launch errors,
 * src/kernels/gamma_smc_flow.cu:365-369).
 */
int gsmc_set_copy_wait_polls(int64_t polls, int64_t* previous);

/*
 * Bit-pack genotypes on the device: packed[h * n_words + w] bit b =
 * G[h][64w + b] & 1, n_words = ceil(n_sites / 64); host in, host out.
 * Replaces _core.bitpack / bitpack_kernel (src/kernels/bitpack.cu:11-38).
 */
int gsmc_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites,
                 uint64_t* packed);

/* Inverse of gsmc_bitpack (_core.unpack, src/kernels/bitpack.cu:43-60). */
int gsmc_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites,
                uint8_t* G);

/*
 * Copy the context's scan tables for one layer back to the host, for tests:
 * table 0..4 = fwd_hom, fwd_het, bwd_hom, bwd_het, chunk; out receives
 * 2 x 2550 floats (log10 mean grid, then log10 CV grid) of that layer.
 * No reference counterpart (debug view of FlowFieldDeviceCacheView).
 */
int gsmc_ctx_table_layer(const gsmc_ctx* ctx, int table, int layer, float* out);

#ifdef __cplusplus
}
#endif

#endif /* GSMC_B200_H */
