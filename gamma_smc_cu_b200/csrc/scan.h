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

// Output selection of a task.  kTaskSummary replaces the per-pair outputs by
// per-warp partial reductions over the task's pairs at each core site: the
// sum, minimum and maximum of the posterior means go to out[0], out[1] and
// out[2] at (s - out_row0) * ldo + out_off + (warp within the tile).
enum TaskFlags { kTaskCI = 1, kTaskPosterior = 2, kTaskSummary = 4 };

// One unit of scan work: up to (tile width x pairs per thread) pairs over one
// padded window.  Forward over [ps, ce), backward over [pe-1 .. cs], posterior
// at core rows [cs, ce).  The task's pairs are (pi[j], pj[j]), j <
// pair_count.  Output element (s, pair j of the task) is
// out[k][out_off + (s - out_row0) * ldo + j] for each selected output k
// (0 mean, 1 lower, 2 upper, 3 alpha, 4 beta).
//
// Speculative chunks: a long window may be cut into chunks whose forward
// pass starts some sites before the chunk at (0, 0) instead of at the
// window's start (and whose backward pass starts some sites after it).  Such
// a task records, for each of its pairs, the states at its chunk boundaries:
// at the left boundary (bl) the forward state after site cs-1 from its burn-in
// (kind 1) and the backward state after applying site cs (kind 2); at the
// right boundary (br) the forward state after site ce-1 (kind 0) and the
// backward state after applying site ce from its burn-in (kind 3).  Kind k of
// pair j of the task is at b[k * bstride + j].  A chunk's result is exact when
// its neighbours' states equal its own bit for bit (the speculative trajectory
// has joined the exact one); pairs where they do not are recomputed.
struct Task {
  int32_t ps, cs, ce, pe;
  const int32_t* pi;
  const int32_t* pj;
  int32_t pair_count;
  int32_t out_row0;
  int32_t flags;        // TaskFlags
  float unscale;        // 2 * Ne of the task's job
  int64_t out_off;
  int64_t ldo;
  float* out[5];
  float2* bl;           // left-boundary records, or null
  float2* br;           // right-boundary records, or null
  int64_t bstride;
};
static_assert(sizeof(Task) == 128, "a warp copies a Task as 32 words");

// Head of a device task list: CTAs take task numbers from `next` (zero when
// the list is uploaded) until it reaches `count`.  Tasks follow at
// kTaskListHead bytes.
struct TaskListHead {
  int next;
  int count;
};
constexpr size_t kTaskListHead = 128;

struct ScanArgs {
  const ulonglong2* geno;   // [n_groups][n_haps]: 128 sites per entry, bit b of .x/.y = site 128g+b / 128g+64+b
  int64_t n_haps;
  const SiteCode* code;     // [n_sites], with kCodePad zero entries before and after
  const float4* site_tab;   // [2 directions][L][hom, het][2450][2]
  const float4* chunk_tab;  // [2450][2]
  int L;
  int* next;                // task counter (device memory, zero at launch)
  const int* count;         // number of tasks (device or mapped host memory)
  const Task* tasks;        // the tasks (device or mapped host memory)
  float2* fwd;              // forward-state slots, one per task slot of the grid
  int64_t slot_rows;        // sites per slot (max core length of the tasks)
};

// Launch shape of the scan: `width` threads (32 = one warp, 128 = the whole
// CTA) share a pair tile and take tasks together; each thread carries
// `pairs_per_thread` independent pair chains.  A tile holds width x
// pairs_per_thread pairs and owns one forward-state slot.
struct ScanShape {
  int width;             // 32 or 128
  int pairs_per_thread;  // 1 or 2
};

// Threads per CTA of the scan kernels.
int scan_threads();
// Pairs of one task tile and tiles (forward-state slots) per CTA for a shape.
int scan_tile_pairs(ScanShape shape);
int scan_tiles_per_cta(ScanShape shape);
// Whether a shape has a compiled kernel.
bool scan_shape_valid(ScanShape shape);

// Resident CTAs of the persistent scan kernel of `shape` on the current device.
int scan_resident_ctas(ScanShape shape);

// Launch the persistent scan over the task list of args with `grid`
// CTAs; CTA b's tile t owns forward-state slot b * tiles_per_cta + t of
// slot_rows x tile pairs float2.  `summary`: every task is a kTaskSummary task.
cudaError_t launch_scan(const ScanArgs& args, int grid, ScanShape shape, cudaStream_t stream,
                        bool summary = false);

// A window decoded in speculative chunks: its chunk boundaries are records
// first_bnd .. first_bnd + n_bnd - 1 of the launch's record buffer, and
// `repair` is the window decoded whole for the launch's pair 0 (its pi / pj
// and out_off advance by the pair index, pair_count is set to 1).
struct SpecWindow {
  int32_t first_bnd;
  int32_t n_bnd;
  int32_t pad[2];
  Task repair;
};

// A job of an executor run whose window was cut into chunks: its boundary
// records start at float2 `rec_off` of the run's record buffer, laid out
// [boundary][4 kinds][n_pairs] as the context's speculative chunks.
struct ExecCheck {
  int64_t rec_off;
  int32_t n_bnd;
  int32_t n_pairs;
  int32_t job;
  int32_t pad;
};

// For every pair of every checked job: compare its boundary records bit for
// bit and set flags[job] = 1 when any differ (the job's chunked outputs may
// then differ from its whole-window decode).
cudaError_t launch_exec_verify(const float2* rec, const ExecCheck* checks, int n_checks,
                               int max_pairs, int32_t* flags, cudaStream_t stream);

// For every (window, pair) of a speculative launch over n_pairs pairs:
// compare the boundary records (rec: [boundary][4 kinds][n_pairs] float2) bit
// for bit and append a one-pair repair task to the list at `head` for each
// pair whose speculative chunks did not join the exact trajectory.
cudaError_t launch_spec_verify(const float2* rec, int64_t n_pairs, const SpecWindow* win,
                               int n_win, TaskListHead* head, Task* repairs, int max_repairs,
                               cudaStream_t stream);

// *acc += *count (one thread), for statistics kept on the device.
cudaError_t launch_add_count(const int* count, int* acc, cudaStream_t stream);

// Fold per-warp partials (sum, min, max) of a summary launch -- rows x cols,
// row pitch ld -- into per-site accumulators acc_sum (float64), acc_min,
// acc_max [rows], in a fixed order (deterministic); `first` overwrites
// instead of accumulating.
cudaError_t launch_summary_fold(const float* p_sum, const float* p_min, const float* p_max,
                                int64_t rows, int64_t cols, int64_t ld, double* acc_sum,
                                float* acc_min, float* acc_max, bool first, cudaStream_t stream);
// site_mean[s] = acc_sum[s] / n_pairs rounded to float32.
cudaError_t launch_summary_finish(const double* acc_sum, int64_t rows, double n_pairs,
                                  float* site_mean, cudaStream_t stream);

// counts[k] = sites where haplotypes 2k and 2k+1 differ (scan layout input).
cudaError_t launch_het_counts(const ulonglong2* geno, int64_t n_haps, int64_t n_groups,
                              long long* counts, cudaStream_t stream);

// Pack [n_haps x n_sites] uint8 genotypes.  scan_layout: word-major 128-site
// groups for the scan; otherwise the reference's row-major uint64 words.
cudaError_t launch_bitpack(const uint8_t* G, int64_t n_haps, int64_t n_sites, void* out,
                           bool scan_layout, cudaStream_t stream);
cudaError_t launch_unpack(const uint64_t* packed, int64_t n_haps, int64_t n_sites, uint8_t* G,
                          cudaStream_t stream);

}  // namespace gsmc
