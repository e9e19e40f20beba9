// Uncached flow-field forward/backward: gamma_smc_cu.gamma_smc_flow_fb.
//
// Instead of the precomputed multi-step tables, every gap is integrated on
// the flow field itself (src/kernels/gamma_smc_flow.cu:29-163, 168-398): one
// recombination step of the per-bp rate, then ceil(10 x scaled rho of the
// rest of the gap) sub-steps that each apply the hom emission (beta += mu)
// and a recombination step, then the site's emission.  The backward pass
// applies the same segment in the opposite order and combines with the
// stored forward states like the cached scan.
//
// The 51 x 50 (u, v) grid -- 20,400 bytes, interleaved as float2 so a corner
// is one 8-byte shared-memory read -- is staged once per CTA by a TMA bulk
// copy (cp.async.bulk into shared memory, completion on an mbarrier).  The
// wait for it is bounded: if the copy has not landed after a set number of
// polls (UncachedArgs::wait_polls) the CTA records an error, waits (again
// bounded) for the copy to finish and skips its pairs.  One thread per pair
// walks all sites forward (states to a [S][P] float2 buffer) and back.
//
// The float arithmetic follows the reference expression by expression --
// including the default contraction of the lines around __exp10f/__log10f --
// so the outputs match its kernel bit for bit.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fwd.h"
#include "scan_device.cuh"
#include "uncached.h"

namespace gsmc {
namespace {

constexpr int kGridCells = kRows * kCols;            // 2550
constexpr unsigned kFlowBytes = kGridCells * sizeof(float2);  // 20400, a multiple of 16
// After giving up on the copy, a CTA still waits this many polls for it to
// land before it exits, so that no bulk copy into its shared memory is in
// flight when the CTA's shared memory is released.
constexpr long long kDrainPolls = 1ll << 26;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t copy_landed(unsigned b) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(b)
      : "memory");
  return done;
}

// Stage the flow field into shared memory with one bulk copy; false if it did
// not complete within `polls` polls of its mbarrier.  On false the CTA has
// recorded the error in *error and, within a second bounded wait, let the
// copy finish, so it may exit.
__device__ bool stage_flow(float2* s_flow, uint64_t* bar, const float2* g_flow, long long polls,
                           int* error) {
  const unsigned b = smem_addr(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kFlowBytes)
        : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_addr(s_flow)), "l"(g_flow), "r"(kFlowBytes), "r"(b)
        : "memory");
  }
  uint32_t done = 0;
  for (long long i = 0; i < polls && !done; ++i) done = copy_landed(b);
  if (done) return true;
  if (threadIdx.x == 0) atomicExch(error, 1);
  for (long long i = 0; i < kDrainPolls && !done; ++i) done = copy_landed(b);
  return false;
}

// Bilinear (u, v) at (m, c) from the staged grid, the scan's interpolation.
__device__ __forceinline__ float2 flow_at(const float2* s_flow, float m, float c) {
  float fm = __fmul_rn(__fsub_rn(m, kMLo), kMInv);
  float fc = __fmul_rn(__fsub_rn(c, kCLo), kCInv);
  fm = fmaxf(0.0f, fminf(fm, (float)(kRows - 1)));
  fc = fmaxf(0.0f, fminf(fc, (float)(kCols - 1)));
  const float rf = floor_small(fminf(fm, (float)kPatchRows - 0.5f));
  const float qf = floor_small(fminf(fc, (float)kPatchCols - 0.5f));
  const float wm = __fsub_rn(fm, rf), wc = __fsub_rn(fc, qf);
  const int base = (int)rf * kCols + (int)qf;
  const float2 v00 = s_flow[base], v01 = s_flow[base + 1];
  const float2 v10 = s_flow[base + kCols], v11 = s_flow[base + kCols + 1];
  const float vc = __fsub_rn(1.0f, wc), vm = __fsub_rn(1.0f, wm);
  float2 r;
  r.x = __fmaf_rn(wm, __fmaf_rn(wc, v11.x, __fmul_rn(vc, v10.x)),
                  __fmul_rn(vm, __fmaf_rn(wc, v01.x, __fmul_rn(vc, v00.x))));
  r.y = __fmaf_rn(wm, __fmaf_rn(wc, v11.y, __fmul_rn(vc, v10.y)),
                  __fmul_rn(vm, __fmaf_rn(wc, v01.y, __fmul_rn(vc, v00.y))));
  return r;
}

__device__ __forceinline__ void recomb_step(const float2* s_flow, float rho, float& m, float& c) {
  const float2 d = flow_at(s_flow, m, c);
  m = __fmaf_rn(d.x, rho, m);
  c = __fmaf_rn(d.y, rho, c);
  m = fmaxf(kMLo, fminf(m, kMHi));
  c = fmaxf(kCLo, fminf(c, kCHi));
}

// Rest of a gap: sub-steps of at most 0.1 scaled recombination, each a hom
// emission then a recombination step (src/kernels/gamma_smc_flow.cu:63-95).
__device__ __forceinline__ void advance(const float2* s_flow, float rho_total, float mu_total,
                                        float& m, float& c) {
  if (rho_total < 1e-12f) return;
  const int n_iter = max(1, (int)ceilf(rho_total * (1.0f / 0.1f)));
  const float inv_n = __frcp_rn((float)n_iter);
  const float rho_per = rho_total * inv_n;
  const float mu_per = mu_total * inv_n;
  for (int i = 0; i < n_iter; ++i) {
    // as the reference writes it (default contraction around the intrinsics)
    const float a_log = -2.0f * c;
    float b_log = a_log - m;
    const float b_lin = __exp10f(b_log) + mu_per;
    b_log = __log10f(b_lin);
    m = a_log - b_log;
    recomb_step(s_flow, rho_per, m, c);
  }
}

// Observed site: hom emission always, het adds alpha + 1 (:141-158).
__device__ __forceinline__ void emit(bool het, float mu, float& m, float& c) {
  float a_log = -2.0f * c;
  float b_log = a_log - m;
  b_log = __log10f(__exp10f(b_log) + mu);
  if (het) a_log = __log10f(__exp10f(a_log) + 1.0f);
  m = a_log - b_log;
  c = -0.5f * a_log;
}

// The segment of `seg` base pairs entering a site: one per-bp recombination
// step, then the rest of the gap.
__device__ __forceinline__ void segment(const float2* s_flow, int seg, float rho, float mu,
                                       float& m, float& c) {
  if (rho >= 1e-12f) recomb_step(s_flow, rho, m, c);
  if (seg > 1) advance(s_flow, rho * (float)(seg - 1), mu * (float)(seg - 1), m, c);
}

// Pair p over sites: forward from (0, 0) before site s0 through site c1 - 1,
// states stored for [c0, c1); backward from (0, 0) after site e1 - 1 down
// through site c0, posteriors written for [c0, c1).  Boundary records (each
// optional): fspec = forward state after c0 - 1, fend = after c1 - 1;
// bspec = backward state after applying site c1 (reached from e1),
// bend = after applying site c0.
template <bool CI>
__device__ __forceinline__ void uncached_walk(const UncachedArgs& a, const float2* s_flow, int p,
                                              int s0, int c0, int c1, int e1, float2* fspec,
                                              float2* fend, float2* bspec, float2* bend) {
  const int hi = a.pi[p], hj = a.pj[p];
  if (hi < 0 || hi >= a.n_haps || hj < 0 || hj >= a.n_haps) return;
  const ulonglong2* gi = a.geno + hi;
  const ulonglong2* gj = a.geno + hj;
  const int64_t P = a.n_pairs;
  float m = 0.0f, c = 0.0f;
  uint64_t x = 0;
  for (int s = s0; s < c1; ++s) {
    if ((s & 63) == 0 || s == s0) x = word_at(gi, a.n_haps, s) ^ word_at(gj, a.n_haps, s);
    const bool het = (x >> (s & 63)) & 1ull;
    segment(s_flow, a.seg[s], a.rho, a.mu, m, c);
    emit(het, a.mu, m, c);
    if (s >= c0)
      __stcs(a.fwd + (int64_t)s * P + p, make_float2(m, c));
    else if (s == c0 - 1 && fspec)
      *fspec = make_float2(m, c);
  }
  if (fend) *fend = make_float2(m, c);
  m = 0.0f;
  c = 0.0f;
  Task t;  // output addressing for the shared combine
  t.unscale = a.unscale;
  t.out[0] = a.mean;
  t.out[1] = a.lower;
  t.out[2] = a.upper;
  t.out[3] = t.out[4] = nullptr;
  for (int s = e1 - 1; s >= c0; --s) {
    if (s < c1) {
      if (s == c1 - 1 && bspec) *bspec = make_float2(m, c);
      const float2 f = __ldlu(a.fwd + (int64_t)s * P + p);
      combine_store(t, (int64_t)s * a.ldo + p, f, m, c, CI, false);
    }
    if ((s & 63) == 63 || s == e1 - 1) x = word_at(gi, a.n_haps, s) ^ word_at(gj, a.n_haps, s);
    const bool het = (x >> (s & 63)) & 1ull;
    emit(het, a.mu, m, c);
    segment(s_flow, a.seg[s], a.rho, a.mu, m, c);
  }
  if (bend) *bend = make_float2(m, c);
}

// One thread per pair over all sites.
template <bool CI>
__global__ void __launch_bounds__(256) uncached_fb_kernel(const UncachedArgs a) {
  __shared__ __align__(16) float2 s_flow[kGridCells];
  __shared__ __align__(8) uint64_t bar;
  if (!stage_flow(s_flow, &bar, a.flow, a.wait_polls, a.error)) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  uncached_walk<CI>(a, s_flow, p, 0, 0, a.n_sites, a.n_sites, nullptr, nullptr, nullptr, nullptr);
}

// Speculative site chunks: thread (pair p, chunk k = blockIdx.y) decodes sites
// [c0, c1) with `burn_in` sites of burn-in on each inner side and writes the
// four boundary records rec[boundary][kind][pair] (kind 0 = forward end of the
// left chunk, 1 = forward burn-in of the right chunk, 2 = backward end of the
// right chunk, 3 = backward burn-in of the left chunk).
template <bool CI>
__global__ void __launch_bounds__(256) uncached_chunk_kernel(const UncachedArgs a, UncachedSpec sp) {
  __shared__ __align__(16) float2 s_flow[kGridCells];
  __shared__ __align__(8) uint64_t bar;
  if (!stage_flow(s_flow, &bar, a.flow, a.wait_polls, a.error)) return;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  const int k = blockIdx.y, K = sp.k_chunks, S = a.n_sites;
  const int c0 = (int)((int64_t)S * k / K), c1 = (int)((int64_t)S * (k + 1) / K);
  const int s0 = k == 0 ? 0 : max(0, c0 - sp.burn_in);
  const int e1 = k == K - 1 ? S : min(S, c1 + sp.burn_in);
  const int64_t P = a.n_pairs;
  float2* left = k > 0 ? sp.rec + (int64_t)(k - 1) * 4 * P + p : nullptr;
  float2* right = k < K - 1 ? sp.rec + (int64_t)k * 4 * P + p : nullptr;
  uncached_walk<CI>(a, s_flow, p, s0, c0, c1, e1, left ? left + P : nullptr, right,
                    right ? right + 3 * P : nullptr, left ? left + 2 * P : nullptr);
}

__device__ __forceinline__ bool same_state(float2 a, float2 b) {
  return __float_as_int(a.x) == __float_as_int(b.x) && __float_as_int(a.y) == __float_as_int(b.y);
}

// Pairs with any boundary whose records differ (bitwise) go on the repair list.
__global__ void uncached_verify_kernel(const UncachedArgs a, UncachedSpec sp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  const int64_t P = a.n_pairs;
  for (int b = 0; b + 1 < sp.k_chunks; ++b) {
    const float2* r = sp.rec + (int64_t)b * 4 * P + p;
    if (!same_state(r[0], r[P]) || !same_state(r[2 * P], r[3 * P])) {
      sp.repair_list[atomicAdd(sp.repair_count, 1)] = p;
      return;
    }
  }
}

// Listed pairs decoded again over all sites.
template <bool CI>
__global__ void __launch_bounds__(256) uncached_repair_kernel(const UncachedArgs a, UncachedSpec sp) {
  const int n = *sp.repair_count;
  if ((int)(blockIdx.x * blockDim.x) >= n) return;  // whole CTAs leave before staging
  __shared__ __align__(16) float2 s_flow[kGridCells];
  __shared__ __align__(8) uint64_t bar;
  if (!stage_flow(s_flow, &bar, a.flow, a.wait_polls, a.error)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) atomicAdd(sp.repaired_total, n);
  if (t >= n) return;
  uncached_walk<CI>(a, s_flow, sp.repair_list[t], 0, 0, a.n_sites, a.n_sites, nullptr, nullptr,
                    nullptr, nullptr);
}

}  // namespace

cudaError_t launch_uncached_fb(const UncachedArgs& a, cudaStream_t stream) {
  if (a.n_pairs <= 0 || a.n_sites <= 0) return cudaSuccess;
  // every CTA stages its own grid copy: small pair counts get 32-thread CTAs
  // on as many SMs as possible rather than a few SMs doing everything
  const int threads = chain_cta_threads(a.n_pairs, 256);
  const unsigned grid = (unsigned)((a.n_pairs + threads - 1) / threads);
  if (a.lower && a.upper)
    uncached_fb_kernel<true><<<grid, threads, 0, stream>>>(a);
  else
    uncached_fb_kernel<false><<<grid, threads, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_uncached_spec(const UncachedArgs& a, const UncachedSpec& sp, cudaStream_t stream) {
  if (a.n_pairs <= 0 || a.n_sites <= 0) return cudaSuccess;
  if (sp.k_chunks <= 1) return launch_uncached_fb(a, stream);
  const bool ci = a.lower && a.upper;
  const int threads = chain_cta_threads((int64_t)a.n_pairs * sp.k_chunks, 256);
  const dim3 grid((unsigned)((a.n_pairs + threads - 1) / threads), (unsigned)sp.k_chunks);
  cudaError_t e = cudaMemsetAsync(sp.repair_count, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  if (ci)
    uncached_chunk_kernel<true><<<grid, threads, 0, stream>>>(a, sp);
  else
    uncached_chunk_kernel<false><<<grid, threads, 0, stream>>>(a, sp);
  const unsigned pg = (unsigned)((a.n_pairs + 127) / 128);
  uncached_verify_kernel<<<pg, 128, 0, stream>>>(a, sp);
  if (ci)
    uncached_repair_kernel<true><<<pg, 128, 0, stream>>>(a, sp);
  else
    uncached_repair_kernel<false><<<pg, 128, 0, stream>>>(a, sp);
  return cudaGetLastError();
}

}  // namespace gsmc
