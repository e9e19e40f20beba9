// Forward-only (filtered) Gamma-SMC posterior: FlowContext.run_fwd.
//
// The reference runs this path with a half-precision copy of its hom
// multi-step table (src/bindings.cpp:2098-2107, 2794-2849 ->
// src/kernels/gamma_smc_flow.cu:1136-1295): each gap of k base pairs is one
// bilinear lookup in layer k-1 (full 1000-step chunks first), a het site adds
// one to alpha in closed form, and every site writes the filtered mean (and
// Wilson-Hilferty bounds).  There is no backward pass and no forward-state
// buffer.
//
// Here the half table is stored in the patch layout of the scan tables: the
// four corners of log10-mean and of log10-CV of one interpolation cell are
// eight halves, one 16-byte load per lookup.  The arithmetic (truncation,
// fused multiply-adds, __exp10f/__log10f, exp2f) is the reference's, so the
// outputs are bit-identical to its kernel.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fwd.h"
#include "scan_device.cuh"

namespace gsmc {
namespace {

__device__ __forceinline__ void half_patch_lookup(const uint4* __restrict__ layer, float& m,
                                                  float& c) {
  float fm = __fmul_rn(__fsub_rn(m, kMLo), kMInv);
  float fc = __fmul_rn(__fsub_rn(c, kCLo), kCInv);
  fm = fmaxf(0.0f, fminf(fm, (float)(kRows - 1)));
  fc = fmaxf(0.0f, fminf(fc, (float)(kCols - 1)));
  const float rf = floor_small(fminf(fm, (float)kPatchRows - 0.5f));
  const float qf = floor_small(fminf(fc, (float)kPatchCols - 0.5f));
  const float wm = __fsub_rn(fm, rf), wc = __fsub_rn(fc, qf);
  const int idx = __float_as_int(__fadd_rn(__fmaf_rn(rf, (float)kPatchCols, qf), 8388608.0f)) -
                  0x4B000000;
  const uint4 v = __ldg(layer + idx);
  const float2 m0 = __half22float2(*reinterpret_cast<const __half2*>(&v.x));  // (r,q) (r,q+1)
  const float2 m1 = __half22float2(*reinterpret_cast<const __half2*>(&v.y));  // (r+1,q) (r+1,q+1)
  const float2 c0 = __half22float2(*reinterpret_cast<const __half2*>(&v.z));
  const float2 c1 = __half22float2(*reinterpret_cast<const __half2*>(&v.w));
  const float vc = __fsub_rn(1.0f, wc), vm = __fsub_rn(1.0f, wm);
  m = __fmaf_rn(wm, __fmaf_rn(wc, m1.y, __fmul_rn(vc, m1.x)),
                __fmul_rn(vm, __fmaf_rn(wc, m0.y, __fmul_rn(vc, m0.x))));
  c = __fmaf_rn(wm, __fmaf_rn(wc, c1.y, __fmul_rn(vc, c1.x)),
                __fmul_rn(vm, __fmaf_rn(wc, c0.y, __fmul_rn(vc, c0.x))));
}

// Pair p's filtered scan over sites [s0, s1), starting from (m, c) = (0, 0)
// before site s0, with outputs from site s_out on (row s of the outputs).
// spec_rec (if set) receives the state after site s_out - 1, end_rec the
// state after site s1 - 1.
template <bool CI>
__device__ __forceinline__ void fwd_walk(const FwdArgs& a, int p, int s0, int s_out, int s1,
                                         float2* spec_rec, float2* end_rec) {
  const int hi = a.pi[p], hj = a.pj[p];
  if (hi < 0 || hi >= a.n_haps || hj < 0 || hj >= a.n_haps) return;  // outputs untouched
  const ulonglong2* gi = a.geno + hi;
  const ulonglong2* gj = a.geno + hj;
  const uint4* chunk = a.tab + (size_t)(a.L - 1) * kPatches;
  float m = 0.0f, c = 0.0f;
  uint64_t x = word_at(gi, a.n_haps, s0) ^ word_at(gj, a.n_haps, s0);
  float* out = a.mean + (int64_t)s_out * a.ldo + p;
  FwdCode nx = a.code[s0];
  for (int s = s0; s < s1; ++s) {
    const FwdCode sc = nx;
    if (s + 1 < a.n_sites) nx = a.code[s + 1];
    if ((s & 63) == 0) x = word_at(gi, a.n_haps, s) ^ word_at(gj, a.n_haps, s);
    // gap transition (none at site 0 or for a zero gap)
    for (int u = 0; u < sc.chunks; ++u) half_patch_lookup(chunk, m, c);
    if (sc.layer >= 0) half_patch_lookup(a.tab + (size_t)sc.layer * kPatches, m, c);
    // het emission: alpha + 1 in closed form.  These lines, the mean and the
    // bounds are left to the compiler's default contraction, written as the
    // reference writes them (src/kernels/gamma_smc_flow.cu:1243-1271), so the
    // intrinsics' inlined multiplies fuse the same way.
    if ((x >> (s & 63)) & 1ull) {
      const float alpha = __exp10f(-2.0f * c) + 1.0f;
      const float a_log = __log10f(alpha);
      const float b_log = -2.0f * c - m;
      m = a_log - b_log;
      c = -0.5f * a_log;
    }
    if (s < s_out) {  // burn-in of a speculative chunk: no output
      if (s == s_out - 1 && spec_rec) *spec_rec = make_float2(m, c);
      continue;
    }
    const float mg = exp2f(m * 3.321928094887362f) * a.two_ne;
    __stcs(out, mg);
    if (CI) {
      const float alpha = __exp10f(-2.0f * c);
      const float inv9a = __frcp_rn(9.0f * alpha);
      const float sq = __fsqrt_rn(inv9a);
      const float base = 1.0f - inv9a;
      const float lo = fmaxf(base - 1.96f * sq, 0.0f);
      const float up = base + 1.96f * sq;
      __stcs(a.lower + (out - a.mean), fmaxf(mg * lo * lo * lo, 0.0f));
      __stcs(a.upper + (out - a.mean), mg * up * up * up);
    }
    out += a.ldo;
  }
  if (end_rec) *end_rec = make_float2(m, c);
}

// One thread per pair over all sites.
template <bool CI>
__global__ void __launch_bounds__(128) fwd_only_kernel(const FwdArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  fwd_walk<CI>(a, p, 0, 0, a.n_sites, nullptr, nullptr);
}

// Speculative site chunks: thread (pair p, chunk k = blockIdx.y) writes sites
// [c0, c1) after a burn-in from (0, 0) at c0 - burn; records its state after
// c0 - 1 (speculative) and after c1 - 1 (to check the next chunk against).
// rec: [boundary][2][n_pairs], kind 0 = end of the left chunk, 1 = the right
// chunk's burn-in.
template <bool CI>
__global__ void __launch_bounds__(128) fwd_chunk_kernel(const FwdArgs a, FwdSpec sp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  const int k = blockIdx.y, K = sp.k_chunks;
  const int c0 = (int)((int64_t)a.n_sites * k / K), c1 = (int)((int64_t)a.n_sites * (k + 1) / K);
  const int s0 = k == 0 ? 0 : max(0, c0 - sp.burn_in);
  float2* spec = k > 0 ? sp.rec + ((int64_t)(k - 1) * 2 + 1) * a.n_pairs + p : nullptr;
  float2* end = k < K - 1 ? sp.rec + (int64_t)k * 2 * a.n_pairs + p : nullptr;
  fwd_walk<CI>(a, p, s0, c0, c1, spec, end);
}

// Pairs whose chunks did not all join the exact trajectory (bitwise) go on
// the repair list.
__global__ void fwd_verify_kernel(const FwdArgs a, FwdSpec sp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  for (int b = 0; b + 1 < sp.k_chunks; ++b) {
    const float2 e = sp.rec[(int64_t)b * 2 * a.n_pairs + p];
    const float2 q = sp.rec[((int64_t)b * 2 + 1) * a.n_pairs + p];
    if (__float_as_int(e.x) != __float_as_int(q.x) || __float_as_int(e.y) != __float_as_int(q.y)) {
      sp.repair_list[atomicAdd(sp.repair_count, 1)] = p;
      return;
    }
  }
}

// Listed pairs decoded again over all sites; counts them into the total.
template <bool CI>
__global__ void __launch_bounds__(128) fwd_repair_kernel(const FwdArgs a, FwdSpec sp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = *sp.repair_count;
  if (t == 0 && n > 0) atomicAdd(sp.repaired_total, n);
  if (t >= n) return;
  fwd_walk<CI>(a, sp.repair_list[t], 0, 0, a.n_sites, nullptr, nullptr);
}

// float32 patches -> half patches, round to nearest even (__float2half_rn).
__global__ void to_half_kernel(const float* __restrict__ src, __half* __restrict__ dst, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = __float2half_rn(src[i]);
}

}  // namespace

// Threads per CTA for one thread per pair: as many as keep every SM busy
// (warps spread over all SMs before SMs get more of them), 32..128.
int chain_cta_threads(int64_t n_pairs, int max_threads) {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t t = n_pairs / std::max(1, 2 * sms);
  t = (t + 31) / 32 * 32;
  return (int)std::max<int64_t>(32, std::min<int64_t>(t, max_threads));
}

cudaError_t launch_fwd_only(const FwdArgs& a, cudaStream_t stream) {
  if (a.n_pairs <= 0 || a.n_sites <= 0) return cudaSuccess;
  const int threads = chain_cta_threads(a.n_pairs, 128);
  const unsigned grid = (unsigned)((a.n_pairs + threads - 1) / threads);
  if (a.lower && a.upper)
    fwd_only_kernel<true><<<grid, threads, 0, stream>>>(a);
  else
    fwd_only_kernel<false><<<grid, threads, 0, stream>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fwd_spec(const FwdArgs& a, const FwdSpec& sp, cudaStream_t stream) {
  if (a.n_pairs <= 0 || a.n_sites <= 0) return cudaSuccess;
  if (sp.k_chunks <= 1) return launch_fwd_only(a, stream);
  const bool ci = a.lower && a.upper;
  const int threads = chain_cta_threads((int64_t)a.n_pairs * sp.k_chunks, 128);
  const dim3 grid((unsigned)((a.n_pairs + threads - 1) / threads), (unsigned)sp.k_chunks);
  cudaError_t e = cudaMemsetAsync(sp.repair_count, 0, sizeof(int), stream);
  if (e != cudaSuccess) return e;
  if (ci)
    fwd_chunk_kernel<true><<<grid, threads, 0, stream>>>(a, sp);
  else
    fwd_chunk_kernel<false><<<grid, threads, 0, stream>>>(a, sp);
  const unsigned pg = (unsigned)((a.n_pairs + 127) / 128);
  fwd_verify_kernel<<<pg, 128, 0, stream>>>(a, sp);
  if (ci)
    fwd_repair_kernel<true><<<pg, 128, 0, stream>>>(a, sp);
  else
    fwd_repair_kernel<false><<<pg, 128, 0, stream>>>(a, sp);
  return cudaGetLastError();
}

cudaError_t launch_to_half(const float* src, void* dst, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  to_half_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(src, static_cast<__half*>(dst), n);
  return cudaGetLastError();
}

}  // namespace gsmc
