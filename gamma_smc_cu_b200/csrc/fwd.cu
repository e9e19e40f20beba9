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

// One thread per pair over all sites.
template <bool CI>
__global__ void __launch_bounds__(128) fwd_only_kernel(const FwdArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n_pairs) return;
  const int hi = a.pi[p], hj = a.pj[p];
  if (hi < 0 || hi >= a.n_haps || hj < 0 || hj >= a.n_haps) return;  // outputs untouched
  const ulonglong2* gi = a.geno + hi;
  const ulonglong2* gj = a.geno + hj;
  const uint4* chunk = a.tab + (size_t)(a.L - 1) * kPatches;
  float m = 0.0f, c = 0.0f;
  uint64_t x = 0;
  float* out = a.mean + p;
  FwdCode nx = a.code[0];
  for (int s = 0; s < a.n_sites; ++s) {
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

cudaError_t launch_to_half(const float* src, void* dst, size_t n, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  to_half_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(src, static_cast<__half*>(dst), n);
  return cudaGetLastError();
}

}  // namespace gsmc
