// Fused Gamma-SMC forward/backward scan for sm_100a.
//
// One thread owns one (pair, window) and walks the window's sites: forward
// from the padded start to the core end, storing its (m, c) state at core
// sites, then backward from the padded end to the core start, combining with
// the stored forward state and writing the posterior at core sites.  Sites are
// shared by every pair, so the table layer chosen by the gap is the same for
// all threads of the launch at a given site; only hom/het differs per pair.
//
// Table lookups read one 32-byte patch (four corners of m and of c) per step,
// as two 16-byte read-only loads from a single sector; the patch tables stay
// in L2 and the touched patches of the current layer in L1.  The arithmetic is
// the reference's cached FB (src/kernels/gamma_smc_flow.cu:112-131, 160-163,
// 408-514, 567-609, 632-669, 678-754, 762-839) with every fused multiply-add
// written explicitly, so results are bit-identical to it.
#include <cuda_runtime.h>
#include <stdint.h>

#include "scan.h"
#include "tables.h"

namespace gsmc {
namespace {

// Grid bounds and steps as the scan kernels hard-code them
// (src/kernels/gamma_smc_flow.cu:10-17).
constexpr float kMLo = -5.0f;
constexpr float kMHi = 2.0f;
constexpr float kCLo = -2.0f;
constexpr float kCHi = 0.0f;
constexpr float kMStep = (kMHi - kMLo) / (kRows - 1);
constexpr float kCStep = (kCHi - kCLo) / (kCols - 1);
constexpr float kMInv = 1.0f / kMStep;
constexpr float kCInv = 1.0f / kCStep;

// Bilinear lookup of (m, c) in one patch layer.
__device__ __forceinline__ void patch_lookup(const float4* __restrict__ layer, float& m,
                                             float& c) {
  float fm = (m - kMLo) * kMInv;
  float fc = (c - kCLo) * kCInv;
  fm = fmaxf(0.0f, fminf(fm, (float)(kRows - 1)));
  fc = fmaxf(0.0f, fminf(fc, (float)(kCols - 1)));
  const int r = min((int)fm, kPatchRows - 1);
  const int q = min((int)fc, kPatchCols - 1);
  const float wm = fm - (float)r;
  const float wc = fc - (float)q;
  const float4* p = layer + 2 * (r * kPatchCols + q);
  const float4 a = __ldg(p);      // m corners: (r,q) (r,q+1) (r+1,q) (r+1,q+1)
  const float4 b = __ldg(p + 1);  // c corners
  const float vc = 1.0f - wc, vm = 1.0f - wm;
  m = __fmaf_rn(wm, __fmaf_rn(wc, a.w, vc * a.z), vm * __fmaf_rn(wc, a.y, vc * a.x));
  c = __fmaf_rn(wm, __fmaf_rn(wc, b.w, vc * b.z), vm * __fmaf_rn(wc, b.y, vc * b.x));
}

// 10^x by the bit construction upstream gamma_smc uses (Schraudolph 1999,
// "A fast, compact approximation of the exponential function"): the float
// with bits trunc(C2 * x * ln10 + C1) (src/kernels/gamma_smc_flow.cu:112-121).
__device__ __forceinline__ float pow10_bits(float x) {
  const float kLn10 = 2.30258509299f;
  const float kC1 = 1064872507.1541044f;
  const float kC2 = 12102203.161561485f;
  return __int_as_float(__float2int_rz(__fmaf_rn(kC2, x * kLn10, kC1)));
}

__device__ __forceinline__ bool het_bit(uint64_t lo, uint64_t hi, int64_t s) {
  const uint64_t w = (s & 64) ? hi : lo;
  return ((w >> (s & 63)) & 1ull) != 0;
}

template <bool CI, bool POST>
__global__ void __launch_bounds__(kScanThreads) fb_scan_kernel(const ScanArgs a) {
  const int64_t p = (int64_t)blockIdx.x * kScanThreads + threadIdx.x;
  if (p >= a.n_pairs) return;
  const Window w = a.win[blockIdx.y];
  const int64_t nh = a.n_haps;
  const int32_t hi = a.pi[p], hj = a.pj[p];
  // Device-side pair indices are not validated by the host: skip bad ones
  // (their outputs are left untouched) instead of reading out of bounds.
  if (hi < 0 || hi >= nh || hj < 0 || hj >= nh) return;
  const ulonglong2* gi = a.geno + hi;
  const ulonglong2* gj = a.geno + hj;
  const size_t layer_sz = (size_t)kPatches * 2;
  const size_t table_sz = layer_sz * a.L;
  const float4* fwd_hom = a.site_tab + kScanFwdHom * table_sz;
  const float4* fwd_het = a.site_tab + kScanFwdHet * table_sz;
  const float4* bwd_hom = a.site_tab + kScanBwdHom * table_sz;
  const float4* bwd_het = a.site_tab + kScanBwdHet * table_sz;
  float2* fwd = a.fwd + w.fwd_off + p;

  // Forward sweep: state starts at (0, 0); a window that does not start at
  // site 0 enters its first site with a 1-bp step.
  float m = 0.0f, c = 0.0f;
  int64_t group = -1;
  uint64_t x0 = 0, x1 = 0;
  for (int64_t s = w.ps; s < w.ce; ++s) {
    if ((s >> 7) != group) {
      group = s >> 7;
      const ulonglong2 u = __ldg(gi + group * nh);
      const ulonglong2 v = __ldg(gj + group * nh);
      x0 = u.x ^ v.x;
      x1 = u.y ^ v.y;
    }
    SiteCode sc = a.code[s];
    if (s == w.ps && w.ps > 0) sc = SiteCode{0, 0};
    for (int k = 0; k < sc.chunks; ++k) patch_lookup(a.chunk_tab, m, c);
    patch_lookup((het_bit(x0, x1, s) ? fwd_het : fwd_hom) + (size_t)sc.layer * layer_sz, m, c);
    if (s >= w.cs) fwd[(s - w.cs) * a.n_pairs] = make_float2(m, c);
  }

  // Backward sweep with the posterior combine at core sites.
  const float unscale = a.unscale;
  m = 0.0f;
  c = 0.0f;
  group = -1;
  for (int64_t s = w.pe - 1; s >= w.cs; --s) {
    if (s < w.ce) {
      const float2 f = fwd[(s - w.cs) * a.n_pairs];
      const float ab = -2.0f * c;
      const float ba = pow10_bits(ab), bb = pow10_bits(ab - m);
      const float af = -2.0f * f.y;
      const float fa = pow10_bits(af), fb = pow10_bits(af - f.x);
      const float a_s = fa + ba - 1.0f;
      const float b_s = fb + bb - 1.0f;
      const float mg = __fdiv_rn(a_s, fmaxf(b_s, 1e-10f)) * unscale;
      const int64_t o = w.out_off + (s - w.out_row0) * a.ldo + a.col0 + p;
      a.mean[o] = mg;
      if constexpr (CI) {
        // Wilson-Hilferty 95% bounds (src/kernels/gamma_smc_flow.cu:724-733).
        const float inv9a = __frcp_rn(9.0f * fmaxf(a_s, 1.0f));
        const float sq = __fsqrt_rn(inv9a);
        const float base = 1.0f - inv9a;
        const float lo = fmaxf(__fmaf_rn(-1.96f, sq, base), 0.0f);
        const float up = __fmaf_rn(1.96f, sq, base);
        a.lower[o] = fmaxf(mg * lo * lo * lo, 0.0f);
        a.upper[o] = mg * up * up * up;
      }
      if constexpr (POST) {
        a.alpha[o] = a_s;
        a.beta[o] = b_s;
      }
    }
    if (s == w.cs) break;
    if ((s >> 7) != group) {
      group = s >> 7;
      const ulonglong2 u = __ldg(gi + group * nh);
      const ulonglong2 v = __ldg(gj + group * nh);
      x0 = u.x ^ v.x;
      x1 = u.y ^ v.y;
    }
    const SiteCode sc = a.code[s];
    patch_lookup((het_bit(x0, x1, s) ? bwd_het : bwd_hom) + (size_t)sc.layer * layer_sz, m, c);
    for (int k = 0; k < sc.chunks; ++k) patch_lookup(a.chunk_tab, m, c);
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

cudaError_t launch_scan(const ScanArgs& args, bool ci, bool posterior, cudaStream_t stream) {
  if (args.n_pairs <= 0 || args.n_windows <= 0) return cudaSuccess;
  const dim3 grid((unsigned)((args.n_pairs + kScanThreads - 1) / kScanThreads),
                  (unsigned)args.n_windows);
  if (ci) {
    if (posterior) fb_scan_kernel<true, true><<<grid, kScanThreads, 0, stream>>>(args);
    else fb_scan_kernel<true, false><<<grid, kScanThreads, 0, stream>>>(args);
  } else {
    if (posterior) fb_scan_kernel<false, true><<<grid, kScanThreads, 0, stream>>>(args);
    else fb_scan_kernel<false, false><<<grid, kScanThreads, 0, stream>>>(args);
  }
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
