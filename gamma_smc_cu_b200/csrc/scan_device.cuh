// Device-side pieces of the Gamma-SMC scan shared by the scan kernels:
// table-patch lookup, the 10^x bit construction, the posterior combine and
// the per-task forward/backward walk (see scan.cu for the kernels).
#pragma once

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

// floor(x) for 0 <= x < 2^23 in two full-rate adds: x + 2^23 lands in
// [2^23, 2^24), where floats are the integers, and rounding the sum down keeps
// 2^23 + floor(x) exactly.
__device__ __forceinline__ float floor_small(float x) {
  return __fsub_rn(__fadd_rd(x, 8388608.0f), 8388608.0f);
}

// Two float32 lanes in one 64-bit register pair, the operands of sm_100's
// packed FP32 instructions (add/sub/mul/fma.rn.f32x2).  Each lane is rounded
// exactly as the scalar instruction rounds it, so the packed arithmetic below
// is bit-identical to the scalar expressions it stands for, at one issued
// instruction where the scalar form needs two.  The scan state is such a
// pair: lo = log10 mean m, hi = log10 CV c.
struct f2 {
  unsigned long long v;
};

__device__ __forceinline__ f2 pack2(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float lo_of(f2 a) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
  return lo;
}
__device__ __forceinline__ float hi_of(f2 a) {
  float lo, hi;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
  return hi;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
// rounded toward -infinity (the packed floor_small)
__device__ __forceinline__ f2 add2_rd(f2 a, f2 b) {
  f2 r;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}
__device__ __forceinline__ f2 as_f2(float2 v) { return pack2(v.x, v.y); }
__device__ __forceinline__ float2 as_float2(f2 v) { return make_float2(lo_of(v), hi_of(v)); }

// Bilinear lookup of a state (m, c) in one patch layer, identical to the
// reference's clamp / truncate / keep-the-upper-cell interpolation
// (src/kernels/gamma_smc_flow.cu:408-431).  Split in two so independent work
// can be scheduled between the load and its use.
struct Fetch {
  f2 p00, p01, p10, p11;  // (m, c) at corners (r,q) (r,q+1) (r+1,q) (r+1,q+1)
  f2 w;                   // {wm, wc}: weights of the upper row / column
};

// 49 * bits(2^23 + r) + bits(2^23 + q) = 49 r + q + kIdxBias (mod 2^32); see
// patch_fetch.
constexpr unsigned kIdxBias = 50u * 0x4B000000u;

__device__ __forceinline__ Fetch patch_fetch(const float4* __restrict__ layer, f2 s) {
  const f2 f = mul2(sub2(s, pack2(kMLo, kCLo)), pack2(kMInv, kCInv));
  const float fm = fmaxf(0.0f, fminf(lo_of(f), (float)(kRows - 1)));
  const float fc = fmaxf(0.0f, fminf(hi_of(f), (float)(kCols - 1)));
  // Lower-left corner: the reference truncates (fm >= 0, so floor) and moves
  // an index that lands on the last row/column down by one.  floor(min(x,
  // last - 0.5)) is both at once, and the weight stays x - corner.
  const f2 k23 = pack2(8388608.0f, 8388608.0f);
  const f2 big = add2_rd(pack2(fminf(fm, (float)kPatchRows - 0.5f),
                               fminf(fc, (float)kPatchCols - 0.5f)), k23);
  Fetch r;
  r.w = sub2(pack2(fm, fc), sub2(big, k23));
  // The bits of 2^23 + k are 0x4B000000 + k, so 49 * bits(2^23 + rf) +
  // bits(2^23 + qf) is the patch index rf * 49 + qf (< 2450) plus
  // 50 * 0x4B000000 mod 2^32 = 0xA6000000, with no further wrap: the index in
  // one integer multiply-add, its bias folded into the layer address.
  const unsigned t =
      __float_as_uint(lo_of(big)) * (unsigned)kPatchCols + __float_as_uint(hi_of(big));
  const unsigned long long addr = reinterpret_cast<unsigned long long>(layer) -
                                  (unsigned long long)kIdxBias * 32ull +
                                  (unsigned long long)t * 32ull;
  // One 256-bit read-only load of the 32-byte patch into four (m, c) pairs.
  // Patches are 32-byte aligned: table bases come from cudaMalloc and every
  // layer, hom/het half and patch offset is a multiple of 32 bytes.
  asm("ld.global.nc.v4.b64 {%0, %1, %2, %3}, [%4];"
      : "=l"(r.p00.v), "=l"(r.p01.v), "=l"(r.p10.v), "=l"(r.p11.v)
      : "l"(addr));
  return r;
}

// m = fma(wm, fma(wc, m11, vc * m10), vm * fma(wc, m01, vc * m00)), and the
// same for c, with vm = 1 - wm, vc = 1 - wc: both lanes at once.
__device__ __forceinline__ f2 patch_interp(const Fetch& f) {
  const f2 v = sub2(pack2(1.0f, 1.0f), f.w);
  const float wm = lo_of(f.w), wc = hi_of(f.w), vm = lo_of(v), vc = hi_of(v);
  const f2 wc2 = pack2(wc, wc), vc2 = pack2(vc, vc);
  const f2 hi_row = fma2(wc2, f.p11, mul2(vc2, f.p10));
  const f2 lo_row = fma2(wc2, f.p01, mul2(vc2, f.p00));
  return fma2(pack2(wm, wm), hi_row, mul2(pack2(vm, vm), lo_row));
}

__device__ __forceinline__ f2 patch_lookup(const float4* __restrict__ layer, f2 s) {
  return patch_interp(patch_fetch(layer, s));
}

// 10^x by the bit construction upstream gamma_smc uses (Schraudolph 1999,
// "A fast, compact approximation of the exponential function"): the float
// whose bits are trunc(C2 * (x * ln10) + C1) (src/kernels/gamma_smc_flow.cu:
// 112-121).
constexpr float kLn10 = 2.30258509299f;
constexpr float kPowC1 = 1064872507.1541044f;
constexpr float kPowC2 = 12102203.161561485f;

__device__ __forceinline__ float pow10_bits(float x) {
  return __int_as_float(__float2int_rz(__fmaf_rn(kPowC2, __fmul_rn(x, kLn10), kPowC1)));
}

// Two arguments at once: the multiply and the multiply-add packed, the
// truncations one by one.
__device__ __forceinline__ f2 pow10_bits2(f2 x) {
  const f2 y = fma2(pack2(kPowC2, kPowC2), mul2(x, pack2(kLn10, kLn10)), pack2(kPowC1, kPowC1));
  return pack2(__int_as_float(__float2int_rz(lo_of(y))), __int_as_float(__float2int_rz(hi_of(y))));
}

// {10^(-2c), 10^(-2c - m)}: a state's Gamma shape and rate terms
// (mc_to_ab, src/kernels/gamma_smc_flow.cu:123-131).
__device__ __forceinline__ f2 mc_to_ab(f2 s) {
  const float a = -2.0f * hi_of(s);
  return pow10_bits2(pack2(a, __fsub_rn(a, lo_of(s))));
}

__device__ __forceinline__ uint64_t word_at(const ulonglong2* g, int64_t nh, int s) {
  const ulonglong2 v = __ldg(g + (int64_t)(s >> 7) * nh);
  return (s & 64) ? v.y : v.x;
}

// Posterior at one core site from the forward state f and the backward state
// b (src/kernels/gamma_smc_flow.cu:708-722): alpha = af + ab - 1,
// beta = bf + bb - 1, mean = alpha / max(beta, 1e-10) * 2 Ne.
__device__ __forceinline__ float posterior(f2 f, f2 b, float unscale, float& a_s, float& b_s) {
  const f2 ab = sub2(add2(mc_to_ab(f), mc_to_ab(b)), pack2(1.0f, 1.0f));
  a_s = lo_of(ab);
  b_s = hi_of(ab);
  return __fmul_rn(__fdiv_rn(a_s, fmaxf(b_s, 1e-10f)), unscale);
}

// Posterior combine at one core site, stored per pair
// (src/kernels/gamma_smc_flow.cu:708-734).
__device__ __forceinline__ void combine_store(const Task& t, int64_t o, f2 f, f2 b, bool ci,
                                              bool post) {
  float a_s, b_s;
  const float mg = posterior(f, b, t.unscale, a_s, b_s);
  __stcs(t.out[0] + o, mg);
  if (ci) {
    // Wilson-Hilferty 95% bounds (src/kernels/gamma_smc_flow.cu:724-733).
    const float inv9a = __frcp_rn(__fmul_rn(9.0f, fmaxf(a_s, 1.0f)));
    const float sq = __fsqrt_rn(inv9a);
    const float base = __fsub_rn(1.0f, inv9a);
    const float lo = fmaxf(__fmaf_rn(-1.96f, sq, base), 0.0f);
    const float up = __fmaf_rn(1.96f, sq, base);
    __stcs(t.out[1] + o, fmaxf(__fmul_rn(__fmul_rn(__fmul_rn(mg, lo), lo), lo), 0.0f));
    __stcs(t.out[2] + o, __fmul_rn(__fmul_rn(__fmul_rn(mg, up), up), up));
  }
  if (post) {
    __stcs(t.out[3] + o, a_s);
    __stcs(t.out[4] + o, b_s);
  }
}

// The same from scalar states (the uncached kernels).
__device__ __forceinline__ void combine_store(const Task& t, int64_t o, float2 f, float m, float c,
                                              bool ci, bool post) {
  combine_store(t, o, as_f2(f), pack2(m, c), ci, post);
}

// Forward states are read back this many sites ahead of their use so the
// DRAM latency of that stream is hidden behind the scan's own lookups (one
// site of lookups, combine and the other warps' work covers it; each deeper
// slot costs registers, and registers cost resident CTAs).  They and the
// outputs are single-use streams: stored with evict-first (.cs) and read with
// last-use (.lu) hints so they do not displace table patches.
constexpr int kFwdPrefetch = 1;
constexpr int kThreads = 128;

// One task: this thread's NP pairs over the task's padded window.  WIDTH
// threads (a warp or the whole CTA) share the task; the forward states live in
// the tile's slot, rows of WIDTH * NP pairs.
// SUMMARY selects the per-warp reductions of kTaskSummary tasks (a separate
// instantiation, so the per-pair kernels carry none of its registers).
template <int NP, int WIDTH, bool SUMMARY = false>
__device__ __forceinline__ void scan_task(const ScanArgs& a, const Task& t, float2* slot) {
  static_assert(WIDTH == 32 || WIDTH == kThreads, "a task is run by one warp or one CTA");
  constexpr int kRow = WIDTH * NP;
  const int64_t nh = a.n_haps;
  const int ps = t.ps, cs = t.cs, ce = t.ce, pe = t.pe;
  const bool ci = (t.flags & kTaskCI) != 0, post = (t.flags & kTaskPosterior) != 0;
  constexpr bool summary = SUMMARY;
  const int j0 = threadIdx.x & (WIDTH - 1);
  // Warps with no pair leave; lanes past the last pair of a partly filled warp
  // walk along on pair (0, 0) with nothing stored (summary reductions need
  // every lane of the warp).
  if ((j0 & ~31) >= t.pair_count) return;

  const ulonglong2* gi[NP];
  const ulonglong2* gj[NP];
  bool live[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    const int j = j0 + k * WIDTH;
    int hi = 0, hj = 0;
    live[k] = j < t.pair_count;
    if (live[k]) {
      hi = t.pi[j];
      hj = t.pj[j];
      // Device-side pair indices are not validated by the host: a bad pair is
      // skipped (outputs untouched) instead of reading out of bounds.
      if (hi < 0 || hi >= nh || hj < 0 || hj >= nh) {
        live[k] = false;
        hi = hj = 0;
      }
    }
    gi[k] = a.geno + hi;
    gj[k] = a.geno + hj;
  }
  // code[-2..-1] and code[n_sites..n_sites+1] exist (zero padding), so the
  // two-sites-ahead code prefetches below never leave the array.
  const SiteCode* __restrict__ code = a.code;
  const float4* __restrict__ fwd_tab = a.site_tab;
  const float4* __restrict__ bwd_tab = a.site_tab + (size_t)a.L * kLayerF4;
  const float4* __restrict__ chunk = a.chunk_tab;

  // ---- forward: [ps, ce); states stored for [cs, ce) ----
  f2 st[NP];
  uint32_t x[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    st[k] = pack2(0.0f, 0.0f);
    x[k] = (uint32_t)((word_at(gi[k], nh, ps) ^ word_at(gj[k], nh, ps)) >> (ps & 63));
  }
  float2* fp = slot + j0;
  // Gap codes run two sites ahead: `cur` is this site's, `nx` the next one's.
  // het bits: 32-bit halves of the pair's XORed genotype words (a 32-bit
  // shift per site); the loops below run in 32-site blocks and reload at each
  // block's first site (the first site of the task comes preloaded)
  auto reload = [&](int s) {
#pragma unroll
    for (int k = 0; k < NP; ++k)
      x[k] = (uint32_t)((word_at(gi[k], nh, s) ^ word_at(gj[k], nh, s)) >> (s & 32));
  };
  auto fwd_step = [&](SiteCode sc) {
    if (sc.chunks) {
      for (int u = 0; u < sc.chunks; ++u) {
#pragma unroll
        for (int k = 0; k < NP; ++k) st[k] = patch_lookup(chunk, st[k]);
      }
    }
    const float4* layer = fwd_tab + sc.layer;
    Fetch f[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int het = (int)(x[k] & 1u);
      x[k] >>= 1;
      f[k] = patch_fetch(layer + het * kHetF4, st[k]);
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) st[k] = patch_interp(f[k]);
  };
  int s = ps;
  // a window that does not start at site 0 enters its first site by 1 bp
  SiteCode cur = ps > 0 ? SiteCode{0, 0} : code[s];
  SiteCode nx = code[s + 1];
  {
    const SiteCode nx2 = code[s + 2];
    fwd_step(cur);
    cur = nx;
    nx = nx2;
  }
  if (s >= cs) {
#pragma unroll
    for (int k = 0; k < NP; ++k) __stcs(fp + k * WIDTH, as_float2(st[k]));
    fp += kRow;
  }
  for (++s; s < cs;) {
    if ((s & 31) == 0) reload(s);
    for (const int e = min(cs, (s | 31) + 1); s < e; ++s) {
      const SiteCode nx2 = code[s + 2];
      fwd_step(cur);
      cur = nx;
      nx = nx2;
    }
  }
  // boundary records of a speculative chunk (see Task); lanes past the task's
  // last pair write nothing
  auto record = [&](float2* b, int kind) {
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int j = j0 + k * WIDTH;
      if (j < t.pair_count) b[kind * t.bstride + j] = as_float2(st[k]);
    }
  };
  if (t.bl) record(t.bl, 1);
  while (s < ce) {
    if ((s & 31) == 0 && s != ps) reload(s);
    for (const int e = min(ce, (s | 31) + 1); s < e; ++s) {
      const SiteCode nx2 = code[s + 2];
      fwd_step(cur);
      cur = nx;
      nx = nx2;
#pragma unroll
      for (int k = 0; k < NP; ++k) __stcs(fp + k * WIDTH, as_float2(st[k]));
      fp += kRow;
    }
  }
  if (t.br) record(t.br, 0);

  // ---- backward: [pe-1 .. cs]; posterior at core sites ----
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    st[k] = pack2(0.0f, 0.0f);
    x[k] = (uint32_t)((word_at(gi[k], nh, pe - 1) ^ word_at(gj[k], nh, pe - 1)) >> ((pe - 1) & 32))
           << (31 - ((pe - 1) & 31));
  }
  // Backward step at site s: the het/hom site table first, then any full
  // 1000-bp chunks.
  auto bwd_fetch = [&](SiteCode sc, Fetch* f) {
    const float4* layer = bwd_tab + sc.layer;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int het = (int)(x[k] >> 31);
      x[k] <<= 1;
      f[k] = patch_fetch(layer + het * kHetF4, st[k]);
    }
  };
  auto bwd_finish = [&](SiteCode sc, const Fetch* f) {
#pragma unroll
    for (int k = 0; k < NP; ++k) st[k] = patch_interp(f[k]);
    if (sc.chunks) {
      for (int u = 0; u < sc.chunks; ++u) {
#pragma unroll
        for (int k = 0; k < NP; ++k) st[k] = patch_lookup(chunk, st[k]);
      }
    }
  };
  s = pe - 1;
  cur = code[s];
  nx = code[s - 1];
  while (s >= ce) {
    if ((s & 31) == 31 && s != pe - 1) reload(s);
    for (const int e = max(ce, s & ~31); s >= e; --s) {
      const SiteCode nx2 = code[s - 2];
      Fetch f[NP];
      bwd_fetch(cur, f);
      bwd_finish(cur, f);
      cur = nx;
      nx = nx2;
    }
  }
  if (t.br) record(t.br, 3);
  // forward-state ring: q[i] holds the state of site s - i
  const float2* fq = slot + (int64_t)(ce - 1 - cs) * kRow + j0;
  f2 q[kFwdPrefetch][NP];
#pragma unroll
  for (int i = 0; i < kFwdPrefetch; ++i) {
#pragma unroll
    for (int k = 0; k < NP; ++k)
      q[i][k] = (ce - 1 - i >= cs) ? as_f2(__ldlu(fq + k * WIDTH)) : pack2(0.0f, 0.0f);
    fq -= kRow;
  }
  int64_t o = t.out_off + (int64_t)(ce - 1 - t.out_row0) * t.ldo + j0;
  s = ce - 1;
  while (s >= cs) {
  if ((s & 31) == 31 && s != pe - 1) reload(s);
  // unrolled by the ring depth so the ring rotation is register renaming
#pragma unroll kFwdPrefetch
  for (const int e = max(cs, s & ~31); s >= e; --s) {
    f2 f[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) f[k] = q[0][k];
#pragma unroll
    for (int i = 0; i + 1 < kFwdPrefetch; ++i) {
#pragma unroll
      for (int k = 0; k < NP; ++k) q[i][k] = q[i + 1][k];
    }
    const bool ahead = s - kFwdPrefetch >= cs;
#pragma unroll
    for (int k = 0; k < NP; ++k)
      q[kFwdPrefetch - 1][k] = ahead ? as_f2(__ldlu(fq + k * WIDTH)) : pack2(0.0f, 0.0f);
    fq -= kRow;
    const SiteCode sc = cur;
    const SiteCode nx2 = code[s - 2];
    const bool more = s > cs;
    // The combine runs before the next lookup is issued: holding the patch
    // registers across it costs more occupancy than the overlap gains.
    if constexpr (summary) {
      // sum / min / max of the posterior means over the warp's live pairs,
      // in a fixed shuffle order; lane 0 stores the warp's partials
      float vs = 0.0f, vmin = __int_as_float(0x7f800000), vmax = -__int_as_float(0x7f800000);
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        float a_s, b_s;
        const float mg = posterior(f[k], st[k], t.unscale, a_s, b_s);
        if (live[k]) {
          vs = __fadd_rn(vs, mg);
          vmin = fminf(vmin, mg);
          vmax = fmaxf(vmax, mg);
        }
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        vs = __fadd_rn(vs, __shfl_xor_sync(0xffffffffu, vs, d));
        vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, d));
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, d));
      }
      if ((threadIdx.x & 31) == 0) {
        const int64_t po = t.out_off + (int64_t)(s - t.out_row0) * t.ldo + (j0 >> 5);
        t.out[0][po] = vs;
        t.out[1][po] = vmin;
        t.out[2][po] = vmax;
      }
    } else {
#pragma unroll
      for (int k = 0; k < NP; ++k)
        if (live[k]) combine_store(t, o + k * WIDTH, f[k], st[k], ci, post);
    }
    o -= t.ldo;
    if (more) {
      Fetch fe[NP];
      bwd_fetch(sc, fe);
      bwd_finish(sc, fe);
    }
    cur = nx;
    nx = nx2;
  }
  }
  if (t.bl) {
    // the backward state after applying site cs itself, for the left neighbour
    Fetch fe[NP];
    const SiteCode scs = code[cs];
    bwd_fetch(scs, fe);
    bwd_finish(scs, fe);
    record(t.bl, 2);
  }
}

}  // namespace
}  // namespace gsmc
