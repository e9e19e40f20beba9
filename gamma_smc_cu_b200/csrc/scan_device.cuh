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

// Bilinear lookup of (m, c) in one patch layer, identical to the reference's
// clamp / truncate / keep-the-upper-cell interpolation.  Split in two so
// independent work can be scheduled between the loads and their use.
struct Fetch {
  float4 a, b;  // m corners and c corners of the patch
  float wm, wc;
  int idx;      // patch index within the layer
};

// Hint the patch a pair will most likely read at its next site (same cell,
// next site's layer, next site's hom/het half) into L1.  Compiled only with
// GSMC_PREFETCH_NEXT: on the chromosome job the extra instructions cost more
// than the hits gained (304 ms against 282 ms per job when measured), so the
// default build emits nothing here.
__device__ __forceinline__ void prefetch_patch(const float4* p) {
#ifdef GSMC_PREFETCH_NEXT
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
#else
  (void)p;
#endif
}

// floor(x) for 0 <= x < 2^23 in two full-rate adds: x + 2^23 lands in
// [2^23, 2^24), where floats are the integers, and rounding the sum down keeps
// 2^23 + floor(x) exactly.
__device__ __forceinline__ float floor_small(float x) {
  return __fsub_rn(__fadd_rd(x, 8388608.0f), 8388608.0f);
}

// Address of patch 0 of `layer` minus 0x4B000000 patches (unsigned, wraps):
// adding (0x4B000000 + index) patches gives the patch.
__device__ __forceinline__ uint64_t biased(const float4* layer) {
  return reinterpret_cast<uint64_t>(layer) - ((uint64_t)0x4B000000u << 5);
}

// Lookup of (m, c) in the hom (het = 0) or het (het = 1) half of the layer
// whose biased base is layer_bias.
__device__ __forceinline__ Fetch patch_fetch(uint64_t layer_bias, int het, float m, float c) {
  const float fm = __fmul_rn(__fsub_rn(m, kMLo), kMInv);
  const float fc = __fmul_rn(__fsub_rn(c, kCLo), kCInv);
  // Lower-left corner: the reference clamps x to [0, last], truncates (x >= 0,
  // so floor) and moves an index that lands on the last row/column down by
  // one.  floor(max(0, min(x, last - 0.5))) is all of it at once -- equal to
  // floor(min(clamp(x), last - 0.5)) for every x, NaN included -- and starts
  // from the unclamped x, so the index does not wait for the weight's clamp.
  // The floor is (y +rd 2^23) - 2^23 (floor_small); the biased sums are kept
  // for the patch index below.
  const float rb = __fadd_rd(fmaxf(0.0f, fminf(fm, (float)kPatchRows - 0.5f)), 8388608.0f);
  const float qb = __fadd_rd(fmaxf(0.0f, fminf(fc, (float)kPatchCols - 0.5f)), 8388608.0f);
  const float rf = __fsub_rn(rb, 8388608.0f);
  const float qf = __fsub_rn(qb, 8388608.0f);
  Fetch f;
  // Weight clamp(x, 0, last) - floor as one saturated subtract: for x < 0 the
  // floor is 0 and both give +0 (x is never -0: it is (v - lo) * step, and
  // v - lo rounds an exact zero to +0); inside [0, last] the clamp does
  // nothing and x - floor lies in [0, 1]; above last the reference's weight is
  // last - (last - 1) = 1 and x - (last - 1) > 1 saturates to 1.  The two
  // differ only for x = NaN (the reference's clamp gives last, .sat gives 0),
  // and x is never NaN: every table value is clamped to the grid when the
  // tables are built (NaN included), so the states -- 0 at the start of a
  // window, then bilinear blends of table values -- stay finite.
  f.wm = __saturatef(__fsub_rn(fm, rf));
  f.wc = __saturatef(__fsub_rn(fc, qf));
  // rf * 49 + qf is an exact integer below 2450, so rf * 49 + (qf + 2^23) is
  // exact too and sits in the low mantissa bits: the patch index needs no
  // conversion instruction.
  const uint32_t bits = (uint32_t)__float_as_int(__fmaf_rn(rf, (float)kPatchCols, qb));
  const int idx = (int)(bits - 0x4B000000u);
  // The het half of a layer starts kPatches patches after the hom half, so
  // the half is one more integer add on the biased index, and the address is
  // one wide multiply-add from the biased layer base.
  const uint32_t key = bits + (uint32_t)(het * kPatches);
  // One 256-bit read-only load of the 32-byte patch: m corners (r,q) (r,q+1)
  // (r+1,q) (r+1,q+1), then the c corners.  Patches are 32-byte aligned:
  // table bases come from cudaMalloc and every layer, hom/het half and patch
  // offset is a multiple of 32 bytes.
  f.idx = idx;
  const float4* p = reinterpret_cast<const float4*>(layer_bias + ((uint64_t)key << 5));
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(f.a.x), "=f"(f.a.y), "=f"(f.a.z), "=f"(f.a.w), "=f"(f.b.x), "=f"(f.b.y),
        "=f"(f.b.z), "=f"(f.b.w)
      : "l"(p));
  return f;
}

__device__ __forceinline__ void patch_interp(const Fetch& f, float& m, float& c) {
  const float vc = __fsub_rn(1.0f, f.wc), vm = __fsub_rn(1.0f, f.wm);
  m = __fmaf_rn(f.wm, __fmaf_rn(f.wc, f.a.w, __fmul_rn(vc, f.a.z)),
                __fmul_rn(vm, __fmaf_rn(f.wc, f.a.y, __fmul_rn(vc, f.a.x))));
  c = __fmaf_rn(f.wm, __fmaf_rn(f.wc, f.b.w, __fmul_rn(vc, f.b.z)),
                __fmul_rn(vm, __fmaf_rn(f.wc, f.b.y, __fmul_rn(vc, f.b.x))));
}

__device__ __forceinline__ void patch_lookup(const float4* __restrict__ layer, float& m,
                                             float& c) {
  const Fetch f = patch_fetch(biased(layer), 0, m, c);
  patch_interp(f, m, c);
}

// 10^x by the bit construction upstream gamma_smc uses (Schraudolph 1999,
// "A fast, compact approximation of the exponential function"): the float
// whose bits are trunc(C2 * (x * ln10) + C1) (src/kernels/gamma_smc_flow.cu:
// 112-121).
__device__ __forceinline__ float pow10_bits(float x) {
  const float kLn10 = 2.30258509299f;
  const float kC1 = 1064872507.1541044f;
  const float kC2 = 12102203.161561485f;
  return __int_as_float(__float2int_rz(__fmaf_rn(kC2, __fmul_rn(x, kLn10), kC1)));
}

__device__ __forceinline__ uint64_t word_at(const ulonglong2* g, int64_t nh, int s) {
  const ulonglong2 v = __ldg(g + (int64_t)(s >> 7) * nh);
  return (s & 64) ? v.y : v.x;
}

// Posterior at one core site: forward state f, backward state (m, c) ->
// alpha, beta and the mean in generations (src/kernels/gamma_smc_flow.cu:708-722).
__device__ __forceinline__ float posterior(float2 f, float m, float c, float unscale, float& a_s,
                                           float& b_s) {
  const float ab = -2.0f * c;
  const float ba = pow10_bits(ab), bb = pow10_bits(__fsub_rn(ab, m));
  const float af = -2.0f * f.y;
  const float fa = pow10_bits(af), fb = pow10_bits(__fsub_rn(af, f.x));
  a_s = __fsub_rn(__fadd_rn(fa, ba), 1.0f);
  b_s = __fsub_rn(__fadd_rn(fb, bb), 1.0f);
  return __fmul_rn(__fdiv_rn(a_s, fmaxf(b_s, 1e-10f)), unscale);
}

// Posterior combine at one core site, stored per pair
// (src/kernels/gamma_smc_flow.cu:708-734).
__device__ __forceinline__ void combine_store(const Task& t, int64_t o, float2 f, float m, float c,
                                              bool ci, bool post) {
  float a_s, b_s;
  const float mg = posterior(f, m, c, t.unscale, a_s, b_s);
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
  // Lanes past the last pair walk along on pair (0, 0) with nothing stored
  // (summary reductions need every lane of the warp).  In a CTA-wide task
  // every warp stays, even one with no pair: the task's warps meet at a
  // barrier at each 32-site block (below).  A warp-wide task's empty warp
  // leaves.
  if (WIDTH != kThreads && (j0 & ~31) >= t.pair_count) return;
  // CTA-wide tasks: the warps meet at the start of every 32-site block, so
  // they walk within one block of each other and read the same table layers;
  // the patches one warp brings into L1 are there when the others need them.
  // (Chromosome job 210 -> 183 ms, full-posterior slice 42 -> 32 ms; without
  // it the warps drift apart over a window and L1 hits stay near 51%.)
  auto meet = [] {
    if constexpr (WIDTH == kThreads) __syncthreads();
  };

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
  float m[NP], c[NP];
  uint32_t x[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    m[k] = 0.0f;
    c[k] = 0.0f;
    x[k] = (uint32_t)((word_at(gi[k], nh, ps) ^ word_at(gj[k], nh, ps)) >> (ps & 63));
  }
  float2* fp = slot + j0;
  // Gap codes run two sites ahead: `cur` is this site's, `nx` the next one's
  // (already in registers, so the next-site prefetch does not wait on it).
  // het bits: 32-bit halves of the pair's XORed genotype words (a 32-bit
  // shift per site); the loops below run in 32-site blocks and reload at each
  // block's first site (the first site of the task comes preloaded)
  auto reload = [&](int s) {
#pragma unroll
    for (int k = 0; k < NP; ++k)
      x[k] = (uint32_t)((word_at(gi[k], nh, s) ^ word_at(gj[k], nh, s)) >> (s & 32));
  };
  auto fwd_step = [&](int s, SiteCode sc, int next_layer) {
    if (sc.chunks) {
      for (int u = 0; u < sc.chunks; ++u) {
#pragma unroll
        for (int k = 0; k < NP; ++k) patch_lookup(chunk, m[k], c[k]);
      }
    }
    const float4* layer = fwd_tab + sc.layer;
    const uint64_t lb = biased(layer);
    Fetch f[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int het = (int)(x[k] & 1u);
      x[k] >>= 1;
      f[k] = patch_fetch(lb, het, m[k], c[k]);
      prefetch_patch(fwd_tab + next_layer + (int)(x[k] & 1u) * kHetF4 + kPatchF4 * f[k].idx);
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) patch_interp(f[k], m[k], c[k]);
  };
  int s = ps;
  // a window that does not start at site 0 enters its first site by 1 bp
  SiteCode cur = ps > 0 ? SiteCode{0, 0} : code[s];
  SiteCode nx = code[s + 1];
  {
    const SiteCode nx2 = code[s + 2];
    fwd_step(s, cur, nx.layer);
    cur = nx;
    nx = nx2;
  }
  if (s >= cs) {
#pragma unroll
    for (int k = 0; k < NP; ++k) __stcs(fp + k * WIDTH, make_float2(m[k], c[k]));
    fp += kRow;
  }
  for (++s; s < cs;) {
    meet();
    if ((s & 31) == 0) reload(s);
    for (const int e = min(cs, (s | 31) + 1); s < e; ++s) {
      const SiteCode nx2 = code[s + 2];
      fwd_step(s, cur, nx.layer);
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
      if (j < t.pair_count) b[kind * t.bstride + j] = make_float2(m[k], c[k]);
    }
  };
  if (t.bl) record(t.bl, 1);
  while (s < ce) {
    meet();
    if ((s & 31) == 0 && s != ps) reload(s);
    for (const int e = min(ce, (s | 31) + 1); s < e; ++s) {
      const SiteCode nx2 = code[s + 2];
      fwd_step(s, cur, nx.layer);
      cur = nx;
      nx = nx2;
#pragma unroll
      for (int k = 0; k < NP; ++k) __stcs(fp + k * WIDTH, make_float2(m[k], c[k]));
      fp += kRow;
    }
  }
  if (t.br) record(t.br, 0);

  // ---- backward: [pe-1 .. cs]; posterior at core sites ----
#pragma unroll
  for (int k = 0; k < NP; ++k) {
    m[k] = 0.0f;
    c[k] = 0.0f;
    x[k] = (uint32_t)((word_at(gi[k], nh, pe - 1) ^ word_at(gj[k], nh, pe - 1)) >> ((pe - 1) & 32))
           << (31 - ((pe - 1) & 31));
  }
  // Backward step at site s: the het/hom site table first, then any full
  // 1000-bp chunks.
  auto bwd_fetch = [&](int s, SiteCode sc, int next_layer, Fetch* f) {
    const uint64_t lb = biased(bwd_tab + sc.layer);
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const int het = (int)(x[k] >> 31);
      x[k] <<= 1;
      f[k] = patch_fetch(lb, het, m[k], c[k]);
      prefetch_patch(bwd_tab + next_layer + (int)(x[k] >> 31) * kHetF4 + kPatchF4 * f[k].idx);
    }
  };
  auto bwd_finish = [&](SiteCode sc, const Fetch* f) {
#pragma unroll
    for (int k = 0; k < NP; ++k) patch_interp(f[k], m[k], c[k]);
    if (sc.chunks) {
      for (int u = 0; u < sc.chunks; ++u) {
#pragma unroll
        for (int k = 0; k < NP; ++k) patch_lookup(chunk, m[k], c[k]);
      }
    }
  };
  s = pe - 1;
  cur = code[s];
  nx = code[s - 1];
  while (s >= ce) {
    meet();
    if ((s & 31) == 31 && s != pe - 1) reload(s);
    for (const int e = max(ce, s & ~31); s >= e; --s) {
      const SiteCode nx2 = code[s - 2];
      Fetch f[NP];
      bwd_fetch(s, cur, nx.layer, f);
      bwd_finish(cur, f);
      cur = nx;
      nx = nx2;
    }
  }
  if (t.br) record(t.br, 3);
  // forward-state ring: q[i] holds the state of site s - i
  const float2* fq = slot + (int64_t)(ce - 1 - cs) * kRow + j0;
  float2 q[kFwdPrefetch][NP];
#pragma unroll
  for (int i = 0; i < kFwdPrefetch; ++i) {
#pragma unroll
    for (int k = 0; k < NP; ++k)
      q[i][k] = (ce - 1 - i >= cs) ? __ldlu(fq + k * WIDTH) : make_float2(0.0f, 0.0f);
    fq -= kRow;
  }
  int64_t o = t.out_off + (int64_t)(ce - 1 - t.out_row0) * t.ldo + j0;
  s = ce - 1;
  while (s >= cs) {
  meet();
  if ((s & 31) == 31 && s != pe - 1) reload(s);
  // unrolled by the ring depth so the ring rotation is register renaming
#pragma unroll kFwdPrefetch
  for (const int e = max(cs, s & ~31); s >= e; --s) {
    float2 f[NP];
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
      q[kFwdPrefetch - 1][k] = ahead ? __ldlu(fq + k * WIDTH) : make_float2(0.0f, 0.0f);
    fq -= kRow;
    const SiteCode sc = cur;
    const SiteCode nx2 = code[s - 2];
    float mb[NP], cb[NP];
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      mb[k] = m[k];
      cb[k] = c[k];
    }
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
        const float mg = posterior(f[k], mb[k], cb[k], t.unscale, a_s, b_s);
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
        if (live[k]) combine_store(t, o + k * WIDTH, f[k], mb[k], cb[k], ci, post);
    }
    o -= t.ldo;
    if (more) {
      Fetch fe[NP];
      bwd_fetch(s, sc, nx.layer, fe);
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
    bwd_fetch(cs, scs, 0, fe);
    bwd_finish(scs, fe);
    record(t.bl, 2);
  }
}

}  // namespace
}  // namespace gsmc
