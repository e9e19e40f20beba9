// CPU oracle for the Gamma-SMC cached forward/backward scan.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// path in gamma_smc_cu_b200/csrc: only tests/, __graft_entry__.smoke() and the
// CPU-baseline leg of bench.py load it.  The product never links or calls it.
//
// It restates, in plain C++ (FP32, explicit fmaf where nvcc contracts), the
// reference's algorithm:
//   * flow-field text loader          src/flow_field.cpp:8-54
//   * entropy CV cap + clip_mc        src/flow_field.cpp:80-166
//   * 12-table multi-step cache build src/flow_field.cpp:205-388
//   * cached FB kernels (full + block) src/kernels/gamma_smc_flow.cu:112-131,
//     160-163, 408-514, 567-609, 632-669, 678-754, 762-839
//   * bitpack                         src/kernels/bitpack.cu:11-30
//   * forward-only half-table kernel  src/kernels/gamma_smc_flow.cu:1136-1256
//     (run_fwd, src/bindings.cpp:2794-2849)
//   * uncached flow-field FB          src/kernels/gamma_smc_flow.cu:29-163,
//     168-398 (gamma_smc_flow_fb, src/bindings.cpp:2159-2300)
//
// Build: see oracle/Makefile (-O3 -mfma -ffp-contract=off -fopenmp).  The
// builder must not contract a*b+c into FMA, because the reference's table
// builder is compiled by g++ for plain x86-64, which has no FMA instructions;
// the scan uses explicit fmaf() exactly where nvcc's default -fmad=true
// contracts the reference's expressions.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kMeanN = 51;          // log10(mean) grid rows   (flow_field.h:6)
constexpr int kCvN = 50;            // log10(cv) grid columns  (flow_field.h:7)
constexpr int kGrid = kMeanN * kCvN;  // 2550 cells            (flow_field.h:8)

// Table order inside the oracle's flat table buffer [12][n_steps][2550].
enum Table {
  T_MISSING_M = 0, T_MISSING_C, T_CHUNK_M, T_CHUNK_C,
  T_FWD_HOM_M, T_FWD_HOM_C, T_FWD_HET_M, T_FWD_HET_C,
  T_BWD_HOM_M, T_BWD_HOM_C, T_BWD_HET_M, T_BWD_HET_C, T_COUNT
};

// ---------------------------------------------------------------- builder --

// Bilinear interpolation on the 51x50 grid as the CPU builder does it:
// index by division, clamp, keep the upper-edge cell, no FMA.
// (src/flow_field.cpp:60-78)
float grid_bilinear(const float* t, float m, float c, float m_min, float m_step,
                    float c_min, float c_step) {
  float fm = (m - m_min) / m_step;
  float fc = (c - c_min) / c_step;
  fm = std::max(0.0f, std::min(fm, (float)(kMeanN - 1)));
  fc = std::max(0.0f, std::min(fc, (float)(kCvN - 1)));
  int r = (int)fm, q = (int)fc;
  if (r == kMeanN - 1) r--;
  if (q == kCvN - 1) q--;
  float wm = fm - r, wc = fc - q;
  const float* p = t + r * kCvN + q;
  return (1 - wm) * ((1 - wc) * p[0] + wc * p[1]) +
         wm * ((1 - wc) * p[kCvN] + wc * p[kCvN + 1]);
}

// Entropy cap constants (src/flow_field.cpp:80-83).
constexpr double kEntMeanMax = 4.0;
constexpr double kEntMeanStep = 0.0008;
constexpr double kEntCvMin = -2.0;
constexpr double kEntCvMax = 0.0;

// Digamma by upward recurrence to x >= 6 and the asymptotic series
// (src/flow_field.cpp:85-104); same term order.
double digamma_series(double x) {
  double acc = 0.0;
  for (; x < 6.0; x += 1.0) acc -= 1.0 / x;
  const double i1 = 1.0 / x, i2 = i1 * i1, i4 = i2 * i2, i6 = i4 * i2,
               i8 = i4 * i4, i10 = i8 * i2;
  acc += std::log(x) - 0.5 * i1 - i2 / 12.0 + i4 / 120.0 - i6 / 252.0 +
         i8 / 240.0 - 5.0 * i10 / 660.0;
  return acc;
}

// Differential entropy of Gamma(alpha, beta) given log10 mean / log10 CV
// (src/flow_field.cpp:106-112).
double gamma_entropy(double mean_log10, double cv_log10) {
  const double a_l = -2.0 * cv_log10;
  const double b_l = a_l - mean_log10;
  const double a = std::pow(10.0, a_l);
  const double b = std::pow(10.0, b_l);
  return a - std::log(b) + std::lgamma(a) + (1.0 - a) * digamma_series(a);
}

// Largest log10 CV with entropy <= 1 per 0.0008-wide log10-mean bin:
// 60 bisection steps between the grid's CV bounds (src/flow_field.cpp:114-148).
const std::vector<float>& cv_cap_table() {
  static const std::vector<float> cap = [] {
    const int n = (int)std::llround(kEntMeanMax / kEntMeanStep) + 1;
    std::vector<float> out((size_t)n);
    for (int i = 0; i < n; ++i) {
      const double ml = i * kEntMeanStep;
      double lo = kEntCvMin, hi = kEntCvMax;
      if (gamma_entropy(ml, lo) > 1.0) { out[i] = (float)lo; continue; }
      if (gamma_entropy(ml, hi) <= 1.0) { out[i] = (float)hi; continue; }
      for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (gamma_entropy(ml, mid) > 1.0) hi = mid; else lo = mid;
      }
      out[i] = (float)hi;
    }
    return out;
  }();
  return cap;
}

// Clamp (m, c) to the grid and cap c by the entropy table
// (src/flow_field.cpp:150-166).
inline void clamp_state(float& m, float& c, float mmin, float mmax, float cmin,
                        float cmax) {
  m = std::max(mmin, std::min(m, mmax));
  c = std::max(cmin, std::min(c, cmax));
  if (m >= 0.0f && m <= kEntMeanMax) {
    const std::vector<float>& cap = cv_cap_table();
    const float x = m / (float)kEntMeanStep;
    const int k = (int)x;
    if (k >= (int)cap.size() - 1) { c = std::min(c, cap.back()); return; }
    const float w = x - k;
    c = std::min(c, (1.0f - w) * cap[k] + w * cap[k + 1]);
    c = std::max(cmin, std::min(c, cmax));
  }
}

// Observed-site emission in log10 space: beta += mu, het also alpha += 1
// (src/flow_field.cpp:168-184).
inline void emit_site(bool het, float mu, float& m, float& c) {
  float a_l = -2.0f * c;
  float b_l = a_l - m;
  b_l = log10f(powf(10.0f, b_l) + mu);
  if (het) a_l = log10f(powf(10.0f, a_l) + 1.0f);
  m = a_l - b_l;
  c = -0.5f * a_l;
}

struct Grid {
  float mmin, mmax, cmin, cmax, mstep, cstep;
};

// One flow-field recombination step: clamp, displace by (u, v) * rho, clamp
// (src/flow_field.cpp:246-255 and :286-294).
inline void recomb_step(const float* u, const float* v, const Grid& g, float rho,
                        float& m, float& c) {
  clamp_state(m, c, g.mmin, g.mmax, g.cmin, g.cmax);
  const float du = grid_bilinear(u, m, c, g.mmin, g.mstep, g.cmin, g.cstep);
  const float dv = grid_bilinear(v, m, c, g.mmin, g.mstep, g.cmin, g.cstep);
  m += du * rho;
  c += dv * rho;
  clamp_state(m, c, g.mmin, g.mmax, g.cmin, g.cmax);
}

}  // namespace

extern "C" {

// Parse the flow-field text format (src/flow_field.cpp:8-54):
//   "mean_min mean_max 51" / "cv_min cv_max 50" / 2550 u values / 2550 v values,
// bounds given linearly and returned as log10f.  Returns 0 on success.
int oracle_load_flow_field(const char* path, float* u, float* v, float* bounds) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  float lo, hi;
  int n;
  int rc = 0;
  if (fscanf(f, "%f %f %d", &lo, &hi, &n) != 3 || n != kMeanN) rc = -2;
  if (!rc) { bounds[0] = log10f(lo); bounds[1] = log10f(hi); }
  if (!rc && (fscanf(f, "%f %f %d", &lo, &hi, &n) != 3 || n != kCvN)) rc = -3;
  if (!rc) { bounds[2] = log10f(lo); bounds[3] = log10f(hi); }
  for (int i = 0; !rc && i < kGrid; ++i)
    if (fscanf(f, "%f", &u[i]) != 1) rc = -4;
  for (int i = 0; !rc && i < kGrid; ++i)
    if (fscanf(f, "%f", &v[i]) != 1) rc = -5;
  fclose(f);
  return rc;
}

// Build the 12 multi-step tables [12][n_steps][2550] (src/flow_field.cpp:205-388).
void oracle_build_tables(const float* u, const float* v, const float* bounds,
                         int n_steps, float scaled_rho, float scaled_mu,
                         float* out) {
  Grid g;
  g.mmin = bounds[0]; g.mmax = bounds[1]; g.cmin = bounds[2]; g.cmax = bounds[3];
  g.mstep = (g.mmax - g.mmin) / (kMeanN - 1);
  g.cstep = (g.cmax - g.cmin) / (kCvN - 1);
  (void)cv_cap_table();  // build the static before the parallel region
  const size_t L = (size_t)n_steps * kGrid;
  auto T = [&](int t) { return out + (size_t)t * L; };

  // Per-cell chains: step 0 is one recombination step from the grid point for
  // both the missing and the hom cache; step k>0 compounds from step k-1
  // (missing: recombination only; hom: beta += mu, then recombination).
#pragma omp parallel for schedule(static)
  for (int cell = 0; cell < kGrid; ++cell) {
    const int row = cell / kCvN, col = cell % kCvN;
    float m = g.mmin + row * g.mstep;
    float c = g.cmin + col * g.cstep;
    recomb_step(u, v, g, scaled_rho, m, c);
    T(T_MISSING_M)[cell] = m; T(T_MISSING_C)[cell] = c;
    T(T_CHUNK_M)[cell] = m;   T(T_CHUNK_C)[cell] = c;
    float mm = m, mc = c, hm = m, hc = c;
    for (int k = 1; k < n_steps; ++k) {
      const size_t at = (size_t)k * kGrid + cell;
      recomb_step(u, v, g, scaled_rho, mm, mc);
      T(T_MISSING_M)[at] = mm; T(T_MISSING_C)[at] = mc;
      const float a_l = -2.0f * hc;
      const float b_l = log10f(powf(10.0f, a_l - hm) + scaled_mu);
      hm = a_l - b_l;
      recomb_step(u, v, g, scaled_rho, hm, hc);
      T(T_CHUNK_M)[at] = hm; T(T_CHUNK_C)[at] = hc;
    }
  }

  // Site tables: forward = hom stretch of k+1 steps, then the observed site;
  // backward = observed site from the grid point, then the stretch looked up
  // in the hom cache at layer k.
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)L; ++idx) {
    const int k = (int)(idx / kGrid), cell = (int)(idx % kGrid);
    const int row = cell / kCvN, col = cell % kCvN;
    for (int het = 0; het < 2; ++het) {
      float m = T(T_CHUNK_M)[idx], c = T(T_CHUNK_C)[idx];
      emit_site(het, scaled_mu, m, c);
      clamp_state(m, c, g.mmin, g.mmax, g.cmin, g.cmax);
      T(het ? T_FWD_HET_M : T_FWD_HOM_M)[idx] = m;
      T(het ? T_FWD_HET_C : T_FWD_HOM_C)[idx] = c;

      m = g.mmin + row * g.mstep;
      c = g.cmin + col * g.cstep;
      emit_site(het, scaled_mu, m, c);
      clamp_state(m, c, g.mmin, g.mmax, g.cmin, g.cmax);
      const float* lm = T(T_CHUNK_M) + (size_t)k * kGrid;
      const float* lc = T(T_CHUNK_C) + (size_t)k * kGrid;
      const float nm = grid_bilinear(lm, m, c, g.mmin, g.mstep, g.cmin, g.cstep);
      const float nc = grid_bilinear(lc, m, c, g.mmin, g.mstep, g.cmin, g.cstep);
      T(het ? T_BWD_HET_M : T_BWD_HOM_M)[idx] = nm;
      T(het ? T_BWD_HET_C : T_BWD_HOM_C)[idx] = nc;
    }
  }
}

// bit b of word w of haplotype h = G[h][64w + b] & 1 (src/kernels/bitpack.cu:11-30).
void oracle_bitpack(const uint8_t* G, long long n, long long S, uint64_t* packed) {
  const long long nw = (S + 63) / 64;
  for (long long h = 0; h < n; ++h)
    for (long long w = 0; w < nw; ++w) {
      uint64_t word = 0;
      for (int b = 0; b < 64 && w * 64 + b < S; ++b)
        word |= (uint64_t)(G[h * S + w * 64 + b] & 1u) << b;
      packed[h * nw + w] = word;
    }
}

}  // extern "C"

// ------------------------------------------------------------------- scan --
namespace {

// The scan kernels hard-code the grid bounds (src/kernels/gamma_smc_flow.cu:10-17).
constexpr float kMmin = -5.0f, kMmax = 2.0f, kCmin = -2.0f, kCmax = 0.0f;
constexpr float kMstep = (kMmax - kMmin) / (kMeanN - 1);
constexpr float kCstep = (kCmax - kCmin) / (kCvN - 1);
constexpr float kMinv = 1.0f / kMstep;
constexpr float kCinv = 1.0f / kCstep;

// Table-layer bilinear as the scan does it: index by multiply, clamp, explicit
// FMA nesting (src/kernels/gamma_smc_flow.cu:408-430).
inline float layer_bilinear(const float* t, float m, float c) {
  float fm = (m - kMmin) * kMinv;
  float fc = (c - kCmin) * kCinv;
  fm = fmaxf(0.0f, fminf(fm, (float)(kMeanN - 1)));
  fc = fmaxf(0.0f, fminf(fc, (float)(kCvN - 1)));
  int r = (int)fm, q = (int)fc;
  if (r == kMeanN - 1) r--;
  if (q == kCvN - 1) q--;
  const float wm = fm - (float)r, wc = fc - (float)q;
  const float* p = t + r * kCvN + q;
  return fmaf(wm, fmaf(wc, p[kCvN + 1], (1.0f - wc) * p[kCvN]),
              (1.0f - wm) * fmaf(wc, p[1], (1.0f - wc) * p[0]));
}

inline void layer_apply(const float* tm, const float* tc, int layer, float& m,
                        float& c) {
  const float* pm = tm + (size_t)layer * kGrid;
  const float* pc = tc + (size_t)layer * kGrid;
  const float nm = layer_bilinear(pm, m, c);
  const float nc = layer_bilinear(pc, m, c);
  m = nm;
  c = nc;
}

// Schraudolph-style 10^x used by upstream gamma_smc and mirrored by the
// reference (src/kernels/gamma_smc_flow.cu:112-121): the float bits are
// trunc(C2 * (x * ln10) + C1), with the multiply-add fused as nvcc does.
inline float pow10_bits(float x) {
  const float kLn10 = 2.30258509299f;
  const float kC1 = 1064872507.1541044f;
  const float kC2 = 12102203.161561485f;
  const int bits = (int)fmaf(kC2, x * kLn10, kC1);
  float out;
  std::memcpy(&out, &bits, sizeof(out));
  return out;
}

inline void state_to_ab(float m, float c, float& a, float& b) {
  const float a_l = -2.0f * c;
  a = pow10_bits(a_l);
  b = pow10_bits(a_l - m);
}

// max(1, round-half-even(delta)) (src/kernels/gamma_smc_flow.cu:160-163).
inline int seg_steps_of(double delta) {
  const double r = std::nearbyint(delta);
  if (!(r >= 1.0)) return 1;
  if (r > 2147483647.0) return 2147483647;
  return (int)r;
}

struct TableView {
  const float *chunk_m, *chunk_c, *fh_m, *fh_c, *fx_m, *fx_c, *bh_m, *bh_c,
      *bx_m, *bx_c;
  int L;
};

// Forward: full chunks of L steps first, the observed-site table last
// (src/kernels/gamma_smc_flow.cu:471-489).
inline void forward_segment(const TableView& t, int seg, bool het, float& m,
                            float& c) {
  while (seg > t.L) {
    layer_apply(t.chunk_m, t.chunk_c, t.L - 1, m, c);
    seg -= t.L;
  }
  layer_apply(het ? t.fx_m : t.fh_m, het ? t.fx_c : t.fh_c, seg - 1, m, c);
}

// Backward: site table on the remainder first, full chunks after
// (src/kernels/gamma_smc_flow.cu:491-514).
inline void backward_segment(const TableView& t, int seg, bool het, float& m,
                             float& c) {
  int rem = seg;
  while (rem > t.L) rem -= t.L;
  layer_apply(het ? t.bx_m : t.bh_m, het ? t.bx_c : t.bh_c, rem - 1, m, c);
  for (seg -= rem; seg > 0; seg -= t.L) layer_apply(t.chunk_m, t.chunk_c, t.L - 1, m, c);
}

}  // namespace

extern "C" {

// The scan's table-layer bilinear on one [51 x 50] grid, exposed for the
// upper-boundary known answers of tests/unit/test_gamma_smc_flow.py:140-158.
float oracle_layer_bilinear(const float* grid, float m, float c) {
  return layer_bilinear(grid, m, c);
}

// One window [w0, w0 + wlen) of the cached FB scan for P pairs: the
// block kernels (src/kernels/gamma_smc_flow.cu:632-669, 762-839), which with
// w0 = 0 and wlen = S are the full-sequence kernels (:567-609, :678-754).
// Outputs are window-local, site-major [wlen][P]; lower/upper/alpha/beta may be
// null.  tables is the [12][L][2550] buffer of oracle_build_tables.
int oracle_fb_window(const uint64_t* packed, long long n_words,
                     const double* pos, long long S, long long w0, long long wlen,
                     const int* pi, const int* pj, long long P, float Ne,
                     const float* tables, int L, float* mean, float* lower,
                     float* upper, float* alpha, float* beta, int n_threads) {
  if (w0 < 0 || wlen < 0 || w0 + wlen > S || L <= 0) return -1;
  const size_t LS = (size_t)L * kGrid;
  TableView t;
  t.chunk_m = tables + T_CHUNK_M * LS; t.chunk_c = tables + T_CHUNK_C * LS;
  t.fh_m = tables + T_FWD_HOM_M * LS; t.fh_c = tables + T_FWD_HOM_C * LS;
  t.fx_m = tables + T_FWD_HET_M * LS; t.fx_c = tables + T_FWD_HET_C * LS;
  t.bh_m = tables + T_BWD_HOM_M * LS; t.bh_c = tables + T_BWD_HOM_C * LS;
  t.bx_m = tables + T_BWD_HET_M * LS; t.bx_c = tables + T_BWD_HET_C * LS;
  t.L = L;
  const bool ci = lower && upper;
  const float unscale = 2.0f * Ne;
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
#pragma omp parallel
  {
    std::vector<float> fwd((size_t)wlen * 2);
#pragma omp for schedule(dynamic, 16)
    for (long long p = 0; p < P; ++p) {
      const uint64_t* hi = packed + (long long)pi[p] * n_words;
      const uint64_t* hj = packed + (long long)pj[p] * n_words;
      auto het_at = [&](long long s) { return ((hi[s >> 6] ^ hj[s >> 6]) >> (s & 63)) & 1u; };
      float m = 0.0f, c = 0.0f;
      double prev = (w0 == 0) ? -1.0 : pos[w0] - 1.0;
      for (long long s = 0; s < wlen; ++s) {
        const double x = pos[w0 + s];
        const int seg = seg_steps_of(x - prev);
        prev = x;
        forward_segment(t, seg, het_at(w0 + s) != 0, m, c);
        fwd[2 * s] = m;
        fwd[2 * s + 1] = c;
      }
      m = 0.0f; c = 0.0f;
      for (long long s = wlen - 1; s >= 0; --s) {
        const long long gs = w0 + s;
        float ba, bb, fa, fb;
        state_to_ab(m, c, ba, bb);
        state_to_ab(fwd[2 * s], fwd[2 * s + 1], fa, fb);
        const float a_s = fa + ba - 1.0f;
        const float b_s = fb + bb - 1.0f;
        const float mg = (a_s / fmaxf(b_s, 1e-10f)) * unscale;
        const size_t o = (size_t)s * P + p;
        mean[o] = mg;
        if (ci) {
          // Wilson-Hilferty 95% bounds (src/kernels/gamma_smc_flow.cu:724-733);
          // base -/+ 1.96*sq are fused by nvcc.
          const float inv9a = 1.0f / (9.0f * fmaxf(a_s, 1.0f));
          const float sq = sqrtf(inv9a);
          const float base = 1.0f - inv9a;
          const float lo = fmaxf(fmaf(-1.96f, sq, base), 0.0f);
          const float up = fmaf(1.96f, sq, base);
          lower[o] = fmaxf(mg * lo * lo * lo, 0.0f);
          upper[o] = mg * up * up * up;
        }
        if (alpha) alpha[o] = a_s;
        if (beta) beta[o] = b_s;
        int seg;
        if (gs == 0) seg = seg_steps_of(pos[0] + 1.0);
        else if (s == 0 && w0 > 0) seg = 1;
        else seg = seg_steps_of(pos[gs] - pos[gs - 1]);
        backward_segment(t, seg, het_at(gs) != 0, m, c);
      }
    }
  }
  return 0;
}

// Forward-only filtered posterior (the reference's run_fwd: the half copy of
// the hom multi-step table, src/kernels/gamma_smc_flow.cu:1136-1256).  hom_m /
// hom_c are that table [L][2550] already rounded through float16 by the
// caller.  exp10f / log10f / exp2f stand in for the device's __exp10f /
// __log10f / exp2f, which differ by a few ulp.  Outputs [S][P].
void oracle_fwd_only(const uint64_t* packed, long long n_words, const double* pos,
                     long long S, const int* pi, const int* pj, long long P, float two_ne,
                     const float* hom_m, const float* hom_c, int L, float* mean,
                     float* lower, float* upper, int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
#pragma omp parallel for schedule(dynamic, 16)
  for (long long p = 0; p < P; ++p) {
    const uint64_t* hi = packed + (long long)pi[p] * n_words;
    const uint64_t* hj = packed + (long long)pj[p] * n_words;
    float m = 0.0f, c = 0.0f;
    double prev = 0.0;
    for (long long s = 0; s < S; ++s) {
      const double x = pos[s];
      const double g = x - prev + 0.5;
      int gap = g >= 2147483647.0 ? 2147483647 : (int)g;  // truncation, as the reference
      prev = x;
      if (s > 0 && gap > 0) {
        while (gap > L) {
          layer_apply(hom_m, hom_c, L - 1, m, c);
          gap -= L;
        }
        layer_apply(hom_m, hom_c, gap - 1, m, c);
      }
      if ((((hi[s >> 6] ^ hj[s >> 6]) >> (s & 63)) & 1u) != 0) {
        const float alpha = exp10f(-2.0f * c) + 1.0f;
        const float a_log = log10f(alpha);
        const float b_log = fmaf(-2.0f, c, -m);
        m = a_log - b_log;
        c = -0.5f * a_log;
      }
      const float mg = exp2f(m * 3.321928094887362f) * two_ne;
      const size_t o = (size_t)s * P + p;
      mean[o] = mg;
      if (lower && upper) {
        const float alpha = exp10f(-2.0f * c);
        const float inv9a = 1.0f / (9.0f * alpha);
        const float sq = sqrtf(inv9a);
        const float base = 1.0f - inv9a;
        const float lo = fmaxf(fmaf(-1.96f, sq, base), 0.0f);
        const float up = fmaf(1.96f, sq, base);
        lower[o] = fmaxf(mg * lo * lo * lo, 0.0f);
        upper[o] = mg * up * up * up;
      }
    }
  }
}

// Uncached flow-field FB (gamma_smc_flow_fb): each gap integrated on the
// 51 x 50 (u, v) grid.  u / v are the flow field [2550]; rho / mu the scaled
// per-bp rates.  libm exp10f / log10f stand in for __exp10f / __log10f.
namespace {
inline float flow_bilinear(const float* t, float m, float c) { return layer_bilinear(t, m, c); }

inline void o_recomb(const float* u, const float* v, float rho, float& m, float& c) {
  const float du = flow_bilinear(u, m, c), dv = flow_bilinear(v, m, c);
  m = fmaf(du, rho, m);
  c = fmaf(dv, rho, c);
  m = std::max(-5.0f, std::min(m, 2.0f));
  c = std::max(-2.0f, std::min(c, 0.0f));
}

inline void o_segment(const float* u, const float* v, int seg, float rho, float mu, float& m,
                      float& c) {
  if (rho >= 1e-12f) o_recomb(u, v, rho, m, c);
  if (seg <= 1) return;
  const float rt = rho * (float)(seg - 1), mt = mu * (float)(seg - 1);
  if (rt < 1e-12f) return;
  const int n_iter = std::max(1, (int)std::ceil(rt * (1.0f / 0.1f)));
  const float inv_n = 1.0f / (float)n_iter;
  const float rp = rt * inv_n, mp = mt * inv_n;
  for (int i = 0; i < n_iter; ++i) {
    const float a_log = -2.0f * c;
    const float b_log = log10f(exp10f(a_log - m) + mp);
    m = a_log - b_log;
    o_recomb(u, v, rp, m, c);
  }
}

inline void o_emit(bool het, float mu, float& m, float& c) {
  float a_log = -2.0f * c;
  const float b_log = log10f(exp10f(a_log - m) + mu);
  if (het) a_log = log10f(exp10f(a_log) + 1.0f);
  m = a_log - b_log;
  c = -0.5f * a_log;
}
}  // namespace

void oracle_flow_fb(const uint64_t* packed, long long n_words, const double* pos, long long S,
                    const int* pi, const int* pj, long long P, const float* u, const float* v,
                    float rho, float mu, float Ne, float* mean, float* lower, float* upper,
                    int n_threads) {
#ifdef _OPENMP
  if (n_threads > 0) omp_set_num_threads(n_threads);
#else
  (void)n_threads;
#endif
  const float unscale = 2.0f * Ne;
  std::vector<int> seg((size_t)S);
  for (long long s = 0; s < S; ++s)
    seg[s] = seg_steps_of(s == 0 ? pos[0] + 1.0 : pos[s] - pos[s - 1]);
#pragma omp parallel
  {
    std::vector<float> fwd((size_t)S * 2);
#pragma omp for schedule(dynamic, 16)
    for (long long p = 0; p < P; ++p) {
      const uint64_t* hi = packed + (long long)pi[p] * n_words;
      const uint64_t* hj = packed + (long long)pj[p] * n_words;
      auto het_at = [&](long long s) { return ((hi[s >> 6] ^ hj[s >> 6]) >> (s & 63)) & 1u; };
      float m = 0.0f, c = 0.0f;
      for (long long s = 0; s < S; ++s) {
        o_segment(u, v, seg[s], rho, mu, m, c);
        o_emit(het_at(s) != 0, mu, m, c);
        fwd[2 * s] = m;
        fwd[2 * s + 1] = c;
      }
      m = 0.0f;
      c = 0.0f;
      for (long long s = S - 1; s >= 0; --s) {
        float ba, bb, fa, fb;
        state_to_ab(m, c, ba, bb);
        state_to_ab(fwd[2 * s], fwd[2 * s + 1], fa, fb);
        const float a_s = fa + ba - 1.0f, b_s = fb + bb - 1.0f;
        const float mg = (a_s / fmaxf(b_s, 1e-10f)) * unscale;
        const size_t o = (size_t)s * P + p;
        mean[o] = mg;
        if (lower && upper) {
          const float inv9a = 1.0f / (9.0f * fmaxf(a_s, 1.0f));
          const float sq = sqrtf(inv9a);
          const float base = 1.0f - inv9a;
          const float lo = fmaxf(fmaf(-1.96f, sq, base), 0.0f);
          lower[o] = fmaxf(mg * lo * lo * lo, 0.0f);
          const float up = fmaf(1.96f, sq, base);
          upper[o] = mg * up * up * up;
        }
        o_emit(het_at(s) != 0, mu, m, c);
        o_segment(u, v, seg[s], rho, mu, m, c);
      }
    }
  }
}

}  // extern "C"
