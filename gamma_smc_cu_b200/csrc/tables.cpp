// Host construction of the multi-step flow-field tables the scan reads.
//
// The scan advances a pair's Gamma state (m, c) = (log10 mean, log10 CV) over a
// gap of k base pairs plus the observed site with ONE bilinear lookup into a
// precomputed table layer k-1.  Building those layers is a per-grid-cell chain
// of k flow-field steps; it runs once per (Ne, mu, rho, n_steps).
//
// The arithmetic is the reference's, step for step, in FP32 with the C
// library's powf/log10f and no FMA contraction (this file is compiled with
// -ffp-contract=off), so the layers are bit-identical to the reference's
// build_flow_field_cache (src/flow_field.cpp:205-388).  Cells are independent
// chains, so the build is split across host threads by cell; the result does
// not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "tables.h"

namespace gsmc {
namespace {

struct GridSpec {
  float m_lo, m_hi, c_lo, c_hi, m_step, c_step;
};

// Grid bilinear with the upper-edge cell kept, indexed by division
// (src/flow_field.cpp:60-78).
float interp(const float* f, float m, float c, const GridSpec& g) {
  float x = (m - g.m_lo) / g.m_step;
  float y = (c - g.c_lo) / g.c_step;
  x = std::max(0.0f, std::min(x, (float)(kRows - 1)));
  y = std::max(0.0f, std::min(y, (float)(kCols - 1)));
  int i = (int)x;
  int j = (int)y;
  if (i == kRows - 1) --i;
  if (j == kCols - 1) --j;
  const float wx = x - i, wy = y - j;
  const float* row0 = f + i * kCols + j;
  const float* row1 = row0 + kCols;
  return (1 - wx) * ((1 - wy) * row0[0] + wy * row0[1]) +
         wx * ((1 - wy) * row1[0] + wy * row1[1]);
}

// log10 CV cap keeping the Gamma's differential entropy <= 1, tabulated in
// FP64 on 5001 log10-mean points 0, 0.0008, ..., 4 (src/flow_field.cpp:80-148).
constexpr double kCapMeanHi = 4.0;
constexpr double kCapMeanStep = 0.0008;

double psi(double x) {  // digamma: recurrence to x >= 6, then asymptotic series
  double r = 0.0;
  while (x < 6.0) {
    r -= 1.0 / x;
    x += 1.0;
  }
  const double a = 1.0 / x;
  const double a2 = a * a;
  const double a4 = a2 * a2;
  const double a6 = a4 * a2;
  const double a8 = a4 * a4;
  const double a10 = a8 * a2;
  r += std::log(x) - 0.5 * a - a2 / 12.0 + a4 / 120.0 - a6 / 252.0 + a8 / 240.0 -
       5.0 * a10 / 660.0;
  return r;
}

double entropy(double mean_l, double cv_l) {
  const double al = -2.0 * cv_l;
  const double bl = al - mean_l;
  const double a = std::pow(10.0, al);
  const double b = std::pow(10.0, bl);
  return a - std::log(b) + std::lgamma(a) + (1.0 - a) * psi(a);
}

std::vector<float> make_cv_cap() {
  const int n = (int)std::llround(kCapMeanHi / kCapMeanStep) + 1;
  std::vector<float> cap(n);
  for (int i = 0; i < n; ++i) {
    const double ml = i * kCapMeanStep;
    double lo = -2.0, hi = 0.0;
    if (entropy(ml, lo) > 1.0) {
      cap[i] = (float)lo;
    } else if (entropy(ml, hi) <= 1.0) {
      cap[i] = (float)hi;
    } else {
      for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        (entropy(ml, mid) > 1.0 ? hi : lo) = mid;
      }
      cap[i] = (float)hi;
    }
  }
  return cap;
}

const std::vector<float>& cv_cap() {
  static const std::vector<float> cap = make_cv_cap();
  return cap;
}

}  // namespace

// The same cap kept in float64 (the bisection's final upper bound), for the
// float64 table build.
const std::vector<double>& cv_cap_f64() {
  static const std::vector<double> cap = [] {
    const int n = (int)std::llround(kCapMeanHi / kCapMeanStep) + 1;
    std::vector<double> out(n);
    for (int i = 0; i < n; ++i) {
      const double ml = i * kCapMeanStep;
      double lo = -2.0, hi = 0.0;
      if (entropy(ml, lo) > 1.0) {
        out[i] = lo;
      } else if (entropy(ml, hi) <= 1.0) {
        out[i] = hi;
      } else {
        for (int it = 0; it < 60; ++it) {
          const double mid = 0.5 * (lo + hi);
          (entropy(ml, mid) > 1.0 ? hi : lo) = mid;
        }
        out[i] = hi;
      }
    }
    return out;
  }();
  return cap;
}

namespace {

// Grid clamp plus the entropy cap (src/flow_field.cpp:150-166).
inline void clip(float& m, float& c, const GridSpec& g, const std::vector<float>& cap) {
  m = std::max(g.m_lo, std::min(m, g.m_hi));
  c = std::max(g.c_lo, std::min(c, g.c_hi));
  if (!(m >= 0.0f && m <= kCapMeanHi)) return;
  const float x = m / (float)kCapMeanStep;
  const int i = (int)x;
  if (i >= (int)cap.size() - 1) {
    c = std::min(c, cap.back());
    return;
  }
  const float w = x - i;
  c = std::min(c, (1.0f - w) * cap[i] + w * cap[i + 1]);
  c = std::max(g.c_lo, std::min(c, g.c_hi));
}

// One recombination step of the flow field (src/flow_field.cpp:246-255).
inline void flow(const FlowField& ff, const GridSpec& g, const std::vector<float>& cap,
                 float rho, float& m, float& c) {
  clip(m, c, g, cap);
  const float du = interp(ff.u, m, c, g);
  const float dv = interp(ff.v, m, c, g);
  m += du * rho;
  c += dv * rho;
  clip(m, c, g, cap);
}

// Observed-site emission: beta += mu; a het site also alpha += 1
// (src/flow_field.cpp:168-184).
inline void observe(bool het, float mu, float& m, float& c) {
  float al = -2.0f * c;
  float bl = al - m;
  bl = log10f(powf(10.0f, bl) + mu);
  if (het) al = log10f(powf(10.0f, al) + 1.0f);
  m = al - bl;
  c = -0.5f * al;
}

template <class F>
void parallel_for(long long n, int threads, F&& body) {
  if (threads <= 1 || n < 2) {
    body(0LL, n);
    return;
  }
  std::vector<std::thread> pool;
  const long long per = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    const long long lo = t * per, hi = std::min(n, lo + per);
    if (lo >= hi) break;
    pool.emplace_back([&body, lo, hi] { body(lo, hi); });
  }
  for (auto& th : pool) th.join();
}

}  // namespace

int load_flow_field(const char* path, FlowField* ff, char* err, size_t err_len) {
  FILE* f = std::fopen(path, "r");
  if (!f) {
    std::snprintf(err, err_len, "Failed to load flow field from: %s", path);
    return -1;
  }
  float lo = 0, hi = 0;
  int n = 0;
  bool ok = std::fscanf(f, "%f %f %d", &lo, &hi, &n) == 3 && n == kRows;
  if (ok) {
    ff->m_lo = log10f(lo);
    ff->m_hi = log10f(hi);
    ok = std::fscanf(f, "%f %f %d", &lo, &hi, &n) == 3 && n == kCols;
  }
  if (ok) {
    ff->c_lo = log10f(lo);
    ff->c_hi = log10f(hi);
  }
  for (int i = 0; ok && i < kCells; ++i) ok = std::fscanf(f, "%f", &ff->u[i]) == 1;
  for (int i = 0; ok && i < kCells; ++i) ok = std::fscanf(f, "%f", &ff->v[i]) == 1;
  std::fclose(f);
  if (!ok) std::snprintf(err, err_len, "Failed to load flow field from: %s", path);
  return ok ? 0 : -1;
}

void build_layers(const FlowField& ff, int n_steps, float scaled_rho, float scaled_mu,
                  int threads, HostLayers* out) {
  GridSpec g;
  g.m_lo = ff.m_lo;
  g.m_hi = ff.m_hi;
  g.c_lo = ff.c_lo;
  g.c_hi = ff.c_hi;
  g.m_step = (g.m_hi - g.m_lo) / (kRows - 1);
  g.c_step = (g.c_hi - g.c_lo) / (kCols - 1);
  const std::vector<float>& cap = cv_cap();
  if (threads <= 0) threads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));

  const size_t n = (size_t)n_steps * kCells;
  for (int t = 0; t < kNumHostTables; ++t) out->t[t].assign(n, 0.0f);
  out->n_steps = n_steps;

  // Hom cache, layer k = k+1 base pairs: layer 0 is one recombination step
  // from the grid point; each further layer adds beta += mu and one more step.
  // The missing-data cache (recombination only) is built alongside.
  float* hom_m = out->t[kHomMean].data();
  float* hom_c = out->t[kHomCv].data();
  float* mis_m = out->t[kMissingMean].data();
  float* mis_c = out->t[kMissingCv].data();
  parallel_for(kCells, threads, [&](long long lo, long long hi) {
    for (long long cell = lo; cell < hi; ++cell) {
      const int row = (int)cell / kCols, col = (int)cell % kCols;
      float m = g.m_lo + row * g.m_step;
      float c = g.c_lo + col * g.c_step;
      flow(ff, g, cap, scaled_rho, m, c);
      float hm = m, hc = c, xm = m, xc = c;
      hom_m[cell] = hm;
      hom_c[cell] = hc;
      mis_m[cell] = xm;
      mis_c[cell] = xc;
      for (int k = 1; k < n_steps; ++k) {
        const size_t at = (size_t)k * kCells + cell;
        flow(ff, g, cap, scaled_rho, xm, xc);
        mis_m[at] = xm;
        mis_c[at] = xc;
        const float al = -2.0f * hc;
        const float bl = al - hm;
        hm = al - log10f(powf(10.0f, bl) + scaled_mu);
        flow(ff, g, cap, scaled_rho, hm, hc);
        hom_m[at] = hm;
        hom_c[at] = hc;
      }
    }
  });

  // Observed-site layers.  Forward: stretch of k+1 bp from the hom cache, then
  // the site.  Backward: the site at the grid point, then the stretch as a
  // lookup into hom layer k.
  parallel_for((long long)n, threads, [&](long long lo, long long hi) {
    for (long long at = lo; at < hi; ++at) {
      const int k = (int)(at / kCells);
      const int cell = (int)(at % kCells);
      const int row = cell / kCols, col = cell % kCols;
      const float* lm = hom_m + (size_t)k * kCells;
      const float* lc = hom_c + (size_t)k * kCells;
      for (int het = 0; het <= 1; ++het) {
        float m = hom_m[at], c = hom_c[at];
        observe(het != 0, scaled_mu, m, c);
        clip(m, c, g, cap);
        out->t[het ? kFwdHetMean : kFwdHomMean][at] = m;
        out->t[het ? kFwdHetCv : kFwdHomCv][at] = c;

        m = g.m_lo + row * g.m_step;
        c = g.c_lo + col * g.c_step;
        observe(het != 0, scaled_mu, m, c);
        clip(m, c, g, cap);
        const float bm = interp(lm, m, c, g);
        const float bc = interp(lc, m, c, g);
        out->t[het ? kBwdHetMean : kBwdHomMean][at] = bm;
        out->t[het ? kBwdHetCv : kBwdHomCv][at] = bc;
      }
    }
  });
}

void scaled_rates(double Ne, double mu, double rho, float* scaled_rho, float* scaled_mu) {
  // FlowContext narrows to float (src/bindings.cpp:2575) and ensure_cache
  // forms 4.0f * Ne * rate in float (src/bindings.cpp:2044-2045).
  const float ne = (float)Ne;
  *scaled_rho = 4.0f * ne * (float)rho;
  *scaled_mu = 4.0f * ne * (float)mu;
}

// Scan layout: one 32-byte patch per interpolation cell (r, q), r < 50,
// q < 49, holding the four corners of m then of c:
//   {m[r][q], m[r][q+1], m[r+1][q], m[r+1][q+1]}, {c[r][q], ..., c[r+1][q+1]}
// so one lookup is a single 256-bit load of one 32-byte sector (the
// forward-only path's half-precision table converts the same layout).
void pack_patches(const float* m, const float* c, float* dst) {
  for (int r = 0; r < kPatchRows; ++r)
    for (int q = 0; q < kPatchCols; ++q) {
      const int a = r * kCols + q;
      const int corner[4] = {a, a + 1, a + kCols, a + kCols + 1};
      float* p = dst + (size_t)(r * kPatchCols + q) * 8;
      for (int k = 0; k < 4; ++k) {
        p[k] = m[corner[k]];
        p[4 + k] = c[corner[k]];
      }
    }
}

void build_scan_layout(const HostLayers& h, std::vector<float>* site, std::vector<float>* chunk,
                       int threads) {
  const int L = h.n_steps;
  const size_t per_layer = (size_t)kPatches * 8;
  site->assign((size_t)kScanTables * L * per_layer, 0.0f);
  static const int kSrc[kScanTables][2] = {{kFwdHomMean, kFwdHomCv},
                                           {kFwdHetMean, kFwdHetCv},
                                           {kBwdHomMean, kBwdHomCv},
                                           {kBwdHetMean, kBwdHetCv}};
  if (threads <= 0) threads = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  parallel_for((long long)kScanTables * L, threads, [&](long long lo, long long hi) {
    for (long long tl = lo; tl < hi; ++tl) {
      const int t = (int)(tl / L), k = (int)(tl % L);
      pack_patches(h.t[kSrc[t][0]].data() + (size_t)k * kCells,
                      h.t[kSrc[t][1]].data() + (size_t)k * kCells,
                      site->data() + scan_layer_offset(t, k, L) * 4);
    }
  });
  chunk->assign(per_layer, 0.0f);
  pack_patches(h.t[kHomMean].data() + (size_t)(L - 1) * kCells,
                  h.t[kHomCv].data() + (size_t)(L - 1) * kCells, chunk->data());
}

}  // namespace gsmc
