// Optional GPU build of the scan tables in float64.
//
// The default build (tables.cpp) reproduces the reference's host builder bit
// for bit: float32 states rounded at every one of the up to 1000 compounded
// steps (src/flow_field.cpp:205-388).  This build carries every cell's state
// in float64 through the whole chain, evaluates the flow-field bilinear, the
// entropy cap (its bisection kept in float64), the emissions (exp10/log10)
// and the backward lookups in float64, and rounds to float32 only when a
// table entry is stored.  The scan then reads the same table layout, so the
// two builds differ only in the tables' last bits; its effect on the
// posteriors is measured by the tests and the benchmark against the
// posterior-mean tolerance.
//
// Structure: the hom multi-step layers are independent per-cell chains (one
// thread per grid cell, the flow field staged in shared memory); the
// observed-site layers are independent per (layer, cell); a last kernel
// packs the patches of the scan layout.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "tables_gpu.h"

namespace gsmc {
namespace {

constexpr int kCapN = 5001;  // log10 mean 0, 0.0008, ..., 4
constexpr double kCapStep = 0.0008;
constexpr double kCapMeanHi = 4.0;

struct GridD {
  double m_lo, m_hi, c_lo, c_hi, m_step, c_step;
};

// Lower-left cell and weights of (m, c), the upper-edge cell kept.
__device__ __forceinline__ int cell_of(double m, double c, const GridD& g, double* wx, double* wy) {
  double x = (m - g.m_lo) / g.m_step;
  double y = (c - g.c_lo) / g.c_step;
  x = fmax(0.0, fmin(x, (double)(kRows - 1)));
  y = fmax(0.0, fmin(y, (double)(kCols - 1)));
  int i = (int)x, j = (int)y;
  if (i == kRows - 1) --i;
  if (j == kCols - 1) --j;
  *wx = x - i;
  *wy = y - j;
  return i * kCols + j;
}

__device__ __forceinline__ double bilerp(const double* f, int b, double wx, double wy) {
  return (1.0 - wx) * ((1.0 - wy) * f[b] + wy * f[b + 1]) +
         wx * ((1.0 - wy) * f[b + kCols] + wy * f[b + kCols + 1]);
}

// Grid clamp plus the entropy cap on log10 CV.
__device__ __forceinline__ void clip_d(double& m, double& c, const GridD& g,
                                      const double* __restrict__ cap) {
  m = fmax(g.m_lo, fmin(m, g.m_hi));
  c = fmax(g.c_lo, fmin(c, g.c_hi));
  if (!(m >= 0.0 && m <= kCapMeanHi)) return;
  const double x = m / kCapStep;
  const int i = (int)x;
  if (i >= kCapN - 1) {
    c = fmin(c, __ldg(cap + kCapN - 1));
    return;
  }
  const double w = x - i;
  c = fmin(c, (1.0 - w) * __ldg(cap + i) + w * __ldg(cap + i + 1));
  c = fmax(g.c_lo, fmin(c, g.c_hi));
}

// One recombination step of the flow field.
__device__ __forceinline__ void flow_d(const double* u, const double* v, const GridD& g,
                                      const double* cap, double rho, double& m, double& c) {
  clip_d(m, c, g, cap);
  double wx, wy;
  const int b = cell_of(m, c, g, &wx, &wy);
  const double du = bilerp(u, b, wx, wy), dv = bilerp(v, b, wx, wy);
  m += du * rho;
  c += dv * rho;
  clip_d(m, c, g, cap);
}

// Observed site: beta += mu, and a het site alpha += 1.
__device__ __forceinline__ void observe_d(bool het, double mu, double& m, double& c) {
  double al = -2.0 * c;
  const double bl = log10(exp10(al - m) + mu);
  if (het) al = log10(exp10(al) + 1.0);
  m = al - bl;
  c = -0.5 * al;
}

// Hom layers: layer k is k + 1 base pairs from the grid point (one
// recombination step, then k times beta += mu and a step).  One thread per
// cell; hom[k][cell] = (m, c).
__global__ void __launch_bounds__(128) hom_chain_kernel(const double* __restrict__ uv,
                                                       const double* __restrict__ cap, GridD g,
                                                       int L, double rho, double mu,
                                                       double2* __restrict__ hom) {
  __shared__ double u[kCells], v[kCells];
  for (int i = threadIdx.x; i < kCells; i += blockDim.x) {
    u[i] = uv[i];
    v[i] = uv[kCells + i];
  }
  __syncthreads();
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= kCells) return;
  double m = g.m_lo + (cell / kCols) * g.m_step;
  double c = g.c_lo + (cell % kCols) * g.c_step;
  flow_d(u, v, g, cap, rho, m, c);
  hom[cell] = make_double2(m, c);
  for (int k = 1; k < L; ++k) {
    const double al = -2.0 * c;
    m = al - log10(exp10(al - m) + mu);
    flow_d(u, v, g, cap, rho, m, c);
    hom[(size_t)k * kCells + cell] = make_double2(m, c);
  }
}

// Observed-site layers, one thread per (layer, cell): forward = hom layer k
// then the site; backward = the site at the grid point, then a lookup in hom
// layer k.  out[t][k][cell] for t = fwd hom m, c, fwd het m, c, bwd hom m, c,
// bwd het m, c; hom_f = hom layers rounded to float32 ([2][L][cell]).
__global__ void site_kernel(const double2* __restrict__ hom, const double* __restrict__ cap,
                            GridD g, int L, double mu, float* __restrict__ out,
                            float* __restrict__ hom_f) {
  const int64_t at = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = (int64_t)L * kCells;
  if (at >= n) return;
  const int k = (int)(at / kCells), cell = (int)(at % kCells);
  const double2 h = hom[at];
  hom_f[at] = (float)h.x;
  hom_f[n + at] = (float)h.y;
  const double2* layer = hom + (size_t)k * kCells;
  for (int het = 0; het <= 1; ++het) {
    double m = h.x, c = h.y;
    observe_d(het != 0, mu, m, c);
    clip_d(m, c, g, cap);
    out[(size_t)(2 * het) * n + at] = (float)m;
    out[(size_t)(2 * het + 1) * n + at] = (float)c;
    m = g.m_lo + (cell / kCols) * g.m_step;
    c = g.c_lo + (cell % kCols) * g.c_step;
    observe_d(het != 0, mu, m, c);
    clip_d(m, c, g, cap);
    double wx, wy;
    const int b = cell_of(m, c, g, &wx, &wy);
    const double2 a = layer[b], e = layer[b + 1];
    const double2 d = layer[b + kCols], f = layer[b + kCols + 1];
    const double bm = (1.0 - wx) * ((1.0 - wy) * a.x + wy * e.x) + wx * ((1.0 - wy) * d.x + wy * f.x);
    const double bc = (1.0 - wx) * ((1.0 - wy) * a.y + wy * e.y) + wx * ((1.0 - wy) * d.y + wy * f.y);
    out[(size_t)(4 + 2 * het) * n + at] = (float)bm;
    out[(size_t)(4 + 2 * het + 1) * n + at] = (float)bc;
  }
}

// Scan layout: thread per (table t, layer k, patch p) writes the patch's
// four m corners, then its four c corners (pack_patches's layout).  Tables t < 4 are
// the scan's fwd hom, fwd het, bwd hom, bwd het; the last kPatches threads
// write the chunk table (hom layer L - 1).
__global__ void pack_kernel(const float* __restrict__ out, const float* __restrict__ hom_f,
                            int L, float* __restrict__ site, float* __restrict__ chunk) {
  const int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t per = (int64_t)L * kPatches;
  if (id >= 4 * per + kPatches) return;
  const int64_t n = (int64_t)L * kCells;
  const float* m;
  const float* c;
  float* dst;
  int p;
  if (id < 4 * per) {
    const int t = (int)(id / per);
    const int k = (int)((id % per) / kPatches);
    p = (int)(id % kPatches);
    m = out + (size_t)(2 * t) * n + (size_t)k * kCells;
    c = out + (size_t)(2 * t + 1) * n + (size_t)k * kCells;
    const size_t layer_f4 = ((size_t)(t / 2) * L + k) * kLayerF4 + (size_t)(t % 2) * kHetF4;
    dst = site + layer_f4 * 4 + (size_t)p * 8;
  } else {
    p = (int)(id - 4 * per);
    m = hom_f + (size_t)(L - 1) * kCells;
    c = hom_f + n + (size_t)(L - 1) * kCells;
    dst = chunk + (size_t)p * 8;
  }
  const int r = p / kPatchCols, q = p % kPatchCols;
  const int a = r * kCols + q;
  const int corner[4] = {a, a + 1, a + kCols, a + kCols + 1};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    dst[i] = m[corner[i]];
    dst[4 + i] = c[corner[i]];
  }
}

}  // namespace

int build_tables_gpu_f64(const FlowField& ff, int L, double scaled_rho, double scaled_mu,
                         float4* site, float4* chunk, std::vector<float>* hom_m,
                         std::vector<float>* hom_c, std::string* err) {
  const std::vector<double>& cap = cv_cap_f64();
  GridD g;
  g.m_lo = ff.m_lo;
  g.m_hi = ff.m_hi;
  g.c_lo = ff.c_lo;
  g.c_hi = ff.c_hi;
  g.m_step = (g.m_hi - g.m_lo) / (kRows - 1);
  g.c_step = (g.c_hi - g.c_lo) / (kCols - 1);
  std::vector<double> uv(2 * kCells);
  for (int i = 0; i < kCells; ++i) {
    uv[i] = ff.u[i];
    uv[kCells + i] = ff.v[i];
  }
  const int64_t n = (int64_t)L * kCells;
  double* d_uv = nullptr;
  double* d_cap = nullptr;
  double2* d_hom = nullptr;
  float* d_out = nullptr;
  float* d_homf = nullptr;
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&d_uv, uv.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_cap, cap.size() * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&d_hom, (size_t)n * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, (size_t)8 * n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&d_homf, (size_t)2 * n * sizeof(float));
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_uv, uv.data(), uv.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_cap, cap.data(), cap.size() * sizeof(double), cudaMemcpyHostToDevice,
                        st);
  if (e == cudaSuccess) {
    hom_chain_kernel<<<(kCells + 127) / 128, 128, 0, st>>>(d_uv, d_cap, g, L, scaled_rho,
                                                           scaled_mu, d_hom);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    site_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_hom, d_cap, g, L, scaled_mu,
                                                            d_out, d_homf);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    const int64_t total = 4 * (int64_t)L * kPatches + kPatches;
    pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(
        d_out, d_homf, L, reinterpret_cast<float*>(site), reinterpret_cast<float*>(chunk));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    hom_m->resize((size_t)n);
    hom_c->resize((size_t)n);
    e = cudaMemcpyAsync(hom_m->data(), d_homf, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost,
                        st);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hom_c->data(), d_homf + n, (size_t)n * sizeof(float),
                        cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d_uv);
  cudaFree(d_cap);
  cudaFree(d_hom);
  cudaFree(d_out);
  cudaFree(d_homf);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *err = std::string("CUDA error: ") + cudaGetErrorString(e) + " (float64 table build)";
    return -1;
  }
  return 0;
}

}  // namespace gsmc
