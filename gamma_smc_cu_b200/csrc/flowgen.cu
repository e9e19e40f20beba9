// Flow-field generation on the GPU in float64.
//
// The flow field is the 51 x 50 grid of (u, v) drift coefficients of the
// Gamma-SMC state (log10 mean, log10 CV) per unit of scaled time.  The
// reference computes it with numpy/scipy, one grid cell after another
// (python/gamma_smc_cu/demographic.py:17-208): for the Gamma(alpha, beta) of
// each cell it evaluates the change of the coalescence-time distribution
// after one recombination ("distribution difference", :17-44 for constant Ne,
// :47-130 for piecewise-constant Ne) on a 1001-point time grid (:133-143),
// and least-squares fits it with the derivatives of the Gamma density with
// respect to log10 alpha and log10 beta (:178-197).
//
// Here one CTA fits one cell: its threads evaluate the time points in
// parallel (regularised incomplete gamma functions, digamma and the 1F1
// needed by the beta ~ 1 cells), and the two-column least-squares problem is
// solved by Gram-Schmidt with one reorthogonalisation (numerically as stable
// as the SVD solver the reference calls, for a full-rank 2-column system).
//
// Special functions, from published methods:
//   * P(a, x), Q(a, x): power series for x < a + 1, Lentz's continued
//     fraction otherwise (Press et al., Numerical Recipes, 3rd ed., 6.2);
//   * P^-1(a, p): Halley's method from the Wilson-Hilferty / small-a starting
//     values of the same section;
//   * digamma: upward recurrence to x >= 10, then the Stirling-type
//     asymptotic series with Bernoulli-number coefficients;
//   * 1F1(a; a+1; z) = a * sum_n z^n / (n! (a + n)), summed in log scale.
// lgamma, exp, log, sqrt, pow are CUDA's double-precision functions.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "flowgen.h"

namespace gsmc {
namespace {

constexpr double kEps = 1e-16;
constexpr double kTiny = 1e-300;
constexpr int kMaxIter = 200000;
constexpr double kLn10 = 2.302585092994045684;
constexpr double kLogMax = 709.782712893384;  // log(DBL_MAX)

// log(x^a e^-x / Gamma(a)).  For a >= 10 it is written as a (log1p(y) - y) +
// log(a / 2 pi) / 2 - (Stirling correction of lgamma(a)), y = x/a - 1, which
// avoids the cancellation of a log x against lgamma(a) for large a
// (Temme's form, as in DiDonato & Morris, ACM TOMS 12 (1986) 377).
__device__ double log_prefactor(double a, double x) {
  if (a < 10.0) return -x + a * log(x) - lgamma(a);
  const double y = (x - a) / a;
  double l1;  // log1p(y) - y
  if (fabs(y) < 0.1) {
    double s = 0.0, pw = -y * y;
    for (int k = 2; k < 60; ++k) {
      const double term = pw / k;
      s += term;
      pw *= -y;
      if (fabs(term) < 1e-17 * fabs(s)) break;
    }
    l1 = s;
  } else {
    l1 = log1p(y) - y;
  }
  const double ia = 1.0 / a, ia2 = ia * ia;
  // lgamma(a) - ((a - 1/2) log a - a + log(2 pi) / 2), Bernoulli series
  const double corr = ia * (1.0 / 12 - ia2 * (1.0 / 360 - ia2 * (1.0 / 1260 - ia2 * (1.0 / 1680 -
                      ia2 / 1188))));
  return a * l1 + 0.5 * log(a / (2.0 * 3.14159265358979323846)) - corr;
}

// Regularised lower / upper incomplete gamma; *upper selects Q.
__device__ double inc_gamma(double a, double x, bool upper) {
  if (!(x > 0.0)) return upper ? 1.0 : 0.0;
  if (!isfinite(x)) return upper ? 0.0 : 1.0;
  const double lp = log_prefactor(a, x);
  if (x < a + 1.0) {
    double ap = a, del = 1.0 / a, sum = del;
    for (int n = 0; n < kMaxIter; ++n) {
      ap += 1.0;
      del *= x / ap;
      sum += del;
      if (fabs(del) < fabs(sum) * kEps) break;
    }
    const double p = sum * exp(lp);
    return upper ? 1.0 - p : p;
  }
  double b = x + 1.0 - a, c = 1.0 / kTiny, d = 1.0 / b, h = d;
  for (int i = 1; i < kMaxIter; ++i) {
    const double an = -i * (i - a);
    b += 2.0;
    d = an * d + b;
    if (fabs(d) < kTiny) d = kTiny;
    c = b + an / c;
    if (fabs(c) < kTiny) c = kTiny;
    d = 1.0 / d;
    const double del = d * c;
    h *= del;
    if (fabs(del - 1.0) < kEps) break;
  }
  const double q = exp(lp) * h;
  return upper ? q : 1.0 - q;
}

// x with P(a, x) = p, 0 < p < 1 (Halley's iteration, stopped when the step
// is below 1e-15 x or after 100 steps); NaN only if it leaves the positive
// reals' finite range.
__device__ double inv_inc_gamma(double a, double p) {
  const double a1 = a - 1.0;
  double x;
  if (a > 1.0) {
    const double pp = p < 0.5 ? p : 1.0 - p;
    const double t = sqrt(-2.0 * log(pp));
    x = (2.30753 + t * 0.27061) / (1.0 + t * (0.99229 + t * 0.04481)) - t;
    if (p < 0.5) x = -x;
    x = fmax(1e-3, a * pow(1.0 - 1.0 / (9.0 * a) - x / (3.0 * sqrt(a)), 3.0));
  } else {
    const double t = 1.0 - a * (0.253 + a * 0.12);
    x = p < t ? pow(p / t, 1.0 / a) : 1.0 - log(1.0 - (p - t) / (1.0 - t));
  }
  for (int j = 0; j < 100; ++j) {
    if (x <= 0.0) return 0.0;
    const double err = inc_gamma(a, x, false) - p;
    const double dens = exp(log_prefactor(a, x) - log(x));  // Gamma(a, 1) density at x
    const double u = err / dens;
    const double step = u / (1.0 - 0.5 * fmin(1.0, u * (a1 / x - 1.0)));
    x -= step;
    if (x <= 0.0) x = 0.5 * (x + step);
    if (fabs(step) < 1e-15 * x) break;
  }
  return isfinite(x) ? x : nan("");
}

__device__ double digamma(double x) {
  double r = 0.0;
  while (x < 10.0) {
    r -= 1.0 / x;
    x += 1.0;
  }
  const double f = 1.0 / (x * x);
  // -1/12, 1/120, -1/252, 1/240, -1/132, 691/32760, -1/12 (B_2k / 2k)
  const double s = f * (-1.0 / 12 + f * (1.0 / 120 + f * (-1.0 / 252 + f * (1.0 / 240 +
                   f * (-1.0 / 132 + f * (691.0 / 32760 + f * (-1.0 / 12)))))));
  return r + log(x) - 0.5 / x + s;
}

// log 1F1(a; a+1; z); +inf when the value is beyond double range.
__device__ double log_hyp1f1_a_a1(double a, double z) {
  // terms T_n = z^n / (n! (a + n)); scaled by exp(-shift) to stay in range
  double logsum = -INFINITY;
  double lt = -log(a);      // log |T_0|
  double sum = 0.0, shift = lt;
  const bool neg = z < 0.0;
  const double lz = log(fabs(z));
  for (int n = 0; n < kMaxIter; ++n) {
    if (n > 0) lt += lz - log((double)n) + log((a + n - 1.0) / (a + n));
    if (z == 0.0 && n > 0) break;
    const double sign = (neg && (n & 1)) ? -1.0 : 1.0;
    if (lt - shift > 600.0) {  // rescale the running sum
      sum *= exp(shift - lt);
      shift = lt;
    }
    const double term = sign * exp(lt - shift);
    sum += term;
    if (n > 0 && fabs(term) < 1e-17 * fabs(sum) && n > fabs(z)) break;
  }
  if (!(sum > 0.0)) return -INFINITY;
  logsum = log(a) + shift + log(sum);
  return logsum;
}

// numpy's exp(where(x > -700, x, -700))
__device__ double clamp_exp(double x) { return exp(x > -700.0 ? x : -700.0); }

// Distribution difference at time t (constant Ne), demographic.py:17-44.
__device__ double dist_diff_const(double t, double alpha, double beta, double lgam_a,
                                  double lgam_a1) {
  t = fmax(t, 1e-15);
  const double bm1 = beta - 1.0, bp1 = beta + 1.0;
  double term_m;
  if (bm1 > 1e-10) {
    const double log_r = alpha * (log(beta) - log(bm1));
    term_m = exp(-t + log_r) * inc_gamma(alpha, bm1 * t, false);
  } else {
    const double base = -t + alpha * log(t * beta) - lgam_a1;
    const double lh = log_hyp1f1_a_a1(alpha, -bm1 * t);
    // scipy's 1F1 overflows to inf beyond double range; the reference then
    // maps the non-finite term to 0
    term_m = lh > kLogMax ? 0.0 : exp(base + lh);
    if (!isfinite(term_m)) term_m = 0.0;
  }
  const double log_r_p = alpha * (log(beta) - log(bp1));
  const double term_p = exp(-t + log_r_p) * inc_gamma(alpha, bp1 * t, false);
  double res = term_m - term_p;
  const double gpdf = clamp_exp(alpha * log(beta) - lgam_a + (alpha - 1.0) * log(t) - beta * t);
  const double gsf = inc_gamma(alpha, beta * t, true);
  res += (exp(-2.0 * t) / 2.0 - 0.5 - t) * gpdf;
  res += (1.0 - exp(-2.0 * t)) * gsf;
  return res;
}

// Distribution difference for piecewise-constant N(t), demographic.py:47-130.
__device__ double dist_diff_demo(double t, double alpha, double beta, double lgam_a,
                                 const FlowGenEpochs& ep) {
  t = fmax(t, 1e-15);
  const int M = ep.n;
  double I_plus = 0.0, I_minus = 0.0;
  for (int k = 0; k < M; ++k) {
    const double a_k = ep.t_bounds[k];
    const double b_k_max = k < M - 1 ? ep.t_bounds[k + 1] : 1e15;
    const double b_k = fmin(t, b_k_max);
    if (!(t > a_k + 1e-15)) break;  // epochs start in increasing order
    const double lam_k = ep.lam[k], L_k = ep.L_bounds[k], t_k = ep.t_bounds[k];
    const double c_plus = beta - lam_k;
    const double log_coeff_plus = L_k - lam_k * t_k;
    if (fabs(c_plus) > 1e-10 && c_plus > 0.0) {
      const double log_scale = log_coeff_plus + alpha * (log(beta) - log(c_plus));
      if (log_scale > -500.0) {
        const double gi_b = inc_gamma(alpha, c_plus * fmax(b_k, 1e-30), false);
        const double gi_a = a_k > 1e-15 ? inc_gamma(alpha, c_plus * fmax(a_k, 1e-30), false) : 0.0;
        I_plus += exp(log_scale) * (gi_b - gi_a);
      }
    } else if (fabs(c_plus) <= 1e-10 && alpha > 0.0) {
      const double coeff = exp(log_coeff_plus + alpha * log(beta) - lgam_a);
      const double b_term = pow(fmax(b_k, 1e-30), alpha);
      const double a_term = a_k > 1e-15 ? pow(fmax(a_k, 1e-30), alpha) : 0.0;
      I_plus += coeff * (b_term - a_term) / alpha;
    }
    const double c_minus = beta + lam_k;
    const double log_scale_m = -L_k + lam_k * t_k + alpha * (log(beta) - log(c_minus));
    if (log_scale_m > -500.0) {
      const double gi_b = inc_gamma(alpha, c_minus * fmax(b_k, 1e-30), false);
      const double gi_a = a_k > 1e-15 ? inc_gamma(alpha, c_minus * fmax(a_k, 1e-30), false) : 0.0;
      I_minus += exp(log_scale_m) * (gi_b - gi_a);
    }
  }
  // epoch of t: last start <= t (searchsorted 'right' - 1, clipped)
  int e = 0;
  while (e + 1 < M && ep.t_bounds[e + 1] <= t) ++e;
  const double Lam = ep.L_bounds[e] + ep.lam[e] * (t - ep.t_bounds[e]);
  const double gpdf = clamp_exp(alpha * log(beta) - lgam_a + (alpha - 1.0) * log(t) - beta * t);
  const double gsf = inc_gamma(alpha, beta * t, true);
  double res = exp(-Lam) * (I_plus - I_minus);
  res += (exp(-2.0 * Lam) / 2.0 - 0.5 - Lam) * gpdf;
  res += (1.0 - exp(-2.0 * Lam)) * gsf;
  return res;
}

// Block-wide sums of up to three values (all threads get the results).
__device__ void block_sum3(double& a, double& b, double& c, double* red) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, d);
    b += __shfl_xor_sync(0xffffffffu, b, d);
    c += __shfl_xor_sync(0xffffffffu, c, d);
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[3 * w] = a;
    red[3 * w + 1] = b;
    red[3 * w + 2] = c;
  }
  __syncthreads();
  a = b = c = 0.0;
  for (int i = 0; i < nw; ++i) {  // same order in every thread
    a += red[3 * i];
    b += red[3 * i + 1];
    c += red[3 * i + 2];
  }
}

__device__ double block_max(double v, double* red) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, d));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  v = -INFINITY;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) v = fmax(v, red[i]);
  return v;
}

constexpr int kGenThreads = 256;

// One CTA per grid cell (row i = blockIdx.y, column j = blockIdx.x).
__global__ void __launch_bounds__(kGenThreads) flow_field_kernel(const FlowGenArgs a,
                                                                 const FlowGenEpochs ep) {
  extern __shared__ double sm[];
  const int n_t = 2 * a.n_steps + 1;
  double* times = sm;            // [n_t]
  double* col_a = times + n_t;   // d_la, then the orthogonalised column
  double* col_b = col_a + n_t;   // d_lb
  double* rhs = col_b + n_t;     // delta * sqrt(dt)
  double* wcol = rhs + n_t;      // second column after Gram-Schmidt
  __shared__ double red[3 * (kGenThreads / 32)];
  __shared__ double s_tmax;
  __shared__ int s_skip;
  const int cell = blockIdx.y * a.cv_n + blockIdx.x;
  const double alpha = a.alpha[cell], beta = a.beta[cell];
  double* u_out = a.u + cell;
  double* v_out = a.v + cell;
  if (threadIdx.x == 0) {
    s_skip = (alpha < 1e-8 || beta < 1e-8 || alpha > 1e8) ? 1 : 0;
    double tm = 0.0;
    if (!s_skip) {
      tm = inv_inc_gamma(alpha, 1.0 - 1e-3) / beta;
      if (!isfinite(tm)) tm = alpha / beta * 5.0;
      tm = fmax(tm, 0.1);
    }
    s_tmax = tm;
    *u_out = 0.0;
    *v_out = 0.0;
  }
  __syncthreads();
  if (s_skip) return;
  // time grid: linspace(1e-10, t_max, n+1) then n steps of t_max_exp/(n-1)
  // (numpy's i * step + start, no fused multiply-add)
  const int n = a.n_steps;
  const double tmax = s_tmax;
  const double step1 = (tmax - 1e-10) / (double)n;
  const double step2 = a.t_max_exp / (double)(n > 1 ? n - 1 : 1);
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
    double t;
    if (k < n)
      t = __dadd_rn(__dmul_rn((double)k, step1), 1e-10);
    else if (k == n)
      t = tmax;
    else
      t = __dadd_rn(tmax, __dmul_rn((double)(k - n), step2));
    times[k] = t;
  }
  __syncthreads();
  const double lgam_a = lgamma(alpha), lgam_a1 = lgamma(alpha + 1.0);
  const double dig = digamma(alpha);
  const double lb = log(beta);
  double gmax_local = -INFINITY;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
    const double t = times[k];
    const double sq = k + 1 < n_t ? sqrt(times[k + 1] - t) : 0.0;
    const double delta = ep.n > 0 ? dist_diff_demo(t, alpha, beta, lgam_a, ep)
                                  : dist_diff_const(t, alpha, beta, lgam_a, lgam_a1);
    const double lt = log(fmax(t, 1e-30));
    const double gpdf = clamp_exp(alpha * lb - lgam_a + (alpha - 1.0) * lt - beta * t);
    col_a[k] = gpdf * (lb - dig + lt) * sq * alpha / kLn10;
    col_b[k] = gpdf * (alpha / beta - t) * sq * beta / kLn10;
    rhs[k] = delta * sq;
    wcol[k] = gpdf;  // kept for the row selection below
    gmax_local = fmax(gmax_local, gpdf);
  }
  const double gmax = block_max(gmax_local, red);
  // rows with gpdf > max * 1e-12 take part; a non-finite value in them makes
  // the reference's solver fail and leave the cell at 0
  double n_good = 0.0, bad = 0.0, dummy = 0.0;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
    const bool good = wcol[k] > gmax * 1e-12;
    if (good) {
      n_good += 1.0;
      if (!isfinite(col_a[k]) || !isfinite(col_b[k]) || !isfinite(rhs[k])) bad += 1.0;
    } else {
      col_a[k] = col_b[k] = rhs[k] = 0.0;  // excluded rows add nothing below
    }
  }
  block_sum3(n_good, bad, dummy, red);
  if (n_good < 3.0 || bad > 0.0) return;
  // Gram-Schmidt with one reorthogonalisation: A = [a1 a2] = Q R
  double s11 = 0.0, s12 = 0.0, s1b = 0.0;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
    s11 += col_a[k] * col_a[k];
    s12 += col_a[k] * col_b[k];
    s1b += col_a[k] * rhs[k];
  }
  block_sum3(s11, s12, s1b, red);
  const double r11 = sqrt(s11);
  if (!(r11 > 0.0)) return;
  double r12 = s12 / r11;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x)
    wcol[k] = col_b[k] - (r12 / r11) * col_a[k];
  double t12 = 0.0, z0 = 0.0, z1 = 0.0;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) t12 += col_a[k] * wcol[k];
  block_sum3(t12, z0, z1, red);
  const double r12b = t12 / r11;
  r12 += r12b;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) wcol[k] -= (r12b / r11) * col_a[k];
  double s22 = 0.0, s2b = 0.0, z2 = 0.0;
  for (int k = threadIdx.x; k < n_t; k += blockDim.x) {
    s22 += wcol[k] * wcol[k];
    s2b += wcol[k] * rhs[k];
  }
  block_sum3(s22, s2b, z2, red);
  const double r22 = sqrt(s22);
  if (threadIdx.x == 0) {
    double x1 = 0.0, x0 = 0.0;
    if (r22 > 0.0) {
      x1 = (s2b / r22) / r22;
      x0 = (s1b / r11 - r12 * x1) / r11;
    } else {
      x0 = (s1b / r11) / r11;  // rank one: the single-column fit
    }
    *u_out = (x0 - x1) / a.calibration;
    *v_out = (-0.5 * x0) / a.calibration;
  }
}

}  // namespace

size_t flow_field_smem_bytes(int n_steps) { return (size_t)5 * (2 * n_steps + 1) * sizeof(double); }

cudaError_t launch_flow_field(const FlowGenArgs& a, const FlowGenEpochs& ep, cudaStream_t stream) {
  const size_t smem = flow_field_smem_bytes(a.n_steps);
  cudaError_t e = cudaFuncSetAttribute(flow_field_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)a.cv_n, (unsigned)a.mean_n);
  flow_field_kernel<<<grid, kGenThreads, smem, stream>>>(a, ep);
  return cudaGetLastError();
}

}  // namespace gsmc
