// C entry points over the reference's own table builder, for the oracle only.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the reference's unmodified src/flow_field.cpp (read in place from a
// reference checkout) into oracle/_ref/libref_tables.so, so the tests can pin
// the oracle's restated builder against the reference's compiled builder.
// Wraps load_flow_field (src/flow_field.cpp:8-54) and build_flow_field_cache
// (src/flow_field.cpp:205-388); table order matches oracle_build_tables.
#include <cstring>

#include "gamma_smc_cu/flow_field.h"

extern "C" int ref_load_flow_field(const char* path, float* u, float* v,
                                   float* bounds) {
  FlowFieldData ff;
  if (!load_flow_field(path, ff)) return -1;
  std::memcpy(u, ff.u, sizeof(ff.u));
  std::memcpy(v, ff.v, sizeof(ff.v));
  bounds[0] = ff.mean_log10_min;
  bounds[1] = ff.mean_log10_max;
  bounds[2] = ff.cv_log10_min;
  bounds[3] = ff.cv_log10_max;
  return 0;
}

extern "C" void ref_build_tables(const float* u, const float* v,
                                 const float* bounds, int n_steps,
                                 float scaled_rho, float scaled_mu, float* out) {
  FlowFieldData ff;
  std::memcpy(ff.u, u, sizeof(ff.u));
  std::memcpy(ff.v, v, sizeof(ff.v));
  ff.mean_log10_min = bounds[0];
  ff.mean_log10_max = bounds[1];
  ff.cv_log10_min = bounds[2];
  ff.cv_log10_max = bounds[3];
  FlowFieldCache c = build_flow_field_cache(ff, n_steps, scaled_rho, scaled_mu);
  const float* src[12] = {c.missing_mean,      c.missing_cv,
                          c.mean,              c.cv,
                          c.fwd_hom_site_mean, c.fwd_hom_site_cv,
                          c.fwd_het_site_mean, c.fwd_het_site_cv,
                          c.bwd_hom_site_mean, c.bwd_hom_site_cv,
                          c.bwd_het_site_mean, c.bwd_het_site_cv};
  const size_t n = (size_t)n_steps * FF_GRID;
  for (int t = 0; t < 12; ++t) std::memcpy(out + t * n, src[t], n * sizeof(float));
  free_flow_field_cache(c);
}
