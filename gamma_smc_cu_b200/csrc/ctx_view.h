// Read-only view of a context's resident device data, for entry points that
// live outside capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gsmc_b200.h"
#include "scan.h"

namespace gsmc {

struct CtxView {
  int device;
  int64_t n_haps;
  int64_t n_sites;
  const ulonglong2* geno;
  const SiteCode* code;
  const float4* site_tab;
  const float4* chunk_tab;
  int L;
  float ne;
};

// Fills *out; false for a null context.
bool ctx_view(const gsmc_ctx* ctx, CtxView* out);

// Records `msg` as this thread's gsmc_last_error() and returns `code`.
int set_error(int code, const char* msg);

}  // namespace gsmc
