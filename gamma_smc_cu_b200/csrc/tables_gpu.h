// Optional float64 GPU build of the scan tables (tables_gpu.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "tables.h"

namespace gsmc {

// Build the scan tables of L layers for (scaled_rho, scaled_mu) on the
// current device in float64 and write them, rounded to float32, into the
// device arrays site ([4][L][2450] patches) and chunk ([2450]
// patches of hom layer L - 1); the hom layers (float32) also go to the host
// vectors.  0 on success, else -1 with *err set.
int build_tables_gpu_f64(const FlowField& ff, int L, double scaled_rho, double scaled_mu,
                         float4* site, float4* chunk, std::vector<float>* hom_m,
                         std::vector<float>* hom_c, std::string* err);

}  // namespace gsmc
