// Flow-field grid, host table build and the scan's device table layout.
#pragma once

#include <cstddef>
#include <vector>

namespace gsmc {

// 51 x 50 grid over log10 mean x log10 CV (include/gamma_smc_cu/flow_field.h:6-8).
constexpr int kRows = 51;
constexpr int kCols = 50;
constexpr int kCells = kRows * kCols;
// Interpolation cells: the lower-left corner index is clamped to rows < 50 and
// columns < 49, so there are 50 x 49 distinct 2 x 2 patches.
constexpr int kPatchRows = kRows - 1;
constexpr int kPatchCols = kCols - 1;
constexpr int kPatches = kPatchRows * kPatchCols;

struct FlowField {
  float u[kCells];
  float v[kCells];
  float m_lo, m_hi, c_lo, c_hi;  // log10 bounds read from the file header
};

// Host tables in the reference's layout, [n_steps][2550] each.
enum HostTable {
  kMissingMean = 0, kMissingCv, kHomMean, kHomCv,
  kFwdHomMean, kFwdHomCv, kFwdHetMean, kFwdHetCv,
  kBwdHomMean, kBwdHomCv, kBwdHetMean, kBwdHetCv,
  kNumHostTables
};

struct HostLayers {
  int n_steps = 0;
  std::vector<float> t[kNumHostTables];
};

// Scan tables on the device: [direction][n_steps][hom, het][kPatches][8]
// floats (patches of pack_patches), so the hom and het patches of one
// layer are adjacent and a pair's
// het bit selects between them with one multiply-add.  Offsets below are in
// float4 units (two per patch).
enum ScanTable { kScanFwdHom = 0, kScanFwdHet, kScanBwdHom, kScanBwdHet, kScanTables };
constexpr int kPatchF4 = 2;                         // float4 per patch
constexpr int kHetF4 = kPatches * kPatchF4;         // hom -> het of one layer
constexpr int kLayerF4 = 2 * kHetF4;                // one layer (hom + het)
// Layer offsets are int32 float4 indices: cap the cache depth accordingly.
constexpr int kMaxCacheSteps = 100000;

inline size_t scan_layer_offset(int table, int layer, int L) {
  const int dir = table / 2, het = table % 2;
  return ((size_t)dir * L + layer) * kLayerF4 + (size_t)het * kHetF4;
}

// The entropy cap on log10 CV at log10 mean 0, 0.0008, ..., 4 in float64
// (the float64 table build's copy of the builder's float table).
const std::vector<double>& cv_cap_f64();

int load_flow_field(const char* path, FlowField* ff, char* err, size_t err_len);
void scaled_rates(double Ne, double mu, double rho, float* scaled_rho, float* scaled_mu);
void build_layers(const FlowField& ff, int n_steps, float scaled_rho, float scaled_mu,
                  int threads, HostLayers* out);
// 2450 patches of 8 floats (four m corners, then four c corners) from one
// [51 x 50] (m, c) layer.
void pack_patches(const float* m, const float* c, float* dst);
void build_scan_layout(const HostLayers& h, std::vector<float>* site,
                       std::vector<float>* chunk, int threads);

}  // namespace gsmc
