// lw_features.cuh -- per-layer inputs of the learned gas optics.
//
// The network maps the intensive state of one layer to the 140 g-point
// optical depths per molecule of dry air and the 140 Planck fractions.  Gas
// optical depth in RRTMG-LW is a sum of column amounts colamt = coldry * vmr
// times interpolated absorption coefficients (radlw_main.F90:838-858,
// 4023-6840), so taug / coldry depends only on intensive quantities:
//   x0 = ln p [hPa]          x1 = T [K]
//   x2 = ln h2o vmr          x3 = ln o3 vmr
//   x4 = co2 [ppmv]          x5 = ch4 [ppmv]        x6 = n2o [ppmv]
// (O2, CO and the CFCs enter at their prescribed constant mixing ratios.)
// Slot 7 of the feature vector is the constant 1 that carries the first
// layer's bias.  The same function feeds training-data extraction, the
// network kernel and the out-of-envelope test of the gas-optics kernel, so
// all three see bit-identical features.
#pragma once

#include <cmath>

namespace lw {

constexpr int SG_NFEAT = 8;      // 7 features + constant 1
constexpr int SG_NOUT = 280;     // 140 log(taug/coldry) + 140 Planck fractions
constexpr int SG_NOUTP = 288;    // padded: [0,140) tau, [140,144) 0, [144,284) frac, [284,288) 0
constexpr int SG_HID = 128;

// Normalisation and training envelope, float[SG_NORM_FLOATS] in device memory:
//   [0,8) input mean, [8,16) input std, [16,24) envelope low, [24,32) envelope high,
//   [32,320) output mean (padded layout), [320,608) output std.
constexpr int SG_IN_MEAN = 0, SG_IN_STD = 8, SG_ENV_LO = 16, SG_ENV_HI = 24;
constexpr int SG_OUT_MEAN = 32, SG_OUT_STD = 32 + SG_NOUTP;
constexpr int SG_NORM_FLOATS = 32 + 2 * SG_NOUTP;

__host__ __device__ inline void layer_features(double pavel, double tavel, double h2ovmr, double o3vmr,
                                               double co2, double ch4, double n2o, float* x) {
  x[0] = (float)log(pavel);
  x[1] = (float)tavel;
  x[2] = (float)log(fmax(h2ovmr, 1.0e-12));
  x[3] = (float)log(fmax(o3vmr, 1.0e-14));
  x[4] = (float)(co2 * 1.0e6);
  x[5] = (float)(ch4 * 1.0e6);
  x[6] = (float)(n2o * 1.0e6);
  x[7] = 1.0f;
}

// true when every feature lies inside the training envelope
__device__ __forceinline__ bool in_envelope(const float* x, const float* norm) {
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 7; ++j) ok = ok && x[j] >= __ldg(norm + SG_ENV_LO + j) && x[j] <= __ldg(norm + SG_ENV_HI + j);
  return ok;
}

// output column of g-point g (0..139): tau part, frac part
__host__ __device__ constexpr int sg_tau_col(int g) { return g; }
__host__ __device__ constexpr int sg_frac_col(int g) { return 144 + g; }

}  // namespace lw
