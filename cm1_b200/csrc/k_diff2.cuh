// k_diff2.cuh -- arguments of the 2nd-order diffusion kernels (k_diff2.cu).
#pragma once
#include "cm1g_common.cuh"

namespace cm1g {

constexpr int kDiff2MaxScalars = 1 + 2 * 8;   // theta, up to 8 q arrays and 8 tracers

struct Diff2Args {
  float kdiff2;
  int bbc, tbc, momentum;
  float cgs1, cgs2, cgs3, cgt1, cgt2, cgt3;   // rf extrapolation to the bottom and top w-levels
  const float *ua, *va, *wa, *rho;
  float *uten, *vten, *wten;
  // scratch: rr, divx, t11, t22, t33, t12 (s-arrays); rf, t13, t23 (w-arrays)
  float *rr, *divx, *t11, *t22, *t33, *t12, *rf, *t13, *t23;
  int nsc;
  const float *s[kDiff2MaxScalars];
  float *sten[kDiff2MaxScalars];
};

void launch_diff2(const DGrid &g, const Diff2Args &a, cudaStream_t st, int64_t *nl);

}  // namespace cm1g
