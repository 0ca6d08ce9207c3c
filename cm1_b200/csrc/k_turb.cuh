// k_turb.cuh -- arguments of the Smagorinsky LES kernels (k_turb.cu).
#pragma once
#include "cm1g_common.cuh"

namespace cm1g {

struct TurbArgs {
  float csm;                                  // Smagorinsky constant (uniform csm of turbsmag)
  float prinv;                                // 1/Prandtl number (turb.F:3421-3422)
  float cgs1, cgs2, cgs3, cgt1, cgt2, cgt3;   // rf extrapolation to the bottom and top w-levels
  int tconfig, bcturbs, bbc, tbc;
  const float *ua, *va, *wa, *rho, *tha;
  float *uten, *vten, *wten;
  // scalars: theta (s = th0 - th0r + tha), then numq q arrays and npt tracers
  const float *qa, *pta;
  float *thten, *qten, *ptten;
  int numq, npt;
  // scratch: rho*S_ij, then the stresses (s-shaped t11, t22, t33, t12 in
  // place; w-shaped t13, t23 formed from s13, s23); kmh, kmv (w-shaped)
  float *t11, *t22, *t33, *t12, *s13, *s23, *t13, *t23, *kmh, *kmv;
  // face coefficients of turbs' x/y fluxes, -0.125*(rho+rho)*(sum of khh)
  // (s-shaped, faces i or j = 1 .. n+1), shared by every scalar
  float *cx, *cy;
};

void launch_turbsmag(const DGrid &g, const TurbArgs &a, cudaStream_t st, int64_t *nl);

}  // namespace cm1g
