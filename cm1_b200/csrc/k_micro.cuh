// k_micro.cuh -- arguments of the Kessler microphysics kernels (k_micro.cu).
#pragma once
#include "cm1g_common.cuh"

namespace cm1g {

// constants of constants.F:65-175 that the Kessler routines read
struct MicroConsts {
  float eps, reps, rd, rv, cp, cv, cpv, cvv, cpl, cpi;
  float lv1, lv2, cpdcv, rovcp, rddcv, cpdrd, p00, rp00;
};

struct MicroArgs {
  float *th3d, *pp3d, *prs, *rho;
  float *qv, *qc, *qr;
  float *vr;              // fall speed of rain (s-array scratch)
  float *rain, *prate;    // (ib:ie,jb:je)
  int *err;               // set to 1 when satadj does not converge in 100 iterations
  float dt, converge;     // converge = 2*tsmall (satadj with nrk = 4)
  int eqtset;
  MicroConsts c;
};

// per-level chunk count of k_mp_point's budget partials
int mp_chunks(const DGrid &g);
// part: 5 x nk x mp_chunks doubles; colbud: 2 x ni x nj doubles; qb: the
// seven FP64 budgets (tcond, tevac, tauto, taccr, tevar, train, erain)
void launch_kessler(const DGrid &g, const MicroArgs &a, double *part, double *colbud, double *qb, cudaStream_t st,
                    int64_t *nl);

}  // namespace cm1g
