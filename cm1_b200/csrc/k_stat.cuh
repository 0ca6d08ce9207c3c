// k_stat.cuh -- job and output-program records of the device statistics
// package (k_stat.cu); built by the host (cm1g_api.cu) in statpack's order.
#pragma once
#include "cm1g_common.cuh"

namespace cm1g {

// point expressions of a job (per level: max/min kinds first, then sums)
enum StatKind {
  SK_FIELD = 0,  // a field (src, stag)
  SK_PRATE,      // 2-D surface precipitation rate (zero when absent)
  SK_PP,         // pressure perturbation prs - p00*pi0**cpdrd
  SK_DIV,        // rho0-weighted divergence
  SK_RH,         // relative humidity
  SK_THE,        // equivalent potential temperature
  SK_WSP,        // horizontal wind speed
  SK_WLEV,       // w interpolated to a height (k0, r1, r2)
  SK_PSFC,       // surface pressure extrapolated from levels 1-3
  SK_CFL,        // Courant number
  SK_VORT,       // vertical vorticity at level k0
  SK_CLOUD,      // sum of the cloud species (level max decides the cloud levels)
  SK_FIRST_SUM,
  SK_MASS = SK_FIRST_SUM,  // dry-air mass
  SK_TMOIS,      // total moisture
  SK_QMAS,       // mass of one species (qn)
  SK_TMF,        // upward and downward mass flux
  SK_MOE,        // momentum (3 sums)
  SK_ENER        // energy terms ek, ei, ep, le (4 sums)
};

// fields of SK_FIELD
enum StatSrc { SF_U = 0, SF_V, SF_W, SF_PPI, SF_THA, SF_PRS, SF_Q, SF_PT };

struct StatJob {
  int kind, src, stag, qn;
  int klo, nlev;      // levels klo .. klo+nlev-1
  int i0, ie, j0, je; // i-j range of one level
  int k0;             // fixed level of SK_WLEV / SK_VORT
  float r1, r2;       // interpolation weights of SK_WLEV
};

struct StatLev {
  float vmax, vmin;
  int imax, imin;     // first location in the level (linear index over the i-j range)
  double s[4];
};
// records: [job][level][chunk]

// output operations: one per rstat entry
enum StatOpKind {
  SO_HOST = 0,    // filled by the host (time, budgets)
  SO_ZERO,        // a constant 0 (maxmin2d of a zero field)
  SO_MAX, SO_MIN, // over the job's levels
  SO_LEVMAX, SO_LEVMIN,   // one level (k)
  SO_ZF_KMAX, SO_ZF_KMIN, SO_ZH_KMAX, SO_ZH_KMIN,   // height of the job's first max / min level
  SO_CFL, SO_VORT, SO_QCTOP, SO_QCBOT,
  SO_SUM,         // sum k of the job's levels; arg 1: x dx*dy*dz, 2: x dx x dy
  SO_ENER_TOTAL
};

struct StatOp {
  int op, job, k, arg;
};

struct StatFields {
  const float *ua, *va, *wa, *ppi, *tha, *prs, *rho, *qa, *pta, *prate;
  long qstride;       // elements between consecutive q / tracer arrays
};

struct StatConsts {
  float p00, eps, reps, rd, rv, cp, cv, cvv, cpl, cpi, cpdrd, g, lv1, ls1;
  float dtdx, dtdy, dtdz, cgs1, cgs2, cgs3, maxz;
  int ptype, imoist, numq, nqv, nql1, nql2, nx, ny;   // q indices 0-based (-1: none)
  unsigned cloudmask;                                 // bit n: q n is a cloud species
  const float *zh, *zf;                               // level heights (device, index k)
};

// chunks of one level of npl points (the first grid dimension of k_stat_levels)
int stat_chunks(int npl);
void launch_stat(const DGrid &g, const StatFields &f, const StatConsts &s, const StatJob *jobs, int njobs,
                 StatLev *lev, int maxlev, int nch, const StatOp *ops, int nops, float *rstat, cudaStream_t st,
                 int64_t *nl);

}  // namespace cm1g
