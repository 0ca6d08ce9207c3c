// k_stat.cu -- the statistics package (statpack.F:10-658) on the device.
//
// statpack evaluates a fixed list of domain statistics: extrema of fields
// and of derived quantities (maxmin / maxmin2d, maxmin.F:5-228), the CFL
// number (calccfl, misclibs.F:2584-2718), vertical vorticity maxima
// (vertvort, misclibs.F:2424-2576), cloud top and base (cloud,
// misclibs.F:2344-2416) and FP64 budgets (calcmass, totmois, totq, calcener,
// calcmoe, tmf; misclibs.F:3134-3636).  Every one of them is a reduction over
// the points of one model level followed by a reduction over the levels, so
// the device form is two launches:
//
//   k_stat_levels  one block per (job, level, chunk of 4096 points): the
//                  block evaluates the job's point expression (a constant of
//                  an unrolled loop) and reduces its chunk to the max and
//                  min (value and first location in the reference's loop
//                  order) and up to four FP64 sums;
//   k_stat_finish  one warp per rstat entry: it combines the chunks and
//                  levels with the reference's tie rule (the value of the
//                  strict comparisons from the same initial values, the
//                  first level holding it) and FP64 sums, and writes rstat
//                  in statpack's order.
//
// The host copies rstat back with one small device-to-host copy.  Point
// expressions keep the reference's operand order and kinds (binary32 where
// the Fortran is real, binary64 where it declares double precision); the
// library is compiled with --fmad=false.
#include "cm1g_common.cuh"
#include "k_stat.cuh"

namespace cm1g {

__device__ __forceinline__ long st_off(const DGrid &g, int stag, int i, int j, int k) {
  return stag == 2 ? iU(g, i, j, k) : stag == 3 ? iV(g, i, j, k) : iS(g, i, j, k);
}

// rslf (cm1libs.F:16-62): saturation mixing ratio over liquid
__device__ __forceinline__ float st_rslf(float p, float t, const StatConsts &s) {
  if (s.ptype == 4) return 380.00f * expf(17.2693882f - 4097.8531f / (t - 35.86f)) / p;
  float esl = 611.2f * expf(17.67f * (t - 273.15f) / (t - 29.65f));
  esl = fminf(esl, p * 0.5f);
  return s.eps * esl / (p - esl);
}

// relative humidity as statpack.F:364-371 forms it
__device__ __forceinline__ float st_rh(const DGrid &g, const StatFields &f, const StatConsts &s, long o, int k,
                                       float *tx_out) {
  const float tx = (LDG(&g.th0[k]) + LDG(&f.tha[o])) * (LDG(&g.pi0[k]) + LDG(&f.ppi[o]));
  const float prs = LDG(&f.prs[o]);
  const float qvs = st_rslf(prs, tx, s);
  const float qv = LDG(&f.qa[(long)s.nqv * f.qstride + o]);
  if (tx_out) *tx_out = tx;
  return qv * (1.0f + qvs * s.reps) / (qvs * (1.0f + qv * s.reps));
}

// value of a max/min job at (i, j, k)
__device__ __forceinline__ float st_value(const DGrid &g, const StatJob &jb, const StatFields &f, const StatConsts &s,
                                          int i, int j, int k, float aux) {
  switch (jb.kind) {
    case SK_FIELD: {
      const float *a = jb.src == SF_U ? f.ua : jb.src == SF_V ? f.va : jb.src == SF_W ? f.wa
                     : jb.src == SF_PPI ? f.ppi : jb.src == SF_THA ? f.tha : jb.src == SF_PRS ? f.prs
                     : jb.src == SF_Q ? f.qa + (long)jb.qn * f.qstride : f.pta + (long)jb.qn * f.qstride;
      return LDG(&a[st_off(g, jb.stag, i, j, k)]);
    }
    case SK_PRATE:
      return f.prate ? LDG(&f.prate[i2(g, i, j)]) : 0.0f;
    case SK_PP:   // statpack.F:236-242, aux = p00*(pi0**cpdrd) of the level
      return LDG(&f.prs[iS(g, i, j, k)]) - aux;
    case SK_DIV: {  // statpack.F:297-309 (axisymm = 0)
      const long o = iS(g, i, j, k), ou = iU(g, i, j, k), ov = iV(g, i, j, k);
      const float r0 = LDG(&g.rho0[k]);
      const float ta = 0.5f * ((r0 + r0) * LDG(&f.ua[ou + 1]) - (r0 + r0) * LDG(&f.ua[ou])) * g.rdx *
                       LDG(&g.uh[i - g.ib]);
      const float tb = 0.5f * ((r0 + r0) * LDG(&f.va[ov + g.NI]) - (r0 + r0) * LDG(&f.va[ov])) * g.rdy *
                       LDG(&g.vh[j - g.jb]);
      const long pl = (long)g.NI * g.NJ;
      const float tc = 0.5f * ((r0 + LDG(&g.rho0[k + 1])) * LDG(&f.wa[o + pl]) -
                               (r0 + LDG(&g.rho0[k - 1])) * LDG(&f.wa[o])) * g.rdz * LDG(&g.mh[k]);
      return (ta + tb) + tc;
    }
    case SK_RH:
      return st_rh(g, f, s, iS(g, i, j, k), k, nullptr);
    case SK_THE: {  // calcthe (misclibs.F:2300-2336), cpm = cp, l0 = 2.555e6
      const long o = iS(g, i, j, k);
      float tx;
      const float rh = st_rh(g, f, s, o, k, &tx);
      const float qv = LDG(&f.qa[(long)s.nqv * f.qstride + o]);
      const float cpm = s.cp;
      return tx * powf(s.p00 * (1.0f + qv * s.reps) / LDG(&f.prs[o]), s.rd / cpm) *
             powf(rh, -(qv * s.rv / cpm)) * expf(2.555e6f * qv / (cpm * tx));
    }
    case SK_WSP: {  // statpack.F:437-441 (umove = vmove = 0)
      const long ou = iU(g, i, j, k), ov = iV(g, i, j, k);
      const float a = 0.0f + 0.5f * (LDG(&f.ua[ou]) + LDG(&f.ua[ou + 1]));
      const float b = 0.0f + 0.5f * (LDG(&f.va[ov]) + LDG(&f.va[ov + g.NI]));
      return sqrtf(a * a + b * b);
    }
    case SK_WLEV: {  // statpack.F:180-188; jb.k0 = nkm
      const long o = iS(g, i, j, jb.k0);
      return jb.r1 * LDG(&f.wa[o]) + jb.r2 * LDG(&f.wa[o + (long)g.NI * g.NJ]);
    }
    case SK_PSFC: {  // statpack.F:425-430
      const long o = iS(g, i, j, 1), pl = (long)g.NI * g.NJ;
      return (s.cgs1 * LDG(&f.prs[o]) + s.cgs2 * LDG(&f.prs[o + pl])) + s.cgs3 * LDG(&f.prs[o + 2 * pl]);
    }
    case SK_CFL: {  // calccfl (misclibs.F:2618-2665)
      const long o = iS(g, i, j, k), ou = iU(g, i, j, k), ov = iV(g, i, j, k);
      const float cu = (LDG(&f.ua[ou]) + LDG(&f.ua[ou + 1])) * s.dtdx * LDG(&g.uh[i - g.ib]);
      const float cv = (LDG(&f.va[ov]) + LDG(&f.va[ov + g.NI])) * s.dtdy * LDG(&g.vh[j - g.jb]);
      const float cw = (LDG(&f.wa[o]) + LDG(&f.wa[o + (long)g.NI * g.NJ])) * s.dtdz * LDG(&g.mh[k]);
      if (s.nx > 1 && s.ny > 1) return sqrtf((cu * cu + cv * cv) + cw * cw);
      if (s.nx > 1) return sqrtf(cu * cu + cw * cw);
      return sqrtf(cv * cv + cw * cw);
    }
    case SK_VORT: {  // vertvort (misclibs.F:2497-2505), jb.k0 = the level
      const int kk = jb.k0;
      const float dv = LDG(&f.va[iV(g, i, j, kk)]) - LDG(&f.va[iV(g, i - 1, j, kk)]);
      const float du = LDG(&f.ua[iU(g, i, j, kk)]) - LDG(&f.ua[iU(g, i, j - 1, kk)]);
      return dv * g.rdx * LDG(&g.uf[i - g.ib]) - du * g.rdy * LDG(&g.vf[j - g.jb]);
    }
    case SK_CLOUD: {  // statpack.F:406-418: sum of the cloud species
      const long o = iS(g, i, j, k);
      float q = 0.0f;
      for (int n = 0; n < s.numq; n++)
        if (s.cloudmask & (1u << n)) q = q + LDG(&f.qa[(long)n * f.qstride + o]);
      return q;
    }
    default:
      return 0.0f;
  }
}

// FP64 sums of the budget jobs at (i, j, k)
__device__ __forceinline__ void st_sums(const DGrid &g, const StatJob &jb, const StatFields &f, const StatConsts &s,
                                        int i, int j, int k, double *acc) {
  const long o = iS(g, i, j, k);
  const float rho = LDG(&f.rho[o]);
  const float ruh = LDG(&g.ruh[i - g.ib]), rvh = LDG(&g.rvh[j - g.jb]), rmh = LDG(&g.rmh[k]);
  float qv = 0.0f, ql = 0.0f;
  if (jb.kind == SK_TMOIS || jb.kind == SK_ENER || jb.kind == SK_MOE) {
    if (s.imoist) {
      qv = LDG(&f.qa[(long)s.nqv * f.qstride + o]);
      for (int n = s.nql1; n >= 0 && n <= s.nql2; n++) ql = ql + LDG(&f.qa[(long)n * f.qstride + o]);
    }
  }
  switch (jb.kind) {
    case SK_MASS:   // calcmass (misclibs.F:3160-3166)
      acc[0] = acc[0] + (double)(rho * ruh * rvh * rmh);
      break;
    case SK_TMOIS:  // totmois (misclibs.F:3224-3230), qi = 0
      acc[0] = acc[0] + (double)(rho * ((qv + ql) + 0.0f) * ruh * rvh * rmh);
      break;
    case SK_QMAS:   // totq (misclibs.F:3297-3303)
      acc[0] = acc[0] + (double)(rho * LDG(&f.qa[(long)jb.qn * f.qstride + o]) * ruh * rvh * rmh);
      break;
    case SK_TMF: {  // tmf (misclibs.F:3588-3596): mf is double precision, formed in binary32
      const double mf = (double)(rho * 0.5f * (LDG(&f.wa[o]) + LDG(&f.wa[o + (long)g.NI * g.NJ])) * ruh * rvh);
      acc[0] = acc[0] + fmax(mf, 0.0);
      acc[1] = acc[1] + fmin(mf, 0.0);
      break;
    }
    case SK_MOE: {  // calcmoe (misclibs.F:3488-3502), umove = vmove = 0, vr = 0
      const double qtot = (double)((qv + ql) + 0.0f);
      const double tem = (double)(ruh * rvh * rmh);
      const long ou = iU(g, i, j, k), ov = iV(g, i, j, k);
      const double rt = (double)rho * tem * (1.0 + qtot);
      acc[0] = acc[0] + rt * (double)(0.0f + 0.5f * (LDG(&f.ua[ou]) + LDG(&f.ua[ou + 1])));
      acc[1] = acc[1] + rt * (double)(0.0f + 0.5f * (LDG(&f.va[ov]) + LDG(&f.va[ov + g.NI])));
      acc[2] = (acc[2] + rt * (double)(0.5f * (LDG(&f.wa[o]) + LDG(&f.wa[o + (long)g.NI * g.NJ])))) -
               (double)rho * tem * (double)ql * 0.0;
      break;
    }
    case SK_ENER: {  // calcener (misclibs.F:3374-3393), umove = vmove = 0, qi = 0, vr = 0
      const double tem = (double)(ruh * rvh * rmh);
      const long ou = iU(g, i, j, k), ov = iV(g, i, j, k), pl = (long)g.NI * g.NJ;
      const float u1 = LDG(&f.ua[ou]), u2 = LDG(&f.ua[ou + 1]), v1 = LDG(&f.va[ov]), v2 = LDG(&f.va[ov + g.NI]);
      const float w1 = LDG(&f.wa[o]), w2 = LDG(&f.wa[o + pl]);
      const double ww = (double)(0.5f * (w1 + w2));
      const double qtot = (double)((qv + ql) + 0.0f);
      const float ke = (0.5f * (u1 * u1 + u2 * u2) + 0.5f * (v1 * v1 + v2 * v2)) + 0.5f * (w1 * w1 + w2 * w2);
      acc[0] = (acc[0] + (double)rho * tem * (1.0 + qtot) * 0.5 * (double)ke) +
               (double)(ql * rho) * tem * 0.5 * (0.0 - 2.0 * ww * 0.0);
      const double tmp = (double)((LDG(&g.th0[k]) + LDG(&f.tha[o])) * (LDG(&g.pi0[k]) + LDG(&f.ppi[o])));
      acc[1] = acc[1] + (double)rho * tem * (double)(s.cv + s.cvv * qv) * tmp;
      acc[2] = acc[2] + (double)rho * tem * (1.0 + qtot) * (double)s.g * (double)s.zh[k];
      acc[3] = (acc[3] + (double)rho * tem * (double)ql * ((double)s.cpl * tmp - (double)s.lv1)) +
               (double)rho * tem * 0.0 * ((double)s.cpi * tmp - (double)s.ls1);
      break;
    }
    default:
      break;
  }
}

// the better of two (value, linear index) candidates: larger (smaller for
// the min) value, the lower index on a tie
__device__ __forceinline__ void st_pick_max(float &v, int &ix, float v2, int ix2) {
  if (v2 > v || (v2 == v && ix2 < ix)) { v = v2; ix = ix2; }
}
__device__ __forceinline__ void st_pick_min(float &v, int &ix, float v2, int ix2) {
  if (v2 < v || (v2 == v && ix2 < ix)) { v = v2; ix = ix2; }
}

static const int ST_NT = 256;                 // threads of a level-chunk block
static const int ST_PPT = 16;                 // points per thread
static const int ST_CHUNK = ST_NT * ST_PPT;   // points of one block

int stat_chunks(int npl) { return npl > 0 ? (npl + ST_CHUNK - 1) / ST_CHUNK : 1; }

// One chunk of one level of one job, with the job's kind a constant so that
// the unrolled point loop issues its loads ahead of their use.
struct StatShared {
  float rv[2][ST_NT];
  int ri[2][ST_NT];
  double rd[ST_NT];
};

template <int KIND>
__device__ __forceinline__ void st_chunk(const DGrid &g, const StatJob &jb, const StatFields &f, const StatConsts &s,
                                         int k, int t0, int npl, int ni, float aux, StatLev *out, StatShared &sh) {
  constexpr bool sums = KIND >= SK_FIRST_SUM;
  float vmax = -1.0e30f, vmin = 1.0e30f;
  int imax = 0x7fffffff, imin = 0x7fffffff;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  StatJob j2 = jb;
  j2.kind = KIND;
  // (ii, jj): offsets of point t in the level's i-j range, advanced by
  // ST_NT points per step without a division
  const int tt = t0 + (int)threadIdx.x;
  int jj = tt / ni, ii = tt - jj * ni;
#pragma unroll 4
  for (int r = 0; r < ST_PPT; r++) {
    const int t = t0 + r * ST_NT + (int)threadIdx.x;
    const int i = jb.i0 + ii, j = jb.j0 + jj;
    ii += ST_NT;
    while (ii >= ni) { ii -= ni; jj++; }
    if (t < npl) {
      if (sums) {
        st_sums(g, j2, f, s, i, j, k, acc);
      } else {
        const float v = st_value(g, j2, f, s, i, j, k, aux);
        if (v > vmax) { vmax = v; imax = t; }   // strict: the first point of this thread's scan
        if (v < vmin) { vmin = v; imin = t; }
      }
    }
  }
  float (&rv)[2][ST_NT] = sh.rv;
  int (&ri)[2][ST_NT] = sh.ri;
  double (&rd)[ST_NT] = sh.rd;
  const int tid = threadIdx.x;
  StatLev o;
  if (!sums) {
    rv[0][tid] = vmax; ri[0][tid] = imax; rv[1][tid] = vmin; ri[1][tid] = imin;
    __syncthreads();
    for (int h = ST_NT / 2; h > 0; h >>= 1) {
      if (tid < h) {
        float a = rv[0][tid]; int ia = ri[0][tid];
        st_pick_max(a, ia, rv[0][tid + h], ri[0][tid + h]);
        rv[0][tid] = a; ri[0][tid] = ia;
        float b = rv[1][tid]; int ib = ri[1][tid];
        st_pick_min(b, ib, rv[1][tid + h], ri[1][tid + h]);
        rv[1][tid] = b; ri[1][tid] = ib;
      }
      __syncthreads();
    }
    o.vmax = rv[0][0]; o.imax = ri[0][0]; o.vmin = rv[1][0]; o.imin = ri[1][0];
    for (int q = 0; q < 4; q++) o.s[q] = 0.0;
  } else {
    for (int q = 0; q < 4; q++) {
      rd[tid] = acc[q];
      __syncthreads();
      for (int h = ST_NT / 2; h > 0; h >>= 1) {
        if (tid < h) rd[tid] = rd[tid] + rd[tid + h];
        __syncthreads();
      }
      o.s[q] = rd[0];
      __syncthreads();
    }
    o.vmax = -1.0e30f; o.vmin = 1.0e30f; o.imax = o.imin = 0x7fffffff;
  }
  if (tid == 0) *out = o;
}

// grid: x = chunk of a level, y = level, z = job
__global__ void __launch_bounds__(ST_NT) k_stat_levels(DGrid g, StatFields f, StatConsts s, const StatJob *jobs,
                                                       StatLev *lev, int maxlev, int nch) {
  const StatJob jb = jobs[blockIdx.z];
  const int kl = (int)blockIdx.y;
  if (kl >= jb.nlev) return;
  const int ni = jb.ie - jb.i0 + 1, nj = jb.je - jb.j0 + 1;
  const int npl = (ni > 0 && nj > 0) ? ni * nj : 0;
  const int t0 = (int)blockIdx.x * ST_CHUNK;   // chunks past npl write the neutral record
  const int k = jb.klo + kl;
  float aux = 0.0f;
  if (jb.kind == SK_PP) aux = s.p00 * powf(LDG(&g.pi0[k]), s.cpdrd);
  StatLev *out = lev + ((long)blockIdx.z * maxlev + kl) * nch + blockIdx.x;
  __shared__ StatShared sh;
  switch (jb.kind) {
    case SK_FIELD: st_chunk<SK_FIELD>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_PRATE: st_chunk<SK_PRATE>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_PP:    st_chunk<SK_PP>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_DIV:   st_chunk<SK_DIV>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_RH:    st_chunk<SK_RH>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_THE:   st_chunk<SK_THE>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_WSP:   st_chunk<SK_WSP>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_WLEV:  st_chunk<SK_WLEV>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_PSFC:  st_chunk<SK_PSFC>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_CFL:   st_chunk<SK_CFL>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_VORT:  st_chunk<SK_VORT>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_CLOUD: st_chunk<SK_CLOUD>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_MASS:  st_chunk<SK_MASS>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_TMOIS: st_chunk<SK_TMOIS>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_QMAS:  st_chunk<SK_QMAS>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_TMF:   st_chunk<SK_TMF>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    case SK_MOE:   st_chunk<SK_MOE>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
    default:       st_chunk<SK_ENER>(g, jb, f, s, k, t0, npl, ni, aux, out, sh); break;
  }
}

// Warp reductions over the (level, chunk) records of a job, records in
// increasing order: the max/min with the first level that holds it, and
// the sums of one component.
__device__ __forceinline__ void warp_best(float &v, int &lv, bool is_max) {
  for (int o = 16; o > 0; o >>= 1) {
    const float v2 = __shfl_down_sync(0xffffffffu, v, o);
    const int l2 = __shfl_down_sync(0xffffffffu, lv, o);
    if (is_max ? (v2 > v || (v2 == v && l2 < lv)) : (v2 < v || (v2 == v && l2 < lv))) { v = v2; lv = l2; }
  }
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// The output program: one warp per rstat entry, statpack's order.
__global__ void k_stat_finish(DGrid g, StatConsts s, const StatJob *jobs, const StatLev *lev, int maxlev, int nch,
                              const StatOp *ops, int nops, float *rstat) {
  const int p = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int lane = (int)(threadIdx.x & 31);
  if (p >= nops) return;
  const StatOp op = ops[p];
  const int jx = op.job >= 0 ? op.job : 0;
  const StatJob jb = jobs[jx];
  const StatLev *L = lev + (long)jx * maxlev * nch;
  const int nrec = jb.nlev * nch;
  float r = 0.0f;
  switch (op.op) {
    case SO_MAX: case SO_ZF_KMAX: case SO_ZH_KMAX: case SO_CFL: {
      // maxmin.F:62-75: strict comparison from -1e30 in level order, level 1
      // if none; calccfl: cfl(k) from -1, fmax from -99999999
      float v = -1.0e30f; int lv = 0x7fffffff;
      for (int q = lane; q < nrec; q += 32) {
        const float x = L[q].vmax;
        if (x > v) { v = x; lv = q / nch; }
      }
      warp_best(v, lv, true);
      if (op.op == SO_MAX) r = v;
      else if (op.op == SO_CFL) r = fmaxf(-99999999.0f, v > -1.0f ? v : -1.0f);
      else {
        const int kmax = (lv == 0x7fffffff) ? 1 : jb.klo + lv;
        r = op.op == SO_ZF_KMAX ? s.zf[kmax] : s.zh[kmax];
      }
      break;
    }
    case SO_MIN: case SO_ZF_KMIN: case SO_ZH_KMIN: {
      float v = 1.0e30f; int lv = 0x7fffffff;
      for (int q = lane; q < nrec; q += 32) {
        const float x = L[q].vmin;
        if (x < v) { v = x; lv = q / nch; }
      }
      warp_best(v, lv, false);
      if (op.op == SO_MIN) r = v;
      else {
        const int kmin = (lv == 0x7fffffff) ? 1 : jb.klo + lv;
        r = op.op == SO_ZF_KMIN ? s.zf[kmin] : s.zh[kmin];
      }
      break;
    }
    case SO_LEVMAX: case SO_VORT: {   // maxmin2d of one level; vertvort: max(-9999999, ...)
      const StatLev *Lk = L + (long)(op.k - jb.klo) * nch;
      if (op.op == SO_VORT) Lk = L;
      float v = -1.0e30f; int lv = 0x7fffffff;
      for (int q = lane; q < nch; q += 32) if (Lk[q].vmax > v) { v = Lk[q].vmax; lv = q; }
      warp_best(v, lv, true);
      r = op.op == SO_VORT ? fmaxf(-9999999.0f, v) : v;
      break;
    }
    case SO_LEVMIN: {
      const StatLev *Lk = L + (long)(op.k - jb.klo) * nch;
      float v = 1.0e30f; int lv = 0x7fffffff;
      for (int q = lane; q < nch; q += 32) if (Lk[q].vmin < v) { v = Lk[q].vmin; lv = q; }
      warp_best(v, lv, false);
      r = v;
      break;
    }
    case SO_QCTOP: case SO_QCBOT: {  // cloud (misclibs.F:2364-2400), clwsat = 1e-6
      float top = 0.0f, bot = s.maxz;
      for (int q = lane; q < nrec; q += 32) {
        const bool cl = L[q].vmax >= 1.e-6f;
        const float z = s.zh[jb.klo + q / nch];
        top = fmaxf(top, cl ? z : 0.0f);
        bot = fminf(bot, cl ? z : s.maxz);
      }
      for (int o = 16; o > 0; o >>= 1) {
        top = fmaxf(top, __shfl_down_sync(0xffffffffu, top, o));
        bot = fminf(bot, __shfl_down_sync(0xffffffffu, bot, o));
      }
      if (bot == s.maxz) bot = 0.0f;
      r = op.op == SO_QCTOP ? top : bot;
      break;
    }
    case SO_SUM: {  // the levels' sums, then the volume factor of the budget
      double t = 0.0;
      for (int q = lane; q < nrec; q += 32) t = t + L[q].s[op.k];
      t = warp_sum(t);
      if (op.arg == 1) t = t * (double)(g.dx * g.dy * g.dz);
      else if (op.arg == 2) t = t * (double)g.dx * (double)g.dy;
      r = (float)t;
      break;
    }
    case SO_ENER_TOTAL: {  // calcener: et = ek + ei + ep + le of the scaled terms
      double e[4];
      for (int c = 0; c < 4; c++) {
        double t = 0.0;
        for (int q = lane; q < nrec; q += 32) t = t + L[q].s[c];
        e[c] = warp_sum(t) * (double)(g.dx * g.dy * g.dz);
      }
      r = (float)(((e[0] + e[1]) + e[2]) + e[3]);
      break;
    }
    default:  // SO_ZERO, and SO_HOST (filled by the host)
      r = 0.0f;
      break;
  }
  if (lane == 0) rstat[p] = r;
}

void launch_stat(const DGrid &g, const StatFields &f, const StatConsts &s, const StatJob *jobs, int njobs,
                 StatLev *lev, int maxlev, int nch, const StatOp *ops, int nops, float *rstat, cudaStream_t st,
                 int64_t *nl) {
  if (njobs > 0) {
    dim3 grid((unsigned)nch, (unsigned)maxlev, (unsigned)njobs);
    { ProfScope _ps("k_stat_levels", st); k_stat_levels<<<grid, ST_NT, 0, st>>>(g, f, s, jobs, lev, maxlev, nch); }
    if (nl) *nl += 1;
  }
  const int wpb = 8;
  { ProfScope _ps("k_stat_finish", st);
    k_stat_finish<<<(unsigned)((nops + wpb - 1) / wpb), 32 * wpb, 0, st>>>(g, s, jobs, lev, maxlev, nch, ops, nops,
                                                                            rstat); }
  if (nl) *nl += 1;
}

}  // namespace cm1g
