// k_micro.cu -- Kessler warm-rain microphysics (ptype=1) on the device: the
// branch of mp_driver that cm1.F runs after solve2 (mp_driver.F:108-233).
//
// After the three pdefq clips of qv, qc and qr (k_pdefq, k_misc.cu) the
// scheme is two launches:
//
//   k_mp_fall   one thread per column: rain fall speeds (k_fallout,
//               kessler.F:441-462), the surface energy flux of the falling
//               rain (geterain, kessler.F:529-558) and the sedimentation of
//               qr in nfall sub-steps with its surface rain, precipitation
//               rate and budget (fallout, kessler.F:470-516);
//   k_mp_point  one thread per point: autoconversion, accretion and rain
//               evaporation (kessler, kessler.F:10-133) followed by the
//               saturation adjustment (satadj, kessler.F:142-432); both
//               read and write only their own point, so they fuse.
//
// The FP64 budgets (qbudget 1-7 of the reference: condensation,
// evaporation, autoconversion, accretion, rain evaporation, surface rain and
// the rain's energy flux) are summed per level or column in fixed order and
// added by k_mp_budget.  The point arithmetic keeps the Fortran's operand
// order (the library is built with --fmad=false); the powers and
// exponentials are evaluated in binary64 and rounded to binary32.
#include "cm1g_common.cuh"
#include "k_micro.cuh"

namespace cm1g {

// Powers and exponentials in binary64, rounded once to binary32: within
// 0.5 ulp (plus ~2^-50 relative) of the exact value, so they agree with a
// correctly rounded binary32 library, as the reference's runs use, except in
// rare double-rounding cases.  The scheme forms pi' and theta' as small
// differences of such values (pp3d = (p/p00)^(rd/cp) - pi0), where one ulp
// of the power is a visible part of the perturbation's range.
__device__ __forceinline__ float mp_powf(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float mp_expf(float x) { return (float)exp((double)x); }

// saturation mixing ratio over liquid of the Kessler routines
// (kessler.F:58-62, 200-204, 258-263): Bolton's esl, capped at p/2
__device__ __forceinline__ float mp_esl(float t, float p) {
  float esl = 611.2f * mp_expf(17.67f * (t - 273.15f) / (t - 29.65f));
  return fminf(esl, p * 0.5f);
}

// --- fall speeds, geterain and fallout: one thread per column -------------
__global__ void k_mp_fall(DGrid g, MicroArgs a, double *colbud) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y;
  if (i > g.ni) return;
  const int nk = g.nk;
  const long pl = (long)g.NI * g.NJ;
  const long oc = iS(g, i, j, 0);
  const MicroConsts &m = a.c;
  const float dt = a.dt;
  float *qr = a.qr, *vr = a.vr;
  const float *rho = a.rho;
  // k_fallout (kessler.F:452-458)
  for (int k = 1; k <= nk; k++) {
    const long o = oc + k * pl;
    const float q = qr[o], r = rho[o];
    vr[o] = (q > 1.0e-12f) ? 14.34f * mp_powf(r * q, 0.1346f) * sqrtf(1.15f / r) : 0.0f;
  }
  const float ruh = LDG(&g.ruh[i - g.ib]), rvh = LDG(&g.rvh[j - g.jb]);
  // geterain (kessler.F:547-550) at k = 1, T of mp_driver.F:98-108, rr = rho
  {
    const long o = oc + pl;
    const float t1 = (LDG(&g.th0[1]) + a.th3d[o]) * (LDG(&g.pi0[1]) + a.pp3d[o]);
    colbud[(long)(j - 1) * g.ni + (i - 1)] =
        (double)(dt * vr[o] * rho[o] * qr[o] * (m.cpl * t1 - m.lv1) * ruh * rvh);
  }
  // fallout (kessler.F:493-512)
  float crmax = 0.0f;
  for (int k = 1; k <= nk; k++) crmax = fmaxf(crmax, vr[oc + k * pl] * dt * g.rdz * LDG(&g.mh[k]));
  const int nfall = max(1, (int)(crmax + 1.0f));
  for (int k = nk - 1; k >= 1; k--)
    if (qr[oc + k * pl] < 1.0e-8f) vr[oc + k * pl] = vr[oc + (k + 1) * pl];
  const float dtfall = dt / (float)nfall;
  double bud = 0.0;
  float rain = a.rain[i2(g, i, j)], prate = 0.0f;
  for (int n = 1; n <= nfall; n++) {
    // rq(k) = rho vq max(0,q); q(k) += dtfall (rq(k+1) - rq(k)) rdz mh / rho,
    // marching down the column with rq(k+1) carried from the level above
    float rqk1 = 0.0f;                       // rq(nk+1)
    float rq1 = 0.0f;
    for (int k = nk; k >= 1; k--) {
      const long o = oc + k * pl;
      const float rk = rho[o] * vr[o] * fmaxf(0.0f, qr[o]);
      qr[o] = qr[o] + dtfall * (rqk1 - rk) * g.rdz * LDG(&g.mh[k]) / rho[o];
      rqk1 = rk;
      rq1 = rk;
    }
    rain = rain + 0.1f * dtfall * rq1;
    prate = rq1;
    const long o1 = oc + pl;
    bud = bud + (double)(dtfall * rho[o1] * vr[o1] * fmaxf(0.0f, qr[o1]) * ruh * rvh);
  }
  a.rain[i2(g, i, j)] = rain;
  a.prate[i2(g, i, j)] = prate;
  colbud[(long)g.ni * g.nj + (long)(j - 1) * g.ni + (i - 1)] = bud;
}

// --- kessler + satadj: one thread per point --------------------------------
static const int MP_NT = 128;

__global__ void __launch_bounds__(MP_NT) k_mp_point(DGrid g, MicroArgs a, double *part, int nchunk) {
  __shared__ double red[MP_NT];
  const int k = 1 + (int)blockIdx.y;
  const long npl = (long)g.ni * g.nj;
  const long t = (long)blockIdx.x * MP_NT + threadIdx.x;
  const MicroConsts &m = a.c;
  const float dt = a.dt;
  double b[5] = {0.0, 0.0, 0.0, 0.0, 0.0};   // kessler ar, cr, er; satadj cond, evap
  if (t < npl) {
    const int i = 1 + (int)(t % g.ni), j = 1 + (int)(t / g.ni);
    const long o = iS(g, i, j, k);
    const float th0 = LDG(&g.th0[k]), pi0 = LDG(&g.pi0[k]);
    const float rr = a.rho[o];                 // rho at the entry of mp_driver (budgets)
    float rho = rr;
    float th3 = a.th3d[o], pp3 = a.pp3d[o], prs = a.prs[o];
    float qv = a.qv[o], qc = a.qc[o], qr = a.qr[o];
    const float tem = LDG(&g.ruh[i - g.ib]) * LDG(&g.rvh[j - g.jb]) * LDG(&g.rmh[k]);
    // ---- kessler (kessler.F:39-118)
    {
      const float tmp = (th0 + th3) * (pi0 + pp3);
      float qvnew = qv, qcnew = qc, qrnew = qr;
      float ar = 0.0f, cr = 0.0f, er = 0.0f;
      if (qcnew > 0.0f) {
        ar = fmaxf(0.001f * (qcnew - 0.001f), 0.0f);
        ar = ar * dt;
      }
      if (qcnew > 0.0f && qrnew > 0.0f) {
        cr = 2.2f * qcnew * mp_powf(qrnew, 0.875f);
        cr = cr * dt;
      }
      if (qrnew > 0.0f) {
        const float esl = mp_esl(tmp, prs);
        const float qvs = m.eps * esl / (prs - esl);
        if (qvnew < qvs) {
          er = (1.6f + 30.3922f * mp_powf(rho * qrnew, 0.2046f)) * (1.0f - (qvnew / qvs)) *
               mp_powf(rho * qrnew, 0.525f) / ((2.03e4f + 9.584e6f / (qvs * prs)) * rho);
          er = fminf(er * dt, qrnew);
          if ((qvnew + er) > qvs) er = qvs - qvnew;
        }
      }
      if ((ar + cr) > qcnew) {
        const float term1 = ar + cr;
        ar = qcnew * ar / term1;
        cr = qcnew * cr / term1;
      }
      qvnew = qvnew + er;
      qcnew = qcnew - (ar + cr);
      qrnew = qrnew + (ar + cr - er);
      if (er > 1.0e-7f) {
        if (a.eqtset == 2) {
          const float cpml = m.cp + m.cpv * qvnew + m.cpl * (qcnew + qrnew);
          const float cvml = m.cv + m.cvv * qvnew + m.cpl * (qcnew + qrnew);
          const float rm = m.rd + m.rv * qvnew;
          th3 = th3 - er * ((m.lv1 - m.lv2 * tmp) / (m.cpdcv * cvml * (pi0 + pp3)) -
                            (th0 + th3) * (m.rv / cvml) * (1.0f - m.rovcp * cpml / rm));
          pp3 = mp_powf(rho * rm * (th0 + th3) * m.rp00, m.rddcv) - pi0;
          prs = m.p00 * mp_powf(pi0 + pp3, m.cpdrd);
        } else {
          th3 = th3 - er * ((m.lv1 - m.lv2 * tmp) / (m.cp * (pi0 + pp3)));
          rho = prs / (m.rd * (th0 + th3) * (pi0 + pp3) * (1.0f + qvnew * m.reps));
        }
      }
      b[0] = (double)(rr * ar * tem);
      b[1] = (double)(rr * cr * tem);
      b[2] = (double)(rr * er * tem);
      qv = qvnew; qc = qcnew; qr = qrnew;
    }
    // ---- satadj (kessler.F:168-355), nrk = 4
    if (a.eqtset == 2) {
      float tnew = (th0 + th3) * (pi0 + pp3);
      float esl = mp_esl(tnew, prs);
      float qvs = m.eps * esl / (prs - esl);
      if (qc > 1.0e-12f || qv > qvs) {
        float qvnew = qv, qcnew = qc;
        float ql = 0.0f;
        ql = ql + qc;                          // q(nql1) .. q(nql2) = qc, qr
        ql = ql + qr;
        ql = fmaxf(0.0f, ql);
        const float qi = fmaxf(0.0f, 0.0f);
        const float cvml = m.cv + m.cvv * qvnew + m.cpl * ql + m.cpi * qi;
        const float lhv = m.lv1 - m.lv2 * tnew;
        const float t1 = (lhv - m.rv * tnew) / cvml;
        const float d1 = t1 * 17.67f * 243.5f;
        float tlast = tnew, pnew = 0.0f;
        int n = 0;
        bool doit = true;
        while (doit) {   // ends: after convergence, or at n = 100 with the error flag
          n = n + 1;
          const float tm = tnew - 29.65f;
          float dqv = (qvs - qvnew) / (1.0f + d1 * qvs / (tm * tm));
          dqv = fminf(dqv, qcnew);
          if ((qvnew + dqv) < 1.0e-20f) dqv = 1.0e-20f - qvnew;
          qvnew = qvnew + dqv;
          qcnew = qcnew - dqv;
          tnew = tnew - dqv * t1;
          pnew = rho * (m.rd + m.rv * qvnew) * tnew;
          doit = false;
          if (fabsf(tnew - tlast) > a.converge) {
            tlast = tnew;
            esl = mp_esl(tnew, prs);
            qvs = m.eps * esl / (pnew - esl);
            doit = true;
          }
          if (n == 100) {
            if (a.err) atomicOr(a.err, 1);
            doit = false;
          }
        }
        b[3] = (double)(rr * fmaxf(qcnew - qc, 0.0f) * tem);
        b[4] = (double)(rr * fmaxf(qvnew - qv, 0.0f) * tem);
        prs = pnew;
        pp3 = mp_powf(pnew * m.rp00, m.rovcp) - pi0;
        th3 = tnew / (pi0 + pp3) - th0;
        qc = qcnew;
        qv = qvnew;
      }
    } else {
      float qvnew = qv, qcnew = qc;
      const float tnew = (th0 + th3) * (pi0 + pp3);
      const float esl = mp_esl(tnew, prs);
      const float qvs = m.eps * esl / (prs - esl);
      const float lhv = m.lv1 - m.lv2 * tnew;
      const float tm = tnew - 29.65f;
      float dqv = (qvs - qvnew) / (1.0f + lhv * qvs * 17.67f * 243.5f / (m.cp * (tm * tm)));
      if ((qvnew + dqv) < 1.0e-20f) dqv = 1.0e-20f - qvnew;
      dqv = fminf(dqv, fmaxf(0.0f, qcnew));
      qvnew = qvnew + dqv;
      qcnew = qcnew - dqv;
      b[3] = (double)(rr * fmaxf(qcnew - qc, 0.0f) * tem);
      b[4] = (double)(rr * fmaxf(qvnew - qv, 0.0f) * tem);
      th3 = th3 - dqv * (lhv / (m.cp * (pi0 + pp3)));
      qc = qcnew;
      qv = qvnew;
      rho = prs / (m.rd * (th0 + th3) * (pi0 + pp3) * (1.0f + qvnew * m.reps));
    }
    a.th3d[o] = th3; a.pp3d[o] = pp3; a.prs[o] = prs; a.rho[o] = rho;
    a.qv[o] = qv; a.qc[o] = qc; a.qr[o] = qr;
  }
  // per-block sums of the five budgets, level k, chunk blockIdx.x
  for (int q = 0; q < 5; q++) {
    red[threadIdx.x] = b[q];
    __syncthreads();
    for (int h = MP_NT / 2; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[((long)q * g.nk + (k - 1)) * nchunk + blockIdx.x] = red[0];
    __syncthreads();
  }
}

// qbudget += the step's budgets: block q adds budget q's partial sums (per
// level and chunk for kessler/satadj, per column for fallout/geterain) in a
// fixed order; qb[0..6] = tcond, tevac, tauto, taccr, tevar, train, erain.
static const int MB_NT = 256;

__global__ void __launch_bounds__(MB_NT) k_mp_budget(DGrid g, const double *part, int nchunk, const double *colbud,
                                                     double *qb) {
  __shared__ double red[MB_NT];
  const int q = (int)blockIdx.x;
  const double *src;
  long n;
  if (q < 5) { src = part + (long)q * g.nk * nchunk; n = (long)g.nk * nchunk; }
  else { src = colbud + (q == 5 ? (long)g.ni * g.nj : 0L); n = (long)g.ni * g.nj; }   // 5 fallout, 6 geterain
  double s = 0.0;
  for (long t = threadIdx.x; t < n; t += MB_NT) s = s + src[t];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = MB_NT / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double tot = red[0];
  if (q < 5) {
    // kessler: tauto/taccr/tevar += bud(k)*dum, dum = dx*dy*dz (kessler.F:120-132);
    // satadj: tcond/tevac likewise (kessler.F:388-396); part order ar, cr, er, cond, evap
    const int dst = q < 3 ? 2 + q : q - 3;
    qb[dst] = qb[dst] + tot * (double)(g.dx * g.dy * g.dz);
  } else if (q == 5) {
    qb[5] = qb[5] + tot * (double)(g.dx * g.dy);            // fallout: tem = dx*dy (kessler.F:514-517)
  } else {
    qb[6] = qb[6] + tot * (double)g.dx * (double)g.dy;      // geterain: bud(j)*dx*dy (kessler.F:553-555)
  }
}

int mp_chunks(const DGrid &g) { return (int)(((long)g.ni * g.nj + MP_NT - 1) / MP_NT); }

void launch_kessler(const DGrid &g, const MicroArgs &a, double *part, double *colbud, double *qb, cudaStream_t st,
                    int64_t *nl) {
  {
    dim3 grid((g.ni + 127) / 128, g.nj);
    ProfScope _ps("k_mp_fall", st);
    k_mp_fall<<<grid, 128, 0, st>>>(g, a, colbud);
  }
  const int nch = mp_chunks(g);
  {
    dim3 grid(nch, g.nk);
    ProfScope _ps("k_mp_point", st);
    k_mp_point<<<grid, MP_NT, 0, st>>>(g, a, part, nch);
  }
  {
    ProfScope _ps("k_mp_budget", st);
    k_mp_budget<<<7, MB_NT, 0, st>>>(g, part, nch, colbud, qb);
  }
  if (nl) *nl += 3;
}

}  // namespace cm1g
