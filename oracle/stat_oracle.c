/*
 * stat_oracle.c -- CPU restatement of CM1 r21.1's statistics package
 * (statpack, src/statpack.F:10-658) for the fields of the dynamical core.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of cm1g_statpack.  tests/ and
 * bench.py's CPU arms may call it; the product never links it.  Parity of
 * the large step itself is unpinned (see cm1_oracle.c); this file follows
 * the serial loop order of each cited routine literally: per-level extrema
 * with strict comparisons (maxmin.F:43-75), per-level FP64 sums in (j, i)
 * order then over the levels (misclibs.F:3134-3636), binary32 point
 * arithmetic in the Fortran's evaluation order (build with
 * -ffp-contract=off).
 *
 * Same scope as cm1g_stat_setup: no terrain, axisymm=0, umove=vmove=0,
 * adapt_dt=0, no turbulence, no ice, bbc != 3.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include "../include/cm1g.h"

typedef struct {
  int ni, nj, nk, ib, jb, NI, NJ;
  float dx, dy, dz, rdx, rdy, rdz;
  int ibw, ibe, ibs, ibn;
  const cm1g_grid_t *gr;
} SG;

/* index of an s- (or w-) point, a u-point, a v-point and a 2-D point */
static long sI(const SG *g, int i, int j, int k) { return (long)(i - g->ib) + (long)g->NI * ((long)(j - g->jb) + (long)g->NJ * k); }
static long uI(const SG *g, int i, int j, int k) { return (long)(i - g->ib) + (long)(g->NI + 1) * ((long)(j - g->jb) + (long)g->NJ * k); }
static long vI(const SG *g, int i, int j, int k) { return (long)(i - g->ib) + (long)g->NI * ((long)(j - g->jb) + (long)(g->NJ + 1) * k); }

/* maxmin (maxmin.F:5-119) over a level range of a point function */
typedef float (*PointFn)(const SG *g, const void *ctx, int i, int j, int k);

static void maxmin_fn(const SG *g, PointFn f, const void *ctx, int i1, int i2, int j1, int j2, int k1, int k2,
                      float *fmax, float *fmin, int *kmax, int *kmin) {
  float mx = -1.e30f, mn = 1.e30f;
  *kmax = 1; *kmin = 1;
  for (int k = k1; k <= k2; k++) {
    float tmax = -1.e30f, tmin = 1.e30f;
    for (int j = j1; j <= j2; j++)
      for (int i = i1; i <= i2; i++) {
        float v = f(g, ctx, i, j, k);
        if (v > tmax) tmax = v;
        if (v < tmin) tmin = v;
      }
    if (tmax > mx) { mx = tmax; *kmax = k; }
    if (tmin < mn) { mn = tmin; *kmin = k; }
  }
  *fmax = mx; *fmin = mn;
}

typedef struct { const float *a; int stag; } FieldCtx;
static float pf_field(const SG *g, const void *c, int i, int j, int k) {
  const FieldCtx *x = (const FieldCtx *)c;
  long o = x->stag == 2 ? uI(g, i, j, k) : x->stag == 3 ? vI(g, i, j, k) : sI(g, i, j, k);
  return x->a[o];
}

typedef struct {
  const float *ua, *va, *wa, *ppi, *tha, *prs, *rho, *qa, *prate;
  long ns;
  float p00, eps, reps, rd, rv, cp, cpdrd, dtdx, dtdy, dtdz, cgs1, cgs2, cgs3, r1, r2;
  int ptype, nqv, nkm, nx, ny, numq, cloud[CM1G_MAXQ];
} StCtx;

static float pf_prate(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c; (void)k;
  return x->prate ? x->prate[(long)(i - g->ib) + (long)g->NI * (j - g->jb)] : 0.0f;
}
/* statpack.F:236-242 */
static float pf_pp(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c;
  return x->prs[sI(g, i, j, k)] - x->p00 * powf(g->gr->pi0[sI(g, i, j, k)], x->cpdrd);
}
/* statpack.F:297-309 */
static float pf_div(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c;
  const float *r0 = g->gr->rho0;
  float a = 0.5f * ((r0[sI(g, i, j, k)] + r0[sI(g, i + 1, j, k)]) * x->ua[uI(g, i + 1, j, k)] -
                    (r0[sI(g, i, j, k)] + r0[sI(g, i - 1, j, k)]) * x->ua[uI(g, i, j, k)]) * g->rdx * g->gr->uh[i - g->ib];
  float b = 0.5f * ((r0[sI(g, i, j, k)] + r0[sI(g, i, j + 1, k)]) * x->va[vI(g, i, j + 1, k)] -
                    (r0[sI(g, i, j, k)] + r0[sI(g, i, j - 1, k)]) * x->va[vI(g, i, j, k)]) * g->rdy * g->gr->vh[j - g->jb];
  float d = 0.5f * ((r0[sI(g, i, j, k)] + r0[sI(g, i, j, k + 1)]) * x->wa[sI(g, i, j, k + 1)] -
                    (r0[sI(g, i, j, k)] + r0[sI(g, i, j, k - 1)]) * x->wa[sI(g, i, j, k)]) * g->rdz *
            g->gr->mh[sI(g, i, j, k)];
  return a + b + d;
}
/* rslf (cm1libs.F:16-62) */
static float rslf(const StCtx *x, float p, float t) {
  if (x->ptype == 4) return 380.00f * expf(17.2693882f - 4097.8531f / (t - 35.86f)) / p;
  float esl = 611.2f * expf(17.67f * (t - 273.15f) / (t - 29.65f));
  esl = fminf(esl, p * 0.5f);
  return x->eps * esl / (p - esl);
}
/* statpack.F:364-371 */
static float pf_rh(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c;
  long o = sI(g, i, j, k);
  float qvs = rslf(x, x->prs[o], (g->gr->th0[o] + x->tha[o]) * (g->gr->pi0[o] + x->ppi[o]));
  float qv = x->qa[x->nqv * x->ns + o];
  return qv * (1.0f + qvs * x->reps) / (qvs * (1.0f + qv * x->reps));
}
/* calcthe (misclibs.F:2300-2336); levels above 10 km copy the one below */
static float pf_the(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c;
  long o = sI(g, i, j, k);
  float tx = (g->gr->th0[o] + x->tha[o]) * (g->gr->pi0[o] + x->ppi[o]);
  float cpm = x->cp;
  float qv = x->qa[x->nqv * x->ns + o];
  float rh = pf_rh(g, c, i, j, k);
  return tx * powf(x->p00 * (1.0f + qv * x->reps) / x->prs[o], x->rd / cpm) * powf(rh, -(qv * x->rv / cpm)) *
         expf(2.555e6f * qv / (cpm * tx));
}
/* statpack.F:437-441 */
static float pf_wsp(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c;
  float a = 0.0f + 0.5f * (x->ua[uI(g, i, j, k)] + x->ua[uI(g, i + 1, j, k)]);
  float b = 0.0f + 0.5f * (x->va[vI(g, i, j, k)] + x->va[vI(g, i, j + 1, k)]);
  return sqrtf(a * a + b * b);
}
/* statpack.F:180-188 */
static float pf_wlev(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c; (void)k;
  return x->r1 * x->wa[sI(g, i, j, x->nkm)] + x->r2 * x->wa[sI(g, i, j, x->nkm + 1)];
}
/* statpack.F:425-430 */
static float pf_psfc(const SG *g, const void *c, int i, int j, int k) {
  const StCtx *x = (const StCtx *)c; (void)k;
  return x->cgs1 * x->prs[sI(g, i, j, 1)] + x->cgs2 * x->prs[sI(g, i, j, 2)] + x->cgs3 * x->prs[sI(g, i, j, 3)];
}

static int emit(float *rstat, int n, float v) { rstat[n] = v; return n + 1; }

int oracle_statpack(const cm1g_config_t *cfg, const cm1g_grid_t *gr, const cm1g_stat_opts_t *o, double mtime,
                    float dt, const float *ua, const float *va, const float *wa, const float *ppi, const float *tha,
                    const float *prs, const float *rho, const float *qa, const float *pta, const float *prate,
                    const double *qbudget, const double *asq, const double *bsq, float *rstat, int *nstat) {
  SG G, *g = &G;
  memset(g, 0, sizeof G);
  g->ni = cfg->ni; g->nj = cfg->nj; g->nk = cfg->nk;
  g->ib = 1 - cfg->ngxy; g->jb = 1 - cfg->ngxy;
  g->NI = cfg->ni + 2 * cfg->ngxy; g->NJ = cfg->nj + 2 * cfg->ngxy;
  g->dx = cfg->dx; g->dy = cfg->dy; g->dz = cfg->dz;
  g->rdx = 1.0f / cfg->dx; g->rdy = 1.0f / cfg->dy; g->rdz = 1.0f / cfg->dz;
  g->ibw = cfg->wbc != 1; g->ibe = cfg->ebc != 1; g->ibs = cfg->sbc != 1; g->ibn = cfg->nbc != 1;
  g->gr = gr;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const int moist = cfg->imoist == 1, numq = moist ? cfg->numq : 0, npt = cfg->iptra ? cfg->npt : 0;
  const long ns = (long)g->NI * g->NJ * (nk + 2);
  /* constants.F:65-175 */
  const int tc = cfg->testcase;
  const float rd = (tc == 4 || tc == 5) ? 287.0f : 287.04f;
  const float cp = tc == 4 ? 1015.0f : tc == 5 ? 1004.0f : 1005.7f;
  const float cpv = 1870.0f, rv = 461.5f, gg = 9.81f, cpl = 4190.0f, cpi = 2106.0f;
  const float cv = cp - rd, cvv = cpv - rv;
  const float xlv = tc == 4 ? 2.47e6f : tc == 5 ? 2.50e6f : 2501000.0f, xls = 2834000.0f, to = 273.15f;
  const float lv1 = (tc == 4 || tc == 5) ? xlv : xlv + (cpl - cpv) * to;
  const float ls1 = xls + (cpi - cpv) * to;
  (void)ls1;
  StCtx X;
  memset(&X, 0, sizeof X);
  X.ua = ua; X.va = va; X.wa = wa; X.ppi = ppi; X.tha = tha; X.prs = prs; X.rho = rho; X.qa = qa;
  X.prate = prate; X.ns = ns;
  X.p00 = 1.0e5f; X.eps = rd / rv; X.reps = rv / rd; X.rd = rd; X.rv = rv; X.cp = cp; X.cpdrd = cp / rd;
  X.dtdx = 0.5f * dt * g->rdx; X.dtdy = 0.5f * dt * g->rdy; X.dtdz = 0.5f * dt * g->rdz;
  X.cgs1 = o->cgs1; X.cgs2 = o->cgs2; X.cgs3 = o->cgs3;
  X.ptype = o->ptype; X.nqv = moist ? cfg->nqv - 1 : 0; X.nx = ni; X.ny = nj; X.numq = numq;
  const float *zh = o->zh, *zf = o->zf;
  float fx, fn;
  int kx, kn, n = 0;

  n = emit(rstat, n, (float)mtime);
  if (o->stat_w) {           /* statpack.F:136-144 */
    FieldCtx f = {wa, 4};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, nk + 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    n = emit(rstat, n, zf[kx]); n = emit(rstat, n, zf[kn]);
  }
  if (o->stat_wlevs && o->maxz >= 10000.0f) {   /* statpack.F:146-212 */
    const float zl[5] = {500.0f, 1000.0f, 2500.0f, 5000.0f, 10000.0f};
    for (int m = 0; m < 5; m++) {
      if (zl[m] < zf[nk + 1]) {
        int nkm = nk + 1;
        while (zf[nkm] > zl[m] && nkm > 1) nkm--;
        X.r2 = (zl[m] - zf[nkm]) / (zf[nkm + 1] - zf[nkm]);
        X.r1 = 1.0f - X.r2;
        X.nkm = nkm;
        maxmin_fn(g, pf_wlev, &X, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
      } else {
        fx = 0.0f; fn = 0.0f;
      }
      n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    }
  }
  if (o->stat_u) {           /* statpack.F:214-217 */
    FieldCtx f = {ua, 2};
    maxmin_fn(g, pf_field, &f, 1, ni + 1, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    maxmin_fn(g, pf_field, &f, 1, ni + 1, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_v) {           /* statpack.F:218-222 */
    FieldCtx f = {va, 3};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj + 1, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj + 1, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_pipert) {      /* statpack.F:227 */
    FieldCtx f = {ppi, 1};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_prspert) {
    maxmin_fn(g, pf_pp, &X, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_thpert) {      /* statpack.F:245-248 */
    FieldCtx f = {tha, 1};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (moist && o->stat_q) {  /* statpack.F:250-261 */
    for (int q = 0; q < numq; q++) {
      FieldCtx f = {qa + q * ns, 1};
      maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
      n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    }
    maxmin_fn(g, pf_prate, &X, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_div) {
    maxmin_fn(g, pf_div, &X, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (moist && o->stat_rh) {
    maxmin_fn(g, pf_rh, &X, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  for (int q = 0; q < npt; q++) {   /* statpack.F:389-407 */
    FieldCtx f = {pta + q * ns, 1};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (moist && o->stat_the) {       /* statpack.F:411-415: dum4 over all levels, copies above 10 km */
    int kt = 0;
    while (kt < nk && zh[kt + 1] <= 10000.0f) kt++;
    if (kt < 1) kt = 1;
    maxmin_fn(g, pf_the, &X, 1, ni, 1, nj, 1, kt, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    maxmin_fn(g, pf_the, &X, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (moist && o->stat_cloud) {     /* cloud (misclibs.F:2344-2416), clwsat = 1e-6 */
    float top = 0.0f, bot = o->maxz;
    for (int k = 1; k <= nk; k++) {
      float qctop = 0.0f, qcbot = o->maxz;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          float qci = 0.0f;
          for (int q = 0; q < numq; q++) if (o->cloudvar[q]) qci = qci + qa[q * ns + sI(g, i, j, k)];
          if (qci >= 1.e-6f) { qctop = fmaxf(qctop, zh[k]); qcbot = fminf(qcbot, zh[k]); }
        }
      top = fmaxf(top, qctop);
      bot = fminf(bot, qcbot);
    }
    if (bot == o->maxz) bot = 0.0f;
    n = emit(rstat, n, top); n = emit(rstat, n, bot);
  }
  if (o->stat_sfcprs) {             /* statpack.F:424-432 */
    FieldCtx f = {prs, 1};
    maxmin_fn(g, pf_field, &f, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    maxmin_fn(g, pf_psfc, &X, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_wsp) {                /* statpack.F:434-452 */
    maxmin_fn(g, pf_wsp, &X, 1, ni, 1, nj, 1, nk, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
    n = emit(rstat, n, zh[kx]); n = emit(rstat, n, zh[kn]);
    maxmin_fn(g, pf_wsp, &X, 1, ni, 1, nj, 1, 1, &fx, &fn, &kx, &kn);
    n = emit(rstat, n, fx); n = emit(rstat, n, fn);
  }
  if (o->stat_cfl) {                /* calccfl (misclibs.F:2584-2718) */
    float fm = -99999999.0f;
    for (int k = 1; k <= nk; k++) {
      float cfl = -1.0f;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          float cu = (ua[uI(g, i, j, k)] + ua[uI(g, i + 1, j, k)]) * X.dtdx * gr->uh[i - g->ib];
          float cv = (va[vI(g, i, j, k)] + va[vI(g, i, j + 1, k)]) * X.dtdy * gr->vh[j - g->jb];
          float cw = (wa[sI(g, i, j, k)] + wa[sI(g, i, j, k + 1)]) * X.dtdz * gr->mh[sI(g, i, j, k)];
          float w;
          if (X.nx > 1 && X.ny > 1) w = sqrtf((cu * cu + cv * cv) + cw * cw);
          else if (X.nx > 1) w = sqrtf(cu * cu + cw * cw);
          else w = sqrtf(cv * cv + cw * cw);
          if (w > cfl) cfl = w;
        }
      if (cfl > fm) fm = cfl;
    }
    n = emit(rstat, n, fm);
  }
  if (o->stat_vort) {               /* vertvort (misclibs.F:2424-2576), no terrain */
    int kv[6] = {1, nk + 1, nk + 1, nk + 1, nk + 1, nk + 1};
    for (int k = nk; k >= 1; k--)
      for (int m = 1; m <= 5; m++)
        if (zh[k] >= 1000.0f * m) kv[m] = k;
    for (int m = 0; m < 6; m++) {
      float vmax = 0.0f;
      int k = kv[m];
      if (k <= nk) {
        vmax = -9999999.0f;
        for (int j = 1 + g->ibs; j <= nj + 1 - g->ibn; j++)
          for (int i = 1 + g->ibw; i <= ni + 1 - g->ibe; i++) {
            float vort = (va[vI(g, i, j, k)] - va[vI(g, i - 1, j, k)]) * g->rdx * gr->uf[i - g->ib] -
                         (ua[uI(g, i, j, k)] - ua[uI(g, i, j - 1, k)]) * g->rdy * gr->vf[j - g->jb];
            vmax = fmaxf(vmax, vort);
          }
      }
      n = emit(rstat, n, vmax);
    }
  }
  const double dv = (double)(g->dx * g->dy * g->dz);
  /* liquid water of getqli (misclibs.F:923-967), qi = 0 */
#define QL(o) ({ float ql_ = 0.0f; if (o->nql1 > 0) for (int q_ = o->nql1 - 1; q_ <= o->nql2 - 1; q_++) ql_ = ql_ + qa[q_ * ns + (oo)]; ql_; })
  if (o->stat_tmass) {              /* calcmass (misclibs.F:3134-3191) */
    double t = 0.0;
    for (int k = 1; k <= nk; k++) {
      double foo = 0.0;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long oo = sI(g, i, j, k);
          foo = foo + (double)(rho[oo] * gr->ruh[i - g->ib] * gr->rvh[j - g->jb] * gr->rmh[oo]);
        }
      t = t + foo;
    }
    n = emit(rstat, n, (float)(t * dv));
  }
  if (moist && o->stat_tmois) {     /* totmois (misclibs.F:3199-3264) */
    double t = 0.0;
    for (int k = 1; k <= nk; k++) {
      double foo = 0.0;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long oo = sI(g, i, j, k);
          float qv = qa[X.nqv * ns + oo], ql = QL(o);
          foo = foo + (double)(rho[oo] * (qv + ql + 0.0f) * gr->ruh[i - g->ib] * gr->rvh[j - g->jb] * gr->rmh[oo]);
        }
      t = t + foo;
    }
    n = emit(rstat, n, (float)(t * dv));
  }
  if (moist && o->stat_qmass)       /* totq (misclibs.F:3272-3335) */
    for (int q = 0; q < numq; q++) {
      int liq = o->nql1 > 0 && q + 1 >= o->nql1 && q + 1 <= o->nql2;
      if (!(q + 1 == cfg->nqv || liq)) continue;
      double t = 0.0;
      for (int k = 1; k <= nk; k++) {
        double foo = 0.0;
        for (int j = 1; j <= nj; j++)
          for (int i = 1; i <= ni; i++) {
            long oo = sI(g, i, j, k);
            foo = foo + (double)(rho[oo] * qa[q * ns + oo] * gr->ruh[i - g->ib] * gr->rvh[j - g->jb] * gr->rmh[oo]);
          }
        t = t + foo;
      }
      n = emit(rstat, n, (float)(t * dv));
    }
  if (o->stat_tenerg) {             /* calcener (misclibs.F:3343-3454), vr = 0, qi = 0 */
    double ek = 0.0, ei = 0.0, ep = 0.0, le = 0.0;
    for (int k = 1; k <= nk; k++) {
      double f1 = 0.0, f2 = 0.0, f3 = 0.0, f4 = 0.0;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long oo = sI(g, i, j, k);
          double tem = (double)(gr->ruh[i - g->ib] * gr->rvh[j - g->jb] * gr->rmh[oo]);
          float u1 = ua[uI(g, i, j, k)], u2 = ua[uI(g, i + 1, j, k)];
          float v1 = va[vI(g, i, j, k)], v2 = va[vI(g, i, j + 1, k)];
          float w1 = wa[oo], w2 = wa[sI(g, i, j, k + 1)];
          double w = (double)(0.5f * (w1 + w2));
          float qv = moist ? qa[X.nqv * ns + oo] : 0.0f, ql = moist ? QL(o) : 0.0f;
          double qtot = (double)(qv + ql + 0.0f);
          float r = rho[oo];
          f1 = f1 + r * tem * (1.0 + qtot) * 0.5 *
                        (0.5f * (u1 * u1 + u2 * u2) + 0.5f * (v1 * v1 + v2 * v2) + 0.5f * (w1 * w1 + w2 * w2)) +
               (ql * r) * tem * 0.5 * (0.0 - 2.0 * w * 0.0);
          double tmp = (double)((gr->th0[oo] + tha[oo]) * (gr->pi0[oo] + ppi[oo]));
          f2 = f2 + r * tem * (cv + cvv * qv) * tmp;
          f3 = f3 + r * tem * (1.0 + qtot) * gg * zh[k];
          f4 = f4 + r * tem * ql * (cpl * tmp - lv1) + r * tem * 0.0 * (cpi * tmp - ls1);
        }
      ek = ek + f1; ei = ei + f2; ep = ep + f3; le = le + f4;
    }
    ek = ek * dv; ei = ei * dv; ep = ep * dv; le = le * dv;
    n = emit(rstat, n, (float)ek); n = emit(rstat, n, (float)ei);
    n = emit(rstat, n, (float)ep); n = emit(rstat, n, (float)le);
    n = emit(rstat, n, (float)(ek + ei + ep + le));
  }
  if (o->stat_mo) {                 /* calcmoe (misclibs.F:3462-3558), vr = 0 */
    double tmu = 0.0, tmv = 0.0, tmw = 0.0;
    for (int k = 1; k <= nk; k++) {
      double f1 = 0.0, f2 = 0.0, f3 = 0.0;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long oo = sI(g, i, j, k);
          float qv = moist ? qa[X.nqv * ns + oo] : 0.0f, ql = moist ? QL(o) : 0.0f;
          double qtot = qv + ql + 0.0f;
          double tem = gr->ruh[i - g->ib] * gr->rvh[j - g->jb] * gr->rmh[oo];
          float r = rho[oo];
          f1 = f1 + r * tem * (1.0 + qtot) * (0.0f + 0.5f * (ua[uI(g, i, j, k)] + ua[uI(g, i + 1, j, k)]));
          f2 = f2 + r * tem * (1.0 + qtot) * (0.0f + 0.5f * (va[vI(g, i, j, k)] + va[vI(g, i, j + 1, k)]));
          f3 = f3 + r * tem * (1.0 + qtot) * (0.5f * (wa[oo] + wa[sI(g, i, j, k + 1)])) - r * tem * ql * 0.0;
        }
      tmu = tmu + f1; tmv = tmv + f2; tmw = tmw + f3;
    }
    n = emit(rstat, n, (float)(tmu * dv)); n = emit(rstat, n, (float)(tmv * dv)); n = emit(rstat, n, (float)(tmw * dv));
  }
  if (o->stat_tmf) {                /* tmf (misclibs.F:3566-3636) */
    double tu = 0.0, td = 0.0;
    for (int k = 1; k <= nk; k++) {
      double f1 = 0.0, f2 = 0.0;
      for (int j = 1; j <= nj; j++)
        for (int i = 1; i <= ni; i++) {
          long oo = sI(g, i, j, k);
          double mf = rho[oo] * 0.5f * (wa[oo] + wa[sI(g, i, j, k + 1)]) * gr->ruh[i - g->ib] * gr->rvh[j - g->jb];
          f1 = f1 + fmax(mf, 0.0);
          f2 = f2 + fmin(mf, 0.0);
        }
      tu = tu + f1; td = td + f2;
    }
    n = emit(rstat, n, (float)(tu * g->dx * g->dy)); n = emit(rstat, n, (float)(td * g->dx * g->dy));
  }
#undef QL
  /* budgets kept by the caller (NULL: zero) */
  if (moist && o->stat_pcn)
    for (int b = 0; b < o->nbudget; b++) n = emit(rstat, n, qbudget ? (float)qbudget[b] : 0.0f);
  if (moist && o->stat_qsrc) {
    for (int q = 0; q < numq; q++) n = emit(rstat, n, asq ? (float)asq[q] : 0.0f);
    for (int q = 0; q < numq; q++) n = emit(rstat, n, bsq ? (float)bsq[q] : 0.0f);
  }
  *nstat = n;
  return 0;
}
