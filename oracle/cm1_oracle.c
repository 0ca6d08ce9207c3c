/*
 * cm1_oracle.c -- CPU restatement of CM1 r21.1's dynamical-core large step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * library: tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may call it, as the checker or as the timed CPU baseline.
 * The product path (libcm1g.so, cm1_b200) never links or calls it.
 *
 * PARITY UNPINNED: the reference is Fortran and no Fortran compiler exists
 * on the build or GPU machines, and the reference ships no golden vectors
 * for this path.  The restatement is pinned instead by known-answer tests
 * (tests/test_oracle_kat.py) derived from the reference's formulas.
 *
 * Each routine follows the loop nests, index ranges and floating-point
 * evaluation order of the Fortran routine it cites (file:line in the
 * reference tree).  Fortran evaluates `a*b*c` as `(a*b)*c`, default REAL is
 * binary32, constants such as 2.0/6.0 are folded in binary32, and WENO's
 * smoothness weights are binary64 (adv_routines.F:6166-6205).  Build with
 * -ffp-contract=off so that no fused multiply-add changes a rounding.
 *
 * Scope (same as the CUDA path): psolver=3, no terrain, axisymm=0, icor=0,
 * no immersed boundaries, no budgets, no 6th-order diffusion, hadvord*=
 * vadvord*=5, WENO5 for scalars (advwenos 0/1/2), no momentum WENO.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/cm1g.h"

/* ------------------------------------------------------------------ */
/* Fortran-layout array views                                          */
/* ------------------------------------------------------------------ */
typedef struct { float *p; long off, sy, sz; } F3;
#define A3(F, i, j, k) ((F).p[(F).off + (long)(i) + (F).sy * (long)(j) + (F).sz * (long)(k)])

typedef struct { uint8_t *p; long off, sy, sz; } B3;
#define L3(F, i, j, k) ((F).p[(F).off + (long)(i) + (F).sy * (long)(j) + (F).sz * (long)(k)])

/* constants of constants.F:set_constants (constants.F:65-175) */
typedef struct {
  float g, rd, rv, cp, cv, cpv, cvv, cpl, cpi;
  float rovcp, rddcv, cpdrd, reps, repsm1;
} Consts;

static void set_constants(int testcase, Consts *c) {
  if (testcase == 4) {        /* constants.F:72-80 */
    c->g = 9.81f; c->rd = 287.0f; c->cp = 1015.0f; c->cpv = 1870.0f;
  } else if (testcase == 5) { /* constants.F:82-90 */
    c->g = 9.81f; c->rd = 287.0f; c->cp = 1004.0f; c->cpv = 1870.0f;
  } else {                    /* constants.F:103-110 (cm1 defaults) */
    c->g = 9.81f; c->rd = 287.04f; c->cp = 1005.7f; c->cpv = 1870.0f;
  }
  c->rv = 461.5f;             /* constants.F:116-140 */
  c->cv = c->cp - c->rd;
  c->cvv = c->cpv - c->rv;
  c->rovcp = c->rd / c->cp;
  c->rddcv = c->rd / c->cv;
  c->cpdrd = c->cp / c->rd;
  c->reps = c->rv / c->rd;
  c->repsm1 = c->rv / c->rd - 1.0f;
  c->cpl = 4190.0f;           /* constants.F:150-151 */
  c->cpi = 2106.0f;
}

static const float EPSILON_ADV = 1.0e-18f;  /* constants.F:57 */
static const float TH0R = 300.0f;           /* constants.F:15 */
static const float P00 = 1.0e5f;            /* constants.F:17 */
static const float CSMAX = 350.0f;          /* constants.F:45 */

/* The binary32 powers of the pressure/density relations (solve2.F:1580-1606,
 * 1976-2033) and of the Kessler scheme.  The reference, built with gfortran,
 * evaluates real**real with the C library's powf; glibc's powf is not
 * correctly rounded for about 0.1% of the arguments these relations see.
 * Mode 0 (default) calls powf, as the reference build does; mode 1 evaluates
 * the power in binary64 and rounds once (the correctly rounded result for all
 * but vanishingly rare arguments), the choice of the CUDA path.  Comparing the
 * two modes measures how much a last-place choice of the math library moves
 * the model. */
static int g_pow_mode = 0;
void oracle_set_pow_mode(int mode) { g_pow_mode = mode; }
int oracle_get_pow_mode(void) { return g_pow_mode; }
static float opowf(float x, float y) { return g_pow_mode ? (float)pow((double)x, (double)y) : powf(x, y); }

typedef struct {
  int ni, nj, nk, ngxy, ib, ie, jb, je, kb, ke, NI, NJ, NK;
  float dx, dy, dz, rdx, rdy, rdz;
  int wbc, ebc, sbc, nbc, ibw, ibe, ibs, ibn;
  const cm1g_config_t *cfg;
  Consts c;
  /* 1-D metrics, indexed with their Fortran lower bound */
  const float *uh, *ruh, *uf, *ruf, *vh, *rvh, *vf, *rvf;
  F3 mh, rmh, c1, c2, mf, pi0, rho0, rr0, rf0, rrf0, th0, rth0, qv0, qc0, qi0, prs0, u0, v0;
  F3 dtu0, dtv0; /* 2-D (ib:ie,jb:je), k unused */
} OG;

static F3 mkS(const OG *g, const float *p) {
  F3 f; f.p = (float *)p; f.sy = g->NI; f.sz = (long)g->NI * g->NJ;
  f.off = -((long)g->ib + f.sy * g->jb + f.sz * g->kb); return f;
}
static F3 mkU(const OG *g, const float *p) {
  F3 f; f.p = (float *)p; f.sy = g->NI + 1; f.sz = (long)(g->NI + 1) * g->NJ;
  f.off = -((long)g->ib + f.sy * g->jb + f.sz * g->kb); return f;
}
static F3 mkV(const OG *g, const float *p) {
  F3 f; f.p = (float *)p; f.sy = g->NI; f.sz = (long)g->NI * (g->NJ + 1);
  f.off = -((long)g->ib + f.sy * g->jb + f.sz * g->kb); return f;
}
static F3 mkW(const OG *g, const float *p) { return mkS(g, p); }
static F3 mk2(const OG *g, const float *p) {
  F3 f; f.p = (float *)p; f.sy = g->NI; f.sz = 0;
  f.off = -((long)g->ib + f.sy * g->jb); return f;
}
static B3 mkB(const OG *g, uint8_t *p) {
  B3 f; f.p = p; f.sy = g->NI; f.sz = (long)g->NI * g->NJ;
  f.off = -((long)g->ib + f.sy * g->jb + f.sz * g->kb); return f;
}
/* radbcw/e (jb:je,kb:ke) and radbcs/n (ib:ie,kb:ke) */
#define RJK(g, a, j, k) ((a)[((j) - (g)->jb) + (long)(g)->NJ * ((k) - (g)->kb)])
#define RIK(g, a, i, k) ((a)[((i) - (g)->ib) + (long)(g)->NI * ((k) - (g)->kb)])

#define UH(i) (g->uh[(i) - g->ib])
#define RUH(i) (g->ruh[(i) - g->ib])
#define UF(i) (g->uf[(i) - g->ib])
#define RUF(i) (g->ruf[(i) - g->ib])
#define VH(j) (g->vh[(j) - g->jb])
#define RVH(j) (g->rvh[(j) - g->jb])
#define VF(j) (g->vf[(j) - g->jb])
#define RVF(j) (g->rvf[(j) - g->jb])

static long nS(const OG *g) { return (long)g->NI * g->NJ * g->NK; }
static long nU(const OG *g) { return (long)(g->NI + 1) * g->NJ * g->NK; }
static long nV(const OG *g) { return (long)g->NI * (g->NJ + 1) * g->NK; }
static long nW(const OG *g) { return (long)g->NI * g->NJ * (g->NK + 1); }

static char g_err[256];
const char *oracle_last_error(void) { return g_err; }

/* Arrays that cross the C-ABI structs (cm1g_grid_t, cm1g_state_t) are typed
 * float there.  RP/RPC view them as this file's real type, so that the FP64
 * build (oracle/make_r8.py turns every binary32 type, literal and function
 * of this file into binary64) reads the double arrays its caller passes. */
#define RP(p) ((float *)(void *)(p))
#define RPC(p) ((const float *)(const void *)(p))

static int og_setup(OG *g, const cm1g_config_t *cfg, const cm1g_grid_t *gr) {
  memset(g, 0, sizeof(*g));
  g->cfg = cfg;
  g->ni = cfg->ni; g->nj = cfg->nj; g->nk = cfg->nk; g->ngxy = cfg->ngxy;
  g->ib = 1 - g->ngxy; g->ie = g->ni + g->ngxy;
  g->jb = 1 - g->ngxy; g->je = g->nj + g->ngxy;
  g->kb = 0; g->ke = g->nk + 1;
  g->NI = g->ie - g->ib + 1; g->NJ = g->je - g->jb + 1; g->NK = g->ke - g->kb + 1;
  g->dx = cfg->dx; g->dy = cfg->dy; g->dz = cfg->dz;
  g->rdx = 1.0f / cfg->dx; g->rdy = 1.0f / cfg->dy; g->rdz = 1.0f / cfg->dz; /* param.F:6325-6327 */
  g->wbc = cfg->wbc; g->ebc = cfg->ebc; g->sbc = cfg->sbc; g->nbc = cfg->nbc;
  /* param.F:6678-6681 (one rank) */
  g->ibw = (cfg->wbc != 1); g->ibe = (cfg->ebc != 1);
  g->ibs = (cfg->sbc != 1); g->ibn = (cfg->nbc != 1);
  set_constants(cfg->testcase, &g->c);
  if (cfg->psolver != 3 || cfg->terrain_flag || cfg->axisymm || cfg->icor) {
    snprintf(g_err, sizeof g_err, "oracle: only psolver=3, no terrain/axisymm/Coriolis");
    return -1;
  }
  if (cfg->hadvordrs != 5 || cfg->vadvordrs != 5 || cfg->hadvordrv != 5 || cfg->vadvordrv != 5 ||
      cfg->advwenov != 0 || (cfg->advwenos && cfg->weno_order != 5) || cfg->ngxy < 3) {
    snprintf(g_err, sizeof g_err, "oracle: only 5th-order / WENO5 scalar advection");
    return -1;
  }
  if (gr) {
    g->uh = RPC(gr->uh); g->ruh = RPC(gr->ruh); g->uf = RPC(gr->uf); g->ruf = RPC(gr->ruf);
    g->vh = RPC(gr->vh); g->rvh = RPC(gr->rvh); g->vf = RPC(gr->vf); g->rvf = RPC(gr->rvf);
    g->mh = mkS(g, RPC(gr->mh)); g->rmh = mkS(g, RPC(gr->rmh)); g->c1 = mkS(g, RPC(gr->c1)); g->c2 = mkS(g, RPC(gr->c2));
    g->mf = mkW(g, RPC(gr->mf));
    g->pi0 = mkS(g, RPC(gr->pi0)); g->rho0 = mkS(g, RPC(gr->rho0)); g->rr0 = mkS(g, RPC(gr->rr0));
    g->rf0 = mkS(g, RPC(gr->rf0)); g->rrf0 = mkS(g, RPC(gr->rrf0)); g->th0 = mkS(g, RPC(gr->th0));
    g->rth0 = mkS(g, RPC(gr->rth0)); g->qv0 = mkS(g, RPC(gr->qv0)); g->qc0 = mkS(g, RPC(gr->qc0));
    g->qi0 = mkS(g, RPC(gr->qi0)); g->prs0 = mkS(g, RPC(gr->prs0));
    g->u0 = mkU(g, RPC(gr->u0)); g->v0 = mkV(g, RPC(gr->v0));
    g->dtu0 = mk2(g, RPC(gr->dtu0)); g->dtv0 = mk2(g, RPC(gr->dtv0));
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Face-value functions                                                */
/* ------------------------------------------------------------------ */

/* flx3: adv_routines.F:5971-5986 */
static inline float flx3(float s1, float s2, float s3) {
  return ((-1.0f / 6.0f) * s1 + (5.0f / 6.0f) * s2) + (2.0f / 6.0f) * s3;
}

/* flx5: adv_routines.F:6006-6024 (Wicker and Skamarock 2002) */
static inline float flx5(float s1, float s2, float s3, float s4, float s5) {
  return ((((2.0f / 60.0f) * s1 + (-13.0f / 60.0f) * s2) + (47.0f / 60.0f) * s3) +
          (27.0f / 60.0f) * s4) + (-3.0f / 60.0f) * s5;
}

/* weno5: adv_routines.F:6166-6205, siform=2 (Borges et al. 2008).
 * b1..b3 are evaluated in binary32 and stored in binary64; the weights and
 * the final quotient are binary64; the candidate stencils are binary32. */
static inline float weno5f(float s1, float s2, float s3, float s4, float s5, double weps) {
  const float c1312 = 13.0f / 12.0f;
  float t, u;
  t = (s1 - 2.0f * s2) + s3; u = (s1 - 4.0f * s2) + 3.0f * s3;
  double b1 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  t = (s2 - 2.0f * s3) + s4; u = s2 - s4;
  double b2 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  t = (s3 - 2.0f * s4) + s5; u = (3.0f * s3 - 4.0f * s4) + s5;
  double b3 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  double tau = fabs(b1 - b3), r;
  r = fmin(1.0e30, tau / (b1 + weps)); double w1 = (double)0.1f * (1.0 + r * r);
  r = fmin(1.0e30, tau / (b2 + weps)); double w2 = (double)0.6f * (1.0 + r * r);
  r = fmin(1.0e30, tau / (b3 + weps)); double w3 = (double)0.3f * (1.0 + r * r);
  float q1 = ((2.0f / 6.0f) * s1 + (-7.0f / 6.0f) * s2) + (11.0f / 6.0f) * s3;
  float q2 = ((-1.0f / 6.0f) * s2 + (5.0f / 6.0f) * s3) + (2.0f / 6.0f) * s4;
  float q3 = ((2.0f / 6.0f) * s3 + (5.0f / 6.0f) * s4) + (-1.0f / 6.0f) * s5;
  double num = (w1 * (double)q1 + w2 * (double)q2) + w3 * (double)q3;
  double den = (w1 + w2) + w3;
  return (float)(num / den);
}

/* upstrpd: adv_routines.F:6331-6355 (Beets & Koren 1996) */
static inline float upstrpd(float s1, float s2, float s3, double weps) {
  float dd = s2 - s1;
  float rr = (s3 - s2) / (copysignf((float)weps, dd) + dd);
  float phi = fmaxf(0.0f, fminf(rr, fminf((1.0f / 6.0f) + (2.0f / 6.0f) * rr, 1.0f)));
  return s2 + phi * (s2 - s1);
}

/* ------------------------------------------------------------------ */
/* Lateral boundary fills, bc.F (non-MPI branches)                     */
/* ------------------------------------------------------------------ */

/* bcs: bc.F:180-367 */
void oracle_bcs_g(const OG *g, F3 s) {
  int i, j, k, ni = g->ni, nj = g->nj, nk = g->nk, ng = g->ngxy;
  if (g->wbc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(s, 1 - i, j, k) = A3(s, ni + 1 - i, j, k);
  } else if (g->wbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1 - ng; i <= 0; i++)
      A3(s, i, j, k) = A3(s, 1, j, k);
  } else if (g->wbc == 3 || g->wbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1; i <= ng; i++)
      A3(s, 1 - i, j, k) = A3(s, i, j, k);
  }
  if (g->ebc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(s, ni + i, j, k) = A3(s, i, j, k);
  } else if (g->ebc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = ni + 1; i <= ni + ng; i++)
      A3(s, i, j, k) = A3(s, ni, j, k);
  } else if (g->ebc == 3 || g->ebc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1; i <= ng; i++)
      A3(s, ni + i, j, k) = A3(s, ni + 1 - i, j, k);
  }
  if (g->sbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(s, i, 1 - j, k) = A3(s, i, nj + 1 - j, k);
  } else if (g->sbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 1 - ng; j <= 0; j++) for (i = 0; i <= ni + 1; i++)
      A3(s, i, j, k) = A3(s, i, 1, k);
  } else if (g->sbc == 3 || g->sbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(s, i, 1 - j, k) = A3(s, i, j, k);
  }
  if (g->nbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(s, i, nj + j, k) = A3(s, i, j, k);
  } else if (g->nbc == 2) {
    for (k = 1; k <= nk; k++) for (j = nj + 1; j <= nj + ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(s, i, j, k) = A3(s, i, nj, k);
  } else if (g->nbc == 3 || g->nbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(s, i, nj + j, k) = A3(s, i, nj + 1 - j, k);
  }
}

/* bcp: bc.F:372-523 */
void oracle_bcp_g(const OG *g, F3 p) {
  int i, j, k, ni = g->ni, nj = g->nj, nk = g->nk;
  if (g->wbc == 1) { for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) A3(p, 0, j, k) = A3(p, ni, j, k); }
  else if (g->wbc >= 2 && g->wbc <= 4) { for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) A3(p, 0, j, k) = A3(p, 1, j, k); }
  if (g->ebc == 1) { for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) A3(p, ni + 1, j, k) = A3(p, 1, j, k); }
  else if (g->ebc >= 2 && g->ebc <= 4) { for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) A3(p, ni + 1, j, k) = A3(p, ni, j, k); }
  if (g->sbc == 1) { for (k = 1; k <= nk; k++) for (i = 0; i <= ni + 1; i++) A3(p, i, 0, k) = A3(p, i, nj, k); }
  else if (g->sbc >= 2 && g->sbc <= 4) { for (k = 1; k <= nk; k++) for (i = 0; i <= ni + 1; i++) A3(p, i, 0, k) = A3(p, i, 1, k); }
  if (g->nbc == 1) { for (k = 1; k <= nk; k++) for (i = 0; i <= ni + 1; i++) A3(p, i, nj + 1, k) = A3(p, i, 1, k); }
  else if (g->nbc >= 2 && g->nbc <= 4) { for (k = 1; k <= nk; k++) for (i = 0; i <= ni + 1; i++) A3(p, i, nj + 1, k) = A3(p, i, nj, k); }
}

/* bcu: bc.F:528-717 */
void oracle_bcu_g(const OG *g, F3 u) {
  int i, j, k, ni = g->ni, nj = g->nj, nk = g->nk, ng = g->ngxy;
  if (g->wbc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(u, 1 - i, j, k) = A3(u, ni + 1 - i, j, k);
  } else if (g->wbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1 - ng; i <= 0; i++)
      A3(u, i, j, k) = A3(u, 1, j, k);
  } else if (g->wbc == 3 || g->wbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) {
      A3(u, 1, j, k) = 0.0f;
      for (i = 1; i <= ng; i++) A3(u, 1 - i, j, k) = -A3(u, 1 + i, j, k);
    }
  }
  if (g->ebc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(u, ni + 1 + i, j, k) = A3(u, 1 + i, j, k);
  } else if (g->ebc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = ni + 2; i <= ni + 1 + ng; i++)
      A3(u, i, j, k) = A3(u, ni + 1, j, k);
  } else if (g->ebc == 3 || g->ebc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 1; j++) {
      A3(u, ni + 1, j, k) = 0.0f;
      for (i = 1; i <= ng; i++) A3(u, ni + 1 + i, j, k) = -A3(u, ni + 1 - i, j, k);
    }
  }
  if (g->sbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie + 1; i++)
      A3(u, i, 1 - j, k) = A3(u, i, nj + 1 - j, k);
  } else if (g->sbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 1 - ng; j <= 0; j++) for (i = 0; i <= ni + 2; i++)
      A3(u, i, j, k) = A3(u, i, 1, k);
  } else if (g->sbc == 3 || g->sbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 2; i++)
      A3(u, i, 1 - j, k) = A3(u, i, j, k);
  }
  if (g->nbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie + 1; i++)
      A3(u, i, nj + j, k) = A3(u, i, j, k);
  } else if (g->nbc == 2) {
    for (k = 1; k <= nk; k++) for (j = nj + 1; j <= nj + ng; j++) for (i = 0; i <= ni + 2; i++)
      A3(u, i, j, k) = A3(u, i, nj, k);
  } else if (g->nbc == 3 || g->nbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 2; i++)
      A3(u, i, nj + j, k) = A3(u, i, nj + 1 - j, k);
  }
}

/* bcv: bc.F:722-937 (south/north first, then west/east) */
void oracle_bcv_g(const OG *g, F3 v) {
  int i, j, k, ni = g->ni, nj = g->nj, nk = g->nk, ng = g->ngxy;
  if (g->sbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(v, i, 1 - j, k) = A3(v, i, nj + 1 - j, k);
  } else if (g->sbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 1 - ng; j <= 0; j++) for (i = 0; i <= ni + 1; i++)
      A3(v, i, j, k) = A3(v, i, 1, k);
  } else if (g->sbc == 3 || g->sbc == 4) {
    for (k = 1; k <= nk; k++) {
      for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++) A3(v, i, 1 - j, k) = -A3(v, i, j + 1, k);
      for (i = 0; i <= ni + 1; i++) A3(v, i, 1, k) = 0.0f;
    }
  }
  if (g->nbc == 1) {
    for (k = 1; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(v, i, nj + 1 + j, k) = A3(v, i, 1 + j, k);
  } else if (g->nbc == 2) {
    for (k = 1; k <= nk; k++) for (j = nj + 2; j <= nj + 1 + ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(v, i, j, k) = A3(v, i, nj + 1, k);
  } else if (g->nbc == 3 || g->nbc == 4) {
    for (k = 1; k <= nk; k++) {
      for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++) A3(v, i, nj + 1 + j, k) = -A3(v, i, nj + 1 - j, k);
      for (i = 0; i <= ni + 1; i++) A3(v, i, nj + 1, k) = 0.0f;
    }
  }
  if (g->wbc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je + 1; j++) for (i = 1; i <= ng; i++)
      A3(v, 1 - i, j, k) = A3(v, ni + 1 - i, j, k);
  } else if (g->wbc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 2; j++) for (i = 1 - ng; i <= 0; i++)
      A3(v, i, j, k) = A3(v, 1, j, k);
  } else if (g->wbc == 3 || g->wbc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 2; j++) for (i = 1; i <= ng; i++)
      A3(v, 1 - i, j, k) = A3(v, i, j, k);
  }
  if (g->ebc == 1) {
    for (k = 1; k <= nk; k++) for (j = g->jb; j <= g->je + 1; j++) for (i = 1; i <= ng; i++)
      A3(v, ni + i, j, k) = A3(v, i, j, k);
  } else if (g->ebc == 2) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 2; j++) for (i = ni + 1; i <= ni + ng; i++)
      A3(v, i, j, k) = A3(v, ni, j, k);
  } else if (g->ebc == 3 || g->ebc == 4) {
    for (k = 1; k <= nk; k++) for (j = 0; j <= nj + 2; j++) for (i = 1; i <= ng; i++)
      A3(v, ni + i, j, k) = A3(v, ni + 1 - i, j, k);
  }
}

/* bcw: bc.F:942-1146 */
void oracle_bcw_g(const OG *g, F3 w, int flag) {
  int i, j, k, ni = g->ni, nj = g->nj, nk = g->nk, ng = g->ngxy;
  if (g->wbc == 1) {
    for (k = 2; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(w, 1 - i, j, k) = A3(w, ni + 1 - i, j, k);
  } else if (g->wbc == 2) {
    for (k = 2; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1 - ng; i <= 0; i++)
      A3(w, i, j, k) = A3(w, 1, j, k);
  } else if (g->wbc == 3 || g->wbc == 4) {
    for (k = 2; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1; i <= ng; i++)
      A3(w, 1 - i, j, k) = A3(w, i, j, k);
  }
  if (g->ebc == 1) {
    for (k = 2; k <= nk; k++) for (j = g->jb; j <= g->je; j++) for (i = 1; i <= ng; i++)
      A3(w, ni + i, j, k) = A3(w, i, j, k);
  } else if (g->ebc == 2) {
    for (k = 2; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = ni + 1; i <= ni + ng; i++)
      A3(w, i, j, k) = A3(w, ni, j, k);
  } else if (g->ebc == 3 || g->ebc == 4) {
    for (k = 2; k <= nk; k++) for (j = 0; j <= nj + 1; j++) for (i = 1; i <= ng; i++)
      A3(w, ni + i, j, k) = A3(w, ni + 1 - i, j, k);
  }
  if (g->sbc == 1) {
    for (k = 2; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(w, i, 1 - j, k) = A3(w, i, nj + 1 - j, k);
  } else if (g->sbc == 2) {
    for (k = 2; k <= nk; k++) for (j = 1 - ng; j <= 0; j++) for (i = 0; i <= ni + 1; i++)
      A3(w, i, j, k) = A3(w, i, 1, k);
  } else if (g->sbc == 3 || g->sbc == 4) {
    for (k = 2; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(w, i, 1 - j, k) = A3(w, i, j, k);
  }
  if (g->nbc == 1) {
    for (k = 2; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = g->ib; i <= g->ie; i++)
      A3(w, i, nj + j, k) = A3(w, i, j, k);
  } else if (g->nbc == 2) {
    for (k = 2; k <= nk; k++) for (j = nj + 1; j <= nj + ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(w, i, j, k) = A3(w, i, nj, k);
  } else if (g->nbc == 3 || g->nbc == 4) {
    for (k = 2; k <= nk; k++) for (j = 1; j <= ng; j++) for (i = 0; i <= ni + 1; i++)
      A3(w, i, nj + j, k) = A3(w, i, nj + 1 - j, k);
  }
  if (flag == 1) {  /* bc.F:1127-1137 */
    for (j = 0; j <= nj + 1; j++) for (i = 0; i <= ni + 1; i++) {
      A3(w, i, j, 1) = 0.0f; A3(w, i, j, nk + 1) = 0.0f;
    }
  }
}

/* ------------------------------------------------------------------ */
/* Horizontal and vertical fluxes (adv_routines.F)                      */
/* ------------------------------------------------------------------ */

/* hadv_flx5 (adv_routines.F:1335-1481) and hadv_weno5 (204-435).
 * stag 1 scalar, 2 u, 3 v, 4 w.  weno != 0 selects weno5 (scalars only:
 * momentum WENO is outside this build). */
static void hadv5(const OG *g, int stag, int weno, int pdef, double weps,
                  F3 rru, F3 rrv, F3 dumx, F3 dumy, F3 a) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  if (stag == 1) {
    float bmin = (float)weps;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++)
      for (int j = 1; j <= nj + 1; j++)
        for (int i = 1; i <= ni + 1; i++) {
          float s1, s2, s3, s4, s5, r = A3(rru, i, j, k);
          if (r >= 0.0f) { s1 = A3(a, i - 3, j, k); s2 = A3(a, i - 2, j, k); s3 = A3(a, i - 1, j, k); s4 = A3(a, i, j, k); s5 = A3(a, i + 1, j, k); }
          else { s1 = A3(a, i + 2, j, k); s2 = A3(a, i + 1, j, k); s3 = A3(a, i, j, k); s4 = A3(a, i - 1, j, k); s5 = A3(a, i - 2, j, k); }
          if (!weno) A3(dumx, i, j, k) = r * flx5(s1, s2, s3, s4, s5);
          else if (pdef == 1) {
            float bmax = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(s1), fabsf(s2)), fabsf(s3)), fabsf(s4)), fabsf(s5));
            /* bmin is weps in double (adv_routines.F:243: bmin = weps, real) */
            A3(dumx, i, j, k) = (bmax > bmin) ? r * weno5f(s1, s2, s3, s4, s5, weps) : 0.0f;
          } else A3(dumx, i, j, k) = r * weno5f(s1, s2, s3, s4, s5, weps);
          r = A3(rrv, i, j, k);
          if (r >= 0.0f) { s1 = A3(a, i, j - 3, k); s2 = A3(a, i, j - 2, k); s3 = A3(a, i, j - 1, k); s4 = A3(a, i, j, k); s5 = A3(a, i, j + 1, k); }
          else { s1 = A3(a, i, j + 2, k); s2 = A3(a, i, j + 1, k); s3 = A3(a, i, j, k); s4 = A3(a, i, j - 1, k); s5 = A3(a, i, j - 2, k); }
          if (!weno) A3(dumy, i, j, k) = r * flx5(s1, s2, s3, s4, s5);
          else if (pdef == 1) {
            float bmax = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(s1), fabsf(s2)), fabsf(s3)), fabsf(s4)), fabsf(s5));
            A3(dumy, i, j, k) = (bmax > bmin) ? r * weno5f(s1, s2, s3, s4, s5, weps) : 0.0f;
          } else A3(dumy, i, j, k) = r * weno5f(s1, s2, s3, s4, s5, weps);
        }
  } else if (stag == 2) {
    int i1 = g->ibw ? 2 : 1, i2 = g->ibe ? ni : ni + 1;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++)
      for (int j = 1; j <= nj + 1; j++)
        for (int i = i1 - 1; i <= i2; i++) {
          float ubar = 0.5f * (A3(rru, i, j, k) + A3(rru, i + 1, j, k));
          if (ubar >= 0.0f) A3(dumx, i, j, k) = ubar * flx5(A3(a, i - 2, j, k), A3(a, i - 1, j, k), A3(a, i, j, k), A3(a, i + 1, j, k), A3(a, i + 2, j, k));
          else A3(dumx, i, j, k) = ubar * flx5(A3(a, i + 3, j, k), A3(a, i + 2, j, k), A3(a, i + 1, j, k), A3(a, i, j, k), A3(a, i - 1, j, k));
          float vbar = 0.5f * (A3(rrv, i, j, k) + A3(rrv, i - 1, j, k));
          if (vbar >= 0.0f) A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j - 3, k), A3(a, i, j - 2, k), A3(a, i, j - 1, k), A3(a, i, j, k), A3(a, i, j + 1, k));
          else A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j + 2, k), A3(a, i, j + 1, k), A3(a, i, j, k), A3(a, i, j - 1, k), A3(a, i, j - 2, k));
        }
  } else if (stag == 3) {
    int j1 = g->ibs ? 2 : 1, j2 = g->ibn ? nj : nj + 1;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++)
      for (int j = j1 - 1; j <= j2; j++)
        for (int i = 1; i <= ni + 1; i++) {
          float ubar = 0.5f * (A3(rru, i, j, k) + A3(rru, i, j - 1, k));
          if (ubar >= 0.0f) A3(dumx, i, j, k) = ubar * flx5(A3(a, i - 3, j, k), A3(a, i - 2, j, k), A3(a, i - 1, j, k), A3(a, i, j, k), A3(a, i + 1, j, k));
          else A3(dumx, i, j, k) = ubar * flx5(A3(a, i + 2, j, k), A3(a, i + 1, j, k), A3(a, i, j, k), A3(a, i - 1, j, k), A3(a, i - 2, j, k));
          float vbar = 0.5f * (A3(rrv, i, j, k) + A3(rrv, i, j + 1, k));
          if (vbar >= 0.0f) A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j - 2, k), A3(a, i, j - 1, k), A3(a, i, j, k), A3(a, i, j + 1, k), A3(a, i, j + 2, k));
          else A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j + 3, k), A3(a, i, j + 2, k), A3(a, i, j + 1, k), A3(a, i, j, k), A3(a, i, j - 1, k));
        }
  } else { /* stag 4 */
#pragma omp parallel for
    for (int k = 2; k <= nk; k++)
      for (int j = 1; j <= nj + 1; j++)
        for (int i = 1; i <= ni + 1; i++) {
          float cc2 = 0.5f * (A3(g->c2, i - 1, j, k) + A3(g->c2, i, j, k));
          float cc1 = 1.0f - cc2;
          float ubar = cc2 * A3(rru, i, j, k) + cc1 * A3(rru, i, j, k - 1);
          if (ubar >= 0.0f) A3(dumx, i, j, k) = ubar * flx5(A3(a, i - 3, j, k), A3(a, i - 2, j, k), A3(a, i - 1, j, k), A3(a, i, j, k), A3(a, i + 1, j, k));
          else A3(dumx, i, j, k) = ubar * flx5(A3(a, i + 2, j, k), A3(a, i + 1, j, k), A3(a, i, j, k), A3(a, i - 1, j, k), A3(a, i - 2, j, k));
          cc2 = 0.5f * (A3(g->c2, i, j - 1, k) + A3(g->c2, i, j, k));
          cc1 = 1.0f - cc2;
          float vbar = cc2 * A3(rrv, i, j, k) + cc1 * A3(rrv, i, j, k - 1);
          if (vbar >= 0.0f) A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j - 3, k), A3(a, i, j - 2, k), A3(a, i, j - 1, k), A3(a, i, j, k), A3(a, i, j + 1, k));
          else A3(dumy, i, j, k) = vbar * flx5(A3(a, i, j + 2, k), A3(a, i, j + 1, k), A3(a, i, j, k), A3(a, i, j - 1, k), A3(a, i, j - 2, k));
        }
  }
}

/* vadv_flx5 for scalars (adv_routines.F:3269-3297) with the lower-order
 * near-boundary fluxes vadv_lwr_flx_23/_35 (4817-4844, 5001-5029), and
 * vadv_weno5 (2359-2433) with vadv_lwr_weno_23/_35/_35_b (4038-4085,
 * 4220-4249, 4402-4452). */
static void vadv5_s(const OG *g, int weno, int pdefweno, double weps, F3 rrw, F3 dumz, F3 a) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float bmin = (float)weps;
#pragma omp parallel for
  for (int j = 1; j <= nj; j++)
    for (int i = 1; i <= ni; i++) {
      int k;
      if (!weno) {
        for (k = 4; k <= nk - 2; k++) {
          float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * flx5(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
          else A3(dumz, i, j, k) = r * flx5(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2));
        }
        k = 2; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k));
          else A3(dumz, i, j, k) = r * flx3(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1)); }
        k = nk; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * flx3(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k));
          else A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k)); }
        k = 3; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * flx3(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k));
          else A3(dumz, i, j, k) = r * flx5(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2)); }
        k = nk - 1; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * flx5(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
          else A3(dumz, i, j, k) = r * flx3(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1)); }
      } else if (pdefweno == 1) {
        for (k = 3; k <= nk - 1; k++) {
          float r = A3(rrw, i, j, k), s1, s2, s3, s4, s5;
          if (r >= 0.0f) { s1 = A3(a, i, j, k - 3); s2 = A3(a, i, j, k - 2); s3 = A3(a, i, j, k - 1); s4 = A3(a, i, j, k); s5 = A3(a, i, j, k + 1); }
          else { s1 = A3(a, i, j, k + 2); s2 = A3(a, i, j, k + 1); s3 = A3(a, i, j, k); s4 = A3(a, i, j, k - 1); s5 = A3(a, i, j, k - 2); }
          int doit = 0;
          float bmax = fmaxf(fmaxf(fmaxf(fmaxf(fabsf(s1), fabsf(s2)), fabsf(s3)), fabsf(s4)), fabsf(s5));
          if (bmax > bmin) doit = 1;
          if (k == 3 && r > 0.0f) doit = 0;
          if (k == nk - 1 && r < 0.0f) doit = 0;
          A3(dumz, i, j, k) = doit ? r * weno5f(s1, s2, s3, s4, s5, weps) : 0.0f;
        }
        /* vadv_lwr_weno_23 */
        k = 2; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k));
          else A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), weps); }
        k = nk; { float r = A3(rrw, i, j, k);
          if (r > 0.0f) A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), weps);
          else A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k)); }
        /* vadv_lwr_weno_35_b */
        k = 3; { float r = A3(rrw, i, j, k);
          if (r > 0.0f) A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), weps); }
        k = nk - 1; { float r = A3(rrw, i, j, k);
          if (r < 0.0f) A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), weps); }
      } else {
        for (k = 4; k <= nk - 2; k++) {
          float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * weno5f(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1), weps);
          else A3(dumz, i, j, k) = r * weno5f(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2), weps);
        }
        k = 2; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k));
          else A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), weps); }
        k = nk; { float r = A3(rrw, i, j, k);
          if (r > 0.0f) A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), weps);
          else A3(dumz, i, j, k) = r * (A3(g->c1, i, j, k) * A3(a, i, j, k - 1) + A3(g->c2, i, j, k) * A3(a, i, j, k)); }
        /* vadv_lwr_weno_35 */
        k = 3; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), weps);
          else A3(dumz, i, j, k) = r * weno5f(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2), weps); }
        k = nk - 1; { float r = A3(rrw, i, j, k);
          if (r >= 0.0f) A3(dumz, i, j, k) = r * weno5f(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1), weps);
          else A3(dumz, i, j, k) = r * upstrpd(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), weps); }
      }
    }
}

/* vadv_flx5 for u (stag 2) and v (stag 3): adv_routines.F:3299-3364 with
 * vadv_lwr_flx_23 (4863-4976) and _35 (5044-5146). */
static void vadv5_uv(const OG *g, int stag, F3 rrw, F3 dumz, F3 a) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  int ilo = 1, ihi = ni, jlo = 1, jhi = nj;
  if (stag == 2) { ilo = g->ibw ? 2 : 1; ihi = g->ibe ? ni : ni + 1; }
  else { jlo = g->ibs ? 2 : 1; jhi = g->ibn ? nj : nj + 1; }
#pragma omp parallel for
  for (int j = jlo; j <= jhi; j++)
    for (int i = ilo; i <= ihi; i++) {
      int k;
#define WBAR(kk) (stag == 2 ? 0.5f * (A3(rrw, i, j, kk) + A3(rrw, i - 1, j, kk)) : 0.5f * (A3(rrw, i, j, kk) + A3(rrw, i, j - 1, kk)))
#define CC2(kk) (stag == 2 ? 0.5f * (A3(g->c2, i - 1, j, kk) + A3(g->c2, i, j, kk)) : 0.5f * (A3(g->c2, i, j - 1, kk) + A3(g->c2, i, j, kk)))
      for (k = 4; k <= nk - 2; k++) {
        float wbar = WBAR(k);
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
        else A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2));
      }
      k = 2; { float wbar = WBAR(k);
        if (wbar >= 0.0f) { float cc2 = CC2(k), cc1 = 1.0f - cc2; A3(dumz, i, j, k) = wbar * (cc1 * A3(a, i, j, k - 1) + cc2 * A3(a, i, j, k)); }
        else A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1)); }
      k = nk; { float wbar = WBAR(k);
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k));
        else { float cc2 = CC2(k), cc1 = 1.0f - cc2; A3(dumz, i, j, k) = wbar * (cc1 * A3(a, i, j, k - 1) + cc2 * A3(a, i, j, k)); } }
      k = 3; { float wbar = WBAR(k);
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k));
        else A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1), A3(a, i, j, k - 2)); }
      k = nk - 1; { float wbar = WBAR(k);
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k - 3), A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
        else A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1)); }
#undef WBAR
#undef CC2
    }
}

/* vadv_flx5 for w (stag 4): adv_routines.F:3366-3384 with
 * vadv_lwr_flx_23 (4979-5000) and _35 (5148-5172). */
static void vadv5_w(const OG *g, F3 rrw, F3 dumz, F3 a) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
#pragma omp parallel for
  for (int j = 1; j <= nj; j++)
    for (int i = 1; i <= ni; i++) {
      int k;
      for (k = 3; k <= nk - 2; k++) {
        float wbar = 0.5f * (A3(rrw, i, j, k) + A3(rrw, i, j, k + 1));
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1), A3(a, i, j, k + 2));
        else A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k + 3), A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1));
      }
      k = 1; { float wbar = 0.5f * (A3(rrw, i, j, k) + A3(rrw, i, j, k + 1));
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * 0.5f * (A3(a, i, j, k) + A3(a, i, j, k + 1));
        else A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k)); }
      k = nk; { float wbar = 0.5f * (A3(rrw, i, j, k) + A3(rrw, i, j, k + 1));
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
        else A3(dumz, i, j, k) = wbar * 0.5f * (A3(a, i, j, k) + A3(a, i, j, k + 1)); }
      k = 2; { float wbar = 0.5f * (A3(rrw, i, j, k) + A3(rrw, i, j, k + 1));
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1));
        else A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k + 3), A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k), A3(a, i, j, k - 1)); }
      k = nk - 1; { float wbar = 0.5f * (A3(rrw, i, j, k) + A3(rrw, i, j, k + 1));
        if (wbar >= 0.0f) A3(dumz, i, j, k) = wbar * flx5(A3(a, i, j, k - 2), A3(a, i, j, k - 1), A3(a, i, j, k), A3(a, i, j, k + 1), A3(a, i, j, k + 2));
        else A3(dumz, i, j, k) = wbar * flx3(A3(a, i, j, k + 2), A3(a, i, j, k + 1), A3(a, i, j, k)); }
    }
}

/* ------------------------------------------------------------------ */
/* Positive-definite limiter, pdef.F                                    */
/* ------------------------------------------------------------------ */

/* pdefx1: pdef.F:15-112 (no terrain) */
static void pdefx1(const OG *g, F3 rru, F3 advx, F3 dum, F3 s0, F3 s, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    A3(dum, i, j, k) = A3(g->rho0, 1, 1, k) * A3(s0, i, j, k) +
        dt * (A3(advx, i, j, k) + A3(s, i, j, k) * (A3(rru, i + 1, j, k) - A3(rru, i, j, k)) * g->rdx * UH(i));
  if (g->wbc == 2 && g->ibw) {
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
      if (A3(rru, 1, j, k) >= 0.0f) A3(dum, 1, j, k) = A3(g->rho0, 1, j, k) * A3(s0, 1, j, k);
  }
  if (g->ebc == 2 && g->ibe) {
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
      if (A3(rru, ni + 1, j, k) <= 0.0f) A3(dum, ni, j, k) = A3(g->rho0, ni, j, k) * A3(s0, ni, j, k);
  }
  oracle_bcs_g(g, dum);
}

/* pdefx2: pdef.F:117-264 (no terrain, Cartesian) */
static void pdefx2(const OG *g, F3 rru, F3 advx, F3 dum, F3 mass, B3 flag, F3 s0, F3 s, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float rdt = 1.0f / dt, smeps = g->cfg->smeps;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) {
    for (int j = 1; j <= nj; j++) for (int i = -1; i <= ni + 2; i++) { A3(mass, i, j, k) = 0.0f; L3(flag, i, j, k) = 0; }
    for (int j = 1; j <= nj; j++) for (int i = 0; i <= ni + 1; i++) {
      if (A3(dum, i, j, k) < 0.0f) {
        float foo1 = fmaxf(0.0f, A3(dum, i - 1, j, k)), foo2 = fmaxf(0.0f, A3(dum, i + 1, j, k));
        if (foo1 + foo2 > smeps) {
          float foo3 = fmaxf(A3(dum, i, j, k), -(foo1 + foo2)) / (foo1 + foo2);
          A3(mass, i - 1, j, k) = A3(mass, i - 1, j, k) + foo1 * foo3;
          A3(mass, i, j, k) = A3(mass, i, j, k) - (foo1 + foo2) * foo3;
          A3(mass, i + 1, j, k) = A3(mass, i + 1, j, k) + foo2 * foo3;
          if (A3(dum, i - 1, j, k) > smeps) L3(flag, i - 1, j, k) = 1;
          L3(flag, i, j, k) = 1;
          if (A3(dum, i + 1, j, k) > smeps) L3(flag, i + 1, j, k) = 1;
        }
      }
    }
  }
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    if (L3(flag, i, j, k))
      A3(advx, i, j, k) = (A3(dum, i, j, k) + A3(mass, i, j, k) - A3(g->rho0, 1, 1, k) * A3(s0, i, j, k)) * rdt -
                          A3(s, i, j, k) * (A3(rru, i + 1, j, k) - A3(rru, i, j, k)) * g->rdx * UH(i);
}

/* pdefy1: pdef.F:269-353 */
static void pdefy1(const OG *g, F3 rrv, F3 advy, F3 dum, F3 s0, F3 s, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    A3(dum, i, j, k) = A3(g->rho0, 1, 1, k) * A3(s0, i, j, k) +
        dt * (A3(advy, i, j, k) + A3(s, i, j, k) * (A3(rrv, i, j + 1, k) - A3(rrv, i, j, k)) * g->rdy * VH(j));
  if (g->sbc == 2 && g->ibs) {
    for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
      if (A3(rrv, i, 1, k) >= 0.0f) A3(dum, i, 1, k) = A3(g->rho0, i, 1, k) * A3(s0, i, 1, k);
  }
  if (g->nbc == 2 && g->ibn) {
    for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
      if (A3(rrv, i, nj + 1, k) <= 0.0f) A3(dum, i, nj, k) = A3(g->rho0, i, nj, k) * A3(s0, i, nj, k);
  }
  oracle_bcs_g(g, dum);
}

/* pdefy2: pdef.F:358-454 */
static void pdefy2(const OG *g, F3 rrv, F3 advy, F3 dum, F3 mass, B3 flag, F3 s0, F3 s, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float smeps = g->cfg->smeps;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) {
    for (int j = -1; j <= nj + 2; j++) for (int i = 1; i <= ni; i++) { A3(mass, i, j, k) = 0.0f; L3(flag, i, j, k) = 0; }
    for (int j = 0; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) {
      if (A3(dum, i, j, k) < 0.0f) {
        float foo1 = fmaxf(0.0f, A3(dum, i, j - 1, k)), foo2 = fmaxf(0.0f, A3(dum, i, j + 1, k));
        if (foo1 + foo2 > smeps) {
          float foo3 = fmaxf(A3(dum, i, j, k), -(foo1 + foo2)) / (foo1 + foo2);
          A3(mass, i, j - 1, k) = A3(mass, i, j - 1, k) + foo1 * foo3;
          A3(mass, i, j, k) = A3(mass, i, j, k) - (foo1 + foo2) * foo3;
          A3(mass, i, j + 1, k) = A3(mass, i, j + 1, k) + foo2 * foo3;
          if (A3(dum, i, j - 1, k) > smeps) L3(flag, i, j - 1, k) = 1;
          L3(flag, i, j, k) = 1;
          if (A3(dum, i, j + 1, k) > smeps) L3(flag, i, j + 1, k) = 1;
        }
      }
    }
  }
  float rdt = 1.0f / dt;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    if (L3(flag, i, j, k))
      A3(advy, i, j, k) = (A3(dum, i, j, k) + A3(mass, i, j, k) - A3(g->rho0, 1, 1, k) * A3(s0, i, j, k)) * rdt -
                          A3(s, i, j, k) * (A3(rrv, i, j + 1, k) - A3(rrv, i, j, k)) * g->rdy * VH(j);
}

/* pdefz: pdef.F:459-581 */
static void pdefz(const OG *g, F3 rrw, F3 advz, F3 dum, F3 mass, B3 flag, F3 s0, F3 s, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float smeps = g->cfg->smeps;
#pragma omp parallel for
  for (int j = 1; j <= nj; j++)
    for (int i = 1; i <= ni; i++) {
      for (int k = 1; k <= nk; k++)
        A3(dum, i, j, k) = A3(g->rho0, 1, 1, k) * A3(s0, i, j, k) +
            dt * (A3(advz, i, j, k) + A3(s, i, j, k) * (A3(rrw, i, j, k + 1) - A3(rrw, i, j, k)) * g->rdz * A3(g->mh, 1, 1, k));
      A3(dum, i, j, 0) = 0.0f; A3(dum, i, j, nk + 1) = 0.0f;
      for (int k = 0; k <= nk + 1; k++) { A3(mass, i, j, k) = 0.0f; L3(flag, i, j, k) = 0; }
      for (int k = 1; k <= nk; k++) {
        if (A3(dum, i, j, k) < 0.0f) {
          float foo1 = fmaxf(0.0f, A3(dum, i, j, k - 1)), foo2 = fmaxf(0.0f, A3(dum, i, j, k + 1));
          if (foo1 + foo2 > smeps) {
            float foo3 = fmaxf(A3(dum, i, j, k), -(foo1 + foo2)) / (foo1 + foo2);
            A3(mass, i, j, k - 1) = A3(mass, i, j, k - 1) + foo1 * foo3;
            A3(mass, i, j, k) = A3(mass, i, j, k) - (foo1 + foo2) * foo3;
            A3(mass, i, j, k + 1) = A3(mass, i, j, k + 1) + foo2 * foo3;
            if (A3(dum, i, j, k - 1) > smeps) L3(flag, i, j, k - 1) = 1;
            L3(flag, i, j, k) = 1;
            if (A3(dum, i, j, k + 1) > smeps) L3(flag, i, j, k + 1) = 1;
          }
        }
      }
      float rdt = 1.0f / dt;
      for (int k = 1; k <= nk; k++)
        if (L3(flag, i, j, k))
          A3(advz, i, j, k) = (A3(dum, i, j, k) + A3(mass, i, j, k) - A3(g->rho0, 1, 1, k) * A3(s0, i, j, k)) * rdt -
                              A3(s, i, j, k) * (A3(rrw, i, j, k + 1) - A3(rrw, i, j, k)) * g->rdz * A3(g->mh, 1, 1, k);
    }
}

/* ------------------------------------------------------------------ */
/* Advection drivers, adv.F                                             */
/* ------------------------------------------------------------------ */

typedef struct { F3 advx, advy, advz, dumx, dumy, dumz, mass; B3 flag; } Scratch;

/* 6th-order horizontal diffusion (idiff=1, difforder=6), adv.F:342-406 and
 * the advu/advv/advw forms (adv.F:1177-1236, 2115-2174, 3109-3170): the
 * difference stencil of a face between a(-1) and a(0), evaluated as
 * (10 (a0 - am1) - 5 (ap1 - am2)) + (ap2 - am3) like the Fortran. */
static inline float d6(float am3, float am2, float am1, float a0, float ap1, float ap2) {
  return (10.0f * (a0 - am1) - 5.0f * (ap1 - am2)) + (ap2 - am3);
}
/* the mdiff limiter: no flux against the local gradient (adv.F:366-373) */
static inline float d6lim(const OG *g, float f, float a0, float am1) {
  return (g->cfg->mdiff == 1 && f * (a0 - am1) <= 0.0f) ? 0.0f : f;
}
static inline int diff6_on(const OG *g) { return g->cfg->idiff == 1 && g->cfg->difforder == 6; }

static int scratch_alloc(const OG *g, Scratch *w) {
  long n = nS(g);
  float *b = (float *)calloc((size_t)n * 7, sizeof(float));
  uint8_t *f = (uint8_t *)calloc((size_t)n, 1);
  if (!b || !f) { free(b); free(f); return -1; }
  w->advx = mkS(g, b); w->advy = mkS(g, b + n); w->advz = mkS(g, b + 2 * n);
  w->dumx = mkS(g, b + 3 * n); w->dumy = mkS(g, b + 4 * n); w->dumz = mkS(g, b + 5 * n);
  w->mass = mkS(g, b + 6 * n); w->flag = mkB(g, f);
  return 0;
}
static void scratch_free(Scratch *w) { free(w->advx.p); free(w->flag.p); }

/* advs: adv.F:14-903 (Cartesian, no terrain, no diffusion, no budgets) */
static void advs_g(const OG *g, Scratch *w, int nrk, int wflag, F3 rru, F3 rrv, F3 rrw, F3 divx,
                   F3 s0, F3 s, F3 sten, int pdef, int pdefweno, float dt, double weps, F3 rho, F3 ri, int diffit) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  const cm1g_config_t *cfg = g->cfg;
  int doweno = (wflag == 1) && (cfg->advwenos == 1 || (cfg->advwenos == 2 && nrk == 3));
  int doitw = (g->wbc == 2 && g->ibw), doite = (g->ebc == 2 && g->ibe);
  int doits = (g->sbc == 2 && g->ibs), doitn = (g->nbc == 2 && g->ibn);
  F3 advx = w->advx, advy = w->advy, advz = w->advz, dumx = w->dumx, dumy = w->dumy, dumz = w->dumz;

  hadv5(g, 1, doweno, pdef, weps, rru, rrv, dumx, dumy, s);
  /* adv.F:212-268: set hadv to zero at inflow */
  if (doitw) for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
    if (A3(rru, 1, j, k) >= 0.0f) A3(dumx, 1, j, k) = A3(dumx, 2, j, k);
  if (doite) for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
    if (A3(rru, ni + 1, j, k) <= 0.0f) A3(dumx, ni + 1, j, k) = A3(dumx, ni, j, k);
  if (doits) for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
    if (A3(rrv, i, 1, k) >= 0.0f) A3(dumy, i, 1, k) = A3(dumy, i, 2, k);
  if (doitn) for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
    if (A3(rrv, i, nj + 1, k) <= 0.0f) A3(dumy, i, nj + 1, k) = A3(dumy, i, nj, k);
  /* adv.F:271-281 */
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    A3(advx, i, j, k) = -(A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * g->rdx * UH(i);
    A3(advy, i, j, k) = -(A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * g->rdy * VH(j);
  }
  /* adv.F:286-335: subtract the divx piece at inflow */
  if (doitw) for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
    if (A3(rru, 1, j, k) >= 0.0f)
      A3(advx, 1, j, k) = A3(advx, 1, j, k) - A3(s, 1, j, k) * (A3(rru, 2, j, k) - A3(rru, 1, j, k)) * g->rdx * UH(1);
  if (doite) for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
    if (A3(rru, ni + 1, j, k) <= 0.0f)
      A3(advx, ni, j, k) = A3(advx, ni, j, k) - A3(s, ni, j, k) * (A3(rru, ni + 1, j, k) - A3(rru, ni, j, k)) * g->rdx * UH(ni);
  if (doits) for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
    if (A3(rrv, i, 1, k) >= 0.0f)
      A3(advy, i, 1, k) = A3(advy, i, 1, k) - A3(s, i, 1, k) * (A3(rrv, i, 2, k) - A3(rrv, i, 1, k)) * g->rdy * VH(1);
  if (doitn) for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
    if (A3(rrv, i, nj + 1, k) <= 0.0f)
      A3(advy, i, nj, k) = A3(advy, i, nj, k) - A3(s, i, nj, k) * (A3(rrv, i, nj + 1, k) - A3(rrv, i, nj, k)) * g->rdy * VH(nj);
  /* adv.F:342-406: 6th-order diffusion */
  if (diffit == 1) {
    float coef = g->cfg->kdiff6 / 64.0f / dt;   /* adv.F:80-82 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) {
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) {
        float f = d6(A3(s, i - 3, j, k), A3(s, i - 2, j, k), A3(s, i - 1, j, k), A3(s, i, j, k), A3(s, i + 1, j, k),
                     A3(s, i + 2, j, k)) * 0.5f * (A3(rho, i - 1, j, k) + A3(rho, i, j, k));
        A3(dumx, i, j, k) = d6lim(g, f, A3(s, i, j, k), A3(s, i - 1, j, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
        A3(advx, i, j, k) = A3(advx, i, j, k) + coef * (A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * A3(ri, i, j, k) * A3(g->rho0, i, j, k);
      for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) {
        float f = d6(A3(s, i, j - 3, k), A3(s, i, j - 2, k), A3(s, i, j - 1, k), A3(s, i, j, k), A3(s, i, j + 1, k),
                     A3(s, i, j + 2, k)) * 0.5f * (A3(rho, i, j - 1, k) + A3(rho, i, j, k));
        A3(dumy, i, j, k) = d6lim(g, f, A3(s, i, j, k), A3(s, i, j - 1, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
        A3(advy, i, j, k) = A3(advy, i, j, k) + coef * (A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * A3(ri, i, j, k) * A3(g->rho0, i, j, k);
    }
  }
  /* adv.F:426-446 */
  if (pdef == 1) pdefx1(g, rru, advx, dumx, s0, s, dt);
  if (pdef == 1) pdefy1(g, rrv, advy, dumy, s0, s, dt);
  /* adv.F:451-577 */
  vadv5_s(g, doweno, pdefweno, weps, rrw, dumz, s);
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    float mhk = A3(g->mh, 1, 1, k);
    if (k == 1) A3(advz, i, j, k) = -A3(dumz, i, j, 2) * g->rdz * mhk;
    else if (k == nk) A3(advz, i, j, k) = +A3(dumz, i, j, nk) * g->rdz * mhk;
    else A3(advz, i, j, k) = -(A3(dumz, i, j, k + 1) - A3(dumz, i, j, k)) * g->rdz * mhk;
  }
  /* adv.F:614-627 */
  if (pdef == 1) {
    pdefz(g, rrw, advz, dumz, w->mass, w->flag, s0, s, dt);
    pdefx2(g, rru, advx, dumx, w->mass, w->flag, s0, s, dt);
    pdefy2(g, rrv, advy, dumy, w->mass, w->flag, s0, s, dt);
  }
  /* adv.F:650-659 */
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    A3(sten, i, j, k) = A3(sten, i, j, k) + (((A3(advx, i, j, k) + A3(advy, i, j, k)) + A3(advz, i, j, k)) +
                                             A3(s, i, j, k) * A3(divx, i, j, k)) * A3(g->rr0, 1, 1, k);
}

/* advu: adv.F:911-1839 (hadvordrv=vadvordrv=5, no WENO) */
static void advu_g(const OG *g, Scratch *w, F3 divx, F3 rru, F3 u3d, F3 uten, F3 rrv, F3 rrw, F3 rho, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  int i1 = g->ibw ? 2 : 1, i2 = g->ibe ? ni : ni + 1;
  int doits = (g->sbc == 2 && g->ibs), doitn = (g->nbc == 2 && g->ibn);
  F3 advx = w->advx, advy = w->advy, advz = w->advz, dumx = w->dumx, dumy = w->dumy, dumz = w->dumz;
  hadv5(g, 2, 0, 0, 0.0, rru, rrv, dumx, dumy, u3d);
  if (doits) for (int k = 1; k <= nk; k++) for (int i = i1; i <= i2; i++)
    if ((A3(rrv, i, 1, k) + A3(rrv, i - 1, 1, k)) >= 0.0f) A3(dumy, i, 1, k) = A3(dumy, i, 2, k);
  if (doitn) for (int k = 1; k <= nk; k++) for (int i = i1; i <= i2; i++)
    if ((A3(rrv, i, nj + 1, k) + A3(rrv, i - 1, nj + 1, k)) <= 0.0f) A3(dumy, i, nj + 1, k) = A3(dumy, i, nj, k);
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = i1; i <= i2; i++) {
    A3(advx, i, j, k) = -(A3(dumx, i, j, k) - A3(dumx, i - 1, j, k)) * g->rdx * UF(i);
    A3(advy, i, j, k) = -(A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * g->rdy * VH(j);
  }
  if (doits) for (int k = 1; k <= nk; k++) for (int i = i1; i <= i2; i++)
    if ((A3(rrv, i, 1, k) + A3(rrv, i - 1, 1, k)) >= 0.0f)
      A3(advy, i, 1, k) = A3(advy, i, 1, k) - A3(u3d, i, 1, k) * 0.5f *
          ((A3(rrv, i - 1, 2, k) - A3(rrv, i - 1, 1, k)) + (A3(rrv, i, 2, k) - A3(rrv, i, 1, k))) * g->rdy * VH(1);
  if (doitn) for (int k = 1; k <= nk; k++) for (int i = i1; i <= i2; i++)
    if ((A3(rrv, i, nj + 1, k) + A3(rrv, i - 1, nj + 1, k)) <= 0.0f)
      A3(advy, i, nj, k) = A3(advy, i, nj, k) - A3(u3d, i, nj, k) * 0.5f *
          ((A3(rrv, i - 1, nj + 1, k) - A3(rrv, i - 1, nj, k)) + (A3(rrv, i, nj + 1, k) - A3(rrv, i, nj, k))) * g->rdy * VH(nj);
  /* adv.F:1177-1236: 6th-order diffusion */
  if (diff6_on(g)) {
    float coef = g->cfg->kdiff6 / 64.0f / dt;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) {
      float r0 = A3(g->rho0, 1, 1, k);
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 2; i++) {
        float f = d6(A3(u3d, i - 3, j, k), A3(u3d, i - 2, j, k), A3(u3d, i - 1, j, k), A3(u3d, i, j, k),
                     A3(u3d, i + 1, j, k), A3(u3d, i + 2, j, k)) * A3(rho, i - 1, j, k);
        A3(dumx, i, j, k) = d6lim(g, f, A3(u3d, i, j, k), A3(u3d, i - 1, j, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = i1; i <= i2; i++)
        A3(advx, i, j, k) = A3(advx, i, j, k) + coef * (A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * (r0 + r0) /
                                                    (A3(rho, i - 1, j, k) + A3(rho, i, j, k));
      for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
        float f = d6(A3(u3d, i, j - 3, k), A3(u3d, i, j - 2, k), A3(u3d, i, j - 1, k), A3(u3d, i, j, k),
                     A3(u3d, i, j + 1, k), A3(u3d, i, j + 2, k)) * 0.25f *
                  ((A3(rho, i - 1, j - 1, k) + A3(rho, i, j, k)) + (A3(rho, i - 1, j, k) + A3(rho, i, j - 1, k)));
        A3(dumy, i, j, k) = d6lim(g, f, A3(u3d, i, j, k), A3(u3d, i, j - 1, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = i1; i <= i2; i++)
        A3(advy, i, j, k) = A3(advy, i, j, k) + coef * (A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * (r0 + r0) /
                                                    (A3(rho, i - 1, j, k) + A3(rho, i, j, k));
    }
  }
  vadv5_uv(g, 2, rrw, dumz, u3d);
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = i1; i <= i2; i++) {
    float mhk = A3(g->mh, 1, 1, k);
    if (k == 1) A3(advz, i, j, k) = -A3(dumz, i, j, 2) * g->rdz * mhk;
    else if (k == nk) A3(advz, i, j, k) = +A3(dumz, i, j, nk) * g->rdz * mhk;
    else A3(advz, i, j, k) = -(A3(dumz, i, j, k + 1) - A3(dumz, i, j, k)) * g->rdz * mhk;
    A3(uten, i, j, k) = A3(uten, i, j, k) + (((A3(advx, i, j, k) + A3(advy, i, j, k)) + A3(advz, i, j, k)) +
        A3(u3d, i, j, k) * 0.5f * (A3(divx, i, j, k) + A3(divx, i - 1, j, k))) * A3(g->rr0, 1, 1, k);
  }
}

/* advv: adv.F:1847-2770 */
static void advv_g(const OG *g, Scratch *w, F3 divx, F3 rru, F3 rrv, F3 v3d, F3 vten, F3 rrw, F3 rho, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  int j1 = g->ibs ? 2 : 1, j2 = g->ibn ? nj : nj + 1;
  int doitw = (g->wbc == 2 && g->ibw), doite = (g->ebc == 2 && g->ibe);
  F3 advx = w->advx, advy = w->advy, advz = w->advz, dumx = w->dumx, dumy = w->dumy, dumz = w->dumz;
  hadv5(g, 3, 0, 0, 0.0, rru, rrv, dumx, dumy, v3d);
  if (doitw) for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++)
    if ((A3(rru, 1, j, k) + A3(rru, 1, j - 1, k)) >= 0.0f) A3(dumx, 1, j, k) = A3(dumx, 2, j, k);
  if (doite) for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++)
    if ((A3(rru, ni + 1, j, k) + A3(rru, ni + 1, j - 1, k)) <= 0.0f) A3(dumx, ni + 1, j, k) = A3(dumx, ni, j, k);
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++) for (int i = 1; i <= ni; i++) {
    A3(advx, i, j, k) = -(A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * g->rdx * UH(i);
    A3(advy, i, j, k) = -(A3(dumy, i, j, k) - A3(dumy, i, j - 1, k)) * g->rdy * VF(j);
  }
  if (doitw) for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++)
    if ((A3(rru, 1, j, k) + A3(rru, 1, j - 1, k)) >= 0.0f)
      A3(advx, 1, j, k) = A3(advx, 1, j, k) - A3(v3d, 1, j, k) * 0.5f *
          ((A3(rru, 2, j - 1, k) - A3(rru, 1, j - 1, k)) + (A3(rru, 2, j, k) - A3(rru, 1, j, k))) * g->rdx * UH(1);
  if (doite) for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++)
    if ((A3(rru, ni + 1, j, k) + A3(rru, ni + 1, j - 1, k)) <= 0.0f)
      A3(advx, ni, j, k) = A3(advx, ni, j, k) - A3(v3d, ni, j, k) * 0.5f *
          ((A3(rru, ni + 1, j - 1, k) - A3(rru, ni, j - 1, k)) + (A3(rru, ni + 1, j, k) - A3(rru, ni, j, k))) * g->rdx * UH(ni);
  /* adv.F:2115-2174: 6th-order diffusion */
  if (diff6_on(g)) {
    float coef = g->cfg->kdiff6 / 64.0f / dt;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) {
      float r0 = A3(g->rho0, 1, 1, k);
      for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
        float f = d6(A3(v3d, i - 3, j, k), A3(v3d, i - 2, j, k), A3(v3d, i - 1, j, k), A3(v3d, i, j, k),
                     A3(v3d, i + 1, j, k), A3(v3d, i + 2, j, k)) * 0.25f *
                  ((A3(rho, i - 1, j - 1, k) + A3(rho, i, j, k)) + (A3(rho, i - 1, j, k) + A3(rho, i, j - 1, k)));
        A3(dumx, i, j, k) = d6lim(g, f, A3(v3d, i, j, k), A3(v3d, i - 1, j, k));
      }
      for (int j = j1; j <= j2; j++) for (int i = 1; i <= ni; i++)
        A3(advx, i, j, k) = A3(advx, i, j, k) + coef * (A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * (r0 + r0) /
                                                    (A3(rho, i, j - 1, k) + A3(rho, i, j, k));
      for (int j = 1; j <= nj + 2; j++) for (int i = 1; i <= ni; i++) {
        float f = d6(A3(v3d, i, j - 3, k), A3(v3d, i, j - 2, k), A3(v3d, i, j - 1, k), A3(v3d, i, j, k),
                     A3(v3d, i, j + 1, k), A3(v3d, i, j + 2, k)) * A3(rho, i, j - 1, k);
        A3(dumy, i, j, k) = d6lim(g, f, A3(v3d, i, j, k), A3(v3d, i, j - 1, k));
      }
      for (int j = j1; j <= j2; j++) for (int i = 1; i <= ni; i++)
        A3(advy, i, j, k) = A3(advy, i, j, k) + coef * (A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * (r0 + r0) /
                                                    (A3(rho, i, j - 1, k) + A3(rho, i, j, k));
    }
  }
  vadv5_uv(g, 3, rrw, dumz, v3d);
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = j1; j <= j2; j++) for (int i = 1; i <= ni; i++) {
    float mhk = A3(g->mh, 1, 1, k);
    if (k == 1) A3(advz, i, j, k) = -A3(dumz, i, j, 2) * g->rdz * mhk;
    else if (k == nk) A3(advz, i, j, k) = +A3(dumz, i, j, nk) * g->rdz * mhk;
    else A3(advz, i, j, k) = -(A3(dumz, i, j, k + 1) - A3(dumz, i, j, k)) * g->rdz * mhk;
    A3(vten, i, j, k) = A3(vten, i, j, k) + (((A3(advx, i, j, k) + A3(advy, i, j, k)) + A3(advz, i, j, k)) +
        A3(v3d, i, j, k) * 0.5f * (A3(divx, i, j, k) + A3(divx, i, j - 1, k))) * A3(g->rr0, 1, 1, k);
  }
}

/* advw: adv.F:2778-3610 */
static void advw_g(const OG *g, Scratch *w, F3 divx, F3 rru, F3 rrv, F3 rrw, F3 w3d, F3 wten, F3 rho, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  int doitw = (g->wbc == 2 && g->ibw), doite = (g->ebc == 2 && g->ibe);
  int doits = (g->sbc == 2 && g->ibs), doitn = (g->nbc == 2 && g->ibn);
  F3 advx = w->advx, advy = w->advy, advz = w->advz, dumx = w->dumx, dumy = w->dumy, dumz = w->dumz;
  F3 c1 = g->c1, c2 = g->c2;
  hadv5(g, 4, 0, 0, 0.0, rru, rrv, dumx, dumy, w3d);
  if (doitw) for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) {
    float cc2 = 0.5f * (A3(c2, 0, j, k) + A3(c2, 1, j, k)), cc1 = 1.0f - cc2;
    float ubar = cc2 * A3(rru, 1, j, k) + cc1 * A3(rru, 1, j, k - 1);
    if (ubar >= 0.0f) A3(dumx, 1, j, k) = A3(dumx, 2, j, k);
  }
  if (doite) for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) {
    float cc2 = 0.5f * (A3(c2, ni, j, k) + A3(c2, ni + 1, j, k)), cc1 = 1.0f - cc2;
    float ubar = cc2 * A3(rru, ni + 1, j, k) + cc1 * A3(rru, ni + 1, j, k - 1);
    if (ubar <= 0.0f) A3(dumx, ni + 1, j, k) = A3(dumx, ni, j, k);
  }
  if (doits) for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++) {
    float cc2 = 0.5f * (A3(c2, i, 0, k) + A3(c2, i, 1, k)), cc1 = 1.0f - cc2;
    float vbar = cc2 * A3(rrv, i, 1, k) + cc1 * A3(rrv, i, 1, k - 1);
    if (vbar >= 0.0f) A3(dumy, i, 1, k) = A3(dumy, i, 2, k);
  }
  if (doitn) for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++) {
    float cc2 = 0.5f * (A3(c2, i, nj, k) + A3(c2, i, nj + 1, k)), cc1 = 1.0f - cc2;
    float vbar = cc2 * A3(rrv, i, nj + 1, k) + cc1 * A3(rrv, i, nj + 1, k - 1);
    if (vbar <= 0.0f) A3(dumy, i, nj + 1, k) = A3(dumy, i, nj, k);
  }
#pragma omp parallel for
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    A3(advx, i, j, k) = -(A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * g->rdx * UH(i);
    A3(advy, i, j, k) = -(A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * g->rdy * VH(j);
  }
  if (doitw) for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) {
    float cc2 = 0.5f * (A3(c2, 0, j, k) + A3(c2, 1, j, k)), cc1 = 1.0f - cc2;
    float ubar = cc2 * A3(rru, 1, j, k) + cc1 * A3(rru, 1, j, k - 1);
    if (ubar >= 0.0f)
      A3(advx, 1, j, k) = A3(advx, 1, j, k) - A3(w3d, 1, j, k) *
          (A3(c1, 1, j, k) * (A3(rru, 2, j, k - 1) - A3(rru, 1, j, k - 1)) + A3(c2, 1, j, k) * (A3(rru, 2, j, k) - A3(rru, 1, j, k))) * g->rdx * UH(1);
  }
  if (doite) for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) {
    float cc2 = 0.5f * (A3(c2, ni, j, k) + A3(c2, ni + 1, j, k)), cc1 = 1.0f - cc2;
    float ubar = cc2 * A3(rru, ni + 1, j, k) + cc1 * A3(rru, ni + 1, j, k - 1);
    if (ubar <= 0.0f)
      A3(advx, ni, j, k) = A3(advx, ni, j, k) - A3(w3d, ni, j, k) *
          (A3(c1, ni, j, k) * (A3(rru, ni + 1, j, k - 1) - A3(rru, ni, j, k - 1)) + A3(c2, ni, j, k) * (A3(rru, ni + 1, j, k) - A3(rru, ni, j, k))) * g->rdx * UH(ni);
  }
  if (doits) for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++) {
    float cc2 = 0.5f * (A3(c2, i, 0, k) + A3(c2, i, 1, k)), cc1 = 1.0f - cc2;
    float vbar = cc2 * A3(rrv, i, 1, k) + cc1 * A3(rrv, i, 1, k - 1);
    if (vbar >= 0.0f)
      A3(advy, i, 1, k) = A3(advy, i, 1, k) - A3(w3d, i, 1, k) *
          (A3(c1, i, 1, k) * (A3(rrv, i, 2, k - 1) - A3(rrv, i, 1, k - 1)) + A3(c2, i, 1, k) * (A3(rrv, i, 2, k) - A3(rrv, i, 1, k))) * g->rdy * VH(1);
  }
  if (doitn) for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++) {
    float cc2 = 0.5f * (A3(c2, i, nj, k) + A3(c2, i, nj + 1, k)), cc1 = 1.0f - cc2;
    float vbar = cc2 * A3(rrv, i, nj + 1, k) + cc1 * A3(rrv, i, nj + 1, k - 1);
    if (vbar <= 0.0f)
      A3(advy, i, nj, k) = A3(advy, i, nj, k) - A3(w3d, i, nj, k) *
          (A3(c1, i, nj, k) * (A3(rrv, i, nj + 1, k - 1) - A3(rrv, i, nj, k - 1)) + A3(c2, i, nj, k) * (A3(rrv, i, nj + 1, k) - A3(rrv, i, nj, k))) * g->rdy * VH(nj);
  }
  /* adv.F:3109-3170: 6th-order diffusion */
  if (diff6_on(g)) {
    float coef = g->cfg->kdiff6 / 64.0f / dt;
#pragma omp parallel for
    for (int k = 2; k <= nk; k++) {
      float rf = A3(g->rf0, 1, 1, k);
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) {
        float cc2 = 0.5f * (A3(c2, i - 1, j, k) + A3(c2, i, j, k)), cc1 = 1.0f - cc2;
        float f = d6(A3(w3d, i - 3, j, k), A3(w3d, i - 2, j, k), A3(w3d, i - 1, j, k), A3(w3d, i, j, k),
                     A3(w3d, i + 1, j, k), A3(w3d, i + 2, j, k)) * 0.5f *
                  (cc2 * (A3(rho, i - 1, j, k) + A3(rho, i, j, k)) + cc1 * (A3(rho, i - 1, j, k - 1) + A3(rho, i, j, k - 1)));
        A3(dumx, i, j, k) = d6lim(g, f, A3(w3d, i, j, k), A3(w3d, i - 1, j, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
        A3(advx, i, j, k) = A3(advx, i, j, k) + coef * (A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * rf /
                                                    (0.5f * (A3(rho, i, j, k - 1) + A3(rho, i, j, k)));
      for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) {
        float cc2 = 0.5f * (A3(c2, i, j - 1, k) + A3(c2, i, j, k)), cc1 = 1.0f - cc2;
        float f = d6(A3(w3d, i, j - 3, k), A3(w3d, i, j - 2, k), A3(w3d, i, j - 1, k), A3(w3d, i, j, k),
                     A3(w3d, i, j + 1, k), A3(w3d, i, j + 2, k)) * 0.5f *
                  (cc2 * (A3(rho, i, j - 1, k) + A3(rho, i, j, k)) + cc1 * (A3(rho, i, j - 1, k - 1) + A3(rho, i, j, k - 1)));
        A3(dumy, i, j, k) = d6lim(g, f, A3(w3d, i, j, k), A3(w3d, i, j - 1, k));
      }
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
        A3(advy, i, j, k) = A3(advy, i, j, k) + coef * (A3(dumy, i, j + 1, k) - A3(dumy, i, j, k)) * rf /
                                                    (0.5f * (A3(rho, i, j, k - 1) + A3(rho, i, j, k)));
    }
  }
  vadv5_w(g, rrw, dumz, w3d);
#pragma omp parallel for
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    A3(advz, i, j, k) = -(A3(dumz, i, j, k) - A3(dumz, i, j, k - 1)) * g->rdz * A3(g->mf, 1, 1, k);
    A3(wten, i, j, k) = A3(wten, i, j, k) + (((A3(advx, i, j, k) + A3(advy, i, j, k)) + A3(advz, i, j, k)) +
        A3(w3d, i, j, k) * (A3(c2, 1, 1, k) * A3(divx, i, j, k) + A3(c1, 1, 1, k) * A3(divx, i, j, k - 1))) * A3(g->rrf0, 1, 1, k);
  }
}

/* ------------------------------------------------------------------ */
/* Open-radiative boundary pieces, bc.F                                 */
/* ------------------------------------------------------------------ */

/* radbcew / radbcns: bc.F:1948-2046, the Klemp-Wilhelmson phase speeds
 * u -/+ cstar of irbc = 1 (from ua, solve1.F:403-409) and irbc = 2 (from
 * u3d at every small step, sound.F:261-267) */
static void radbcew_kw(const OG *g, float *radbcw, float *radbce, F3 ua) {
  const float cstar = g->cfg->cstar;
  if (g->ibw && g->wbc == 2)
    for (int k = 1; k <= g->nk; k++) for (int j = 1; j <= g->nj; j++) {
      float cbcw = A3(ua, 1, j, k) - cstar;
      RJK(g, radbcw, j, k) = (cbcw < 0.0f) ? cbcw : 0.0f;
    }
  if (g->ibe && g->ebc == 2)
    for (int k = 1; k <= g->nk; k++) for (int j = 1; j <= g->nj; j++) {
      float cbce = A3(ua, g->ni + 1, j, k) + cstar;
      RJK(g, radbce, j, k) = (cbce > 0.0f) ? cbce : 0.0f;
    }
}
static void radbcns_kw(const OG *g, float *radbcs, float *radbcn, F3 va) {
  const float cstar = g->cfg->cstar;
  if (g->ibs && g->sbc == 2)
    for (int k = 1; k <= g->nk; k++) for (int i = 1; i <= g->ni; i++) {
      float cbcs = A3(va, i, 1, k) - cstar;
      RIK(g, radbcs, i, k) = (cbcs < 0.0f) ? cbcs : 0.0f;
    }
  if (g->ibn && g->nbc == 2)
    for (int k = 1; k <= g->nk; k++) for (int i = 1; i <= g->ni; i++) {
      float cbcn = A3(va, i, g->nj + 1, k) + cstar;
      RIK(g, radbcn, i, k) = (cbcn > 0.0f) ? cbcn : 0.0f;
    }
}

/* radbcew4: bc.F:2054-2115 */
/* restrict_openbc_we / restrict_openbc_sn: bc.F:2180-2384, called by
 * sound.F:283-285 and 299-301 with roflux = 1.  The mass fluxes through the
 * open lateral boundaries are summed in binary64 per level (each level over
 * j, resp. i, west/south before east/north) and then over the levels; the
 * outflow points' velocity is scaled by inflow/outflow. */
static void restrict_openbc_we(const OG *g, F3 u3d) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  double fluxout = 0.0, fluxin = 0.0;
  for (int k = 1; k <= nk; k++) {
    double tout = 0.0, tin = 0.0;
    if (g->wbc == 2 && g->ibw)
      for (int j = 1; j <= nj; j++) {
        const float f = A3(g->rho0, 1, j, k) * A3(u3d, 1, j, k) * RVH(j) * A3(g->rmh, 1, j, k);
        tout = tout - (double)fminf(0.0f, f);
        tin = tin + (double)fmaxf(0.0f, f);
      }
    if (g->ebc == 2 && g->ibe)
      for (int j = 1; j <= nj; j++) {
        const float f = A3(g->rho0, ni, j, k) * A3(u3d, ni + 1, j, k) * RVH(j) * A3(g->rmh, ni, j, k);
        tout = tout + (double)fmaxf(0.0f, f);
        tin = tin - (double)fminf(0.0f, f);
      }
    fluxout = fluxout + tout;
    fluxin = fluxin + tin;
  }
  const double t3 = (fluxin + 1.0e-20) / (fluxout + 1.0e-20);
  for (int k = 1; k <= nk; k++)
    for (int j = 1; j <= nj; j++) {
      if (g->wbc == 2 && g->ibw) {
        const double u1 = (double)(A3(g->rho0, 1, j, k) * A3(u3d, 1, j, k));
        if (u1 < 0.0) A3(u3d, 1, j, k) = (float)(u1 * t3 / (double)A3(g->rho0, 1, j, k));
      }
      if (g->ebc == 2 && g->ibe) {
        const double u1 = (double)(A3(g->rho0, ni, j, k) * A3(u3d, ni + 1, j, k));
        if (u1 > 0.0) A3(u3d, ni + 1, j, k) = (float)(u1 * t3 / (double)A3(g->rho0, ni, j, k));
      }
    }
}
static void restrict_openbc_sn(const OG *g, F3 v3d) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  double fluxout = 0.0, fluxin = 0.0;
  for (int k = 1; k <= nk; k++) {
    double tout = 0.0, tin = 0.0;
    if (g->sbc == 2 && g->ibs)
      for (int i = 1; i <= ni; i++) {
        const float f = A3(g->rho0, i, 1, k) * A3(v3d, i, 1, k) * RUH(i) * A3(g->rmh, i, 1, k);
        tout = tout - (double)fminf(0.0f, f);
        tin = tin + (double)fmaxf(0.0f, f);
      }
    if (g->nbc == 2 && g->ibn)
      for (int i = 1; i <= ni; i++) {
        const float f = A3(g->rho0, i, nj, k) * A3(v3d, i, nj + 1, k) * RUH(i) * A3(g->rmh, i, nj, k);
        tout = tout + (double)fmaxf(0.0f, f);
        tin = tin - (double)fminf(0.0f, f);
      }
    fluxout = fluxout + tout;
    fluxin = fluxin + tin;
  }
  const double t3 = (fluxin + 1.0e-20) / (fluxout + 1.0e-20);
  for (int k = 1; k <= nk; k++)
    for (int i = 1; i <= ni; i++) {
      if (g->sbc == 2 && g->ibs) {
        const double u1 = (double)(A3(g->rho0, i, 1, k) * A3(v3d, i, 1, k));
        if (u1 < 0.0) A3(v3d, i, 1, k) = (float)(u1 * t3 / (double)A3(g->rho0, i, 1, k));
      }
      if (g->nbc == 2 && g->ibn) {
        const double u1 = (double)(A3(g->rho0, i, nj, k) * A3(v3d, i, nj + 1, k));
        if (u1 > 0.0) A3(v3d, i, nj + 1, k) = (float)(u1 * t3 / (double)A3(g->rho0, i, nj, k));
      }
    }
}

static void radbcew4(const OG *g, float *radbcw, float *radbce, F3 u1, F3 u2, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float umax = CSMAX;
  if (g->ibw && g->wbc == 2) {
    for (int j = 1; j <= nj; j++) {
      float avgw = 0.0f;
      for (int k = 1; k <= nk; k++) {
        float foo = A3(u1, 3, j, k) - A3(u1, 2, j, k);
        float cbcw = g->dx * RUF(2) * (A3(u1, 2, j, k) - A3(u2, 2, j, k)) / (dt * (copysignf(1.e-10f, foo) + foo));
        cbcw = fmaxf(fminf(cbcw, 0.0f), -umax);
        avgw = avgw + cbcw;
      }
      avgw = avgw / (float)nk;
      for (int k = 1; k <= nk; k++) RJK(g, radbcw, j, k) = avgw;
    }
  }
  if (g->ibe && g->ebc == 2) {
    for (int j = 1; j <= nj; j++) {
      float avge = 0.0f;
      for (int k = 1; k <= nk; k++) {
        float foo = A3(u1, ni, j, k) - A3(u1, ni - 1, j, k);
        float cbce = g->dx * RUF(ni) * (A3(u1, ni, j, k) - A3(u2, ni, j, k)) / (dt * (copysignf(1.e-10f, foo) + foo));
        cbce = fminf(fmaxf(cbce, 0.0f), umax);
        avge = avge + cbce;
      }
      avge = avge / (float)nk;
      for (int k = 1; k <= nk; k++) RJK(g, radbce, j, k) = avge;
    }
  }
}

/* radbcns4: bc.F:2117-2178 */
static void radbcns4(const OG *g, float *radbcs, float *radbcn, F3 v1, F3 v2, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float umax = CSMAX;
  if (g->ibs && g->sbc == 2) {
    for (int i = 1; i <= ni; i++) {
      float avgs = 0.0f;
      for (int k = 1; k <= nk; k++) {
        float foo = A3(v1, i, 3, k) - A3(v1, i, 2, k);
        float cbcs = g->dy * RVF(2) * (A3(v1, i, 2, k) - A3(v2, i, 2, k)) / (dt * (copysignf(1.e-10f, foo) + foo));
        cbcs = fmaxf(fminf(cbcs, 0.0f), -umax);
        avgs = avgs + cbcs;
      }
      avgs = avgs / (float)nk;
      for (int k = 1; k <= nk; k++) RIK(g, radbcs, i, k) = avgs;
    }
  }
  if (g->ibn && g->nbc == 2) {
    for (int i = 1; i <= ni; i++) {
      float avgn = 0.0f;
      for (int k = 1; k <= nk; k++) {
        float foo = A3(v1, i, nj, k) - A3(v1, i, nj - 1, k);
        float cbcn = g->dy * RVF(nj) * (A3(v1, i, nj, k) - A3(v2, i, nj, k)) / (dt * (copysignf(1.e-10f, foo) + foo));
        cbcn = fminf(fmaxf(cbcn, 0.0f), umax);
        avgn = avgn + cbcn;
      }
      avgn = avgn / (float)nk;
      for (int k = 1; k <= nk; k++) RIK(g, radbcn, i, k) = avgn;
    }
  }
}

/* ------------------------------------------------------------------ */
/* Acoustic substeps, sound.F (psolver=3, no terrain, Cartesian)        */
/* ------------------------------------------------------------------ */

typedef struct {
  F3 ua, u3d, uten, va, v3d, vten, wa, w3d, wten, ppi, pp3d, piadv, ppten, ppx, thv, ppterm, rru, rrv, rrw;
  float *radbcw, *radbce, *radbcs, *radbcn;
} SoundArgs;

static void sound_g(const OG *g, const SoundArgs *a, int nrk, float dt) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  const cm1g_config_t *cfg = g->cfg;
  float alph = cfg->alph, kdiv = cfg->kdiv, smeps = cfg->smeps, cp = g->c.cp;
  int nsound = cfg->nsound, nloop = 1;
  float dts = dt;
  /* sound.F:79-101 */
  float beta = 1.0f - alph, asq = alph * alph;
  if (nrk == 1) {
    nloop = (int)lroundf((float)nsound / 3.0f);
    dts = dt / ((float)nloop * 3.0f);
    if (dts > (dt / (float)nsound)) { nloop = nloop + 1; dts = dt / ((float)nloop * 3.0f); }
  } else if (nrk == 2) { nloop = (int)(0.5f * (float)nsound); dts = dt / (float)nsound; }
  else { nloop = nsound; dts = dt / (float)nsound; }

  long ns = nS(g);
  float *buf = (float *)calloc((size_t)ns * 8 + (size_t)g->NI * g->NJ * 2, sizeof(float));
  F3 mm = mkS(g, buf), qk = mkS(g, buf + ns), pk1 = mkS(g, buf + 2 * ns), pk2 = mkS(g, buf + 3 * ns);
  F3 ppd = mkS(g, buf + 4 * ns), fpk = mkS(g, buf + 5 * ns), dum1 = mkS(g, buf + 6 * ns), dum2 = mkS(g, buf + 7 * ns);
  F3 dtu = mk2(g, buf + 8 * ns), dtv = mk2(g, buf + 8 * ns + (long)g->NI * g->NJ);
  F3 u3d = a->u3d, v3d = a->v3d, w3d = a->w3d, pp3d = a->pp3d, rru = a->rru, rrv = a->rrv, rrw = a->rrw;
  F3 thv = a->thv, ppterm = a->ppterm, piadv = a->piadv;

  for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
    A3(dtu, i, j, 0) = dts * A3(g->dtu0, i, j, 0);
    A3(dtv, i, j, 0) = dts * A3(g->dtv0, i, j, 0);
  }
  /* sound.F:115-135 */
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) {
    float mhk = A3(g->mh, 1, 1, k), rr0k = A3(g->rr0, 1, 1, k);
    float tem = dts * g->rdz * mhk;
    float r2 = dts * g->rdz * mhk * rr0k * A3(g->rf0, 1, 1, k + 1);
    float r1 = dts * g->rdz * mhk * rr0k * A3(g->rf0, 1, 1, k);
    float tem1 = dts * g->rdz * cp * A3(g->mf, 1, 1, k);
    float c1a = A3(g->c1, 1, 1, k), c1b = A3(g->c1, 1, 1, k + 1), c2a = A3(g->c2, 1, 1, k), c2b = A3(g->c2, 1, 1, k + 1);
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      A3(qk, i, j, k) = tem * A3(ppterm, i, j, k);
      A3(pk2, i, j, k) = r2 * (-c2b * A3(piadv, i, j, k + 1) + (1.0f - c1b) * A3(piadv, i, j, k));
      A3(pk1, i, j, k) = r1 * (+c1a * A3(piadv, i, j, k - 1) + (c2a - 1.0f) * A3(piadv, i, j, k));
      A3(mm, i, j, k) = tem1 * (c2a * A3(thv, i, j, k) + c1a * A3(thv, i, j, k - 1));
    }
  }
  for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) { A3(pk1, i, j, 1) = 0.0f; A3(pk2, i, j, nk) = 0.0f; }
  /* sound.F:192-250 */
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    if (nrk != 1) {
      A3(u3d, i, j, k) = A3(a->ua, i, j, k);
      A3(v3d, i, j, k) = A3(a->va, i, j, k);
      A3(w3d, i, j, k) = A3(a->wa, i, j, k);
      A3(pp3d, i, j, k) = A3(a->ppi, i, j, k);
    }
    A3(ppd, i, j, k) = A3(a->ppx, i, j, k);
    A3(rru, i, j, k) = 0.0f; A3(rrv, i, j, k) = 0.0f;
    A3(rrw, i, j, k) = A3(a->wa, i, j, k) * beta;
  }

  for (int n = 1; n <= nloop; n++) {
    /* sound.F:261-267 */
    if (cfg->irbc == 2) {
      if (g->ibw || g->ibe) radbcew_kw(g, a->radbcw, a->radbce, u3d);
      if (g->ibs || g->ibn) radbcns_kw(g, a->radbcs, a->radbcn, v3d);
    }
    /* sound.F:273-303 */
    if (cfg->wbc == 2 && g->ibw)
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
        A3(u3d, 1, j, k) = A3(u3d, 1, j, k) + dts * (-RJK(g, a->radbcw, j, k) * (A3(u3d, 2, j, k) - A3(u3d, 1, j, k)) * g->rdx * UH(1) + A3(a->uten, 1, j, k));
    if (cfg->ebc == 2 && g->ibe)
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++)
        A3(u3d, ni + 1, j, k) = A3(u3d, ni + 1, j, k) + dts * (-RJK(g, a->radbce, j, k) * (A3(u3d, ni + 1, j, k) - A3(u3d, ni, j, k)) * g->rdx * UH(ni) + A3(a->uten, ni + 1, j, k));
    if (cfg->roflux == 1) restrict_openbc_we(g, u3d);
    if (cfg->sbc == 2 && g->ibs)
      for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
        A3(v3d, i, 1, k) = A3(v3d, i, 1, k) + dts * (-RIK(g, a->radbcs, i, k) * (A3(v3d, i, 2, k) - A3(v3d, i, 1, k)) * g->rdy * VH(1) + A3(a->vten, i, 1, k));
    if (cfg->nbc == 2 && g->ibn)
      for (int k = 1; k <= nk; k++) for (int i = 1; i <= ni; i++)
        A3(v3d, i, nj + 1, k) = A3(v3d, i, nj + 1, k) + dts * (-RIK(g, a->radbcn, i, k) * (A3(v3d, i, nj + 1, k) - A3(v3d, i, nj, k)) * g->rdy * VH(nj) + A3(a->vten, i, nj + 1, k));
    if (cfg->roflux == 1) restrict_openbc_sn(g, v3d);
    /* sound.F:321-341 */
    float tem1 = g->rdx * cp * 0.5f, tem2 = g->rdy * cp * 0.5f;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
      A3(u3d, i, j, k) = A3(u3d, i, j, k) + A3(dtu, i, j, 0) * (A3(a->uten, i, j, k) -
          tem1 * (A3(ppd, i, j, k) - A3(ppd, i - 1, j, k)) * UF(i) * (A3(thv, i, j, k) + A3(thv, i - 1, j, k)));
      A3(v3d, i, j, k) = A3(v3d, i, j, k) + A3(dtv, i, j, 0) * (A3(a->vten, i, j, k) -
          tem2 * (A3(ppd, i, j, k) - A3(ppd, i, j - 1, k)) * VF(j) * (A3(thv, i, j, k) + A3(thv, i, j - 1, k)));
    }
    /* sound.F:479-502 */
    float temx = dts * 0.5f * g->rdx, temy = dts * 0.5f * g->rdy;
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      float div = (A3(u3d, i + 1, j, k) - A3(u3d, i, j, k)) * g->rdx * UH(i) + (A3(v3d, i, j + 1, k) - A3(v3d, i, j, k)) * g->rdy * VH(j);
      if (fabsf(div) < smeps) div = 0.0f;
      float X = A3(u3d, i, j, k) * (A3(piadv, i, j, k) - A3(piadv, i - 1, j, k)) + A3(u3d, i + 1, j, k) * (A3(piadv, i + 1, j, k) - A3(piadv, i, j, k));
      float Y = A3(v3d, i, j, k) * (A3(piadv, i, j, k) - A3(piadv, i, j - 1, k)) + A3(v3d, i, j + 1, k) * (A3(piadv, i, j + 1, k) - A3(piadv, i, j, k));
      float A = dts * (A3(a->ppten, i, j, k) - A3(ppterm, i, j, k) * div);
      float B = -(X * temx * UH(i)) - Y * temy * VH(j);
      float C = beta * (A3(w3d, i, j, k) * (A3(pk1, i, j, k) + A3(qk, i, j, k)) + A3(w3d, i, j, k + 1) * (A3(pk2, i, j, k) - A3(qk, i, j, k)));
      A3(fpk, i, j, k) = (A + B) + C;
    }
    /* sound.F:659-733: vertically implicit solve for w */
#pragma omp parallel for
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      int k;
      float aa, bb, cc, dd, fwk, r1, mmk;
      k = 2;
      mmk = A3(mm, i, j, k);
      cc = -asq * (-mmk * (A3(pk2, i, j, k) - A3(qk, i, j, k)));
      bb = 1.0f - asq * (+mmk * (-(A3(pk1, i, j, k) + A3(qk, i, j, k)) + (A3(pk2, i, j, k - 1) - A3(qk, i, j, k - 1))));
      fwk = dts * A3(a->wten, i, j, k) + beta * (-mmk * (A3(pp3d, i, j, k) - A3(pp3d, i, j, k - 1)));
      dd = A3(w3d, i, j, k) + fwk + alph * (-mmk * ((A3(pp3d, i, j, k) + A3(fpk, i, j, k)) - (A3(pp3d, i, j, k - 1) + A3(fpk, i, j, k - 1))));
      r1 = 1.0f / bb;
      A3(dum1, i, j, k) = -cc * r1;
      A3(dum2, i, j, k) = dd * r1;
      for (k = 3; k <= nk - 1; k++) {
        mmk = A3(mm, i, j, k);
        aa = -asq * (+mmk * (A3(pk1, i, j, k - 1) + A3(qk, i, j, k - 1)));
        cc = -asq * (-mmk * (A3(pk2, i, j, k) - A3(qk, i, j, k)));
        bb = 1.0f - asq * (+mmk * (-(A3(pk1, i, j, k) + A3(qk, i, j, k)) + (A3(pk2, i, j, k - 1) - A3(qk, i, j, k - 1))));
        fwk = dts * A3(a->wten, i, j, k) + beta * (-mmk * (A3(pp3d, i, j, k) - A3(pp3d, i, j, k - 1)));
        dd = A3(w3d, i, j, k) + fwk + alph * (-mmk * ((A3(pp3d, i, j, k) + A3(fpk, i, j, k)) - (A3(pp3d, i, j, k - 1) + A3(fpk, i, j, k - 1))));
        r1 = 1.0f / (aa * A3(dum1, i, j, k - 1) + bb);
        A3(dum1, i, j, k) = -cc * r1;
        A3(dum2, i, j, k) = (dd - aa * A3(dum2, i, j, k - 1)) * r1;
      }
      k = nk;
      mmk = A3(mm, i, j, k);
      aa = -asq * (+mmk * (A3(pk1, i, j, k - 1) + A3(qk, i, j, k - 1)));
      bb = 1.0f - asq * (+mmk * (-(A3(pk1, i, j, k) + A3(qk, i, j, k)) + (A3(pk2, i, j, k - 1) - A3(qk, i, j, k - 1))));
      fwk = dts * A3(a->wten, i, j, k) + beta * (-mmk * (A3(pp3d, i, j, k) - A3(pp3d, i, j, k - 1)));
      dd = A3(w3d, i, j, k) + fwk + alph * (-mmk * ((A3(pp3d, i, j, k) + A3(fpk, i, j, k)) - (A3(pp3d, i, j, k - 1) + A3(fpk, i, j, k - 1))));
      r1 = 1.0f / (aa * A3(dum1, i, j, k - 1) + bb);
      A3(w3d, i, j, k) = (dd - aa * A3(dum2, i, j, k - 1)) * r1;
      for (k = nk - 1; k >= 2; k--)
        A3(w3d, i, j, k) = A3(dum1, i, j, k) * A3(w3d, i, j, k + 1) + A3(dum2, i, j, k);
    }
    /* sound.F:746-760 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      A3(ppd, i, j, k) = A3(pp3d, i, j, k);
      A3(pp3d, i, j, k) = A3(pp3d, i, j, k) + A3(fpk, i, j, k) +
          alph * (A3(w3d, i, j, k) * (A3(pk1, i, j, k) + A3(qk, i, j, k)) + A3(w3d, i, j, k + 1) * (A3(pk2, i, j, k) - A3(qk, i, j, k)));
      if (fabsf(A3(pp3d, i, j, k)) < smeps) A3(pp3d, i, j, k) = 0.0f;
      A3(dum1, i, j, k) = kdiv * (A3(pp3d, i, j, k) - A3(ppd, i, j, k));
      A3(ppd, i, j, k) = A3(pp3d, i, j, k) + A3(dum1, i, j, k);
    }
    if (n < nloop) oracle_bcp_g(g, ppd);
    /* sound.F:806-835 */
    if (n < nloop) {
#pragma omp parallel for
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
        A3(rru, i, j, k) = A3(rru, i, j, k) + A3(u3d, i, j, k);
        A3(rrv, i, j, k) = A3(rrv, i, j, k) + A3(v3d, i, j, k);
        A3(rrw, i, j, k) = A3(rrw, i, j, k) + A3(w3d, i, j, k);
      }
    } else {
      float tavg = 1.0f / (float)nloop;
#pragma omp parallel for
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
        A3(rru, i, j, k) = (A3(rru, i, j, k) + A3(u3d, i, j, k)) * tavg;
        A3(rrv, i, j, k) = (A3(rrv, i, j, k) + A3(v3d, i, j, k)) * tavg;
        A3(rrw, i, j, k) = (A3(rrw, i, j, k) + A3(w3d, i, j, k) * alph) * tavg;
      }
    }
  }
  /* sound.F:841-852 */
  if (nrk == 3)
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
      A3(a->ppx, i, j, k) = A3(dum1, i, j, k);
  free(buf);
}

/* ------------------------------------------------------------------ */
/* misclibs.F pieces                                                    */
/* ------------------------------------------------------------------ */

/* getdiv: misclibs.F:108-215 (Cartesian, no terrain) */
static void getdiv_g(const OG *g, F3 u, F3 v, F3 w, F3 div) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float smeps = g->cfg->smeps;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    float d = ((A3(u, i + 1, j, k) - A3(u, i, j, k)) * g->rdx * UH(i) + (A3(v, i, j + 1, k) - A3(v, i, j, k)) * g->rdy * VH(j)) +
              (A3(w, i, j, k + 1) - A3(w, i, j, k)) * g->rdz * A3(g->mh, 1, 1, k);
    if (fabsf(d) < smeps) d = 0.0f;
    A3(div, i, j, k) = d;
  }
}

/* getdivx: misclibs.F:222-370 (no terrain) */
static void getdivx_g(const OG *g, F3 rru, F3 rrv, F3 rrw, F3 divx) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) {
    float tem = A3(g->rho0, 1, 1, k);
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) A3(rru, i, j, k) = A3(rru, i, j, k) * tem;
    for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) A3(rrv, i, j, k) = A3(rrv, i, j, k) * tem;
    if (k == 1) {
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) { A3(rrw, i, j, 1) = 0.0f; A3(rrw, i, j, nk + 1) = 0.0f; }
    } else {
      tem = A3(g->rf0, 1, 1, k);
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) A3(rrw, i, j, k) = A3(rrw, i, j, k) * tem;
    }
  }
  getdiv_g(g, rru, rrv, rrw, divx);
}

/* calccflquick: misclibs.F:2726-2814 (nx>1, ny>1) */
static float calccflquick_g(const OG *g, float dt, F3 ua, F3 va, F3 wa) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  float dtdx = 0.5f * dt * g->rdx, dtdy = 0.5f * dt * g->rdy, dtdz = 0.5f * dt * g->rdz;
  float cflmx = -99999999.0f;
  for (int k = 1; k <= nk; k++) {
    float cfl = 0.0f;
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      float a1 = (A3(ua, i, j, k) + A3(ua, i + 1, j, k)) * dtdx * UH(i);
      float a2 = (A3(va, i, j, k) + A3(va, i, j + 1, k)) * dtdy * VH(j);
      float a3 = (A3(wa, i, j, k) + A3(wa, i, j, k + 1)) * dtdz * A3(g->mh, i, j, k);
      float wsp = sqrtf((a1 * a1 + a2 * a2) + a3 * a3);
      cfl = fmaxf(cfl, wsp);
    }
    cflmx = fmaxf(cflmx, cfl);
  }
  return cflmx;
}

/* pdefq: misclibs.F:1037-1117 (pdscheme=1).  Returns the budget change. */
static double pdefq_g(const OG *g, float rmax, F3 rho, F3 q3d) {
  int ni = g->ni, nj = g->nj, nk = g->nk;
  double tem = (double)(g->dx * g->dy * g->dz), asq = 0.0;
  double *budj = (double *)calloc((size_t)nj + 1, sizeof(double));
#pragma omp parallel for
  for (int j = 1; j <= nj; j++) {
    budj[j] = 0.0;
    for (int i = 1; i <= ni; i++) {
      double t1 = 0.0, t2 = 0.0, a1 = 0.0, a2 = 0.0;
      for (int k = 1; k <= nk; k++) {
        t1 = t1 + (double)(A3(rho, i, j, k) * A3(q3d, i, j, k));
        a1 = a1 + (double)(A3(rho, i, j, k) * A3(q3d, i, j, k) * RUH(i) * RVH(j) * A3(g->rmh, i, j, k));
        if (A3(q3d, i, j, k) < rmax) A3(q3d, i, j, k) = 0.0f;
        t2 = t2 + (double)(A3(rho, i, j, k) * A3(q3d, i, j, k));
      }
      double t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20);
      if (t3 < 0.0) t3 = 1.0;
      for (int k = 1; k <= nk; k++) {
        A3(q3d, i, j, k) = (float)(t3 * (double)A3(q3d, i, j, k));
        a2 = a2 + (double)(A3(rho, i, j, k) * A3(q3d, i, j, k) * RUH(i) * RVH(j) * A3(g->rmh, i, j, k));
      }
      budj[j] = budj[j] + a2 - a1;
    }
  }
  for (int j = 1; j <= nj; j++) asq = asq + budj[j] * tem;
  free(budj);
  return asq;
}

/* ------------------------------------------------------------------ */
/* solve2: RK3 large step (solve2.F:296-2052)                          */
/* ------------------------------------------------------------------ */

typedef struct {
  F3 ua, u3d, uten1, va, v3d, vten1, wa, w3d, wten1, ppi, pp3d, ppx, ppten, tha, th3d, thten1, rho, prs;
  F3 qa[CM1G_MAXQ], q3d[CM1G_MAXQ], qten[CM1G_MAXQ];
  F3 pta[CM1G_MAXQ], pt3d[CM1G_MAXQ], ptten[CM1G_MAXQ];
  float *radbcw, *radbce, *radbcs, *radbcn;
  F3 rain, prate;   /* (ib:ie,jb:je), ptype=1 */
} St;

static void st_view(const OG *g, const cm1g_state_t *s, St *t) {
  t->ua = mkU(g, RP(s->ua)); t->u3d = mkU(g, RP(s->u3d)); t->uten1 = mkU(g, RP(s->uten1));
  t->va = mkV(g, RP(s->va)); t->v3d = mkV(g, RP(s->v3d)); t->vten1 = mkV(g, RP(s->vten1));
  t->wa = mkW(g, RP(s->wa)); t->w3d = mkW(g, RP(s->w3d)); t->wten1 = mkW(g, RP(s->wten1));
  t->ppi = mkS(g, RP(s->ppi)); t->pp3d = mkS(g, RP(s->pp3d)); t->ppx = mkS(g, RP(s->ppx)); t->ppten = mkS(g, RP(s->ppten));
  t->tha = mkS(g, RP(s->tha)); t->th3d = mkS(g, RP(s->th3d)); t->thten1 = mkS(g, RP(s->thten1));
  t->rho = mkS(g, RP(s->rho)); t->prs = mkS(g, RP(s->prs));
  long n = nS(g);
  int numq = g->cfg->imoist ? g->cfg->numq : 0, npt = g->cfg->iptra ? g->cfg->npt : 0;
  for (int q = 0; q < numq; q++) { t->qa[q] = mkS(g, RP(s->qa) + q * n); t->q3d[q] = mkS(g, RP(s->q3d) + q * n); t->qten[q] = mkS(g, RP(s->qten) + q * n); }
  for (int q = 0; q < npt; q++) { t->pta[q] = mkS(g, RP(s->pta) + q * n); t->pt3d[q] = mkS(g, RP(s->pt3d) + q * n); t->ptten[q] = mkS(g, RP(s->ptten) + q * n); }
  t->radbcw = RP(s->radbcw); t->radbce = RP(s->radbce); t->radbcs = RP(s->radbcs); t->radbcn = RP(s->radbcn);
  if (g->cfg->ptype == 1) { t->rain = mk2(g, RP(s->rain)); t->prate = mk2(g, RP(s->prate)); }
}

static int check_cfg(const cm1g_config_t *cfg) {
  if (cfg->imoist && cfg->ptype == 0 && (cfg->nqv != 1 || cfg->numq != 1)) return -1;
  if (cfg->ptype == 1 && (!cfg->imoist || cfg->numq != 3 || cfg->nqv != 1 || cfg->nql1 != 2 || cfg->nql2 != 3 ||
                          cfg->efall != 0)) return -1;
  if (cfg->ptype != 0 && cfg->ptype != 1) return -1;
  if (cfg->iptra && (cfg->npt < 0 || cfg->npt > CM1G_MAXQ)) return -1;
  if (cfg->roflux != 0 && cfg->roflux != 1) return -1;
  if ((cfg->wbc == 2 || cfg->ebc == 2 || cfg->sbc == 2 || cfg->nbc == 2) &&
      !(cfg->irbc == 1 || cfg->irbc == 2 || cfg->irbc == 4)) return -1;
  if (cfg->nsound < 2 || (cfg->nsound % 2)) return -1;
  return 0;
}

int oracle_solve2(const cm1g_config_t *cfg, const cm1g_grid_t *gr, cm1g_state_t *state,
                  int nstep, float dt, double mtime, double mass1, double *mass2_out, float *cflmax_out) {
  (void)nstep; (void)mtime;
  OG G, *g = &G;
  if (og_setup(g, cfg, gr) || check_cfg(cfg)) { if (!g_err[0]) snprintf(g_err, sizeof g_err, "oracle: unsupported config"); return -1; }
  St s; st_view(g, state, &s);
  int ni = g->ni, nj = g->nj, nk = g->nk;
  Consts c = g->c;
  long ns = nS(g);
  Scratch w;
  if (scratch_alloc(g, &w)) return -3;
  float *tb = (float *)calloc((size_t)(9 * ns + nU(g) + nV(g) + 2 * nW(g) + nU(g) + nV(g)), sizeof(float));
  if (!tb) { scratch_free(&w); return -3; }
  float *p = tb;
  F3 dum8 = mkS(g, p); p += ns;
  F3 t11 = mkS(g, p); p += ns;
  F3 t22 = mkS(g, p); p += ns;
  F3 thterm = mkS(g, p); p += ns;
  F3 divx = mkS(g, p); p += ns;
  F3 sadv = mkS(g, p); p += ns;
  F3 sten = mkS(g, p); p += ns;
  F3 thten = mkS(g, p); p += ns;
  p += ns; /* spare */
  F3 rru = mkU(g, p); p += nU(g);
  F3 rrv = mkV(g, p); p += nV(g);
  F3 rrw = mkW(g, p); p += nW(g);
  F3 wten = mkW(g, p); p += nW(g);
  F3 uten = mkU(g, p); p += nU(g);
  F3 vten = mkV(g, p); p += nV(g);
  double *dumk3 = (double *)calloc((size_t)nk + 2, sizeof(double));
  double *dumk4 = (double *)calloc((size_t)nk + 2, sizeof(double));
  double mass2 = 0.0;
  float cflmax = 0.0f;
  int numq = cfg->imoist ? cfg->numq : 0, npt = cfg->iptra ? cfg->npt : 0;
  /* 6th-order diffusion: rr = 1/rho as solve3 (solve3.F:660-675) left it at
   * the end of the previous step, then updated after stages 1 and 2 */
  const int diffit = diff6_on(g);
  float *rrbuf = (float *)calloc((size_t)ns, sizeof(float));
  F3 rr = mkS(g, rrbuf);
  if (diffit)
    for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++)
      A3(rr, i, j, k) = 1.0f / A3(s.rho, i, j, k);
  /* irbc = 1: the phase speeds of the step, from ua, as solve1 forms them
   * before solve2 (solve1.F:403-409) */
  if (cfg->irbc == 1) {
    if (g->ibw || g->ibe) radbcew_kw(g, s.radbcw, s.radbce, s.ua);
    if (g->ibs || g->ibn) radbcns_kw(g, s.radbcs, s.radbcn, s.va);
  }

  for (int nrk = 1; nrk <= 3; nrk++) {
    float dttmp = dt / (float)(3 + 1 - nrk);
    /* solve2.F:313-446 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      float th3 = A3(s.th3d, i, j, k), th0 = A3(g->th0, i, j, k), pi0 = A3(g->pi0, i, j, k);
      if (cfg->imoist) {
        float qv = fmaxf(A3(s.q3d[cfg->nqv - 1], i, j, k), 0.0f);
        /* dum2: the liquid species (solve2.F:315-345); no ice */
        float d2 = 0.0f, d3 = 0.0f;
        if (cfg->nql1 > 0) {
          d2 = A3(s.q3d[cfg->nql1 - 1], i, j, k);
          for (int n = cfg->nql1 + 1; n <= cfg->nql2; n++) d2 = d2 + A3(s.q3d[n - 1], i, j, k);
        }
        float qli = fmaxf(0.0f, d2 + d3);
        A3(dum8, i, j, k) = c.g * ((th3 * A3(g->rth0, i, j, k) + c.repsm1 * (qv - A3(g->qv0, i, j, k))) -
                                   ((qli - A3(g->qc0, i, j, k)) - A3(g->qi0, i, j, k)));
        A3(t11, i, j, k) = (th0 + th3) * (1.0f + c.reps * qv) / ((1.0f + qv) + qli);
        if (cfg->eqtset == 2) {
          float cpli = c.cpl * fmaxf(0.0f, d2) + c.cpi * fmaxf(0.0f, d3);
          float cpm = (c.cp + c.cpv * qv) + cpli;
          float cvm = 1.0f / ((c.cv + c.cvv * qv) + cpli);
          A3(thterm, i, j, k) = (th0 + th3) * ((c.rd + c.rv * qv) - c.rovcp * cpm) * cvm;
          A3(t22, i, j, k) = (pi0 + A3(s.pp3d, i, j, k)) * c.rovcp * cpm * cvm;
        } else {
          A3(t22, i, j, k) = (pi0 + A3(s.pp3d, i, j, k)) * c.rddcv;
        }
      } else {
        A3(dum8, i, j, k) = c.g * th3 * A3(g->rth0, i, j, k);
        A3(t11, i, j, k) = th0 + th3;
        A3(t22, i, j, k) = (pi0 + A3(s.pp3d, i, j, k)) * c.rddcv;
      }
    }
    oracle_bcp_g(g, t11);
    /* solve2.F:456-467 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
      A3(uten, i, j, k) = A3(s.uten1, i, j, k);
      A3(vten, i, j, k) = A3(s.vten1, i, j, k);
      A3(wten, i, j, k) = A3(s.wten1, i, j, k);
    }
    /* solve2.F:493-527 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) {
      float r0 = A3(g->rho0, 1, 1, k);
      for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 2; i++) A3(rru, i, j, k) = r0 * A3(s.u3d, i, j, k);
      for (int j = 0; j <= nj + 2; j++) for (int i = 0; i <= ni + 1; i++) A3(rrv, i, j, k) = r0 * A3(s.v3d, i, j, k);
      if (k == 1) {
        for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) { A3(rrw, i, j, 1) = 0.0f; A3(rrw, i, j, nk + 1) = 0.0f; }
      } else {
        for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) A3(rrw, i, j, k) = A3(g->rf0, 1, 1, k) * A3(s.w3d, i, j, k);
      }
    }
    /* solve2.F:588-599 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
      float d = ((A3(rru, i + 1, j, k) - A3(rru, i, j, k)) * g->rdx * UH(i) + (A3(rrv, i, j + 1, k) - A3(rrv, i, j, k)) * g->rdy * VH(j)) +
                (A3(rrw, i, j, k + 1) - A3(rrw, i, j, k)) * g->rdz * A3(g->mh, 1, 1, k);
      if (fabsf(d) < cfg->smeps) d = 0.0f;
      A3(divx, i, j, k) = d;
    }
    /* solve2.F:884-893 */
    advu_g(g, &w, divx, rru, s.u3d, uten, rrv, rrw, s.rho, dttmp);
    advv_g(g, &w, divx, rru, rrv, s.v3d, vten, rrw, s.rho, dttmp);
    advw_g(g, &w, divx, rru, rrv, rrw, s.w3d, wten, s.rho, dttmp);
    /* solve2.F:899-907 */
#pragma omp parallel for
    for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
      A3(wten, i, j, k) = A3(wten, i, j, k) + (A3(g->c1, i, j, k) * A3(dum8, i, j, k - 1) + A3(g->c2, i, j, k) * A3(dum8, i, j, k));
    /* solve2.F:1027-1038 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) { float tem = A3(g->pi0, 1, 1, k);
      for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) A3(sadv, i, j, k) = tem + A3(s.pp3d, i, j, k); }
    /* solve2.F:1119-1134 */
    SoundArgs sa;
    sa.ua = s.ua; sa.u3d = s.u3d; sa.uten = uten; sa.va = s.va; sa.v3d = s.v3d; sa.vten = vten;
    sa.wa = s.wa; sa.w3d = s.w3d; sa.wten = wten; sa.ppi = s.ppi; sa.pp3d = s.pp3d; sa.piadv = sadv;
    sa.ppten = s.ppten; sa.ppx = s.ppx; sa.thv = t11; sa.ppterm = t22; sa.rru = rru; sa.rrv = rrv; sa.rrw = rrw;
    sa.radbcw = s.radbcw; sa.radbce = s.radbce; sa.radbcs = s.radbcs; sa.radbcn = s.radbcn;
    sound_g(g, &sa, nrk, dt);
    /* solve2.F:1252-1256 */
    if (nrk == 3) cflmax = calccflquick_g(g, dt, s.u3d, s.v3d, s.w3d);
    /* solve2.F:1260-1272 */
    if (cfg->irbc == 4) {
      if (g->ibw || g->ibe) radbcew4(g, s.radbcw, s.radbce, s.ua, s.u3d, dttmp);
      if (g->ibs || g->ibn) radbcns4(g, s.radbcs, s.radbcn, s.va, s.v3d, dttmp);
    }
    /* solve2.F:1277-1287 */
    if (cfg->imoist && cfg->eqtset == 2) getdiv_g(g, rru, rrv, rrw, t11);
    /* solve2.F:1303-1307 */
    getdivx_g(g, rru, rrv, rrw, divx);
    /* solve2.F:1320-1355 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
      A3(thten, i, j, k) = (cfg->imoist && cfg->eqtset == 2) ? A3(s.thten1, i, j, k) - A3(t11, i, j, k) * A3(thterm, i, j, k)
                                                            : A3(s.thten1, i, j, k);
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) { float tem = A3(g->th0, 1, 1, k) - TH0R;
      for (int j = g->jb; j <= g->je; j++) for (int i = g->ib; i <= g->ie; i++) A3(sadv, i, j, k) = tem + A3(s.th3d, i, j, k); }
    /* solve2.F:1391-1399 */
    advs_g(g, &w, nrk, 1, rru, rrv, rrw, divx, s.tha, sadv, thten, 0, 0, dttmp, (double)(10.0f * EPSILON_ADV),
           s.rho, rr, diffit);
    /* solve2.F:1419-1425 */
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      float v = A3(s.tha, i, j, k) + dttmp * A3(thten, i, j, k);
      if (fabsf(v) < cfg->smeps) v = 0.0f;
      A3(s.th3d, i, j, k) = v;
    }
    /* solve2.F:1431-1530 */
    for (int n = 0; n < numq; n++) {
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) A3(sten, i, j, k) = A3(s.qten[n], i, j, k);
      int pdef = (nrk == 3);
      double weps = (double)(cfg->qmag[n] * EPSILON_ADV);
      int pdefweno = (n + 1 == cfg->nqv) ? 0 : 1;
      advs_g(g, &w, nrk, 1, rru, rrv, rrw, divx, s.qa[n], s.q3d[n], sten, pdef, pdefweno, dttmp, weps, s.rho, rr, diffit);
#pragma omp parallel for
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        float v = A3(s.qa[n], i, j, k) + dttmp * A3(sten, i, j, k);
        if (fabsf(v) < cfg->smeps) v = 0.0f;
        A3(s.q3d[n], i, j, k) = v;
      }
    }
    /* solve2.F:1556-1656 */
    int dopf = 0;
    if (nrk == 3 || diffit) {   /* solve2.F:1582, 1599 */
#pragma omp parallel for
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        float pi = A3(g->pi0, i, j, k) + A3(s.pp3d, i, j, k);
        float pr = P00 * opowf(pi, c.cpdrd);
        A3(s.prs, i, j, k) = pr;
        if (cfg->imoist)
          A3(s.rho, i, j, k) = pr / ((A3(g->th0, i, j, k) + A3(s.th3d, i, j, k)) * pi * (c.rd + fmaxf(0.0f, A3(s.q3d[cfg->nqv - 1], i, j, k)) * c.rv));
        else
          A3(s.rho, i, j, k) = pr / (c.rd * (A3(g->th0, i, j, k) + A3(s.th3d, i, j, k)) * pi);
      }
      if (cfg->apmasscon == 1 && nrk == 3) {
#pragma omp parallel for
        for (int k = 1; k <= nk; k++) {
          double d3 = 0.0, d4 = 0.0;
          for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
            d3 = d3 + (double)(A3(s.rho, i, j, k) * RUH(i) * RVH(j) * A3(g->rmh, i, j, k));
            d4 = d4 + (double)(A3(g->pi0, i, j, k) + A3(s.pp3d, i, j, k));
          }
          dumk3[k] = d3; dumk4[k] = d4;
        }
        dopf = 1;
      }
    }
    /* solve2.F:1663-1707 */
    oracle_bcu_g(g, s.u3d);
    oracle_bcv_g(g, s.v3d);
    oracle_bcw_g(g, s.w3d, 1);
    if (nrk < 3) {
      oracle_bcp_g(g, s.rho);
      oracle_bcp_g(g, s.pp3d);
      oracle_bcs_g(g, s.th3d);
      for (int n = 0; n < numq; n++) oracle_bcs_g(g, s.q3d[n]);
    }
    /* solve2.F:1880-1970: passive tracers */
    if (cfg->iptra) {
      int pdef = (nrk == 3 && cfg->pdtra == 1);
      for (int n = 0; n < npt; n++) {
        for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) A3(sten, i, j, k) = A3(s.ptten[n], i, j, k);
        advs_g(g, &w, nrk, 1, rru, rrv, rrw, divx, s.pta[n], s.pt3d[n], sten, pdef, 1, dttmp, (double)(1.0f * EPSILON_ADV),
               s.rho, rr, diffit);
#pragma omp parallel for
        for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
          A3(s.pt3d[n], i, j, k) = A3(s.pta[n], i, j, k) + dttmp * A3(sten, i, j, k);
        if (nrk <= 2) oracle_bcs_g(g, s.pt3d[n]);
      }
    }
    /* solve2.F:2036-2046 */
    if (diffit && nrk < 3)
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
        A3(rr, i, j, k) = 1.0f / A3(s.rho, i, j, k);
    /* solve2.F:1976-2033 */
    if (dopf) {
      __float128 temq1 = 0, temq2 = 0;
      for (int k = 1; k <= nk; k++) { temq1 = temq1 + (__float128)dumk3[k]; temq2 = temq2 + (__float128)dumk4[k]; }
      mass2 = (double)temq1;
      double p2 = (double)temq2;
      float tem = (float)((pow(mass1 / mass2, (double)c.rddcv) - 1.0) * p2 / (double)((int64_t)ni * nj * nk));
#pragma omp parallel for
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        A3(s.pp3d, i, j, k) = A3(s.pp3d, i, j, k) + tem;
        float pi = A3(g->pi0, i, j, k) + A3(s.pp3d, i, j, k);
        float pr = P00 * opowf(pi, c.cpdrd);
        A3(s.prs, i, j, k) = pr;
        if (cfg->imoist)
          A3(s.rho, i, j, k) = pr / ((A3(g->th0, i, j, k) + A3(s.th3d, i, j, k)) * pi * (c.rd + fmaxf(0.0f, A3(s.q3d[cfg->nqv - 1], i, j, k)) * c.rv));
        else
          A3(s.rho, i, j, k) = pr / (c.rd * (A3(g->th0, i, j, k) + A3(s.th3d, i, j, k)) * pi);
      }
    }
  }
  /* solve2.F:2064-2075 */
  if (cfg->iptra) for (int n = 0; n < npt; n++) {
    if (cfg->pdtra == 1) pdefq_g(g, 0.0f, s.rho, s.pt3d[n]);
    oracle_bcs_g(g, s.pt3d[n]);
  }
  if (mass2_out) *mass2_out = mass2;
  if (cflmax_out) *cflmax_out = cflmax;
  free(dumk3); free(dumk4); free(tb); free(rrbuf); scratch_free(&w);
  return 0;
}

/* solve3 (dycore part): solve3.F:243-311 and 546-640 */
int oracle_solve3(const cm1g_config_t *cfg, const cm1g_grid_t *gr, cm1g_state_t *state) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  St s; st_view(g, state, &s);
  int ni = g->ni, nj = g->nj, nk = g->nk;
  int numq = cfg->imoist ? cfg->numq : 0, npt = cfg->iptra ? cfg->npt : 0;
  oracle_bcp_g(g, s.pp3d);
  oracle_bcs_g(g, s.th3d);
  for (int n = 0; n < numq; n++) oracle_bcs_g(g, s.q3d[n]);
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    A3(s.ppx, i, j, k) = A3(s.pp3d, i, j, k) + A3(s.ppx, i, j, k);
  oracle_bcp_g(g, s.ppx);
  oracle_bcp_g(g, s.rho);
  for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 2; j++) for (int i = 0; i <= ni + 2; i++) {
    A3(s.ua, i, j, k) = A3(s.u3d, i, j, k);
    A3(s.va, i, j, k) = A3(s.v3d, i, j, k);
    A3(s.wa, i, j, k) = A3(s.w3d, i, j, k);
  }
  for (int n = 0; n < npt; n++)
    for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++)
      A3(s.pta[n], i, j, k) = A3(s.pt3d[n], i, j, k);
  for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    A3(s.ppi, i, j, k) = A3(s.pp3d, i, j, k);
    A3(s.tha, i, j, k) = A3(s.th3d, i, j, k);
  }
  for (int n = 0; n < numq; n++)
    for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++)
      A3(s.qa[n], i, j, k) = A3(s.q3d[n], i, j, k);
  return 0;
}

/* pdefq on one array (misclibs.F:1037) */
int oracle_pdefq(const cm1g_config_t *cfg, const cm1g_grid_t *gr, float rmax, double *asq, const float *rho, float *q3d) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  double d = pdefq_g(g, rmax, mkS(g, rho), mkS(g, q3d));
  if (asq) *asq += d;
  return 0;
}

/* ------------------------------------------------------------------ */
/* 2nd-order diffusion (difforder=2): diff2def + diff2u/v/w/s          */
/* ------------------------------------------------------------------ */

/* rr, rf (solve3.F:660-678), divx and the stress tensor (diff2.F:743-989),
 * then the tendencies (diff2.F:11-735), in solve1's order (solve1.F:686-734) */
int oracle_diff2(const cm1g_config_t *cfg, const cm1g_grid_t *gr, float kdiff2, int idiff, int bbc, int tbc,
                 const float *cgs, const float *cgt, const float *ua_, const float *va_, const float *wa_,
                 const float *rho_, const float *tha_, const float *qa_, const float *pta_, float *uten_,
                 float *vten_, float *wten_, float *thten_, float *qten_, float *ptten_) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  if (idiff < 1) return 0;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const long ns = nS(g);
  F3 ua = mkU(g, ua_), va = mkV(g, va_), wa = mkW(g, wa_), rho = mkS(g, rho_);
  F3 uten = mkU(g, uten_), vten = mkV(g, vten_), wten = mkW(g, wten_);
  float *buf = (float *)calloc((size_t)(6 * ns + 3 * nW(g)), sizeof(float));
  if (!buf) return -3;
  float *p = buf;
  F3 rr = mkS(g, p); p += ns;
  F3 divx = mkS(g, p); p += ns;
  F3 t11 = mkS(g, p); p += ns;
  F3 t22 = mkS(g, p); p += ns;
  F3 t33 = mkS(g, p); p += ns;
  F3 t12 = mkS(g, p); p += ns;
  F3 rf = mkW(g, p); p += nW(g);
  F3 t13 = mkW(g, p); p += nW(g);
  F3 t23 = mkW(g, p);
  const float coef = kdiff2, twdth = 2.0f / 3.0f;
  const float rdx = g->rdx, rdy = g->rdy, rdz = g->rdz;
  const int wbc = cfg->wbc, ebc = cfg->ebc, sbc = cfg->sbc, nbc = cfg->nbc;
  /* solve3.F:660-678 */
  for (int k = 2; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    A3(rr, i, j, k) = 1.0f / A3(rho, i, j, k);
    A3(rf, i, j, k) = (A3(g->c1, i, j, k) * A3(rho, i, j, k - 1) + A3(g->c2, i, j, k) * A3(rho, i, j, k));
  }
  for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    A3(rr, i, j, 1) = 1.0f / A3(rho, i, j, 1);
    A3(rf, i, j, 1) = cgs[0] * A3(rho, i, j, 1) + cgs[1] * A3(rho, i, j, 2) + cgs[2] * A3(rho, i, j, 3);
    A3(rf, i, j, nk + 1) = cgt[0] * A3(rho, i, j, nk) + cgt[1] * A3(rho, i, j, nk - 1) + cgt[2] * A3(rho, i, j, nk - 2);
  }
  /* diff2def (Cartesian) */
  for (int k = 1; k <= nk; k++) {
    for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
      float d = (A3(ua, i + 1, j, k) - A3(ua, i, j, k)) * rdx * UH(i) + (A3(va, i, j + 1, k) - A3(va, i, j, k)) * rdy * VH(j) +
                (A3(wa, i, j, k + 1) - A3(wa, i, j, k)) * rdz * A3(g->mh, 1, 1, k);
      if (fabsf(d) < cfg->smeps) d = 0.0f;
      A3(divx, i, j, k) = d;
    }
    for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
      A3(t11, i, j, k) = coef * A3(rho, i, j, k) * (A3(ua, i + 1, j, k) - A3(ua, i, j, k)) * rdx * UH(i);
      A3(t22, i, j, k) = coef * A3(rho, i, j, k) * (A3(va, i, j + 1, k) - A3(va, i, j, k)) * rdy * VH(j);
      A3(t33, i, j, k) = coef * A3(rho, i, j, k) * (A3(wa, i, j, k + 1) - A3(wa, i, j, k)) * rdz * A3(g->mh, 1, 1, k);
      A3(t12, i, j, k) = coef * ((A3(ua, i, j, k) - A3(ua, i, j - 1, k)) * rdy * VF(j) +
                                 (A3(va, i, j, k) - A3(va, i - 1, j, k)) * rdx * UF(i)) * 0.25f *
                         ((A3(rho, i - 1, j - 1, k) + A3(rho, i, j, k)) + (A3(rho, i - 1, j, k) + A3(rho, i, j - 1, k)));
    }
#define R4(i, j) ((A3(rho, (i) - 1, (j) - 1, k) + A3(rho, i, j, k)) + (A3(rho, (i) - 1, j, k) + A3(rho, i, (j) - 1, k)))
    if (wbc == 3 && g->ibw) { for (int j = 1; j <= nj + 1; j++) A3(t12, 1, j, k) = A3(t12, 2, j, k); }
    else if (wbc == 4 && g->ibw) { for (int j = 1; j <= nj + 1; j++) A3(t12, 1, j, k) = coef * 2.0f * A3(va, 1, j, k) * rdx * UF(1) * 0.25f * R4(1, j); }
    if (ebc == 3 && g->ibe) { for (int j = 1; j <= nj + 1; j++) A3(t12, ni + 1, j, k) = A3(t12, ni, j, k); }
    else if (ebc == 4 && g->ibe) { for (int j = 1; j <= nj + 1; j++) A3(t12, ni + 1, j, k) = -coef * 2.0f * A3(va, ni, j, k) * rdx * UF(ni + 1) * 0.25f * R4(ni + 1, j); }
    if (sbc == 3 && g->ibs) { for (int i = 1; i <= ni + 1; i++) A3(t12, i, 1, k) = A3(t12, i, 2, k); }
    else if (sbc == 4 && g->ibs) { for (int i = 1; i <= ni + 1; i++) A3(t12, i, 1, k) = coef * 2.0f * A3(ua, i, 1, k) * rdy * VF(1) * 0.25f * R4(i, 1); }
    if (nbc == 3 && g->ibn) { for (int i = 1; i <= ni + 1; i++) A3(t12, i, nj + 1, k) = A3(t12, i, nj, k); }
    else if (nbc == 4 && g->ibn) { for (int i = 1; i <= ni + 1; i++) A3(t12, i, nj + 1, k) = -coef * 2.0f * A3(ua, i, nj, k) * rdy * VF(nj + 1) * 0.25f * R4(i, nj + 1); }
#undef R4
    if (k != 1) {
      for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
        A3(t13, i, j, k) = coef * ((A3(ua, i, j, k) - A3(ua, i, j, k - 1)) * rdz * A3(g->mf, 1, 1, k) +
                                   (A3(wa, i, j, k) - A3(wa, i - 1, j, k)) * rdx * UF(i));
        A3(t23, i, j, k) = coef * ((A3(va, i, j, k) - A3(va, i, j, k - 1)) * rdz * A3(g->mf, 1, 1, k) +
                                   (A3(wa, i, j, k) - A3(wa, i, j - 1, k)) * rdy * VF(j));
      }
      if (wbc == 3 && g->ibw) { for (int j = 1; j <= nj; j++) A3(t13, 1, j, k) = A3(t13, 2, j, k); }
      else if (wbc == 4 && g->ibw) { for (int j = 1; j <= nj; j++) A3(t13, 1, j, k) = coef * 2.0f * A3(wa, 1, j, k) * rdx * UF(1); }
      if (ebc == 3 && g->ibe) { for (int j = 1; j <= nj; j++) A3(t13, ni + 1, j, k) = A3(t13, ni, j, k); }
      else if (ebc == 4 && g->ibe) { for (int j = 1; j <= nj; j++) A3(t13, ni + 1, j, k) = -coef * 2.0f * A3(wa, ni, j, k) * rdx * UF(ni + 1); }
      if (sbc == 3 && g->ibs) { for (int i = 1; i <= ni; i++) A3(t23, i, 1, k) = A3(t23, i, 2, k); }
      else if (sbc == 4 && g->ibs) { for (int i = 1; i <= ni; i++) A3(t23, i, 1, k) = coef * 2.0f * A3(wa, i, 1, k) * rdy * VF(1); }
      if (nbc == 3 && g->ibn) { for (int i = 1; i <= ni; i++) A3(t23, i, nj + 1, k) = A3(t23, i, nj, k); }
      else if (nbc == 4 && g->ibn) { for (int i = 1; i <= ni; i++) A3(t23, i, nj + 1, k) = -coef * 2.0f * A3(wa, i, nj, k) * rdy * VF(nj + 1); }
    }
  }
  if (bbc == 1) {
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) A3(t13, i, j, 1) = A3(t13, i, j, 2);
    for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) A3(t23, i, j, 1) = A3(t23, i, j, 2);
  } else if (bbc == 2) {
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++)
      A3(t13, i, j, 1) = coef * 2.0f * (A3(ua, i, j, 1) + 0.0f) * rdz * A3(g->mf, 1, 1, 1);
    for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++)
      A3(t23, i, j, 1) = coef * 2.0f * (A3(va, i, j, 1) + 0.0f) * rdz * A3(g->mf, 1, 1, 1);
  }
  if (tbc == 1) {
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) A3(t13, i, j, nk + 1) = A3(t13, i, j, nk);
    for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) A3(t23, i, j, nk + 1) = A3(t23, i, j, nk);
  } else if (tbc == 2) {
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++)
      A3(t13, i, j, nk + 1) = -coef * 2.0f * A3(ua, i, j, nk) * rdz * A3(g->mf, 1, 1, nk + 1);
    for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++)
      A3(t23, i, j, nk + 1) = -coef * 2.0f * A3(va, i, j, nk) * rdz * A3(g->mf, 1, 1, nk + 1);
  }
  for (int k = 1; k <= nk + 1; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
    A3(t13, i, j, k) = A3(t13, i, j, k) * 0.5f * (A3(rf, i - 1, j, k) + A3(rf, i, j, k));
    A3(t23, i, j, k) = A3(t23, i, j, k) * 0.5f * (A3(rf, i, j - 1, k) + A3(rf, i, j, k));
  }
  /* diff2u */
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) {
    float d0 = 2.0f * A3(t11, i, j, k) - A3(rho, i, j, k) * twdth * A3(divx, i, j, k);
    float dm = 2.0f * A3(t11, i - 1, j, k) - A3(rho, i - 1, j, k) * twdth * A3(divx, i - 1, j, k);
    float fx = (d0 - dm) * rdx * UF(i);
    float fy = (A3(t12, i, j + 1, k) - A3(t12, i, j, k)) * rdy * VH(j);
    float fz = (A3(t13, i, j, k + 1) - A3(t13, i, j, k)) * rdz * A3(g->mh, 1, 1, k);
    A3(uten, i, j, k) = A3(uten, i, j, k) + ((fx + fy) + fz) / (0.5f * (A3(rho, i - 1, j, k) + A3(rho, i, j, k)));
  }
  /* diff2v */
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) {
    float fx = (A3(t12, i + 1, j, k) - A3(t12, i, j, k)) * rdx * UH(i);
    float d0 = 2.0f * A3(t22, i, j, k) - A3(rho, i, j, k) * twdth * A3(divx, i, j, k);
    float dm = 2.0f * A3(t22, i, j - 1, k) - A3(rho, i, j - 1, k) * twdth * A3(divx, i, j - 1, k);
    float fy = (d0 - dm) * rdy * VF(j);
    float fz = (A3(t23, i, j, k + 1) - A3(t23, i, j, k)) * rdz * A3(g->mh, 1, 1, k);
    A3(vten, i, j, k) = A3(vten, i, j, k) + ((fx + fy) + fz) / (0.5f * (A3(rho, i, j - 1, k) + A3(rho, i, j, k)));
  }
  /* diff2w */
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    float fx = (A3(t13, i + 1, j, k) - A3(t13, i, j, k)) * rdx * UH(i);
    float fy = (A3(t23, i, j + 1, k) - A3(t23, i, j, k)) * rdy * VH(j);
    float d0 = 2.0f * A3(t33, i, j, k) - A3(rho, i, j, k) * twdth * A3(divx, i, j, k);
    float dm = 2.0f * A3(t33, i, j, k - 1) - A3(rho, i, j, k - 1) * twdth * A3(divx, i, j, k - 1);
    float fz = (d0 - dm) * rdz * A3(g->mf, 1, 1, k);
    A3(wten, i, j, k) = A3(wten, i, j, k) + ((fx + fy) + fz) / A3(rf, i, j, k);
  }
  /* diff2s: theta, each q, each tracer (idiff = 1) */
  if (idiff == 1) {
    int numq = cfg->imoist ? cfg->numq : 0, npt = cfg->iptra ? cfg->npt : 0;
    int nsc = 1 + numq + npt;
    for (int n = 0; n < nsc; n++) {
      const float *sp = n == 0 ? tha_ : n <= numq ? qa_ + (n - 1) * ns : pta_ + (n - 1 - numq) * ns;
      float *tp = n == 0 ? thten_ : n <= numq ? qten_ + (n - 1) * ns : ptten_ + (n - 1 - numq) * ns;
      F3 s = mkS(g, sp), sten = mkS(g, tp);
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        float dxl = 0.5f * (A3(rho, i, j, k) + A3(rho, i - 1, j, k)) * (A3(s, i, j, k) - A3(s, i - 1, j, k)) * rdx * UF(i);
        float dxr = 0.5f * (A3(rho, i + 1, j, k) + A3(rho, i, j, k)) * (A3(s, i + 1, j, k) - A3(s, i, j, k)) * rdx * UF(i + 1);
        float fx = coef * (dxr - dxl) * rdx * UH(i);
        float dyl = 0.5f * (A3(rho, i, j, k) + A3(rho, i, j - 1, k)) * (A3(s, i, j, k) - A3(s, i, j - 1, k)) * rdy * VF(j);
        float dyr = 0.5f * (A3(rho, i, j + 1, k) + A3(rho, i, j, k)) * (A3(s, i, j + 1, k) - A3(s, i, j, k)) * rdy * VF(j + 1);
        float fy = coef * (dyr - dyl) * rdy * VH(j);
        float dzl = k == 1 ? 0.0f : (A3(s, i, j, k) - A3(s, i, j, k - 1)) * rdz * A3(g->mf, 1, 1, k);
        float dzu = k == nk ? 0.0f : (A3(s, i, j, k + 1) - A3(s, i, j, k)) * rdz * A3(g->mf, 1, 1, k + 1);
        float fz = coef * (A3(rf, i, j, k + 1) * dzu - A3(rf, i, j, k) * dzl) * rdz * A3(g->mh, 1, 1, k);
        A3(sten, i, j, k) = A3(sten, i, j, k) + ((fx + fy) + fz) * A3(rr, i, j, k);
      }
    }
  }
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Kessler microphysics (ptype=1): mp_driver.F:189-233, kessler.F      */
/* ------------------------------------------------------------------ */

typedef struct {
  float eps, lv1, lv2, cpdcv, rp00;
} KConsts;

static KConsts kessler_consts(const OG *g) {
  /* constants.F:115-159 */
  const Consts c = g->c;
  const int tc = g->cfg->testcase;
  const float xlv = tc == 4 ? 2.47e6f : tc == 5 ? 2.50e6f : 2501000.0f, to = 273.15f;
  KConsts k;
  k.eps = c.rd / c.rv;
  k.lv1 = (tc == 4 || tc == 5) ? xlv : xlv + (c.cpl - c.cpv) * to;
  k.lv2 = (tc == 4 || tc == 5) ? 0.0f : c.cpl - c.cpv;
  k.cpdcv = c.cp / c.cv;
  k.rp00 = 1.0f / P00;
  return k;
}

/* k_fallout (kessler.F:441-462) */
static void k_fallout_g(const OG *g, F3 rho, F3 qr, F3 vr) {
#pragma omp parallel for
  for (int k = 1; k <= g->nk; k++) for (int j = 1; j <= g->nj; j++) for (int i = 1; i <= g->ni; i++) {
    A3(vr, i, j, k) = 0.0f;
    if (A3(qr, i, j, k) > 1.0e-12f)
      A3(vr, i, j, k) = 14.34f * opowf(A3(rho, i, j, k) * A3(qr, i, j, k), 0.1346f) * sqrtf(1.15f / A3(rho, i, j, k));
  }
}

/* geterain (kessler.F:529-558) */
static void geterain_g(const OG *g, float dt, float cpx, float lx1, double *erain, F3 t, F3 rr, F3 q, F3 vr) {
  double *bud = (double *)calloc((size_t)g->nj + 1, sizeof(double));
#pragma omp parallel for
  for (int j = 1; j <= g->nj; j++) {
    bud[j] = 0.0;
    for (int i = 1; i <= g->ni; i++)
      bud[j] = bud[j] + (double)(dt * A3(vr, i, j, 1) * A3(rr, i, j, 1) * A3(q, i, j, 1) * (cpx * A3(t, i, j, 1) - lx1) *
                                 RUH(i) * RVH(j));
  }
  for (int j = 1; j <= g->nj; j++) *erain = *erain + bud[j] * (double)g->dx * (double)g->dy;
  free(bud);
}

/* fallout (kessler.F:470-521), nrain = 1 */
static void fallout_g(const OG *g, float dt, double *train, F3 rain, F3 prate, F3 rr, F3 rho, F3 q, F3 vq) {
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  double *bud = (double *)calloc((size_t)nj + 1, sizeof(double));
#pragma omp parallel for
  for (int j = 1; j <= nj; j++) {
    float *rq = (float *)calloc((size_t)nk + 5, sizeof(float));   /* rq(-1:nk+3) at rq[k+1] */
    bud[j] = 0.0;
    for (int i = 1; i <= ni; i++) {
      float crmax = 0.0f;
      for (int k = 1; k <= nk; k++) crmax = fmaxf(crmax, A3(vq, i, j, k) * dt * g->rdz * A3(g->mh, i, j, k));
      int nfall = (int)(crmax + 1.0f);
      if (nfall < 1) nfall = 1;
      for (int k = nk - 1; k >= 1; k--)
        if (A3(q, i, j, k) < 1.0e-8f) A3(vq, i, j, k) = A3(vq, i, j, k + 1);
      float dtfall = dt / (float)nfall;
      for (int n = 1; n <= nfall; n++) {
        for (int k = 1; k <= nk; k++) rq[k + 1] = A3(rho, i, j, k) * A3(vq, i, j, k) * fmaxf(0.0f, A3(q, i, j, k));
        rq[nk + 2] = 0.0f;
        for (int k = 1; k <= nk; k++)
          A3(q, i, j, k) = A3(q, i, j, k) + dtfall * (rq[k + 2] - rq[k + 1]) * g->rdz * A3(g->mh, i, j, k) /
                                                A3(rho, i, j, k);
        A3(rain, i, j, 0) = A3(rain, i, j, 0) + 0.1f * dtfall * rq[2];
        A3(prate, i, j, 0) = rq[2];
        bud[j] = bud[j] + (double)(dtfall * A3(rr, i, j, 1) * A3(vq, i, j, 1) * fmaxf(0.0f, A3(q, i, j, 1)) * RUH(i) *
                                   RVH(j));
      }
    }
    free(rq);
  }
  double tem = (double)(g->dx * g->dy);
  for (int j = 1; j <= nj; j++) *train = *train + bud[j] * tem;
  free(bud);
}

static float esl_of(float t, float p) {
  float esl = 611.2f * expf(17.67f * (t - 273.15f) / (t - 29.65f));
  return fminf(esl, p * 0.5f);
}

/* kessler (kessler.F:10-133) */
static void kessler_g(const OG *g, float dt, double *tauto, double *taccr, double *tevar, F3 tmp, F3 rho, F3 rr,
                      F3 pp3d, F3 th3d, F3 prs, F3 qv3d, F3 qc3d, F3 qr3d) {
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const Consts c = g->c;
  const KConsts K = kessler_consts(g);
  double *bud = (double *)calloc((size_t)3 * (nk + 1), sizeof(double));
#pragma omp parallel for
  for (int k = 1; k <= nk; k++) {
    double b1 = 0.0, b2 = 0.0, b3 = 0.0;
    for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
      const float th0 = A3(g->th0, i, j, k), pi0 = A3(g->pi0, i, j, k);
      A3(tmp, i, j, k) = (th0 + A3(th3d, i, j, k)) * (pi0 + A3(pp3d, i, j, k));
      float qvnew = A3(qv3d, i, j, k), qcnew = A3(qc3d, i, j, k), qrnew = A3(qr3d, i, j, k);
      float ar = 0.0f, cr = 0.0f, er = 0.0f;
      if (qcnew > 0.0f) {
        ar = fmaxf(0.001f * (qcnew - 0.001f), 0.0f);
        ar = ar * dt;
      }
      if (qcnew > 0.0f && qrnew > 0.0f) {
        cr = 2.2f * qcnew * opowf(qrnew, 0.875f);
        cr = cr * dt;
      }
      if (qrnew > 0.0f) {
        float esl = esl_of(A3(tmp, i, j, k), A3(prs, i, j, k));
        float qvs = K.eps * esl / (A3(prs, i, j, k) - esl);
        if (qvnew < qvs) {
          float r = A3(rho, i, j, k);
          er = (1.6f + 30.3922f * opowf(r * qrnew, 0.2046f)) * (1.0f - (qvnew / qvs)) * opowf(r * qrnew, 0.525f) /
               ((2.03e4f + 9.584e6f / (qvs * A3(prs, i, j, k))) * r);
          er = fminf(er * dt, qrnew);
          if ((qvnew + er) > qvs) er = qvs - qvnew;
        }
      }
      if ((ar + cr) > qcnew) {
        float term1 = ar + cr;
        ar = qcnew * ar / term1;
        cr = qcnew * cr / term1;
      }
      qvnew = qvnew + er;
      qcnew = qcnew - (ar + cr);
      qrnew = qrnew + (ar + cr - er);
      if (er > 1.0e-7f) {
        if (g->cfg->eqtset == 2) {
          float cpml = c.cp + c.cpv * qvnew + c.cpl * (qcnew + qrnew);
          float cvml = c.cv + c.cvv * qvnew + c.cpl * (qcnew + qrnew);
          float rm = c.rd + c.rv * qvnew;
          A3(th3d, i, j, k) = A3(th3d, i, j, k) -
              er * ((K.lv1 - K.lv2 * A3(tmp, i, j, k)) / (K.cpdcv * cvml * (pi0 + A3(pp3d, i, j, k))) -
                    (th0 + A3(th3d, i, j, k)) * (c.rv / cvml) * (1.0f - c.rovcp * cpml / rm));
          A3(pp3d, i, j, k) = opowf(A3(rho, i, j, k) * rm * (th0 + A3(th3d, i, j, k)) * K.rp00, c.rddcv) - pi0;
          A3(prs, i, j, k) = P00 * opowf(pi0 + A3(pp3d, i, j, k), c.cpdrd);
        } else {
          A3(th3d, i, j, k) = A3(th3d, i, j, k) - er * ((K.lv1 - K.lv2 * A3(tmp, i, j, k)) / (c.cp * (pi0 + A3(pp3d, i, j, k))));
          A3(rho, i, j, k) = A3(prs, i, j, k) /
              (c.rd * (th0 + A3(th3d, i, j, k)) * (pi0 + A3(pp3d, i, j, k)) * (1.0f + qvnew * c.reps));
        }
      }
      float tem = RUH(i) * RVH(j) * A3(g->rmh, i, j, k);
      b1 = b1 + (double)(A3(rr, i, j, k) * ar * tem);
      b2 = b2 + (double)(A3(rr, i, j, k) * cr * tem);
      b3 = b3 + (double)(A3(rr, i, j, k) * er * tem);
      A3(qv3d, i, j, k) = qvnew;
      A3(qc3d, i, j, k) = qcnew;
      A3(qr3d, i, j, k) = qrnew;
    }
    bud[3 * k] = b1; bud[3 * k + 1] = b2; bud[3 * k + 2] = b3;
  }
  double dum = (double)(g->dx * g->dy * g->dz);
  for (int k = 1; k <= nk; k++) *tauto = *tauto + bud[3 * k] * dum;
  for (int k = 1; k <= nk; k++) *taccr = *taccr + bud[3 * k + 1] * dum;
  for (int k = 1; k <= nk; k++) *tevar = *tevar + bud[3 * k + 2] * dum;
  free(bud);
}

/* satadj (kessler.F:142-432) with nrk = 4; returns 1 when an iteration did
 * not converge (the reference stops the model) */
static int satadj_g(const OG *g, float dt, double *tcond, double *tevac, F3 rho, F3 rr, F3 pp3d, F3 prs, F3 th3d,
                    F3 *q3d) {
  (void)dt;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const Consts c = g->c;
  const KConsts K = kessler_consts(g);
  const cm1g_config_t *cfg = g->cfg;
  const int nqv = cfg->nqv - 1, nqc = cfg->nql1 - 1;
  double *bud = (double *)calloc((size_t)2 * (nk + 1), sizeof(double));
  int iflag = 0;
  if (cfg->eqtset == 2) {
    const float converge = 2.0f * cfg->tsmall;
#pragma omp parallel for reduction(|:iflag)
    for (int k = 1; k <= nk; k++) {
      double b1 = 0.0, b2 = 0.0;
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        const float th0 = A3(g->th0, i, j, k), pi0 = A3(g->pi0, i, j, k);
        float tnew = (th0 + A3(th3d, i, j, k)) * (pi0 + A3(pp3d, i, j, k));
        float esl = esl_of(tnew, A3(prs, i, j, k));
        float qvs = K.eps * esl / (A3(prs, i, j, k) - esl);
        if (A3(q3d[nqc], i, j, k) > 1.0e-12f || A3(q3d[nqv], i, j, k) > qvs) {
          float qvnew = A3(q3d[nqv], i, j, k), qcnew = A3(q3d[nqc], i, j, k);
          float ql = 0.0f, qi = 0.0f;
          for (int n = cfg->nql1; n <= cfg->nql2; n++) ql = ql + A3(q3d[n - 1], i, j, k);
          ql = fmaxf(0.0f, ql);
          qi = fmaxf(0.0f, qi);
          float cvml = c.cv + c.cvv * qvnew + c.cpl * ql + c.cpi * qi;
          float lhv = K.lv1 - K.lv2 * tnew;
          float t1 = (lhv - c.rv * tnew) / cvml;
          float d1 = t1 * 17.67f * 243.5f;
          int n = 0;
          float tlast = tnew, pnew = 0.0f;
          int doit = 1;
          while (doit) {
            n = n + 1;
            float dqv = (qvs - qvnew) / (1.0f + d1 * qvs / ((tnew - 29.65f) * (tnew - 29.65f)));
            dqv = fminf(dqv, qcnew);
            if ((qvnew + dqv) < 1.0e-20f) dqv = 1.0e-20f - qvnew;
            qvnew = qvnew + dqv;
            qcnew = qcnew - dqv;
            tnew = tnew - dqv * t1;
            pnew = A3(rho, i, j, k) * (c.rd + c.rv * qvnew) * tnew;
            doit = 0;
            if (fabsf(tnew - tlast) > converge) {
              tlast = tnew;
              esl = esl_of(tnew, A3(prs, i, j, k));
              qvs = K.eps * esl / (pnew - esl);
              doit = 1;
            }
            if (n == 100) { iflag = 1; doit = 0; }
          }
          float tem = RUH(i) * RVH(j) * A3(g->rmh, i, j, k);
          b1 = b1 + (double)(A3(rr, i, j, k) * fmaxf(qcnew - A3(q3d[nqc], i, j, k), 0.0f) * tem);
          b2 = b2 + (double)(A3(rr, i, j, k) * fmaxf(qvnew - A3(q3d[nqv], i, j, k), 0.0f) * tem);
          A3(prs, i, j, k) = pnew;
          A3(pp3d, i, j, k) = opowf(pnew * K.rp00, c.rovcp) - pi0;
          A3(th3d, i, j, k) = tnew / (pi0 + A3(pp3d, i, j, k)) - th0;
          A3(q3d[nqc], i, j, k) = qcnew;
          A3(q3d[nqv], i, j, k) = qvnew;
        }
      }
      bud[2 * k] = b1; bud[2 * k + 1] = b2;
    }
  } else {
#pragma omp parallel for
    for (int k = 1; k <= nk; k++) {
      double b1 = 0.0, b2 = 0.0;
      for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        const float th0 = A3(g->th0, i, j, k), pi0 = A3(g->pi0, i, j, k);
        float qvnew = A3(q3d[nqv], i, j, k), qcnew = A3(q3d[nqc], i, j, k);
        float tnew = (th0 + A3(th3d, i, j, k)) * (pi0 + A3(pp3d, i, j, k));
        float esl = esl_of(tnew, A3(prs, i, j, k));
        float qvs = K.eps * esl / (A3(prs, i, j, k) - esl);
        float lhv = K.lv1 - K.lv2 * tnew;
        float dqv = (qvs - qvnew) / (1.0f + lhv * qvs * 17.67f * 243.5f / (c.cp * ((tnew - 29.65f) * (tnew - 29.65f))));
        if ((qvnew + dqv) < 1.0e-20f) dqv = 1.0e-20f - qvnew;
        dqv = fminf(dqv, fmaxf(0.0f, qcnew));
        qvnew = qvnew + dqv;
        qcnew = qcnew - dqv;
        float tem = RUH(i) * RVH(j) * A3(g->rmh, i, j, k);
        b1 = b1 + (double)(A3(rr, i, j, k) * fmaxf(qcnew - A3(q3d[nqc], i, j, k), 0.0f) * tem);
        b2 = b2 + (double)(A3(rr, i, j, k) * fmaxf(qvnew - A3(q3d[nqv], i, j, k), 0.0f) * tem);
        A3(th3d, i, j, k) = A3(th3d, i, j, k) - dqv * (lhv / (c.cp * (pi0 + A3(pp3d, i, j, k))));
        A3(q3d[nqc], i, j, k) = qcnew;
        A3(q3d[nqv], i, j, k) = qvnew;
        A3(rho, i, j, k) = A3(prs, i, j, k) /
            (c.rd * (th0 + A3(th3d, i, j, k)) * (pi0 + A3(pp3d, i, j, k)) * (1.0f + qvnew * c.reps));
      }
      bud[2 * k] = b1; bud[2 * k + 1] = b2;
    }
  }
  double dum = (double)(g->dx * g->dy * g->dz);
  for (int k = 1; k <= nk; k++) *tcond = *tcond + bud[2 * k] * dum;
  for (int k = 1; k <= nk; k++) *tevac = *tevac + bud[2 * k + 1] * dum;
  free(bud);
  return iflag;
}

/* The Kessler branch of mp_driver (mp_driver.F:98-233, efall = 0):
 * qbudget[0..6] = qbudget(1..7), asq[0..2] = asq(1..3). */
static int mp_kessler_g(const OG *g, St *s, float dt, double *qbudget, double *asq) {
  const long ns = nS(g);
  const Consts c = g->c;
  const KConsts K = kessler_consts(g);
  float *buf = (float *)calloc((size_t)3 * ns, sizeof(float));
  if (!buf) return -3;
  F3 dum1 = mkS(g, buf), dum3 = mkS(g, buf + ns), vr = mkS(g, buf + 2 * ns);
  for (int k = 1; k <= g->nk; k++) for (int j = 1; j <= g->nj; j++) for (int i = 1; i <= g->ni; i++) {
    A3(dum1, i, j, k) = (A3(g->th0, i, j, k) + A3(s->th3d, i, j, k)) * (A3(g->pi0, i, j, k) + A3(s->pp3d, i, j, k));
    A3(dum3, i, j, k) = A3(s->rho, i, j, k);
  }
  asq[0] += pdefq_g(g, 0.0f, s->rho, s->q3d[0]);
  asq[1] += pdefq_g(g, g->cfg->qsmall, s->rho, s->q3d[1]);
  asq[2] += pdefq_g(g, g->cfg->qsmall, s->rho, s->q3d[2]);
  k_fallout_g(g, s->rho, s->q3d[2], vr);
  geterain_g(g, dt, c.cpl, K.lv1, &qbudget[6], dum1, dum3, s->q3d[2], vr);
  fallout_g(g, dt, &qbudget[5], s->rain, s->prate, dum3, s->rho, s->q3d[2], vr);
  kessler_g(g, dt, &qbudget[2], &qbudget[3], &qbudget[4], dum1, s->rho, dum3, s->pp3d, s->th3d, s->prs, s->q3d[0],
            s->q3d[1], s->q3d[2]);
  int bad = satadj_g(g, dt, &qbudget[0], &qbudget[1], s->rho, dum3, s->pp3d, s->prs, s->th3d, s->q3d);
  free(buf);
  if (bad) { snprintf(g_err, sizeof g_err, "satadj: convergence cannot be reached"); return -4; }
  return 0;
}

/* mp_driver alone (ptype=1), with the budgets it adds to */
int oracle_mp_driver(const cm1g_config_t *cfg, const cm1g_grid_t *gr, cm1g_state_t *state, float dt,
                     double qbudget[7], double asq[3]) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr) || check_cfg(cfg) || cfg->ptype != 1) return -1;
  St s; st_view(g, state, &s);
  return mp_kessler_g(g, &s, dt, qbudget, asq);
}

/* One time step as cm1.F runs it: solve2 (3357), pdefq for ptype=0 (3414)
 * or mp_driver for ptype=1 (3421-3431), solve3 (3432). */
int oracle_step(const cm1g_config_t *cfg, const cm1g_grid_t *gr, cm1g_state_t *state, int nstep, float dt,
                double mtime, double mass1, double *mass2, float *cflmax) {
  int rc = oracle_solve2(cfg, gr, state, nstep, dt, mtime, mass1, mass2, cflmax);
  if (rc) return rc;
  if (cfg->imoist && cfg->ptype == 1) {   /* cm1.F:3421-3431: mp_driver */
    double qb[7] = {0, 0, 0, 0, 0, 0, 0}, asq[3] = {0, 0, 0};
    rc = oracle_mp_driver(cfg, gr, state, dt, qb, asq);
    if (rc) return rc;
  } else if (cfg->imoist) {
    double asq = 0.0;
    long n = (long)(cfg->ni + 2 * cfg->ngxy) * (cfg->nj + 2 * cfg->ngxy) * (cfg->nk + 2);
    rc = oracle_pdefq(cfg, gr, 0.0f, &asq, RPC(state->rho), RP(state->q3d) + (long)(cfg->nqv - 1) * n);
    if (rc) return rc;
  }
  return oracle_solve3(cfg, gr, state);
}

/* ------------------------------------------------------------------ */
/* Per-routine entry points used by the unit parity tests               */
/* ------------------------------------------------------------------ */

int oracle_bc(const cm1g_config_t *cfg, int which, float *a, int flag) {
  OG G, *g = &G;
  if (og_setup(g, cfg, NULL)) return -1;
  switch (which) {
    case 1: oracle_bcs_g(g, mkS(g, a)); break;
    case 2: oracle_bcp_g(g, mkS(g, a)); break;
    case 3: oracle_bcu_g(g, mkU(g, a)); break;
    case 4: oracle_bcv_g(g, mkV(g, a)); break;
    case 5: oracle_bcw_g(g, mkW(g, a), flag); break;
    default: return -1;
  }
  return 0;
}

int oracle_advs(const cm1g_config_t *cfg, const cm1g_grid_t *gr, int nrk, int wflag,
                const float *rru, const float *rrv, const float *rrw, const float *divx,
                const float *s0, const float *s, float *sten, int pdef, int pdefweno, float dt, double weps) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  Scratch w;
  if (scratch_alloc(g, &w)) return -3;
  /* pdef routines write into the halos of dumx/dumy via bcs, the flux arrays
   * are scratch; s, rru, rrv, rrw, divx are read only. */
  advs_g(g, &w, nrk, wflag, mkU(g, rru), mkV(g, rrv), mkW(g, rrw), mkS(g, divx), mkS(g, s0), mkS(g, s), mkS(g, sten),
         pdef, pdefweno, dt, weps, mkS(g, s), mkS(g, s), 0);
  scratch_free(&w);
  return 0;
}

int oracle_advuvw(const cm1g_config_t *cfg_in, const cm1g_grid_t *gr, const float *u3d, const float *v3d,
                  const float *w3d, float *uten, float *vten, float *wten) {
  /* advection alone: the 6th-order diffusion needs rho, which this entry
   * point does not take */
  cm1g_config_t cfgv = *cfg_in;
  const cm1g_config_t *cfg = &cfgv;
  cfgv.idiff = 0;
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  int ni = g->ni, nj = g->nj, nk = g->nk;
  Scratch w;
  if (scratch_alloc(g, &w)) return -3;
  float *tb = (float *)calloc((size_t)(nU(g) + nV(g) + nW(g) + nS(g)), sizeof(float));
  F3 rru = mkU(g, tb), rrv = mkV(g, tb + nU(g)), rrw = mkW(g, tb + nU(g) + nV(g)), divx = mkS(g, tb + nU(g) + nV(g) + nW(g));
  F3 u = mkU(g, u3d), v = mkV(g, v3d), ww = mkW(g, w3d);
  for (int k = 1; k <= nk; k++) {
    float r0 = A3(g->rho0, 1, 1, k);
    for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 2; i++) A3(rru, i, j, k) = r0 * A3(u, i, j, k);
    for (int j = 0; j <= nj + 2; j++) for (int i = 0; i <= ni + 1; i++) A3(rrv, i, j, k) = r0 * A3(v, i, j, k);
    if (k == 1) { for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) { A3(rrw, i, j, 1) = 0.0f; A3(rrw, i, j, nk + 1) = 0.0f; } }
    else for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) A3(rrw, i, j, k) = A3(g->rf0, 1, 1, k) * A3(ww, i, j, k);
  }
  for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    float d = ((A3(rru, i + 1, j, k) - A3(rru, i, j, k)) * g->rdx * UH(i) + (A3(rrv, i, j + 1, k) - A3(rrv, i, j, k)) * g->rdy * VH(j)) +
              (A3(rrw, i, j, k + 1) - A3(rrw, i, j, k)) * g->rdz * A3(g->mh, 1, 1, k);
    if (fabsf(d) < cfg->smeps) d = 0.0f;
    A3(divx, i, j, k) = d;
  }
  advu_g(g, &w, divx, rru, u, mkU(g, uten), rrv, rrw, u, 1.0f);
  advv_g(g, &w, divx, rru, rrv, v, mkV(g, vten), rrw, v, 1.0f);
  advw_g(g, &w, divx, rru, rrv, rrw, ww, mkW(g, wten), ww, 1.0f);
  free(tb); scratch_free(&w);
  return 0;
}

int oracle_sound(const cm1g_config_t *cfg, const cm1g_grid_t *gr, int nrk, float dt, float dttmp,
                 float *ua, float *u3d, const float *uten, float *va, float *v3d, const float *vten,
                 float *wa, float *w3d, const float *wten, float *ppi, float *pp3d, const float *piadv,
                 const float *ppten, float *ppx, const float *thv, const float *ppterm,
                 float *rru, float *rrv, float *rrw, float *radbcw, float *radbce, float *radbcs, float *radbcn) {
  (void)dttmp;
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  SoundArgs a;
  a.ua = mkU(g, ua); a.u3d = mkU(g, u3d); a.uten = mkU(g, uten);
  a.va = mkV(g, va); a.v3d = mkV(g, v3d); a.vten = mkV(g, vten);
  a.wa = mkW(g, wa); a.w3d = mkW(g, w3d); a.wten = mkW(g, wten);
  a.ppi = mkS(g, ppi); a.pp3d = mkS(g, pp3d); a.piadv = mkS(g, piadv); a.ppten = mkS(g, ppten);
  a.ppx = mkS(g, ppx); a.thv = mkS(g, thv); a.ppterm = mkS(g, ppterm);
  a.rru = mkU(g, rru); a.rrv = mkV(g, rrv); a.rrw = mkW(g, rrw);
  a.radbcw = radbcw; a.radbce = radbce; a.radbcs = radbcs; a.radbcn = radbcn;
  sound_g(g, &a, nrk, dt);
  return 0;
}

/* calcmass: misclibs.F:3134-3191 */
int oracle_calcmass(const cm1g_config_t *cfg, const cm1g_grid_t *gr, const float *rho, double *tmass) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  F3 r = mkS(g, rho);
  double tm = 0.0;
  for (int k = 1; k <= g->nk; k++) {
    double foo = 0.0;
    for (int j = 1; j <= g->nj; j++) for (int i = 1; i <= g->ni; i++)
      foo = foo + (double)(A3(r, i, j, k) * RUH(i) * RVH(j) * A3(g->rmh, i, j, k));
    tm = tm + foo;
  }
  *tmass = tm * (double)(g->dx * g->dy * g->dz);
  return 0;
}

/* maxmin: maxmin.F:5-119 (first occurrence in i-fastest order wins) */
int oracle_maxmin(const cm1g_config_t *cfg, const float *a, int stag, float *amax, float *amin, int loc[6]) {
  OG G, *g = &G;
  if (og_setup(g, cfg, NULL)) return -1;
  F3 f = stag == 2 ? mkU(g, a) : stag == 3 ? mkV(g, a) : mkS(g, a);
  int ie = g->ni + (stag == 2), je = g->nj + (stag == 3), ke = g->nk + (stag == 4);
  float mx = -1e30f, mn = 1e30f;
  for (int k = 1; k <= ke; k++) for (int j = 1; j <= je; j++) for (int i = 1; i <= ie; i++) {
    float v = A3(f, i, j, k);
    if (v > mx) { mx = v; loc[0] = i; loc[1] = j; loc[2] = k; }
    if (v < mn) { mn = v; loc[3] = i; loc[4] = j; loc[5] = k; }
  }
  *amax = mx; *amin = mn;
  return 0;
}

/* dtsmall: misclibs.F:817-915, the number of small steps per large step.
   psolver 1/4/5 -> 1; 2 and 3 from the grid spacing.  The reference stops
   the model when nsound exceeds 192 without adapt_dt; here that returns -2.
   psolver 6/7 (which need csound) return -1. */
static int nint_d(double x) { return (int)(x >= 0.0 ? floor(x + 0.5) : ceil(x - 0.5)); }
int oracle_dtsmall(int psolver, int nx, int ny, float min_dx, float min_dy, float min_dz, int adapt_dt,
                   float *dt, double *dbldt, int *nsound) {
  const int max_nsound = 192;
  float dtsm;
  if (psolver == 1 || psolver == 4 || psolver == 5) { *nsound = 1; return 0; }
  if (psolver == 2) {
    if (ny == 1) dtsm = 0.60f * fminf(min_dx, min_dz) / 360.0f;
    else if (nx == 1) dtsm = 0.60f * fminf(min_dy, min_dz) / 360.0f;
    else dtsm = 0.50f * fminf(fminf(min_dx, min_dy), min_dz) / 360.0f;
  } else if (psolver == 3) {
    if (ny == 1) dtsm = 0.60f * min_dx / 360.0f;
    else if (nx == 1) dtsm = 0.60f * min_dy / 360.0f;
    else dtsm = 0.60f * fminf(min_dx, min_dy) / 360.0f;
  } else {
    return -1;
  }
  int ns = nint_d(*dbldt / (double)dtsm);
  if (ns < 4) ns = 4;
  if (ns % 2 != 0) ns = ns + 1;
  if (*dbldt / (double)(float)ns > (double)dtsm) ns = ns + 2;
  if (ns > max_nsound) {
    if (adapt_dt != 1) return -2;
    ns = max_nsound;
    *dbldt = (double)((float)ns * dtsm);
    *dt = (float)*dbldt;
  }
  *nsound = ns;
  return 0;
}

/* Pre-RK tendencies of solve1 (solve1.F:414-486): Rayleigh damping of u, v,
   w, theta toward the base state (irdamp=1, or hrdamp=1) or toward the
   horizontal-mean profiles uavg/vavg/thavg (irdamp=2), else zero; the
   moisture and tracer tendencies are zeroed.  tauh/taus are s-arrays, tauf
   a w-array (param.F:8650-8680). */
int oracle_tendency_init(const cm1g_config_t *cfg, const cm1g_grid_t *gr, int irdamp, float rdalpha,
                         const float *tauh, const float *taus, const float *tauf, const float *uavg,
                         const float *vavg, const float *thavg, const float *ua, const float *va, const float *wa,
                         const float *tha, float *uten1, float *vten1, float *wten1, float *thten1, float *qten,
                         float *ptten) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  F3 th = mkS(g, tauh), ts = mkS(g, taus), tf = mkW(g, tauf);
  F3 u = mkU(g, ua), v = mkV(g, va), w = mkW(g, wa), t = mkS(g, tha);
  F3 ut = mkU(g, uten1), vt = mkV(g, vten1), wt = mkW(g, wten1), tt = mkS(g, thten1);
  for (int k = 1; k <= g->nk; k++)
    for (int j = 1; j <= g->nj + 1; j++)
      for (int i = 1; i <= g->ni + 1; i++) {
        if (irdamp == 1) {
          A3(ut, i, j, k) = -(rdalpha * 0.5f * (A3(th, i - 1, j, k) + A3(th, i, j, k)) * (A3(u, i, j, k) - A3(g->u0, i, j, k)));
          A3(vt, i, j, k) = -(rdalpha * 0.5f * (A3(th, i, j - 1, k) + A3(th, i, j, k)) * (A3(v, i, j, k) - A3(g->v0, i, j, k)));
          A3(wt, i, j, k) = -(rdalpha * A3(tf, i, j, k) * A3(w, i, j, k));
          A3(tt, i, j, k) = -(rdalpha * A3(ts, i, j, k) * A3(t, i, j, k));
        } else if (irdamp == 2) {
          A3(ut, i, j, k) = -(rdalpha * 0.5f * (A3(th, i - 1, j, k) + A3(th, i, j, k)) * (A3(u, i, j, k) - uavg[k]));
          A3(vt, i, j, k) = -(rdalpha * 0.5f * (A3(th, i, j - 1, k) + A3(th, i, j, k)) * (A3(v, i, j, k) - vavg[k]));
          A3(wt, i, j, k) = -(rdalpha * A3(tf, i, j, k) * A3(w, i, j, k));
          A3(tt, i, j, k) = -(rdalpha * A3(ts, i, j, k) * ((A3(g->th0, i, j, k) - thavg[k]) + A3(t, i, j, k)));
        } else {
          A3(ut, i, j, k) = 0.0f; A3(vt, i, j, k) = 0.0f; A3(wt, i, j, k) = 0.0f; A3(tt, i, j, k) = 0.0f;
        }
      }
  const int numq = cfg->imoist ? cfg->numq : 0, npt = cfg->iptra ? cfg->npt : 0;
  for (int n = 0; n < numq + npt; n++) {
    F3 q = mkS(g, (n < numq ? qten : ptten) + (long)(n < numq ? n : n - numq) * nS(g));
    for (int k = 1; k <= g->nk; k++) for (int j = 1; j <= g->nj; j++) for (int i = 1; i <= g->ni; i++)
      A3(q, i, j, k) = 0.0f;
  }
  return 0;
}

/* calcener: misclibs.F:3343-3454 (umove = vmove = 0).  Kinetic, internal,
   potential and latent energy and their total, each an FP64 sum over the
   physical cells.  Operands keep the reference's kinds: the per-cell
   factors are binary32 expressions promoted where a binary64 operand meets
   them.  ql, qi, vr may be NULL (zero); qv may be NULL for a dry run. */
int oracle_calcener(const cm1g_config_t *cfg, const cm1g_grid_t *gr, const float *zh, const float *rho,
                    const float *ua, const float *va, const float *wa, const float *ppi, const float *tha,
                    const float *qv, const float *ql, const float *qi, const float *vr, double out[5]) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  const Consts c = g->c;
  const float xlv = cfg->testcase == 4 ? 2.47e6f : cfg->testcase == 5 ? 2.50e6f : 2501000.0f;
  const float xls = 2834000.0f, to = 273.15f;
  /* constants.F:148-159: testcases 4 and 5 take lv1 = xlv */
  const float lv1 = (cfg->testcase == 4 || cfg->testcase == 5) ? xlv : xlv + (c.cpl - c.cpv) * to;
  const float ls1 = xls + (c.cpi - c.cpv) * to;
  F3 z = mkS(g, zh), r = mkS(g, rho), u = mkU(g, ua), v = mkV(g, va), w = mkW(g, wa), p = mkS(g, ppi), t = mkS(g, tha);
  F3 fv = mkS(g, qv), fl = mkS(g, ql), fi = mkS(g, qi), fr = mkS(g, vr);
  double ek = 0.0, ei = 0.0, ep = 0.0, le = 0.0;
  for (int k = 1; k <= g->nk; k++) {
    double f1 = 0.0, f2 = 0.0, f3 = 0.0, f4 = 0.0;
    for (int j = 1; j <= g->nj; j++)
      for (int i = 1; i <= g->ni; i++) {
        const double tem = (double)(RUH(i) * RVH(j) * A3(g->rmh, i, j, k));
        const float u1 = A3(u, i, j, k), u2 = A3(u, i + 1, j, k), v1 = A3(v, i, j, k), v2 = A3(v, i, j + 1, k);
        const float w1 = A3(w, i, j, k), w2 = A3(w, i, j, k + 1);
        const double ww = (double)(0.5f * (w1 + w2));
        const float q_v = qv ? A3(fv, i, j, k) : 0.0f, q_l = ql ? A3(fl, i, j, k) : 0.0f;
        const float q_i = qi ? A3(fi, i, j, k) : 0.0f, v_r = vr ? A3(fr, i, j, k) : 0.0f;
        const double qtot = (double)((q_v + q_l) + q_i);
        const float rr = A3(r, i, j, k);
        const float ke = (0.5f * (u1 * u1 + u2 * u2) + 0.5f * (v1 * v1 + v2 * v2)) + 0.5f * (w1 * w1 + w2 * w2);
        f1 = (f1 + (double)rr * tem * (1.0 + qtot) * 0.5 * (double)ke) +
             (double)(q_l * rr) * tem * 0.5 * ((double)(v_r * v_r) - 2.0 * ww * (double)v_r);
        const double tmp = (double)((A3(g->th0, i, j, k) + A3(t, i, j, k)) * (A3(g->pi0, i, j, k) + A3(p, i, j, k)));
        f2 = f2 + (double)rr * tem * (double)(c.cv + c.cvv * q_v) * tmp;
        f3 = f3 + (double)rr * tem * (1.0 + qtot) * (double)c.g * (double)A3(z, i, j, k);
        f4 = (f4 + (double)rr * tem * (double)q_l * ((double)c.cpl * tmp - (double)lv1)) +
             (double)rr * tem * (double)q_i * ((double)c.cpi * tmp - (double)ls1);
      }
    ek = ek + f1; ei = ei + f2; ep = ep + f3; le = le + f4;
  }
  const double vol = (double)(g->dx * g->dy * g->dz);
  out[0] = ek * vol; out[1] = ei * vol; out[2] = ep * vol; out[3] = le * vol;
  out[4] = ((out[0] + out[1]) + out[2]) + out[3];
  return 0;
}

/* Exposed face-value functions for known-answer tests. */
float oracle_flx5(float s1, float s2, float s3, float s4, float s5) { return flx5(s1, s2, s3, s4, s5); }
float oracle_flx3(float s1, float s2, float s3) { return flx3(s1, s2, s3); }
float oracle_weno5(float s1, float s2, float s3, float s4, float s5, double weps) { return weno5f(s1, s2, s3, s4, s5, weps); }
float oracle_upstrpd(float s1, float s2, float s3, double weps) { return upstrpd(s1, s2, s3, weps); }
int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* Smagorinsky LES (sgsmodel=2), dry, no terrain, periodic laterals    */
/* ------------------------------------------------------------------ */

/* calcnm (dry, turb.F:5458-5477), calcdef (turb.F:4772-4893, 5366-5390),
 * turbsmag (turb.F:3415-3540) with bcw(kmh/kmv, 1) (bc.F:1126-1137 and the
 * periodic fill), gettau (turb.F:4110-4135, 4190-4200) with sfcstress
 * (turb.F:4537-4562) and the top rows (turb.F:4397-4420), then turbu, turbv,
 * turbw (turbtend.F:1101-1104, 1290-1296, 1408-1416; 1860-1866, 2056-2060,
 * 2170-2180; 2510-2515, 2540-2547, 2575-2580) and turbs/turbsz explicit
 * (turbtend.F:66-104, 380-395, 480-545) in solve1's order
 * (solve1.F:1113-1240).  Loops over the same index ranges as the Fortran;
 * binary32 in its evaluation order; logf and powf from the C library. */
int oracle_turbsmag(const cm1g_config_t *cfg, const cm1g_grid_t *gr, float csm, int tconfig, int bcturbs, int bbc,
                    int tbc, const float *cgs, const float *cgt, const float *ua_, const float *va_, const float *wa_,
                    const float *rho_, const float *tha_, const float *pta_, float *uten_, float *vten_, float *wten_,
                    float *thten_, float *ptten_, float *kmh_out, float *kmv_out) {
  OG G, *g = &G;
  if (og_setup(g, cfg, gr)) return -1;
  if (cfg->wbc != 1 || cfg->ebc != 1 || cfg->sbc != 1 || cfg->nbc != 1 || cfg->imoist) return -2;
  const int ni = g->ni, nj = g->nj, nk = g->nk;
  const int npt = cfg->iptra ? cfg->npt : 0;
  const long ns = nS(g), nw = nW(g);
  F3 ua = mkU(g, ua_), va = mkV(g, va_), wa = mkW(g, wa_), rho = mkS(g, rho_), tha = mkS(g, tha_);
  F3 uten = mkU(g, uten_), vten = mkV(g, vten_), wten = mkW(g, wten_);
  float *buf = (float *)calloc((size_t)(7 * ns + 9 * nw), sizeof(float));
  if (!buf) return -3;
  float *p = buf;
  F3 rr = mkS(g, p); p += ns;
  F3 t11 = mkS(g, p); p += ns;
  F3 t22 = mkS(g, p); p += ns;
  F3 t33 = mkS(g, p); p += ns;
  F3 t12 = mkS(g, p); p += ns;
  F3 sadv = mkS(g, p); p += ns;
  F3 dumx = mkS(g, p); p += ns;
  F3 rf = mkW(g, p); p += nw;
  F3 t13 = mkW(g, p); p += nw;
  F3 t23 = mkW(g, p); p += nw;
  F3 nm = mkW(g, p); p += nw;
  F3 defv = mkW(g, p); p += nw;
  F3 defh = mkW(g, p); p += nw;
  F3 kmh = mkW(g, p); p += nw;
  F3 kmv = mkW(g, p); p += nw;
  F3 dumz = mkW(g, p);
  const float rdx = g->rdx, rdy = g->rdy, rdz = g->rdz, grav = g->c.g;
  const float prandtl = 1.0f / 3.00f, prinv = 1.0f / prandtl, dmin = 1.0e-10f;
  /* rr, rf (solve3.F:660-678) */
  for (int k = 2; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    A3(rr, i, j, k) = 1.0f / A3(rho, i, j, k);
    A3(rf, i, j, k) = (A3(g->c1, i, j, k) * A3(rho, i, j, k - 1) + A3(g->c2, i, j, k) * A3(rho, i, j, k));
  }
  for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    A3(rr, i, j, 1) = 1.0f / A3(rho, i, j, 1);
    A3(rf, i, j, 1) = cgs[0] * A3(rho, i, j, 1) + cgs[1] * A3(rho, i, j, 2) + cgs[2] * A3(rho, i, j, 3);
    A3(rf, i, j, nk + 1) = cgt[0] * A3(rho, i, j, nk) + cgt[1] * A3(rho, i, j, nk - 1) + cgt[2] * A3(rho, i, j, nk - 2);
  }
  /* calcnm, imoist = 0 */
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++)
    A3(nm, i, j, k) = logf((A3(g->th0, i, j, k) + A3(tha, i, j, k)) / (A3(g->th0, i, j, k - 1) + A3(tha, i, j, k - 1))) *
                      grav * rdz * A3(g->mf, i, j, k);
  /* calcdef: rho * S_ij */
  for (int k = 1; k <= nk; k++) {
    const float temz = rdz * A3(g->mh, 1, 1, k);
    for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
      A3(t11, i, j, k) = A3(rho, i, j, k) * (A3(ua, i + 1, j, k) - A3(ua, i, j, k)) * rdx * UH(i);
      A3(t22, i, j, k) = A3(rho, i, j, k) * (A3(va, i, j + 1, k) - A3(va, i, j, k)) * rdy * VH(j);
      A3(t33, i, j, k) = A3(rho, i, j, k) * (A3(wa, i, j, k + 1) - A3(wa, i, j, k)) * temz;
      A3(t12, i, j, k) = 0.5f * ((A3(ua, i, j, k) - A3(ua, i, j - 1, k)) * rdy * VF(j) +
                                 (A3(va, i, j, k) - A3(va, i - 1, j, k)) * rdx * UF(i)) * 0.25f *
                         ((A3(rho, i - 1, j - 1, k) + A3(rho, i, j, k)) + (A3(rho, i - 1, j, k) + A3(rho, i, j - 1, k)));
    }
  }
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
    A3(t13, i, j, k) = 0.5f * ((A3(wa, i, j, k) - A3(wa, i - 1, j, k)) * rdx * UF(i) +
                               (A3(ua, i, j, k) - A3(ua, i, j, k - 1)) * rdz * 0.5f * (A3(g->mf, i - 1, j, k) + A3(g->mf, i, j, k))) *
                       0.5f * (A3(rf, i - 1, j, k) + A3(rf, i, j, k));
    A3(t23, i, j, k) = 0.5f * ((A3(wa, i, j, k) - A3(wa, i, j - 1, k)) * rdy * VF(j) +
                               (A3(va, i, j, k) - A3(va, i, j, k - 1)) * rdz * 0.5f * (A3(g->mf, i, j - 1, k) + A3(g->mf, i, j, k))) *
                       0.5f * (A3(rf, i, j - 1, k) + A3(rf, i, j, k));
  }
#define SQ(x) ((x) * (x))
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    const float c1 = A3(g->c1, i, j, k), c2 = A3(g->c2, i, j, k);
    float tmp11 = (c1 * SQ(A3(t11, i, j, k - 1)) + c2 * SQ(A3(t11, i, j, k)));
    float tmp22 = (c1 * SQ(A3(t22, i, j, k - 1)) + c2 * SQ(A3(t22, i, j, k)));
    float tmp33 = (c1 * SQ(A3(t33, i, j, k - 1)) + c2 * SQ(A3(t33, i, j, k)));
    float tmp12 = 0.25f * (c1 * ((SQ(A3(t12, i, j, k - 1)) + SQ(A3(t12, i + 1, j + 1, k - 1))) +
                                 (SQ(A3(t12, i, j + 1, k - 1)) + SQ(A3(t12, i + 1, j, k - 1)))) +
                           c2 * ((SQ(A3(t12, i, j, k)) + SQ(A3(t12, i + 1, j + 1, k))) +
                                 (SQ(A3(t12, i, j + 1, k)) + SQ(A3(t12, i + 1, j, k)))));
    float tmp13 = 0.5f * (SQ(A3(t13, i, j, k)) + SQ(A3(t13, i + 1, j, k)));
    float tmp23 = 0.5f * (SQ(A3(t23, i, j, k)) + SQ(A3(t23, i, j + 1, k)));
    float rrf = 1.0f / SQ(A3(rf, i, j, k));
    A3(defv, i, j, k) = 4.0f * (tmp13 + tmp23) * rrf;
    A3(defh, i, j, k) = (2.0f * ((tmp11 + tmp22) + tmp33) + 4.0f * tmp12) * rrf;
  }
  /* turbsmag */
  for (int j = 1; j <= nj; j++) for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++) {
    const float rmf = 1.0f / A3(g->mf, i, j, k);
    if (tconfig == 1) {
      float grdscl = opowf(((g->dx * RUH(i)) * (g->dy * RVH(j))) * (g->dz * rmf), 0.33333333f);
      A3(kmh, i, j, k) = SQ(csm * grdscl) * sqrtf(fmaxf(A3(defv, i, j, k) + A3(defh, i, j, k) - A3(nm, i, j, k) * prinv, dmin));
      A3(kmv, i, j, k) = A3(kmh, i, j, k);
    } else {
      float lenh = sqrtf((g->dx * RUH(i)) * (g->dy * RVH(j)));
      float grdscl = g->dz * rmf;
      A3(kmh, i, j, k) = SQ(csm * lenh) * sqrtf(fmaxf(A3(defh, i, j, k), dmin));
      A3(kmv, i, j, k) = SQ(csm * grdscl) * sqrtf(fmaxf(A3(defv, i, j, k) - A3(nm, i, j, k) * prinv, dmin));
    }
  }
  /* bcw(kmh, 1), bcw(kmv, 1): periodic fill of the halo ring, zero bottom and top rows */
  F3 km2[2] = {kmh, kmv};
  for (int m = 0; m < 2; m++) {
    F3 K = km2[m];
    for (int k = 2; k <= nk; k++) {
      for (int j = 1; j <= nj; j++) { A3(K, 0, j, k) = A3(K, ni, j, k); A3(K, ni + 1, j, k) = A3(K, 1, j, k); }
      for (int i = 0; i <= ni + 1; i++) { A3(K, i, 0, k) = A3(K, i, nj, k); A3(K, i, nj + 1, k) = A3(K, i, 1, k); }
    }
    for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) { A3(K, i, j, 1) = 0.0f; A3(K, i, j, nk + 1) = 0.0f; }
  }
  /* gettau */
  for (int k = 1; k <= nk; k++) for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) {
    float tem = (A3(kmh, i, j, k) + A3(kmh, i, j, k + 1));
    A3(t11, i, j, k) = A3(t11, i, j, k) * tem;
    A3(t22, i, j, k) = A3(t22, i, j, k) * tem;
    A3(t33, i, j, k) = A3(t33, i, j, k) * tem;
    if (i >= 1 && j >= 1)   /* the Fortran's i=0/j=0 products are never read */
      A3(t12, i, j, k) = A3(t12, i, j, k) * 0.25f *
                         (((A3(kmh, i - 1, j - 1, k) + A3(kmh, i, j, k)) + (A3(kmh, i - 1, j, k) + A3(kmh, i, j - 1, k))) +
                          ((A3(kmh, i - 1, j - 1, k + 1) + A3(kmh, i, j, k + 1)) + (A3(kmh, i - 1, j, k + 1) + A3(kmh, i, j - 1, k + 1))));
  }
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
    A3(t13, i, j, k) = A3(t13, i, j, k) * (A3(kmv, i - 1, j, k) + A3(kmv, i, j, k));
    A3(t23, i, j, k) = A3(t23, i, j, k) * (A3(kmv, i, j - 1, k) + A3(kmv, i, j, k));
  }
  for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
    if (bbc == 1) { A3(t13, i, j, 1) = A3(t13, i, j, 2); A3(t23, i, j, 1) = A3(t23, i, j, 2); }
    else {
      A3(t13, i, j, 1) = 2.0f * A3(ua, i, j, 1) * rdz * 0.5f * (A3(g->mf, i - 1, j, 1) + A3(g->mf, i, j, 1)) * 0.5f *
                         (A3(rf, i - 1, j, 1) + A3(rf, i, j, 1)) * 0.5f * (A3(kmv, i - 1, j, 2) + A3(kmv, i, j, 2));
      A3(t23, i, j, 1) = 2.0f * A3(va, i, j, 1) * rdz * 0.5f * (A3(g->mf, i, j - 1, 1) + A3(g->mf, i, j, 1)) * 0.5f *
                         (A3(rf, i, j - 1, 1) + A3(rf, i, j, 1)) * 0.5f * (A3(kmv, i, j - 1, 2) + A3(kmv, i, j, 2));
    }
    if (tbc == 1) { A3(t13, i, j, nk + 1) = A3(t13, i, j, nk); A3(t23, i, j, nk + 1) = A3(t23, i, j, nk); }
    else {
      A3(t13, i, j, nk + 1) = -2.0f * A3(ua, i, j, nk) * rdz * 0.5f * (A3(g->mf, i - 1, j, nk + 1) + A3(g->mf, i, j, nk + 1)) *
                              0.5f * (A3(rf, i - 1, j, nk + 1) + A3(rf, i, j, nk + 1)) * 0.5f *
                              (A3(kmv, i - 1, j, nk) + A3(kmv, i, j, nk));
      A3(t23, i, j, nk + 1) = -2.0f * A3(va, i, j, nk) * rdz * 0.5f * (A3(g->mf, i, j - 1, nk + 1) + A3(g->mf, i, j, nk + 1)) *
                              0.5f * (A3(rf, i, j - 1, nk + 1) + A3(rf, i, j, nk + 1)) * 0.5f *
                              (A3(kmv, i, j - 1, nk) + A3(kmv, i, j, nk));
    }
  }
  /* turbu, turbv, turbw */
  const float tem = rdz * 0.5f;
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni + 1; i++) {
    float tx = (A3(t11, i, j, k) - A3(t11, i - 1, j, k)) * rdx * UF(i);
    float ty = (A3(t12, i, j + 1, k) - A3(t12, i, j, k)) * rdy * VH(j);
    float tz = (A3(t13, i, j, k + 1) - A3(t13, i, j, k)) * tem * (A3(g->mh, i - 1, j, k) + A3(g->mh, i, j, k));
    float rru0 = 1.0f / (0.5f * (A3(rho, i - 1, j, k) + A3(rho, i, j, k)));
    A3(uten, i, j, k) = A3(uten, i, j, k) + ((tx + ty) + tz) * rru0;
  }
  for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni; i++) {
    float tx = (A3(t12, i + 1, j, k) - A3(t12, i, j, k)) * rdx * UH(i);
    float ty = (A3(t22, i, j, k) - A3(t22, i, j - 1, k)) * rdy * VF(j);
    float tz = (A3(t23, i, j, k + 1) - A3(t23, i, j, k)) * tem * (A3(g->mh, i, j - 1, k) + A3(g->mh, i, j, k));
    float rrv0 = 1.0f / (0.5f * (A3(rho, i, j - 1, k) + A3(rho, i, j, k)));
    A3(vten, i, j, k) = A3(vten, i, j, k) + ((tx + ty) + tz) * rrv0;
  }
  for (int k = 2; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
    float tx = (A3(t13, i + 1, j, k) - A3(t13, i, j, k)) * rdx * UH(i);
    float ty = (A3(t23, i, j + 1, k) - A3(t23, i, j, k)) * rdy * VH(j);
    float tz = (A3(t33, i, j, k) - A3(t33, i, j, k - 1)) * rdz * A3(g->mf, i, j, k);
    A3(wten, i, j, k) = A3(wten, i, j, k) + ((tx + ty) + tz) / A3(rf, i, j, k);
  }
  /* turbs: theta (s = th0 - th0r + tha), then each tracer */
  if (thten_) {
    for (int n = -1; n < npt; n++) {
      F3 sten = n < 0 ? mkS(g, thten_) : mkS(g, ptten_ + (long)n * ns);
      if (n < 0) {
        for (int k = 1; k <= nk; k++) {
          float t0 = A3(g->th0, 1, 1, k) - 300.0f;
          for (int j = 0; j <= nj + 1; j++) for (int i = 0; i <= ni + 1; i++) A3(sadv, i, j, k) = t0 + A3(tha, i, j, k);
        }
      } else {
        memcpy(sadv.p, pta_ + (long)n * ns, (size_t)ns * sizeof(float));
      }
      F3 s = sadv;
      for (int k = 1; k <= nk; k++) {
        for (int j = 1; j <= nj + 1; j++) for (int i = 1; i <= ni + 1; i++) {
          A3(dumx, i, j, k) = -0.125f * (A3(rho, i, j, k) + A3(rho, i - 1, j, k)) *
                              ((A3(kmh, i, j, k) * prinv + A3(kmh, i - 1, j, k) * prinv) +
                               (A3(kmh, i, j, k + 1) * prinv + A3(kmh, i - 1, j, k + 1) * prinv)) *
                              (A3(s, i, j, k) - A3(s, i - 1, j, k)) * rdx * UF(i);
          A3(t13, i, j, k) = -0.125f * (A3(rho, i, j, k) + A3(rho, i, j - 1, k)) *    /* t13 reused as dumy */
                             ((A3(kmh, i, j, k) * prinv + A3(kmh, i, j - 1, k) * prinv) +
                              (A3(kmh, i, j, k + 1) * prinv + A3(kmh, i, j - 1, k + 1) * prinv)) *
                             (A3(s, i, j, k) - A3(s, i, j - 1, k)) * rdy * VF(j);
        }
      }
      for (int j = 1; j <= nj; j++) {
        for (int k = 2; k <= nk; k++) for (int i = 1; i <= ni; i++)
          A3(dumz, i, j, k) = -(A3(kmv, i, j, k) * prinv) * (A3(s, i, j, k) - A3(s, i, j, k - 1)) * rdz * A3(g->mf, i, j, k) *
                              A3(rf, i, j, k);
        for (int i = 1; i <= ni; i++) {
          if (bcturbs == 1) { A3(dumz, i, j, 1) = 0.0f; A3(dumz, i, j, nk + 1) = 0.0f; }
          else { A3(dumz, i, j, 1) = A3(dumz, i, j, 2); A3(dumz, i, j, nk + 1) = A3(dumz, i, j, nk); }
        }
      }
      for (int k = 1; k <= nk; k++) for (int j = 1; j <= nj; j++) for (int i = 1; i <= ni; i++) {
        float tx = -(A3(dumx, i + 1, j, k) - A3(dumx, i, j, k)) * rdx * UH(i);
        float ty = -(A3(t13, i, j + 1, k) - A3(t13, i, j, k)) * rdy * VH(j);
        float tz = -(A3(dumz, i, j, k + 1) - A3(dumz, i, j, k)) * rdz * A3(g->mh, i, j, k);
        A3(sten, i, j, k) = A3(sten, i, j, k) + ((tx + ty) + tz) * A3(rr, i, j, k);
      }
    }
  }
#undef SQ
  if (kmh_out) memcpy(kmh_out, kmh.p, (size_t)nw * sizeof(float));
  if (kmv_out) memcpy(kmv_out, kmv.p, (size_t)nw * sizeof(float));
  free(buf);
  return 0;
}
