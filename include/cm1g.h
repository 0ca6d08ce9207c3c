/*
 * cm1g.h -- C-ABI of the B200 dynamical-core large step (libcm1g.so).
 *
 * The library advances CM1's dynamical core (RK3 large step, 5th-order /
 * WENO5 advection, split-explicit acoustic substeps, boundary/halo fills)
 * on one NVIDIA B200 (sm_100a).  Every entry point takes plain pointers
 * and sizes; no C++ or torch types cross this boundary.
 *
 * Array layout: exactly the reference's Fortran layout (column-major, i
 * fastest) with explicit lower bounds:
 *   s-points  (ib:ie,   jb:je,   kb:ke)       ib=1-ngxy, ie=ni+ngxy, kb=0, ke=nk+1
 *   u-points  (ib:ie+1, jb:je,   kb:ke)
 *   v-points  (ib:ie,   jb:je+1, kb:ke)
 *   w-points  (ib:ie,   jb:je,   kb:ke+1)
 *   4-D q/tracer arrays are n consecutive s-point arrays.
 * A pointer may address host or device memory; host arrays are staged
 * through device buffers owned by the context (correct but slow: use device
 * pointers for throughput).
 *
 * Errors: every entry point returns 0 on success and a negative CM1G_ERR_*
 * code otherwise; cm1g_last_error() gives the message.  Nothing here calls
 * exit() or stops the process (the reference calls stopcm1 instead).
 *
 * Threading: one host thread per context; calls are ordered on the
 * context's CUDA stream.  Independent contexts may run concurrently.
 */
#ifndef CM1G_H
#define CM1G_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CM1G_VERSION_MAJOR 0
#define CM1G_VERSION_MINOR 1

#define CM1G_OK              0
#define CM1G_ERR_ARG        -1   /* bad argument / unsupported option          */
#define CM1G_ERR_CUDA       -2   /* CUDA runtime error                          */
#define CM1G_ERR_NOMEM      -3   /* device allocation failed                    */
#define CM1G_ERR_NONFINITE  -4   /* NaN/Inf found by a host-side check          */
#define CM1G_ERR_UNSUPPORTED -5  /* option of the reference not built here      */
#define CM1G_ERR_STATE      -6   /* call out of order (e.g. before cm1g_init)   */

#define CM1G_MAXQ 8

/*
 * Globals of the reference's module `input` (src/input.F:44-300) and
 * `constants` (src/constants.F) that the large step reads.  The
 * ISO_C_BINDING module fills this once after `param` has run.
 */
typedef struct cm1g_config {
  int32_t ni, nj, nk;          /* physical cells (one rank: nx=ni, ny=nj, nz=nk) */
  int32_t ngxy;                /* horizontal halo width; 3 for 5th order / WENO5  */
  float   dx, dy, dz;          /* grid spacing (m)                                */
  int32_t wbc, ebc, sbc, nbc;  /* lateral bc: 1 periodic, 2 open-radiative, 3 free-slip wall */
  int32_t hadvordrs, vadvordrs;/* scalar advection order (5)                      */
  int32_t hadvordrv, vadvordrv;/* momentum advection order (5)                    */
  int32_t advwenos;            /* 0 none, 1 WENO every RK stage, 2 final stage   */
  int32_t advwenov;            /* momentum WENO (0 only)                          */
  int32_t weno_order;          /* 5                                               */
  int32_t nsound;              /* acoustic steps per large step (even)            */
  float   alph;                /* vertically implicit forward weight             */
  float   kdiv;                /* divergence damping coefficient                 */
  int32_t imoist;              /* 0 dry, 1 moist (water vapour only)             */
  int32_t eqtset;              /* 1 or 2 (mass/energy-conserving)                 */
  int32_t numq;                /* number of moisture arrays (1 = qv)              */
  int32_t nqv;                 /* 1-based index of qv                             */
  int32_t iptra;               /* passive tracers on/off                          */
  int32_t npt;                 /* number of passive tracers                       */
  int32_t pdtra;               /* positive-definite tracers                       */
  int32_t apmasscon;           /* dry-air mass conservation fix (psolver 3)       */
  int32_t irbc;                /* open-bc phase speed: 1, 2 Klemp-Wilhelmson, 4 Durran-Klemp */
  float   cstar;               /* open-bc phase speed for irbc=1,2                */
  int32_t roflux;              /* 1: restrict outward flux at open bcs to the inflow */
  float   smeps;               /* flush-to-zero threshold (1e-30)                 */
  int32_t testcase;            /* selects the constants set (0 = CM1 defaults)    */
  int32_t psolver;             /* 3 = Klemp-Wilhelmson split-explicit             */
  int32_t terrain_flag;        /* 0 only                                          */
  int32_t axisymm;             /* 0 only                                          */
  int32_t icor;                /* 0 only                                          */
  float   qmag[CM1G_MAXQ];     /* magnitude of each q (param.F), for WENO eps     */
  int32_t idiff;               /* 1: horizontal diffusion inside advection        */
  int32_t difforder;           /* 6 (the advection-embedded 6th-order form) only  */
  int32_t mdiff;               /* 1: monotonic limiter of the 6th-order fluxes    */
  float   kdiff6;              /* 6th-order coefficient: kdiff6/64/dt per step    */
  int32_t ptype;               /* microphysics: 0 water vapour only (pdefq after  */
                               /* solve2), 1 Kessler (numq=3: qv, qc, qr)         */
  int32_t nql1, nql2;          /* 1-based q indices of the liquid species (0 0:   */
                               /* none; Kessler 2 3), param.F:3169-3175           */
  int32_t efall;               /* energy fallout correction of mp_driver: 0 only  */
  float   tsmall, qsmall;      /* cm1.F:311-319 (1e-4, 1e-14): satadj's           */
                               /* convergence 2*tsmall, pdefq floor of qc, qr     */
} cm1g_config_t;

/*
 * Grid metrics and base state (host pointers, Fortran layout), as passed to
 * the reference's sound / adv* / solve2 subroutines.
 */
typedef struct cm1g_grid {
  const float *uh, *ruh;       /* (ib:ie)     */
  const float *uf, *ruf;       /* (ib:ie+1)   */
  const float *vh, *rvh;       /* (jb:je)     */
  const float *vf, *rvf;       /* (jb:je+1)   */
  const float *mh, *rmh, *c1, *c2;           /* s-points */
  const float *mf, *rmf;                     /* w-points */
  const float *pi0, *rho0, *rr0, *rf0, *rrf0, *th0, *rth0;
  const float *qv0, *qc0, *qi0, *prs0;       /* s-points */
  const float *u0;             /* u-points    */
  const float *v0;             /* v-points    */
  const float *dtu0, *dtv0;    /* (ib:ie,jb:je) */
} cm1g_grid_t;

/*
 * Prognostic state and the pre-RK tendencies of solve1 (the arrays solve2
 * and solve3 read and write).  "a" arrays hold time t, "3d" arrays t+dt.
 */
typedef struct cm1g_state {
  float *ua, *u3d, *uten1;     /* u-points */
  float *va, *v3d, *vten1;     /* v-points */
  float *wa, *w3d, *wten1;     /* w-points */
  float *ppi, *pp3d, *ppx, *ppten;   /* s-points */
  float *tha, *th3d, *thten1;        /* s-points */
  float *rho, *prs;                  /* s-points */
  float *qa, *q3d, *qten;            /* numq s-point arrays */
  float *pta, *pt3d, *ptten;         /* npt  s-point arrays */
  float *radbcw, *radbce;            /* (jb:je,kb:ke) */
  float *radbcs, *radbcn;            /* (ib:ie,kb:ke) */
  float *rain, *prate;               /* (ib:ie,jb:je): accumulated surface rain (cm) and
                                        the surface precipitation rate (ptype=1; nrain=1) */
} cm1g_state_t;

typedef struct cm1g_ctx cm1g_ctx_t;
typedef struct cm1g_ens cm1g_ens_t;

const char *cm1g_last_error(void);
int cm1g_version(int32_t *major, int32_t *minor);

/* Context set-up (replaces the module globals set by param/base,
 * src/param.F:10, src/base.F).  Copies the grid/base state to the device. */
int cm1g_init(const cm1g_config_t *cfg, const cm1g_grid_t *grid, cm1g_ctx_t **ctx);
int cm1g_finalize(cm1g_ctx_t *ctx);
/* Order all work of the context on this cudaStream_t (NULL = legacy stream). */
int cm1g_set_stream(cm1g_ctx_t *ctx, void *stream);
/* Number of kernels this context has launched so far. */
int cm1g_launch_count(cm1g_ctx_t *ctx, int64_t *count);

/* RK3 large step: replaces solve2 (src/solve2.F:77-2097; rkloop 296-2052)
 * for psolver=3, no terrain, no axisymmetry, no Coriolis.  mass1 is the
 * initial dry-air mass (apmasscon); mass2 receives the new one.
 * cflmax receives calccflquick's maximum Courant number (misclibs.F:2726). */
int cm1g_solve2(cm1g_ctx_t *ctx, int32_t nstep, float dt, double mtime,
                double mass1, double *mass2, float *cflmax, cm1g_state_t *st);

/* Positive-definite column fix of one q array: replaces pdefq
 * (src/misclibs.F:1037-1117) with pdscheme=1.  asq accumulates the budget. */
int cm1g_pdefq(cm1g_ctx_t *ctx, float rmax, double *asq, const float *rho, float *q3d);

/* End-of-step boundary fills, ppx update and rollover of the dynamical
 * core: replaces the dycore part of solve3 (src/solve3.F:243-311, 540-640). */
int cm1g_solve3(cm1g_ctx_t *ctx, cm1g_state_t *st);

/* One complete large step as the reference's time loop runs it
 * (cm1.F:3357 solve2; cm1.F:3414 pdefq for qv-only moisture or mp_driver's
 * Kessler branch for ptype=1; cm1.F:3432 solve3).  With use_graph != 0
 * the step is captured once in a CUDA graph and replayed (device pointers
 * only). */
int cm1g_step(cm1g_ctx_t *ctx, int32_t nstep, float dt, double mtime,
              double mass1, double *mass2, float *cflmax, cm1g_state_t *st,
              int32_t use_graph);

/* Kessler warm-rain microphysics (ptype=1): replaces the Kessler branch of
 * mp_driver (src/mp_driver.F:189-233) that cm1.F:3421-3431 calls between
 * solve2 and solve3: pdefq of qv, qc, qr; rain fall speeds (k_fallout),
 * geterain, fallout (sedimentation, st->rain += rain, st->prate), kessler
 * (autoconversion, accretion, evaporation) and satadj (saturation
 * adjustment, nrk=4), kessler.F:10-558.  cm1g_step runs it itself when
 * ptype=1.  Where satadj does not converge in 100 iterations the reference
 * stops the model; here the call returns CM1G_ERR_NONFINITE.
 * cm1g_mp_budget reads the FP64 budgets the context has accumulated:
 * qbudget(1..7) (tcond, tevac, tauto, taccr, tevar, train, erain, the
 * reference's qbudget entries 1-7) and asq(1..3) of the three pdefq calls;
 * reset != 0 zeroes them afterwards. */
int cm1g_mp_driver(cm1g_ctx_t *ctx, float dt, cm1g_state_t *st);
int cm1g_mp_budget(cm1g_ctx_t *ctx, double qbudget[7], double asq[3], int32_t reset);

/* Lateral boundary fills: replace bcs, bcp, bcu, bcv, bcw
 * (src/bc.F:180, 372, 528, 722, 942).  flag as in bcw (1: w=0 top/bottom). */
int cm1g_bcs(cm1g_ctx_t *ctx, float *s);
int cm1g_bcp(cm1g_ctx_t *ctx, float *p);
int cm1g_bcu(cm1g_ctx_t *ctx, float *u);
int cm1g_bcv(cm1g_ctx_t *ctx, float *v);
int cm1g_bcw(cm1g_ctx_t *ctx, float *w, int32_t flag);

/* Scalar advection tendency: replaces advs (src/adv.F:14-903) for
 * hadvorder=vadvorder=5 / WENO5, no budgets, and diffit=0 (the 6th-order
 * diffusion of idiff=1 runs inside cm1g_solve2 / cm1g_step only).  Argument
 * meaning follows adv.F:14-19: rru/rrv/rrw are the rho0-weighted fluxes,
 * divx their divergence, s0 the RK base value, s the advected field,
 * sten is incremented by the advective tendency (times rr0).  pdef selects
 * the positive-definite limiter (pdef.F), pdefweno the pdef form of the
 * vertical WENO (adv_routines.F:2359-2433).  All arrays device or host.
 * The arguments kept are those of adv.F:14-19 in their order there (nrk,
 * wflag, ..., divx, rru, rrv, rrw, s0, s, sten, pdef, pdefweno, dt, weps);
 * grid metrics and scratch arrays come from the context. */
int cm1g_advs(cm1g_ctx_t *ctx, int32_t nrk, int32_t wflag,
              const float *divx, const float *rru, const float *rrv, const float *rrw,
              const float *s0, const float *s, float *sten,
              int32_t pdef, int32_t pdefweno, float dt, double weps);

/* Momentum advection tendencies, one routine each: replace advu, advv and
 * advw (src/adv.F:911-912, 1847-1848, 2778-2781) with hadvordrv=vadvordrv=5.
 * The tendency of the routine's component is incremented by the flux-form
 * advection of that component.  The arguments kept are the reference's, in
 * its order (advu: nrk, ..., u3d, uten, ..., v3d, w3d; advv: nrk, ..., v3d,
 * vten, ..., u3d, w3d; advw: nrk, ..., w3d, wten, ..., u3d, v3d).  The mass
 * fluxes rru/rrv/rrw and their divergence divx, which solve2 forms from
 * u3d/v3d/w3d just before these calls (solve2.F:490-628), are formed on the
 * device from the same velocities, so they are not passed.  Advection only:
 * the 6th-order diffusion of idiff=1 (which needs rho and dt) runs inside
 * cm1g_solve2 / cm1g_step. */
int cm1g_advu(cm1g_ctx_t *ctx, int32_t nrk, const float *u3d, float *uten,
              const float *v3d, const float *w3d);
int cm1g_advv(cm1g_ctx_t *ctx, int32_t nrk, const float *v3d, float *vten,
              const float *u3d, const float *w3d);
int cm1g_advw(cm1g_ctx_t *ctx, int32_t nrk, const float *w3d, float *wten,
              const float *u3d, const float *v3d);
/* The three calls of solve2.F:883-893 in one: advu, advv and advw of the
 * same velocities (no single reference routine has this argument list). */
int cm1g_advuvw(cm1g_ctx_t *ctx, int32_t nrk, const float *u3d, const float *v3d,
                const float *w3d, float *uten, float *vten, float *wten);

/* Acoustic substeps of one RK stage: replaces sound (src/sound.F:10-857)
 * with psolver=3.  thv = theta_rho (t11), ppterm (t22), piadv (pi0+pp').
 * On return rru/rrv/rrw hold the small-step-averaged velocities.  The
 * arguments kept are those of sound.F:10-24 in their order there; grid
 * metrics, the base state and the work arrays (dum1..dum4, mm, ppd, fpk, qk,
 * pk1, pk2) come from the context. */
int cm1g_sound(cm1g_ctx_t *ctx, float dt,
               float *radbcw, float *radbce, float *radbcs, float *radbcn,
               float *rru, float *ua, float *u3d, const float *uten,
               float *rrv, float *va, float *v3d, const float *vten,
               float *rrw, float *wa, float *w3d, const float *wten,
               float *ppi, float *pp3d, const float *piadv, const float *ppten, float *ppx,
               const float *thv, const float *ppterm, int32_t nrk, float dttmp);

/* Domain-integrated dry-air mass, FP64 accumulation: replaces calcmass
 * (src/misclibs.F:3134-3191).  tmass = sum(rho*dV). */
int cm1g_calcmass(cm1g_ctx_t *ctx, const float *rho, double *tmass);

/* Energy budget, FP64 accumulation: replaces calcener
 * (src/misclibs.F:3343-3454, argument order of its arrays, umove = vmove = 0).
 * energy receives ek, ei, ep, le and their total et.  zh is the s-level
 * height array; qv, ql, qi, vr may be NULL (zero). */
int cm1g_calcener(cm1g_ctx_t *ctx, const float *zh, const float *rho, const float *ua, const float *va,
                  const float *wa, const float *ppi, const float *tha, const float *qv, const float *ql,
                  const float *qi, const float *vr, double energy[5]);

/* Number of small steps per large step: replaces dtsmall
 * (src/misclibs.F:817-915) with the module values it reads passed in
 * (psolver, nx, ny, min_dx, min_dy, min_dz, adapt_dt).  Host-only, no
 * context.  Where the reference stops the model (nsound > 192 without
 * adapt_dt) it returns CM1G_ERR_ARG; psolver 6/7 return UNSUPPORTED. */
int cm1g_dtsmall(int32_t psolver, int32_t nx, int32_t ny, float min_dx, float min_dy, float min_dz,
                 int32_t adapt_dt, float *dt, double *dbldt, int32_t *nsound);

/* Pre-RK tendencies of solve1 (src/solve1.F:414-486): irdamp 1 damps u, v,
 * w, theta toward the base state (u0/v0 of cm1g_init, as hrdamp=1 does),
 * irdamp 2 toward the horizontal-mean profiles uavg/vavg/thavg(kb:ke), 0
 * zeroes them; qten/ptten are zeroed.  tauh/taus are s-arrays, tauf a
 * w-array (param.F:8650-8680). */
int cm1g_tendency_init(cm1g_ctx_t *ctx, int32_t irdamp, float rdalpha, const float *tauh, const float *taus,
                       const float *tauf, const float *uavg, const float *vavg, const float *thavg,
                       const float *ua, const float *va, const float *wa, const float *tha,
                       float *uten1, float *vten1, float *wten1, float *thten1, float *qten, float *ptten);

/* 2nd-order diffusion with a fixed viscosity kdiff2 (difforder=2): the
 * stress tensor of diff2def (src/diff2.F:743-1221) and the tendencies of
 * diff2u/v/w (idiff >= 1) and diff2s for theta, each q and each tracer
 * (idiff = 1), added to uten1 ... ptten as solve1 does (solve1.F:686-734),
 * with rr = 1/rho and the w-level density rf of solve3.F:660-678 (cgs and cgt
 * the extrapolation weights of rf to the bottom and top w-levels,
 * param.F:9038-9060).  Cartesian grid, no terrain; bbc and tbc 1 (free slip)
 * or 2 (no slip); lateral walls wbc..nbc = 3 (free slip) or 4 (no slip) are
 * honoured.  ua/va/wa are the velocities diff2def is given (u3d, v3d, w3d
 * after solve3); rho, tha, qa, pta need filled halos. */
int cm1g_diff2(cm1g_ctx_t *ctx, float kdiff2, int32_t idiff, int32_t bbc, int32_t tbc, const float cgs[3],
               const float cgt[3], const float *ua, const float *va, const float *wa, const float *rho,
               const float *tha, const float *qa, const float *pta, float *uten1, float *vten1, float *wten1,
               float *thten1, float *qten, float *ptten);

/* Smagorinsky subgrid turbulence of an LES (sgsmodel=2), dry, Cartesian
 * without terrain, periodic lateral boundaries, explicit vertical mixing
 * (doimpl=0): calcnm's dry N^2 and calcdef's deformation (src/turb.F:
 * 1327-1340, 4711-5423, 5432-5480), turbsmag's kmh/kmv for tconfig 1 or 2
 * with a uniform Smagorinsky constant csm (src/turb.F:3375-3621), gettau's
 * stresses with sfcstress's free-slip (bbc=1) or no-slip (bbc=2) bottom and
 * the free-slip/no-slip top (src/turb.F:4059-4582), and the tendencies of
 * turbu/turbv/turbw and turbs for theta and each tracer that solve1 adds to
 * uten1 ... ptten (src/turbtend.F; src/solve1.F:1113-1240), without surface
 * fluxes.  cgs/cgt extrapolate rf to the bottom/top w-levels.  thten1 NULL
 * skips the scalars.  kmh/kmv (w-arrays, may be NULL) receive the eddy
 * viscosities including bcw's zero bottom/top rows and periodic halo.
 * Replaces: the iturb/sgsmodel=2 branch of sfc_and_turb plus the doturb
 * block of solve1 (src/solve1.F:1113). */
int cm1g_turbsmag(cm1g_ctx_t *ctx, float csm, int32_t tconfig, int32_t bcturbs, int32_t bbc, int32_t tbc,
                  const float cgs[3], const float cgt[3], const float *ua, const float *va, const float *wa,
                  const float *rho, const float *tha, const float *qa, const float *pta, float *uten1,
                  float *vten1, float *wten1, float *thten1, float *qten, float *ptten, float *kmh, float *kmv);

/* Domain extrema over the physical cells of an s/u/v/w array: replaces
 * maxmin (src/maxmin.F:5-119).  stag: 1 s, 2 u, 3 v, 4 w.  loc receives
 * 1-based (i,j,k) of the max (loc[0..2]) and of the min (loc[3..5]). */
int cm1g_maxmin(cm1g_ctx_t *ctx, const float *a, int32_t stag,
                float *amax, float *amin, int32_t loc[6]);

/* Statistics package: replaces statpack (src/statpack.F:10-658) for the
 * fields of the dynamical core.  The switches are those of namelist param9
 * after param's checks (src/param.F:6140-6205); the statistics are the
 * reference's, in its order (setup_stat_vars, statpack.F:666-1458).  Not
 * built: adapt_dt's mean time step, stat_rmw (axisymmetric runs), stat_rhi
 * (ice), stat_km/stat_kh (subgrid turbulence), and bbc=3 (surface layer):
 * a non-zero switch for any of them returns CM1G_ERR_UNSUPPORTED (stat_tke
 * adds nothing without turbulence and is accepted).  umove = vmove = 0.
 *   nql1..nql2   1-based q indices of the liquid species (0 0: none);
 *   cloudvar[n]  1: q n+1 counts as cloud for qctop/qcbot;
 *   zh, zf       host arrays (kb:ke) and (kb:ke+1): heights of the s- and
 *                w-levels (sigma and sigmaf without terrain);
 *   maxz         model top; cgs1..cgs3 the surface extrapolation weights
 *                (param.F:9038-9040);
 *   qname        short names of the q arrays ("qv"), budname nbudget names
 *                of 6 characters each (stat_pcn), used by cm1g_stat_name. */
typedef struct cm1g_stat_opts {
  int32_t stat_w, stat_wlevs, stat_u, stat_v, stat_rmw, stat_pipert, stat_prspert, stat_thpert,
          stat_q, stat_tke, stat_km, stat_kh, stat_div, stat_rh, stat_rhi, stat_the, stat_cloud,
          stat_sfcprs, stat_wsp, stat_cfl, stat_vort, stat_tmass, stat_tmois, stat_qmass,
          stat_tenerg, stat_mo, stat_tmf, stat_pcn, stat_qsrc;
  int32_t adapt_dt, bbc, ptype, iice;
  int32_t nql1, nql2;
  int32_t cloudvar[CM1G_MAXQ];
  int32_t nbudget;
  float maxz, cgs1, cgs2, cgs3;
  const float *zh, *zf;
  char qname[CM1G_MAXQ][4];
  const char *budname;
} cm1g_stat_opts_t;

/* Builds the statistics list of opts on the context (once per run, like
 * setup_stat_vars); stat_out receives the number of statistics. */
int cm1g_stat_setup(cm1g_ctx_t *ctx, const cm1g_stat_opts_t *opts, int32_t *stat_out);
/* Name of statistic n (1-based), as setup_stat_vars names it. */
int cm1g_stat_name(cm1g_ctx_t *ctx, int32_t n, char *name, int32_t len);
/* One call of statpack: rstat (host, stat_out floats) receives the
 * statistics, computed on the device with one device-to-host copy of rstat.
 * Fields may be host or device arrays; qa holds numq q arrays and pta npt
 * tracers (NULL when absent); prate (ib:ie,jb:je) may be NULL (zero).
 * qbudget (nbudget), asq and bsq (numq) are copied into their entries when
 * stat_pcn / stat_qsrc are on; dt is the time step calccfl uses. */
int cm1g_statpack(cm1g_ctx_t *ctx, double mtime, float dt, const float *ua, const float *va, const float *wa,
                  const float *ppi, const float *tha, const float *prs, const float *rho, const float *qa,
                  const float *pta, const float *prate, const double *qbudget, const double *asq,
                  const double *bsq, float *rstat);
/* Writes rstat as record nrec (1-based) of the GrADS stats file
 * (cm1out_stats.dat: direct access, record length 4*nstat bytes,
 * statpack.F:620-632). */
int cm1g_stat_write(const char *path, int32_t nrec, const float *rstat, int32_t nstat);

/* Records of output files: field n's physical points as one record per
 * level k1[n]..k2[n], i fastest then j (the GrADS layout of writeout with
 * output_format=1, writeout.F:8901-8995, and the records of restart_write's
 * writer, restart_write.F:2422-2714), the fields one after another.  stag: 1
 * s (a 2-D (ib:ie,jb:je) array is an s-array with k1 = k2 = 0), 2 u, 3 v,
 * 4 w.  The fields leave the device in one gather and one copy; fields and
 * the buffer may be host or device arrays.  cm1g_records_size gives the
 * buffer's length in floats; cm1g_unpack_records is the inverse. */
int cm1g_records_size(cm1g_ctx_t *ctx, int32_t n, const int32_t *stag, const int32_t *k1, const int32_t *k2,
                      int64_t *nvals);
int cm1g_pack_records(cm1g_ctx_t *ctx, int32_t n, const float *const *fields, const int32_t *stag,
                      const int32_t *k1, const int32_t *k2, float *out);
int cm1g_unpack_records(cm1g_ctx_t *ctx, int32_t n, float *const *fields, const int32_t *stag,
                        const int32_t *k1, const int32_t *k2, const float *in);

/* writeout with output_format=1 (writeout.F:20-8752) for the fields this
 * library advances: the switches are writeout's output_* of namelist param6
 * for those fields, the variables follow writeout's order and forms (th =
 * th0+tha, prspert = prs-prs0, pi = (prs/p00)**(rd/cp), pipert = pi-pi0,
 * rhopert = rho-rho0, qvpert = qv-qv0, the other q arrays by qname, upert =
 * ua-u0, vpert = va-v0; rain and prate with ptype=1), gathered on the device
 * and written as time nwrite (1-based) of <prefix>_s.dat, _u.dat, _v.dat and
 * _w.dat (direct access, one record per level of nx*ny points), each with a
 * GrADS descriptor <prefix>_?.ctl (its own layout; not byte-identical to the
 * reference's write_ctl).  prspert needs the grid's prs0 at cm1g_init. */
typedef struct cm1g_writeout_opts {
  int32_t output_rain, output_prate, output_th, output_thpert, output_prs, output_prspert, output_pi,
          output_pipert, output_rho, output_rhopert, output_qv, output_qvpert, output_q, output_u, output_upert,
          output_v, output_vpert, output_w;
  char qname[CM1G_MAXQ][4];
} cm1g_writeout_opts_t;
int cm1g_writeout(cm1g_ctx_t *ctx, const char *prefix, int32_t nwrite, double mtime,
                  const cm1g_writeout_opts_t *opts, const cm1g_state_t *st);

/* Restart of the state the library advances: the dynamical-core part of
 * restart_write / restart_read (restart_write.F:10-2850, restart_read.F).
 * The file holds a header (grid, options, nstep, mtime, dt, dtlast, mass1),
 * a field table, then the fields' records in restart_write's order (rain
 * when ptype=1, rho, prs, ua, va, wa, ppi, tha, ppx, each q, each tracer) and
 * the radiative boundary speeds radbcw/e/s/n per level.  Reading checks the
 * grid and options against the context, fills the halos as the end of a
 * step leaves them and sets u3d, v3d, w3d, pp3d, th3d, q3d, pt3d (when
 * given) equal to the time-t arrays, so that stepping on resumes bit for bit.
 * The tendencies of solve1 and the diagnostics (prate) are not part of it. */
typedef struct cm1g_restart {
  int32_t nstep;
  double mtime;
  float dt, dtlast;
  double mass1;
} cm1g_restart_t;
int cm1g_restart_write(cm1g_ctx_t *ctx, const char *path, const cm1g_restart_t *hdr, const cm1g_state_t *st);
int cm1g_restart_read(cm1g_ctx_t *ctx, const char *path, cm1g_restart_t *hdr, cm1g_state_t *st);

/* Per-kernel device timing, the counterpart of the reference's timestats
 * (src/input.F:359-387, cm1.F:4597-4689).  While enabled, every kernel launch
 * is bracketed by CUDA events (graph replay is bypassed); entries are read
 * back by index until the call returns an error. */
int cm1g_profile(cm1g_ctx_t *ctx, int32_t enable);
int cm1g_profile_read(cm1g_ctx_t *ctx, int32_t index, char *name, int32_t name_len,
                      int64_t *launches, double *total_ms);

/* Ensembles of independent members with uneven grids (no counterpart in the
 * reference, which runs one domain per executable).  Each member is a context
 * from cm1g_init with its own stream; cm1g_ensemble_step advances every member
 * by one large step (solve2 + pdefq + solve3, as cm1g_step), forking the
 * members onto their own streams so that their kernels run concurrently, and
 * with use_graph replays the whole ensemble step as one CUDA graph launch.
 * states, dt, mass1, mass2 and cflmax hold one entry per member; the states
 * must be device arrays.  The ensemble does not own the member contexts. */
int cm1g_ensemble_create(cm1g_ctx_t **members, int32_t n, cm1g_ens_t **ens);
int cm1g_ensemble_step(cm1g_ens_t *ens, cm1g_state_t *states, const float *dt, const double *mass1,
                       double *mass2, float *cflmax, int32_t use_graph);
int cm1g_ensemble_launch_count(cm1g_ens_t *ens, int64_t *kernels_per_step);
int cm1g_ensemble_destroy(cm1g_ens_t *ens);

/* Learned coarse-grid advection closure (no counterpart in the reference).
 * A 7 -> 64 -> 64 -> 6 MLP (ReLU or GELU hidden activation, chosen with
 * cm1g_mlp_set_activation for every later call and launch of the closure
 * kernels; ReLU by default) with BF16 weights and FP32 accumulation
 * predicts the six coefficients (projected to sum to 1) of the face value
 * of theta's horizontal faces from the face's upwind-ordered six-point
 * stencil (normalised) and its Courant number; where the face value leaves
 * the range of the four stencil cells nearest the face, WENO5 is used.  params is an
 * FP32 array of cm1g_mlp_param_count() values: W1[8][64], b1[64],
 * W2[64][64], b2[64], W3[64][8], b3[8].  The building blocks below take
 * device pointers and the caller's stream:
 *   face_features: x[f][8] (6 stencil values, Courant number, 0), mean m[f],
 *     scale d[f], face velocity u[f] of the x-faces (dir 0: (ni+1) x nj x nk)
 *     or y-faces (dir 1: ni x (nj+1) x nk), f = ((k-1)*nfy + j-1)*nfx + i-1;
 *   mlp_forward: y[n][8] outputs before the projection, c[n][6]
 *     coefficients, z1/z2[n][64] pre-activations (each may be NULL);
 *   mlp_backward: grad += d loss / d params from dy = d loss / d y;
 *   closure_loss: *loss += sum_f w (phi_f - target_f)^2, dy of it;
 *   adam: one Adam step on params with grad * grad_scale;
 *   face_phi: phi[f] = m + d sum_k c_k x_k, or NaN outside the range of
 *     stencil cells 2..5 (two on each side of the face) widened by
 *     widen * d on each side (widen = 0: the strict range);
 *   closure_faces: features -> forward -> face_phi in one kernel, the same
 *     phi[f] bit for bit (the form the large step runs).
 * cm1g_closure_set turns the closure on (enable=1) for theta in the
 * context's large step; cm1g_capture_fluxes records theta's final-stage
 * x/y face fluxes and face mass fluxes (u-/v-array layout, device arrays;
 * all NULL stops) for building training targets from fine-grid runs. */
int32_t cm1g_mlp_param_count(void);
/* act 0: ReLU, 1: GELU (z Phi(z)); anything else returns CM1G_ERR_ARG. */
int cm1g_mlp_set_activation(int32_t act);
int32_t cm1g_mlp_get_activation(void);
int cm1g_mlp_forward(const float *params, int32_t n, const float *x, float *y, float *c, float *z1, float *z2,
                     void *stream);
int cm1g_mlp_backward(const float *params, int32_t n, const float *x, const float *z1, const float *z2,
                      const float *dy, float *grad, void *stream);
int cm1g_closure_loss(int32_t n, const float *x, const float *y, const float *m, const float *d,
                      const float *target, const float *w, float *dy, double *loss, void *stream);
int cm1g_adam(int32_t np, float *params, const float *grad, float *m1, float *m2, int32_t step, float lr,
              float grad_scale, void *stream);
int cm1g_face_features(int32_t ni, int32_t nj, int32_t nk, int32_t ngxy, int32_t dir, const float *s,
                       const float *th0, int32_t sadd, const float *vel, float dtdx, float *x, float *m, float *d,
                       float *u, void *stream);
int cm1g_face_phi(int64_t nf, const float *x, const float *c, const float *m, const float *d, float widen,
                  float *phi, void *stream);
int cm1g_closure_faces(int32_t ni, int32_t nj, int32_t nk, int32_t ngxy, int32_t dir, const float *s,
                       const float *th0, int32_t sadd, const float *vel, float dtdx, const float *params,
                       float widen, float *phi, void *stream);
int cm1g_closure_set(cm1g_ctx_t *ctx, const float *params, int32_t enable);
/* Bound of the closure's face values in the large step: the range of the
 * four nearest stencil cells widened by widen * (stencil max - min) on each
 * side (default 0). */
int cm1g_closure_bounds(cm1g_ctx_t *ctx, float widen);
int cm1g_capture_fluxes(cm1g_ctx_t *ctx, float *fx, float *fy, float *rx, float *ry);

/* Largest ni*nj that cm1g_pdefq_noalloc accepts: its scratch array holds one
 * FP64 budget per column, 8 MiB of device memory at this size. */
#define CM1G_PDEFQ_NOALLOC_MAX_COLUMNS (1024 * 1024)

/* Positive-definite column fix without any device allocation.  This entry
 * point has no counterpart in the reference; it exists for host programs
 * that must not allocate device memory after start-up (a memory pool owned
 * by someone else, an embedding that forbids it) and so cannot create a
 * context.  It computes what cm1g_pdefq computes (pdscheme=1), with the
 * reference's pdefq argument list (src/misclibs.F:1037): ruh(ib:ie),
 * rvh(jb:je), rmh/rho/q3d(ib:ie,jb:je,kb:ke), all DEVICE pointers; q3d is
 * updated in place, asq += the column-budget change.  The per-column budget
 * lives in a fixed file-scope device array shared by every call in the
 * process: calls that may overlap on one GPU must be serialized by the
 * caller.  The first call with a given device current looks the array's
 * address up (cudaGetSymbolAddress).  Every call synchronizes `stream` to
 * read asq back, so it cannot be made while that stream is being captured
 * into a CUDA graph.  Any ni x nj up to CM1G_PDEFQ_NOALLOC_MAX_COLUMNS
 * columns is accepted (the columns are spread over a one-dimensional grid);
 * more returns CM1G_ERR_ARG, and a failed launch returns CM1G_ERR_CUDA
 * before asq is touched. */
int cm1g_pdefq_noalloc(const cm1g_config_t *cfg, float rmax, double *asq,
                       const float *ruh, const float *rvh, const float *rmh,
                       const float *rho, float *q3d, void *stream);

/* Launch shapes of the large step.  This has no counterpart in the
 * reference (its loops have no launch shapes).  adv_shape indexes the
 * tile shapes of the scalar passes (cm1g_scal_tile_shape: x and y cells of
 * a tile, levels per block; the block has one more row of threads than the
 * tile has cell rows) and mom_shape those of the momentum pass
 * (cm1g_tile_shape: x and y threads of a block, levels per block);
 * sound_form selects the acoustic kernel: -1 automatic (by the number of
 * columns), 0 tile form with 8 warps over the levels of 32 columns, 1 the
 * same with 4 warps, 2 column sweep with 32 x 4 columns per block, 3 column
 * sweep with 32 x 2.  step_ms is the measured large-step time of the
 * configuration (cm1g_autotune; 0 when not measured). */
typedef struct cm1g_tune {
  int32_t adv_shape, mom_shape, sound_form;
  float step_ms;
} cm1g_tune_t;

/* shape[0..2] = x threads, y threads, levels per block of tile shape
 * `index`; CM1G_ERR_ARG past the end of the table. */
int cm1g_tile_shape(int32_t index, int32_t shape[3]);
/* shape[0..2] = x cells, y cells, levels per block of scalar tile shape
 * `index`; CM1G_ERR_ARG past the end of the table. */
int cm1g_scal_tile_shape(int32_t index, int32_t shape[3]);
int cm1g_set_tune(cm1g_ctx_t *ctx, const cm1g_tune_t *tune);
int cm1g_get_tune(cm1g_ctx_t *ctx, cm1g_tune_t *tune);

/* Autotuner: times the candidate launch shapes of this grid on a scratch
 * copy of st (st itself is left unchanged; device or host pointers), each
 * as `reps` replays of the captured large step after one untimed replay,
 * one choice at a time (acoustic form, then scalar tile, then momentum
 * tile), and keeps the fastest on the context.  Results are cached per
 * device, grid shape and configuration: in the process, and, when
 * cache_path is not NULL, in that text file (one line per entry); a cached
 * entry is applied without timing.  out (may be NULL) receives the choice. */
int cm1g_autotune(cm1g_ctx_t *ctx, float dt, double mass1, const cm1g_state_t *st, int32_t reps,
                  const char *cache_path, cm1g_tune_t *out);

#ifdef __cplusplus
}
#endif

#endif /* CM1G_H */
