// cm1g_api.cu -- the C-ABI of libcm1g.so: context, device buffers, host
// staging, the RK3 orchestration of solve2 and the end-of-step solve3 work.
//
// The context holds the grid descriptor, the vertical profiles on the
// device and every scratch array of the large step.  A large step is a fixed
// sequence of kernel launches on the context's stream, so cm1g_step can
// capture it once in a CUDA graph and replay it.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdarg>
#include <cmath>
#include <vector>
#include <algorithm>
#include <string>
#include <map>
#include <mutex>
#include "cm1g_common.cuh"
#include "k_stat.cuh"
#include "k_micro.cuh"
#include "k_diff2.cuh"
#include "k_turb.cuh"
#include "../../include/cm1g.h"

namespace cm1g {
void launch_bc(const DGrid &g, float *a, int which, int wflag, cudaStream_t st, int64_t *nlaunch);
void launch_bc_batch(const DGrid &g, float *const *arrays, const int *which, const int *wflag, int n,
                     cudaStream_t st, int64_t *nlaunch);
void launch_tend_init(const DGrid &g, const TendIn &t, cudaStream_t st, int64_t *nl);
void launch_closure_faces(int ni, int nj, int nk, int ngxy, int dir, const float *s, const float *th0, int sadd,
                          const float *vel, float dtdx, const float *params, float widen, float *phi, cudaStream_t st);
int mlp_param_count();
int ener_chunks(const DGrid &g);
void launch_recip_rho(const DGrid &g, const float *rho, float *rr, cudaStream_t st, int64_t *nl);
long record_count(const DGrid &g, int stag, int k1, int k2);
void launch_pack_records(const DGrid &g, const float *a, int stag, int k1, int k2, float *out, bool unpack,
                         cudaStream_t st, int64_t *nl, int mode = 0, const float *base = nullptr);
void launch_calcener(const DGrid &g, const EnerIn &e, double *part, double *out, cudaStream_t st, int64_t *nl);
void launch_adv_momentum(const DGrid &g, const float *u, const float *v, const float *w, const float *uten1,
                         const float *vten1, const float *wten1, float *uten, float *vten, float *wten,
                         const float *th3d, const float *qv, float *divx, cudaStream_t st, int64_t *nl,
                         const Diff6 *diff = nullptr, const float *b8 = nullptr, int which = 7);
void launch_advs(const DGrid &g, const float *rru, const float *rrv, const float *rrw, int weighted,
                 const float *divx, const float *s, const float *s0, int sadd, const float *ten1,
                 const float *thterm, float *sten_out, float *snew, int weno, int pdef, int pdefweno,
                 double weps, float dt, int flush, float *scratch, cudaStream_t st, int64_t *nl);
void launch_advs_tiled(const DGrid &g, const float *rru, const float *rrv, const float *rrw, const float *s,
                       const float *s0, int sadd, const float *ten1, const float *thterm, float *snew, int weno,
                       int pdef, int pdefweno, double weps, float dt, int flush, float *scratch, cudaStream_t st,
                       int64_t *nl, const TileExtras *ex = nullptr, const Diff6 *diff = nullptr);
void launch_scal_pass(const DGrid &g, const ScalField *f, int n, const float *rru, const float *rrv,
                      const float *rrw, const float *thterm, int weno, float dt, int *err, cudaStream_t st,
                      int64_t *nl);
void launch_sound(const DGrid &g, int nsound, int nrk, float dt, const float *ua, float *u3d, const float *uten,
                  const float *va, float *v3d, const float *vten, const float *wa, float *w3d, const float *wten,
                  const float *ppi, float *pp3d, const float *piadv, const float *ppten, float *ppx,
                  const float *thv, const float *ppterm, float *rru, float *rrv, float *rrw, float *radbcw,
                  float *radbce, float *radbcs, float *radbcn, float *su, float *sv, float *su2,
                  float *sv2, float *d1, float *d2, float *lu, float *rbnd, cudaStream_t st, int64_t *nl);
int sound_max_nk();
void launch_stage_prep(const DGrid &g, const float *th3d, const float *pp3d, const float *qv, const LiquidIn &liq,
                       int imoist, int eqtset, float *t11, float *t22, float *thterm, float *piadv, cudaStream_t st,
                       int64_t *nl);
void launch_radbc4(const DGrid &g, const float *ua, const float *u3d, const float *va, const float *v3d,
                   float *rw, float *re, float *rs, float *rn, float dt, cudaStream_t st, int64_t *nl);
void launch_radbc_kw(const DGrid &g, const float *ua, const float *va, float *rw, float *re, float *rs, float *rn,
                     cudaStream_t st, int64_t *nl);
int prs_nchunk(const DGrid &g);
void launch_prs_rho(const DGrid &g, const float *pp3d, const float *th3d, const float *qv, int imoist,
                    float *prs, float *rho, double *part3, double *part4, int do_sums, cudaStream_t st, int64_t *nl);
void launch_masscon(const DGrid &g, float *pp3d, const float *th3d, const float *qv, int imoist, float *prs,
                    float *rho, const double *part3, const double *part4, double mass1, double *dev, float *devf,
                    cudaStream_t st, int64_t *nl);
void launch_cfl(const DGrid &g, const float *u, const float *v, const float *w, float dt, int *out,
                cudaStream_t st, int64_t *nl);
void launch_pdefq(const DGrid &g, float rmax, const float *rho, float *q, double *bud, double *asq,
                  cudaStream_t st, int64_t *nl);
void launch_ppx_update(const DGrid &g, const float *pp3d, float *ppx, cudaStream_t st, int64_t *nl);
void launch_copy_batch(const DGrid &g, const float *const *src, float *const *dst, const int *stag, const int *ilo,
                       const int *ihi, const int *jlo, const int *jhi, int n, cudaStream_t st, int64_t *nl);
void launch_level_mass(const DGrid &g, const float *rho, double *lev, cudaStream_t st, int64_t *nl);
void launch_maxmin(const DGrid &g, const float *a, int stag, unsigned long long *om, cudaStream_t st, int64_t *nl);
}  // namespace cm1g

using namespace cm1g;

// ---------------------------------------------------------------------
// kernel timing (cm1g_profile)
// ---------------------------------------------------------------------
namespace cm1g {
struct Profile {
  struct Pending { std::string name; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<std::string> names;
  std::vector<int64_t> count;
  std::vector<double> ms;
  void drain() {
    for (auto &p : pending) {
      float t = 0.f;
      cudaEventSynchronize(p.b);
      cudaEventElapsedTime(&t, p.a, p.b);
      size_t i = 0;
      while (i < names.size() && names[i] != p.name) i++;
      if (i == names.size()) { names.push_back(p.name); count.push_back(0); ms.push_back(0.0); }
      count[i] += 1;
      ms[i] += t;
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    pending.clear();
  }
};
thread_local Profile *g_profile = nullptr;
void prof_record(const char *name, cudaStream_t st, bool begin) {
  Profile *p = g_profile;
  if (begin) {
    Profile::Pending e;
    e.name = name;
    cudaEventCreate(&e.a);
    cudaEventCreate(&e.b);
    cudaEventRecord(e.a, st);
    p->pending.push_back(e);
  } else {
    cudaEventRecord(p->pending.back().b, st);
  }
}
}  // namespace cm1g

static thread_local char g_errbuf[512] = "";

static int set_err(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_errbuf, sizeof g_errbuf, fmt, ap);
  va_end(ap);
  return code;
}

int cm1g::report_error(int code, const char *msg) { return set_err(code, "%s", msg); }

#define CUCHK(x)                                                                                   \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_));    \
  } while (0)

struct cm1g_ctx {
  cm1g_config_t cfg;
  DGrid g;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int64_t nlaunch = 0;
  std::vector<void *> allocs;
  // scratch
  float *t11 = nullptr, *t22 = nullptr, *thterm = nullptr, *piadv = nullptr;
  float *uten = nullptr, *vten = nullptr, *wten = nullptr;
  float *rru = nullptr, *rrv = nullptr, *rrw = nullptr;
  float *su = nullptr, *sv = nullptr, *su2 = nullptr, *sv2 = nullptr, *d1 = nullptr, *d2 = nullptr;
  float *lu = nullptr;   // LU factors of the acoustic column sweep
  float *rbnd = nullptr; // roflux = 1: restricted open-boundary u/v of an acoustic step
  float *sx[2 * (1 + 2 * CM1G_MAXQ)] = {};   // per-scalar stage buffers
  float *pdefscr = nullptr;                   // 6 s-arrays
  float *mdivx = nullptr;                     // divx of the momentum pass
  float *rr = nullptr;                        // 1/rho as solve2 keeps it (6th-order diffusion)
  // learned closure of theta's horizontal faces (cm1g_closure_set)
  bool cl_on = false;
  float *cl_params = nullptr;
  float *cl_phi[2] = {};
  float cl_widen = 0.0f;                      // widening of the face-value bounds (cm1g_closure_bounds)
  long cl_nf[2] = {0, 0};
  // capture of theta's final-stage face fluxes (cm1g_capture_fluxes)
  float *cap_fx = nullptr, *cap_fy = nullptr, *cap_rx = nullptr, *cap_ry = nullptr;
  // the scalar fields of a stage in one fused launch (k_scal_tile); off: one
  // k_advs_tile launch per field (CM1G_SCALAR_PASS=perfield, for comparisons)
  bool scal_fused = true;
  double *part3 = nullptr, *part4 = nullptr, *dscal = nullptr, *bud = nullptr, *lev = nullptr;
  double *ener = nullptr;                     // calcener chunk sums (4 x nk x chunks) and results
  float *fscal = nullptr;
  int *cflbits = nullptr;
  unsigned long long *mm = nullptr;
  // host staging (for host-pointer calls)
  cm1g_state_t dst{};
  bool dst_ready = false;
  std::vector<std::pair<float *, size_t>> stage_pool;
  // graph
  cudaGraphExec_t gexec = nullptr;
  cudaGraph_t graph = nullptr;
  cm1g_state_t gstate{};
  float gdt = 0.f;
  double gmass1 = 0.0;
  int64_t graph_nodes = 0;
  uint64_t gen = 0;                           // bumped when launch shapes or the closure change
  float tuned_ms = 0.0f;                      // measured step time of the launch shapes (autotune)
  Profile *prof = nullptr;
  // statistics package (cm1g_stat_setup / cm1g_statpack)
  bool st_ready = false;
  cm1g_stat_opts_t st_opts{};
  std::vector<StatJob> st_jobs;
  std::vector<StatOp> st_ops;
  std::vector<std::string> st_names;
  StatJob *d_st_jobs = nullptr;
  StatOp *d_st_ops = nullptr;
  StatLev *d_st_lev = nullptr;
  float *d_rstat = nullptr, *d_st_zh = nullptr, *d_st_zf = nullptr;
  int st_cap_jobs = 0, st_cap_ops = 0, st_nch = 1;
  // Kessler microphysics (ptype=1)
  float *b8 = nullptr, *vr = nullptr;         // buoyancy of the stage set-up; rain fall speed
  double *mp_part = nullptr, *mp_colbud = nullptr;
  double *mp_qbud = nullptr;                  // qbudget(1..7) and asq(1..3), accumulated on the device
  int *mp_err = nullptr;
  float *d2s = nullptr;                       // scratch of the 2nd-order diffusion (cm1g_diff2)
  float *les = nullptr;                       // scratch of the Smagorinsky LES tendencies (cm1g_turbsmag)
};

// Makes the context's profile (if any) the active one for the calling thread.
struct ProfActive {
  Profile *saved;
  explicit ProfActive(cm1g_ctx *c) : saved(g_profile) { g_profile = c->prof; }
  ~ProfActive() { g_profile = saved; }
};

static void *dalloc(cm1g_ctx *c, size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    c->allocs.push_back(nullptr);   // the failure is found by the check after the allocations
    return nullptr;
  }
  cudaMemset(p, 0, bytes);
  c->allocs.push_back(p);
  return p;
}

static bool is_device_ptr(const void *p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static void set_constants_(int testcase, Consts *c) {
  // constants.F:65-175 (same binary32 arithmetic as the Fortran)
  if (testcase == 4) { c->g = 9.81f; c->rd = 287.0f; c->cp = 1015.0f; c->cpv = 1870.0f; }
  else if (testcase == 5) { c->g = 9.81f; c->rd = 287.0f; c->cp = 1004.0f; c->cpv = 1870.0f; }
  else { c->g = 9.81f; c->rd = 287.04f; c->cp = 1005.7f; c->cpv = 1870.0f; }
  c->rv = 461.5f;
  c->cv = c->cp - c->rd;
  c->cvv = c->cpv - c->rv;
  c->rovcp = c->rd / c->cp;
  c->rddcv = c->rd / c->cv;
  c->cpdrd = c->cp / c->rd;
  c->reps = c->rv / c->rd;
  c->repsm1 = c->rv / c->rd - 1.0f;
  c->cpl = 4190.0f;
  c->cpi = 2106.0f;
}

extern "C" const char *cm1g_last_error(void) { return g_errbuf; }

extern "C" int cm1g_version(int32_t *major, int32_t *minor) {
  if (major) *major = CM1G_VERSION_MAJOR;
  if (minor) *minor = CM1G_VERSION_MINOR;
  return CM1G_OK;
}

static int check_config(const cm1g_config_t *c) {
  if (c->ni < 4 || c->nj < 4 || c->nk < 6) return set_err(CM1G_ERR_ARG, "grid too small (ni,nj>=4, nk>=6)");
  if (c->ngxy < 3) return set_err(CM1G_ERR_ARG, "ngxy must be >= 3 for 5th order");
  // the per-point kernels index rows with a launch grid's y extent
  if (c->nj + 2 * c->ngxy > 65535) return set_err(CM1G_ERR_UNSUPPORTED, "nj > %d rows is not built", 65535 - 2 * c->ngxy);
  // the scalar pass indexes arrays with 32-bit offsets (an array of 2^31
  // points is 8 GiB; the ~40 arrays of a step would not fit in HBM anyway)
  if ((long long)(c->ni + 2 * c->ngxy + 1) * (c->nj + 2 * c->ngxy + 1) * (c->nk + 3) >= (1LL << 31))
    return set_err(CM1G_ERR_UNSUPPORTED, "arrays of 2^31 points or more are not built");
  // levels index a launch grid's y or z extent
  if (c->nk + 2 > 65535) return set_err(CM1G_ERR_UNSUPPORTED, "nk > 65533 levels is not built");
  if (c->psolver != 3) return set_err(CM1G_ERR_UNSUPPORTED, "psolver=%d: only 3 (sound.F) is built", c->psolver);
  if (c->terrain_flag || c->axisymm || c->icor)
    return set_err(CM1G_ERR_UNSUPPORTED, "terrain, axisymmetric grids and Coriolis are not built");
  if (c->hadvordrs != 5 || c->vadvordrs != 5 || c->hadvordrv != 5 || c->vadvordrv != 5)
    return set_err(CM1G_ERR_UNSUPPORTED, "only 5th-order advection is built");
  if (c->advwenov != 0) return set_err(CM1G_ERR_UNSUPPORTED, "momentum WENO is not built");
  if (c->advwenos && c->weno_order != 5) return set_err(CM1G_ERR_UNSUPPORTED, "only WENO5 is built");
  if (c->nsound < 2 || (c->nsound % 2)) return set_err(CM1G_ERR_ARG, "nsound must be even and >= 2");
  if (c->ptype != 0 && c->ptype != 1)
    return set_err(CM1G_ERR_UNSUPPORTED, "microphysics: ptype=%d is not built (0 water vapour, 1 Kessler)", c->ptype);
  if (c->imoist && c->ptype == 0 && (c->numq != 1 || c->nqv != 1))
    return set_err(CM1G_ERR_UNSUPPORTED, "moisture: ptype=0 is water vapour only (numq=1, nqv=1)");
  if (c->ptype == 1) {   // param.F:3169-3175
    if (!c->imoist || c->numq != 3 || c->nqv != 1 || c->nql1 != 2 || c->nql2 != 3)
      return set_err(CM1G_ERR_ARG, "Kessler needs imoist=1, numq=3, nqv=1, nql1=2, nql2=3");
    if (c->efall != 0) return set_err(CM1G_ERR_UNSUPPORTED, "efall=1 is not built");
    if (!(c->tsmall > 0.0f) || !(c->qsmall >= 0.0f)) return set_err(CM1G_ERR_ARG, "tsmall/qsmall not set");
  }
  if (c->iptra && (c->npt < 0 || c->npt > CM1G_MAXQ)) return set_err(CM1G_ERR_ARG, "npt out of range");
  if (c->roflux != 0 && c->roflux != 1) return set_err(CM1G_ERR_ARG, "roflux must be 0 or 1");
  // the per-level flux sums of one acoustic step are held in shared memory
  if (c->roflux == 1 && c->nk > 6000) return set_err(CM1G_ERR_UNSUPPORTED, "roflux=1 with nk > 6000 is not built");
  if (c->idiff != 0 && c->difforder != 6)
    return set_err(CM1G_ERR_UNSUPPORTED, "diffusion: only the 6th-order form (difforder=6) is built");
  if (c->idiff < 0 || c->idiff > 1) return set_err(CM1G_ERR_UNSUPPORTED, "idiff must be 0 or 1");
  if (c->idiff && !(c->kdiff6 >= 0.0f)) return set_err(CM1G_ERR_ARG, "kdiff6 must be >= 0");
  bool open = c->wbc == 2 || c->ebc == 2 || c->sbc == 2 || c->nbc == 2;
  if (open && !(c->irbc == 1 || c->irbc == 2 || c->irbc == 4))
    return set_err(CM1G_ERR_UNSUPPORTED, "open boundaries: irbc=%d is not built (1, 2 and 4 are)", c->irbc);
  for (int b : {c->wbc, c->ebc, c->sbc, c->nbc})
    if (b < 1 || b > 4) return set_err(CM1G_ERR_ARG, "lateral bc must be 1..4");
  if ((c->wbc == 1) != (c->ebc == 1) || (c->sbc == 1) != (c->nbc == 1))
    return set_err(CM1G_ERR_ARG, "periodic bc must be set on both sides");
  return CM1G_OK;
}

// A 3-D base-state array is horizontally uniform without terrain; return its
// (1,1,k) column, after checking the whole array agrees with it.
static bool column_of(const float *a, const DGrid &g, int nkk, std::vector<float> &out) {
  out.resize(nkk);
  long plane = (long)g.NI * g.NJ;
  for (int k = 0; k < nkk; k++) {
    float v = a[iS(g, 1, 1, k)];
    out[k] = v;
    const float *p = a + plane * k;
    for (long t = 0; t < plane; t++)
      if (!(p[t] == v)) return false;
  }
  return true;
}

extern "C" int cm1g_init(const cm1g_config_t *cfg, const cm1g_grid_t *gr, cm1g_ctx_t **out) {
  if (!cfg || !gr || !out) return set_err(CM1G_ERR_ARG, "null argument");
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(CM1G_ERR_CUDA, "no CUDA device: the library has no CPU path");
  cm1g_ctx *c = new cm1g_ctx();
  c->cfg = *cfg;
  cudaGetDevice(&c->device);
  DGrid &g = c->g;
  memset(&g, 0, sizeof g);
  g.ni = cfg->ni; g.nj = cfg->nj; g.nk = cfg->nk; g.ngxy = cfg->ngxy;
  g.ib = 1 - g.ngxy; g.jb = 1 - g.ngxy;
  g.NI = g.ni + 2 * g.ngxy; g.NJ = g.nj + 2 * g.ngxy; g.NK = g.nk + 2;
  g.dx = cfg->dx; g.dy = cfg->dy; g.dz = cfg->dz;
  g.rdx = 1.0f / cfg->dx; g.rdy = 1.0f / cfg->dy; g.rdz = 1.0f / cfg->dz;
  g.wbc = cfg->wbc; g.ebc = cfg->ebc; g.sbc = cfg->sbc; g.nbc = cfg->nbc;
  g.ibw = cfg->wbc != 1; g.ibe = cfg->ebc != 1; g.ibs = cfg->sbc != 1; g.ibn = cfg->nbc != 1;
  g.smeps = cfg->smeps; g.alph = cfg->alph; g.kdiv = cfg->kdiv;
  g.irbc = cfg->irbc; g.cstar = cfg->cstar; g.roflux = cfg->roflux;
  g.tile_adv = 0; g.tile_mom = 0; g.sound_cfg = -1;
  set_constants_(cfg->testcase, &g.c);

  // vertical profiles from the 3-D base state
  struct { const float *src; const float **dst; int nkk; } prof[] = {
      {gr->mh, &g.mh, g.NK}, {gr->rmh, &g.rmh, g.NK}, {gr->mf, &g.mf, g.NK + 1}, {gr->rho0, &g.rho0, g.NK},
      {gr->rr0, &g.rr0, g.NK}, {gr->rf0, &g.rf0, g.NK}, {gr->rrf0, &g.rrf0, g.NK}, {gr->c1, &g.c1, g.NK},
      {gr->c2, &g.c2, g.NK}, {gr->pi0, &g.pi0, g.NK}, {gr->th0, &g.th0, g.NK}, {gr->rth0, &g.rth0, g.NK},
      {gr->qv0, &g.qv0, g.NK}, {gr->qc0, &g.qc0, g.NK}, {gr->qi0, &g.qi0, g.NK}};
  std::vector<float> col;
  for (auto &p : prof) {
    if (!p.src) { cm1g_finalize(c); return set_err(CM1G_ERR_ARG, "grid array missing"); }
    if (!column_of(p.src, g, p.nkk, col)) {
      cm1g_finalize(c);
      return set_err(CM1G_ERR_UNSUPPORTED, "base state/metric varies horizontally (terrain is not built)");
    }
    col.resize(g.NK + 2, col.back());
    float *d = (float *)dalloc(c, col.size() * sizeof(float));
    if (!d) { cm1g_finalize(c); return set_err(CM1G_ERR_NOMEM, "profile alloc"); }
    cudaMemcpy(d, col.data(), col.size() * sizeof(float), cudaMemcpyHostToDevice);
    *p.dst = d;
  }
  if (gr->prs0 && column_of(gr->prs0, g, g.NK, col)) {   // optional: the output's pressure perturbation
    col.resize(g.NK + 2, col.back());
    float *d = (float *)dalloc(c, col.size() * sizeof(float));
    if (!d) { cm1g_finalize(c); return set_err(CM1G_ERR_NOMEM, "profile alloc"); }
    cudaMemcpy(d, col.data(), col.size() * sizeof(float), cudaMemcpyHostToDevice);
    g.prs0 = d;
  }
  struct { const float *src; const float **dst; size_t n; } h1[] = {
      {gr->uh, &g.uh, (size_t)g.NI}, {gr->ruh, &g.ruh, (size_t)g.NI}, {gr->uf, &g.uf, (size_t)g.NI + 1},
      {gr->ruf, &g.ruf, (size_t)g.NI + 1}, {gr->vh, &g.vh, (size_t)g.NJ}, {gr->rvh, &g.rvh, (size_t)g.NJ},
      {gr->vf, &g.vf, (size_t)g.NJ + 1}, {gr->rvf, &g.rvf, (size_t)g.NJ + 1},
      {gr->dtu0, &g.dtu0, (size_t)g.NI * g.NJ}, {gr->dtv0, &g.dtv0, (size_t)g.NI * g.NJ}};
  for (auto &p : h1) {
    if (!p.src) { cm1g_finalize(c); return set_err(CM1G_ERR_ARG, "grid array missing"); }
    float *d = (float *)dalloc(c, (p.n + 4) * sizeof(float));
    if (!d) { cm1g_finalize(c); return set_err(CM1G_ERR_NOMEM, "metric alloc"); }
    cudaMemcpy(d, p.src, p.n * sizeof(float), cudaMemcpyHostToDevice);
    *p.dst = d;
  }
  // scratch arrays
  const size_t bS = nS(g) * sizeof(float), bU = nU(g) * sizeof(float), bV = nV(g) * sizeof(float),
               bW = nW(g) * sizeof(float);
  c->t11 = (float *)dalloc(c, bS); c->t22 = (float *)dalloc(c, bS); c->thterm = (float *)dalloc(c, bS);
  c->piadv = (float *)dalloc(c, bS);
  c->uten = (float *)dalloc(c, bU); c->vten = (float *)dalloc(c, bV); c->wten = (float *)dalloc(c, bW);
  c->rru = (float *)dalloc(c, bU); c->rrv = (float *)dalloc(c, bV); c->rrw = (float *)dalloc(c, bW);
  c->su = (float *)dalloc(c, bU); c->sv = (float *)dalloc(c, bV);
  c->su2 = (float *)dalloc(c, bU); c->sv2 = (float *)dalloc(c, bV);
  c->d1 = (float *)dalloc(c, bS); c->d2 = (float *)dalloc(c, bS);
  c->lu = (float *)dalloc(c, bS);
  if (cfg->roflux == 1)
    c->rbnd = (float *)dalloc(c, (size_t)2 * (g.NJ + g.NI) * g.NK * sizeof(float));
  int nsc = 1 + (cfg->imoist ? cfg->numq : 0) + (cfg->iptra ? cfg->npt : 0);
  for (int s = 0; s < 2 * nsc; s++) c->sx[s] = (float *)dalloc(c, bS);
  bool pdef_needed = cfg->imoist || (cfg->iptra && cfg->pdtra);
  c->pdefscr = (float *)dalloc(c, (pdef_needed ? 6 : 6) * bS);
  c->mdivx = (float *)dalloc(c, bS);
  if (cfg->idiff == 1) c->rr = (float *)dalloc(c, bS);
  c->ener = (double *)dalloc(c, ((size_t)4 * g.nk * ener_chunks(g) + 8) * sizeof(double));
  // base-state winds (full u/v arrays) for the Rayleigh damping of cm1g_tendency_init
  if (gr->u0 && gr->v0) {
    float *du0 = (float *)dalloc(c, bU), *dv0 = (float *)dalloc(c, bV);
    if (du0 && dv0) {
      cudaMemcpy(du0, gr->u0, bU, cudaMemcpyHostToDevice);
      cudaMemcpy(dv0, gr->v0, bV, cudaMemcpyHostToDevice);
      g.u0 = du0; g.v0 = dv0;
    }
  }
  int nchunk = prs_nchunk(g);
  c->part3 = (double *)dalloc(c, (size_t)(g.nk + 2) * nchunk * sizeof(double));
  c->part4 = (double *)dalloc(c, (size_t)(g.nk + 2) * nchunk * sizeof(double));
  c->dscal = (double *)dalloc(c, 16 * sizeof(double));
  c->bud = (double *)dalloc(c, (size_t)g.ni * g.nj * sizeof(double));
  c->lev = (double *)dalloc(c, (size_t)(g.nk + 2) * sizeof(double));
  c->fscal = (float *)dalloc(c, 16 * sizeof(float));
  c->cflbits = (int *)dalloc(c, 16 * sizeof(int));   // [0] max CFL bits, [1] staging-wait error of k_scal_tile
  {
    const char *sp = getenv("CM1G_SCALAR_PASS");
    c->scal_fused = !(sp && strcmp(sp, "perfield") == 0);
  }
  c->mm = (unsigned long long *)dalloc(c, 4 * sizeof(unsigned long long));
  if (cfg->ptype == 1) {
    c->b8 = (float *)dalloc(c, bS);
    c->vr = (float *)dalloc(c, bS);
    c->mp_part = (double *)dalloc(c, (size_t)5 * g.nk * mp_chunks(g) * sizeof(double));
    c->mp_colbud = (double *)dalloc(c, (size_t)2 * g.ni * g.nj * sizeof(double));
    c->mp_qbud = (double *)dalloc(c, 16 * sizeof(double));
    c->mp_err = (int *)dalloc(c, 4 * sizeof(int));
  }
  for (void *p : c->allocs)
    if (!p) { cm1g_finalize(c); return set_err(CM1G_ERR_NOMEM, "scratch alloc"); }
  if (!c->mm) { cm1g_finalize(c); return set_err(CM1G_ERR_NOMEM, "scratch alloc"); }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cm1g_finalize(c);
    return set_err(CM1G_ERR_CUDA, "stream create");
  }
  c->own_stream = true;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { cm1g_finalize(c); return set_err(CM1G_ERR_CUDA, "init: %s", cudaGetErrorString(e)); }
  *out = c;
  return CM1G_OK;
}

static void drop_graph(cm1g_ctx *c) {
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->gexec = nullptr; c->graph = nullptr;
}

extern "C" int cm1g_finalize(cm1g_ctx_t *c) {
  if (!c) return CM1G_OK;
  drop_graph(c);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->prof) { c->prof->drain(); delete c->prof; }
  for (void *p : c->allocs) if (p) cudaFree(p);
  for (void *p : {(void *)c->d_st_jobs, (void *)c->d_st_ops, (void *)c->d_st_lev, (void *)c->d_rstat,
                  (void *)c->d_st_zh, (void *)c->d_st_zf})
    if (p) cudaFree(p);
  for (auto &b : c->stage_pool) cudaFree(b.first);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return CM1G_OK;
}

extern "C" int cm1g_set_stream(cm1g_ctx_t *c, void *stream) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = (cudaStream_t)stream;
  c->own_stream = false;
  drop_graph(c);
  return CM1G_OK;
}

extern "C" int cm1g_launch_count(cm1g_ctx_t *c, int64_t *count) {
  if (!c || !count) return set_err(CM1G_ERR_ARG, "null argument");
  *count = c->nlaunch;
  return CM1G_OK;
}

// ---------------------------------------------------------------------
// Host staging: arrays given as host pointers go through device buffers.
// ---------------------------------------------------------------------
struct Stager {
  cm1g_ctx *c;
  struct Item { float *host; float *dev; size_t n; bool out; };
  std::vector<Item> items;
  size_t pool_i = 0;
  int err = 0;
  explicit Stager(cm1g_ctx *cc) : c(cc) {}
  float *dev_buffer(size_t n) {
    if (pool_i < c->stage_pool.size() && c->stage_pool[pool_i].second >= n) return c->stage_pool[pool_i++].first;
    float *p = nullptr;
    if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) { err = 1; return nullptr; }
    if (pool_i < c->stage_pool.size()) { cudaFree(c->stage_pool[pool_i].first); c->stage_pool[pool_i] = {p, n}; }
    else c->stage_pool.push_back({p, n});
    pool_i++;
    return p;
  }
  // returns a device pointer for p (n floats); copies in; remembers copy-out
  float *in(const float *p, size_t n, bool out) {
    if (!p || n == 0) return const_cast<float *>(p);
    if (is_device_ptr(p)) return const_cast<float *>(p);
    float *d = dev_buffer(n);
    if (!d) return nullptr;
    cudaMemcpyAsync(d, p, n * sizeof(float), cudaMemcpyHostToDevice, c->stream);
    items.push_back({const_cast<float *>(p), d, n, out});
    return d;
  }
  int finish() {
    for (auto &it : items)
      if (it.out) cudaMemcpyAsync(it.host, it.dev, it.n * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
    return err ? set_err(CM1G_ERR_NOMEM, "staging alloc") : CM1G_OK;
  }
};

static int stage_state(cm1g_ctx *c, Stager &S, const cm1g_state_t *st, cm1g_state_t *d) {
  const DGrid &g = c->g;
  size_t ns = nS(g), nu = nU(g), nv = nV(g), nw = nW(g);
  size_t nq = (c->cfg.imoist ? c->cfg.numq : 0) * ns, npt = (c->cfg.iptra ? c->cfg.npt : 0) * ns;
  size_t nrw = (size_t)g.NJ * g.NK, nrs = (size_t)g.NI * g.NK;
  d->ua = S.in(st->ua, nu, true); d->u3d = S.in(st->u3d, nu, true); d->uten1 = S.in(st->uten1, nu, false);
  d->va = S.in(st->va, nv, true); d->v3d = S.in(st->v3d, nv, true); d->vten1 = S.in(st->vten1, nv, false);
  d->wa = S.in(st->wa, nw, true); d->w3d = S.in(st->w3d, nw, true); d->wten1 = S.in(st->wten1, nw, false);
  d->ppi = S.in(st->ppi, ns, true); d->pp3d = S.in(st->pp3d, ns, true); d->ppx = S.in(st->ppx, ns, true);
  d->ppten = S.in(st->ppten, ns, false);
  d->tha = S.in(st->tha, ns, true); d->th3d = S.in(st->th3d, ns, true); d->thten1 = S.in(st->thten1, ns, false);
  d->rho = S.in(st->rho, ns, true); d->prs = S.in(st->prs, ns, true);
  d->qa = S.in(st->qa, nq, true); d->q3d = S.in(st->q3d, nq, true); d->qten = S.in(st->qten, nq, false);
  d->pta = S.in(st->pta, npt, true); d->pt3d = S.in(st->pt3d, npt, true); d->ptten = S.in(st->ptten, npt, false);
  d->radbcw = S.in(st->radbcw, nrw, true); d->radbce = S.in(st->radbce, nrw, true);
  d->radbcs = S.in(st->radbcs, nrs, true); d->radbcn = S.in(st->radbcn, nrs, true);
  if (c->cfg.ptype == 1) {
    d->rain = S.in(st->rain, (size_t)g.NI * g.NJ, true); d->prate = S.in(st->prate, (size_t)g.NI * g.NJ, true);
  } else {
    d->rain = d->prate = nullptr;
  }
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  return CM1G_OK;
}

static int check_state(const cm1g_ctx *c, const cm1g_state_t *st) {
  const float *req[] = {st->ua, st->u3d, st->uten1, st->va, st->v3d, st->vten1, st->wa, st->w3d, st->wten1,
                        st->ppi, st->pp3d, st->ppx, st->ppten, st->tha, st->th3d, st->thten1, st->rho, st->prs,
                        st->radbcw, st->radbce, st->radbcs, st->radbcn};
  for (const float *p : req) if (!p) return set_err(CM1G_ERR_ARG, "state array missing");
  if (c->cfg.imoist && (!st->qa || !st->q3d || !st->qten)) return set_err(CM1G_ERR_ARG, "moisture arrays missing");
  if (c->cfg.ptype == 1 && (!st->rain || !st->prate)) return set_err(CM1G_ERR_ARG, "Kessler needs rain and prate");
  if (c->cfg.iptra && c->cfg.npt > 0 && (!st->pta || !st->pt3d || !st->ptten))
    return set_err(CM1G_ERR_ARG, "tracer arrays missing");
  return CM1G_OK;
}

// ---------------------------------------------------------------------
// solve2 on device arrays (solve2.F:296-2075)
// ---------------------------------------------------------------------
// learned face values of theta's horizontal faces for one RK stage: features
// of every x- and y-face, the MLP, and the bounded face value (NaN: WENO5)
static void closure_phi(cm1g_ctx *c, const float *th, float dt, cudaStream_t st, int64_t *nl) {
  const DGrid &g = c->g;
  for (int dir = 0; dir < 2; dir++) {
    ProfScope _ps("k_closure_faces", st);
    launch_closure_faces(g.ni, g.nj, g.nk, g.ngxy, dir, th, g.th0, 1, dir ? c->rrv : c->rru,
                         dt * (dir ? g.rdy : g.rdx), c->cl_params, c->cl_widen, c->cl_phi[dir], st);
    if (nl) *nl += 1;
  }
}

static void run_solve2(cm1g_ctx *c, const cm1g_state_t *d, float dt, double mass1) {
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  cudaStream_t st = c->stream;
  int64_t *nl = &c->nlaunch;
  const long ns = nS(g);
  const int numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  const bool open = g.ibw || g.ibe || g.ibs || g.ibn;
  const bool openrad = (cf.wbc == 2 || cf.ebc == 2 || cf.sbc == 2 || cf.nbc == 2) && cf.irbc == 4;
  // scalar list: 0 theta, 1..numq moisture, then tracers
  const int nsc = 1 + numq + npt;
  std::vector<const float *> base(nsc), ten1(nsc);
  std::vector<float *> s3d(nsc);
  base[0] = d->tha; s3d[0] = d->th3d; ten1[0] = d->thten1;
  for (int n = 0; n < numq; n++) { base[1 + n] = d->qa + n * ns; s3d[1 + n] = d->q3d + n * ns; ten1[1 + n] = d->qten + n * ns; }
  for (int n = 0; n < npt; n++) { base[1 + numq + n] = d->pta + n * ns; s3d[1 + numq + n] = d->pt3d + n * ns; ten1[1 + numq + n] = d->ptten + n * ns; }
  auto buf_in = [&](int s, int nrk) -> float * { return nrk == 1 ? s3d[s] : c->sx[2 * s + (nrk - 2)]; };
  auto buf_out = [&](int s, int nrk) -> float * { return nrk == 3 ? s3d[s] : c->sx[2 * s + (nrk - 1)]; };
  const int iqv = cf.nqv;  // scalar index of qv
  // 6th-order diffusion (solve2.F:1393, 1475, 1847, 1940): rho at the start of
  // every stage, rr = 1/rho as solve3 left it, updated after stages 1 and 2
  const bool diffit = cf.idiff == 1 && cf.difforder == 6;
  Diff6 df;
  if (diffit) {
    df.rho = d->rho; df.ri = c->rr; df.mdiff = cf.mdiff;
    launch_recip_rho(g, d->rho, c->rr, st, nl);
  }

  // irbc = 1: the open boundaries' phase speeds of the step, from ua/va, as
  // solve1 forms them before solve2 (solve1.F:403-409)
  if (cf.irbc == 1 && open)
    launch_radbc_kw(g, d->ua, d->va, d->radbcw, d->radbce, d->radbcs, d->radbcn, st, nl);
  for (int nrk = 1; nrk <= 3; nrk++) {
    const float dttmp = dt / (float)(3 + 1 - nrk);
    const float *th_in = buf_in(0, nrk);
    const float *qv_in = cf.imoist ? buf_in(iqv, nrk) : nullptr;
    LiquidIn liq;
    if (cf.imoist && cf.nql1 > 0) {   // liquid species of this stage's input (solve2.F:315-345)
      for (int n = cf.nql1; n <= cf.nql2 && liq.n < 2; n++) liq.q[liq.n++] = buf_in(n, nrk);
      liq.b8 = c->b8;
    }
    launch_stage_prep(g, th_in, d->pp3d, qv_in, liq, cf.imoist, cf.eqtset, c->t11, c->t22, c->thterm, c->piadv, st,
                      nl);
    launch_bc(g, c->t11, 2, 0, st, nl);
    if (diffit) df.coef = cf.kdiff6 / 64.0f / dttmp;   // adv.F:80-82, 962-964
    launch_adv_momentum(g, d->u3d, d->v3d, d->w3d, d->uten1, d->vten1, d->wten1, c->uten, c->vten, c->wten,
                        th_in, qv_in, c->mdivx, st, nl, diffit ? &df : nullptr, liq.b8);
    launch_sound(g, cf.nsound, nrk, dt, d->ua, d->u3d, c->uten, d->va, d->v3d, c->vten, d->wa, d->w3d, c->wten,
                 d->ppi, d->pp3d, c->piadv, d->ppten, d->ppx, c->t11, c->t22, c->rru, c->rrv, c->rrw,
                 d->radbcw, d->radbce, d->radbcs, d->radbcn, c->su, c->sv, c->su2, c->sv2, c->d1, c->d2, c->lu, c->rbnd, st, nl);
    if (nrk == 3) launch_cfl(g, d->u3d, d->v3d, d->w3d, dt, c->cflbits, st, nl);
    if (openrad) launch_radbc4(g, d->ua, d->u3d, d->va, d->v3d, d->radbcw, d->radbce, d->radbcs, d->radbcn, dttmp, st, nl);
    const int weno = (cf.advwenos == 1 || (cf.advwenos == 2 && nrk == 3)) ? 1 : 0;
    // Every field whose stage is a plain update (theta; moisture and tracers
    // except at the final stage's positive-definite pass) in one fused launch;
    // the fields are independent given rru/rrv/rrw, so this equals the
    // reference's sequence of advs calls.  The 6th-order diffusion, the
    // learned closure and the flux capture use the per-field tiles below.
    const bool fused = c->scal_fused && !diffit && !c->cl_on && !(nrk == 3 && c->cap_fx);
    std::vector<char> done(nsc, 0);
    if (fused) {
      std::vector<ScalField> fl;
      auto add = [&](int s, int sadd, double weps, int flush, int pdefweno) {
        ScalField f{};
        f.s = buf_in(s, nrk); f.sbase = base[s]; f.ten1 = ten1[s]; f.snew = buf_out(s, nrk);
        f.weps = weps; f.sadd = sadd; f.flush = flush; f.pdefweno = pdefweno;
        fl.push_back(f);
        done[s] = 1;
      };
      add(0, 1, (double)(10.0f * 1.0e-18f), 1, 0);
      for (int n = 0; n < numq; n++)
        if (nrk < 3) add(1 + n, 0, (double)(cf.qmag[n] * 1.0e-18f), 1, (n + 1 == cf.nqv) ? 0 : 1);
      for (int n = 0; n < npt; n++)
        if (!(nrk == 3 && cf.pdtra == 1)) add(1 + numq + n, 0, (double)(1.0f * 1.0e-18f), 0, 1);
      launch_scal_pass(g, fl.data(), (int)fl.size(), c->rru, c->rrv, c->rrw,
                       (cf.imoist && cf.eqtset == 2) ? c->thterm : nullptr, weno, dttmp, c->cflbits + 1, st, nl);
    }
    // theta (solve2.F:1320-1425)
    TileExtras ex;
    const TileExtras *exp = nullptr;
    if (c->cl_on) {
      closure_phi(c, th_in, dt, st, nl);
      ex.phix = c->cl_phi[0]; ex.phiy = c->cl_phi[1]; exp = &ex;
    }
    if (nrk == 3 && c->cap_fx) {
      ex.capfx = c->cap_fx; ex.capfy = c->cap_fy; ex.caprx = c->cap_rx; ex.capry = c->cap_ry; exp = &ex;
    }
    if (!done[0])
      launch_advs_tiled(g, c->rru, c->rrv, c->rrw, th_in, d->tha, 1, d->thten1,
                        (cf.imoist && cf.eqtset == 2) ? c->thterm : nullptr, buf_out(0, nrk), weno, 0, 0,
                        (double)(10.0f * 1.0e-18f), dttmp, 1, c->pdefscr, st, nl, exp, diffit ? &df : nullptr);
    // moisture (solve2.F:1431-1530)
    for (int n = 0; n < numq; n++) {
      const int s = 1 + n;
      if (done[s]) continue;
      launch_advs_tiled(g, c->rru, c->rrv, c->rrw, buf_in(s, nrk), base[s], 0, ten1[s], nullptr, buf_out(s, nrk),
                        weno, nrk == 3 ? 1 : 0, (n + 1 == cf.nqv) ? 0 : 1, (double)(cf.qmag[n] * 1.0e-18f), dttmp, 1,
                        c->pdefscr, st, nl, nullptr, diffit ? &df : nullptr);
    }
    // pressure, density, mass sums (solve2.F:1536-1656; every stage with the
    // 6th-order diffusion, solve2.F:1582, 1599)
    if (nrk == 3 || diffit)
      launch_prs_rho(g, d->pp3d, buf_out(0, nrk), cf.imoist ? buf_out(iqv, nrk) : nullptr, cf.imoist, d->prs, d->rho,
                     c->part3, c->part4, nrk == 3 && cf.apmasscon == 1, st, nl);
    // the tracers below read rho's halo through the diffusion: fill it where
    // the reference does, before them (solve2.F:1681-1684)
    if (diffit && nrk < 3) launch_bc(g, d->rho, 2, 0, st, nl);
    // passive tracers (solve2.F:1880-1970)
    for (int n = 0; n < npt; n++) {
      const int s = 1 + numq + n;
      if (done[s]) continue;
      const int pdef = (nrk == 3 && cf.pdtra == 1) ? 1 : 0;
      launch_advs_tiled(g, c->rru, c->rrv, c->rrw, buf_in(s, nrk), base[s], 0, ten1[s], nullptr, buf_out(s, nrk),
                        weno, pdef, 1, (double)(1.0f * 1.0e-18f), dttmp, 0, c->pdefscr, st, nl, nullptr,
                        diffit ? &df : nullptr);
    }
    if (diffit && nrk < 3) launch_recip_rho(g, d->rho, c->rr, st, nl);   // solve2.F:2036-2046
    // halo fills of the stage (solve2.F:1663-1707 and the tracers' bcs of
    // solve2.F:1959-1961), batched into one two-phase launch: every array is
    // distinct and nothing between their reference positions and here reads
    // their halos
    {
      std::vector<float *> arr{d->u3d, d->v3d, d->w3d};
      std::vector<int> which{3, 4, 5}, flag{0, 0, 1};
      if (nrk < 3) {
        if (!diffit) { arr.push_back(d->rho); which.push_back(2); flag.push_back(0); }
        arr.push_back(d->pp3d); which.push_back(2); flag.push_back(0);
        for (int s = 0; s < nsc; s++) { arr.push_back(buf_out(s, nrk)); which.push_back(1); flag.push_back(0); }
      }
      launch_bc_batch(g, arr.data(), which.data(), flag.data(), (int)arr.size(), st, nl);
    }
    // dry-air mass fix (solve2.F:1976-2033)
    if (nrk == 3 && cf.apmasscon == 1)
      launch_masscon(g, d->pp3d, buf_out(0, 3), cf.imoist ? buf_out(iqv, 3) : nullptr, cf.imoist, d->prs, d->rho,
                     c->part3, c->part4, mass1, c->dscal, c->fscal, st, nl);
  }
  // tracers after the RK loop (solve2.F:2064-2075)
  std::vector<float *> tr;
  for (int n = 0; n < npt; n++) {
    float *pt = d->pt3d + n * ns;
    if (cf.pdtra == 1) launch_pdefq(g, 0.0f, d->rho, pt, nullptr, nullptr, st, nl);
    tr.push_back(pt);
  }
  if (npt) {
    std::vector<int> which(npt, 1);
    launch_bc_batch(g, tr.data(), which.data(), nullptr, npt, st, nl);
  }
  (void)open;
}

static void run_solve3(cm1g_ctx *c, const cm1g_state_t *d) {
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  cudaStream_t st = c->stream;
  int64_t *nl = &c->nlaunch;
  const long ns = nS(g);
  const int numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  const int ni = g.ni, nj = g.nj;
  // solve3.F:246-311
  {
    std::vector<float *> arr{d->pp3d, d->th3d, d->rho};
    std::vector<int> which{2, 1, 2};
    for (int n = 0; n < numq; n++) { arr.push_back(d->q3d + n * ns); which.push_back(1); }
    launch_bc_batch(g, arr.data(), which.data(), nullptr, (int)arr.size(), st, nl);
  }
  launch_ppx_update(g, d->pp3d, d->ppx, st, nl);
  launch_bc(g, d->ppx, 2, 0, st, nl);
  // solve3.F:546-640 rollover
  {
    std::vector<const float *> src;
    std::vector<float *> dst;
    std::vector<int> stag, ihi, jhi;
    auto add = [&](const float *a, float *b, int sg, int ih, int jh) {
      src.push_back(a); dst.push_back(b); stag.push_back(sg); ihi.push_back(ih); jhi.push_back(jh);
    };
    add(d->u3d, d->ua, 2, ni + 2, nj + 2);
    add(d->v3d, d->va, 3, ni + 2, nj + 2);
    add(d->w3d, d->wa, 4, ni + 2, nj + 2);
    for (int n = 0; n < npt; n++) add(d->pt3d + n * ns, d->pta + n * ns, 1, ni + 1, nj + 1);
    add(d->pp3d, d->ppi, 1, ni + 1, nj + 1);
    add(d->th3d, d->tha, 1, ni + 1, nj + 1);
    for (int n = 0; n < numq; n++) add(d->q3d + n * ns, d->qa + n * ns, 1, ni + 1, nj + 1);
    std::vector<int> lo(src.size(), 0);
    launch_copy_batch(g, src.data(), dst.data(), stag.data(), lo.data(), ihi.data(), lo.data(), jhi.data(),
                      (int)src.size(), st, nl);
  }
}

// mp_driver's Kessler branch (mp_driver.F:189-233): pdefq of qv, qc, qr,
// then fall speeds, geterain and fallout (k_mp_fall), kessler and satadj
// (k_mp_point), and the FP64 budgets.
static void run_kessler(cm1g_ctx *c, const cm1g_state_t *d, float dt) {
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const long ns = nS(g);
  float *qv = d->q3d, *qc = d->q3d + ns, *qr = d->q3d + 2 * ns;
  launch_pdefq(g, 0.0f, d->rho, qv, c->bud, c->mp_qbud + 8, c->stream, &c->nlaunch);
  launch_pdefq(g, cf.qsmall, d->rho, qc, c->bud, c->mp_qbud + 9, c->stream, &c->nlaunch);
  launch_pdefq(g, cf.qsmall, d->rho, qr, c->bud, c->mp_qbud + 10, c->stream, &c->nlaunch);
  MicroArgs a{};
  a.th3d = d->th3d; a.pp3d = d->pp3d; a.prs = d->prs; a.rho = d->rho;
  a.qv = qv; a.qc = qc; a.qr = qr; a.vr = c->vr; a.rain = d->rain; a.prate = d->prate; a.err = c->mp_err;
  a.dt = dt; a.converge = 2.0f * cf.tsmall; a.eqtset = cf.eqtset;
  // constants.F:115-159
  const Consts &k = g.c;
  const int tc = cf.testcase;
  const float xlv = tc == 4 ? 2.47e6f : tc == 5 ? 2.50e6f : 2501000.0f, to = 273.15f;
  MicroConsts &m = a.c;
  m.eps = k.rd / k.rv; m.reps = k.reps; m.rd = k.rd; m.rv = k.rv; m.cp = k.cp; m.cv = k.cv; m.cpv = k.cpv;
  m.cvv = k.cvv; m.cpl = k.cpl; m.cpi = k.cpi;
  m.lv1 = (tc == 4 || tc == 5) ? xlv : xlv + (k.cpl - k.cpv) * to;
  m.lv2 = (tc == 4 || tc == 5) ? 0.0f : k.cpl - k.cpv;
  m.cpdcv = k.cp / k.cv; m.rovcp = k.rovcp; m.rddcv = k.rddcv; m.cpdrd = k.cpdrd;
  m.p00 = 1.0e5f; m.rp00 = 1.0f / 1.0e5f;
  launch_kessler(g, a, c->mp_part, c->mp_colbud, c->mp_qbud, c->stream, &c->nlaunch);
}

static void run_step(cm1g_ctx *c, const cm1g_state_t *d, float dt, double mass1) {
  run_solve2(c, d, dt, mass1);
  if (c->cfg.imoist && c->cfg.ptype == 1)   // cm1.F:3421-3431 (mp_driver)
    run_kessler(c, d, dt);
  else if (c->cfg.imoist)                   // cm1.F:3410-3415 (ptype=0)
    launch_pdefq(c->g, 0.0f, d->rho, d->q3d + (long)(c->cfg.nqv - 1) * nS(c->g), nullptr, nullptr, c->stream,
                 &c->nlaunch);
  run_solve3(c, d);
}

static int fetch_scalars(cm1g_ctx *c, double *mass2, float *cflmax) {
  double dv[2];
  int fl[2] = {0, 0};
  CUCHK(cudaMemcpyAsync(dv, c->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUCHK(cudaMemcpyAsync(fl, c->cflbits, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CUCHK(cudaStreamSynchronize(c->stream));
  if (mass2) *mass2 = c->cfg.apmasscon == 1 ? dv[0] : 0.0;
  float f;
  memcpy(&f, &fl[0], 4);
  if (cflmax) *cflmax = f;
  if (fl[1]) {   // a block of the fused scalar pass gave up waiting for its staged planes
    CUCHK(cudaMemsetAsync(c->cflbits + 1, 0, sizeof(int), c->stream));
    return set_err(CM1G_ERR_CUDA, "scalar pass: staged data did not arrive (bulk-copy wait gave up)");
  }
  // the reference stops the model when the step goes unstable (solve2.F:2082);
  // here a non-finite velocity is returned as an error code instead
  if (!std::isfinite(f)) return set_err(CM1G_ERR_NONFINITE, "non-finite velocity after the large step");
  if (c->mp_err) {   // satadj without convergence (kessler.F:412-426 stops the model)
    int err = 0;
    CUCHK(cudaMemcpy(&err, c->mp_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
      cudaMemset(c->mp_err, 0, sizeof(int));
      return set_err(CM1G_ERR_NONFINITE, "satadj: convergence cannot be reached (unstable step?)");
    }
  }
  return CM1G_OK;
}

// One large step as a CUDA graph: captured on first use (and again when the
// state arrays, dt or mass1 change), then replayed with one launch.
static int graph_step(cm1g_ctx *c, const cm1g_state_t *d, float dt, double mass1) {
  bool same = c->gexec && memcmp(&c->gstate, d, sizeof *d) == 0 && c->gdt == dt && c->gmass1 == mass1;
  if (!same) {
    drop_graph(c);
    int64_t before = c->nlaunch;
    CUCHK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    run_step(c, d, dt, mass1);
    cudaGraph_t gr;
    CUCHK(cudaStreamEndCapture(c->stream, &gr));
    c->graph = gr;
    CUCHK(cudaGraphInstantiate(&c->gexec, gr, 0));
    c->graph_nodes = c->nlaunch - before;
    c->nlaunch = before;
    c->gstate = *d; c->gdt = dt; c->gmass1 = mass1;
  }
  CUCHK(cudaGraphLaunch(c->gexec, c->stream));
  c->nlaunch += c->graph_nodes;
  return CM1G_OK;
}

static int solve_common(cm1g_ctx_t *c, float dt, double mass1, double *mass2, float *cflmax, cm1g_state_t *st,
                        int which, int use_graph) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (!st) return set_err(CM1G_ERR_ARG, "null state");
  int rc = check_state(c, st);
  if (rc) return rc;
  if (!(dt > 0.0f) || !std::isfinite(dt)) return set_err(CM1G_ERR_ARG, "dt must be positive");
  if (c->cfg.apmasscon == 1 && !(mass1 > 0.0)) return set_err(CM1G_ERR_ARG, "mass1 must be positive");
  Stager S(c);
  cm1g_state_t d;
  rc = stage_state(c, S, st, &d);
  if (rc) return rc;
  bool all_device = S.items.empty();
  ProfActive pa(c);
  if (use_graph && all_device && which == 3 && !c->prof) {
    rc = graph_step(c, &d, dt, mass1);
    if (rc) return rc;
  } else {
    if (which == 1) run_solve2(c, &d, dt, mass1);
    else if (which == 2) run_solve3(c, &d);
    else if (which == 4) run_kessler(c, &d, dt);
    else run_step(c, &d, dt, mass1);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
  if (which == 4) {   // satadj's convergence flag only
    int err = 0;
    CUCHK(cudaMemcpyAsync(&err, c->mp_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUCHK(cudaStreamSynchronize(c->stream));
    if (err) {
      cudaMemset(c->mp_err, 0, sizeof(int));
      S.finish();
      return set_err(CM1G_ERR_NONFINITE, "satadj: convergence cannot be reached (unstable step?)");
    }
  } else if (which != 2) {
    rc = fetch_scalars(c, mass2, cflmax);
    if (rc) return rc;
  }
  return S.finish();
}

extern "C" int cm1g_solve2(cm1g_ctx_t *c, int32_t nstep, float dt, double mtime, double mass1, double *mass2,
                           float *cflmax, cm1g_state_t *st) {
  (void)nstep; (void)mtime;
  return solve_common(c, dt, mass1, mass2, cflmax, st, 1, 0);
}

extern "C" int cm1g_solve3(cm1g_ctx_t *c, cm1g_state_t *st) {
  return solve_common(c, 1.0f, 1.0, nullptr, nullptr, st, 2, 0);
}

extern "C" int cm1g_mp_driver(cm1g_ctx_t *c, float dt, cm1g_state_t *st) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (c->cfg.ptype != 1 || !c->cfg.imoist) return set_err(CM1G_ERR_ARG, "cm1g_mp_driver needs ptype=1 (Kessler)");
  return solve_common(c, dt, 1.0, nullptr, nullptr, st, 4, 0);
}

extern "C" int cm1g_mp_budget(cm1g_ctx_t *c, double qbudget[7], double asq[3], int32_t reset) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (!c->mp_qbud) return set_err(CM1G_ERR_ARG, "no microphysics budgets (ptype=0)");
  double h[16];
  CUCHK(cudaMemcpyAsync(h, c->mp_qbud, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  CUCHK(cudaStreamSynchronize(c->stream));
  if (qbudget) for (int q = 0; q < 7; q++) qbudget[q] = h[q];
  if (asq) for (int q = 0; q < 3; q++) asq[q] = h[8 + q];
  if (reset) {
    CUCHK(cudaMemsetAsync(c->mp_qbud, 0, 16 * sizeof(double), c->stream));
    CUCHK(cudaStreamSynchronize(c->stream));
  }
  return CM1G_OK;
}

extern "C" int cm1g_step(cm1g_ctx_t *c, int32_t nstep, float dt, double mtime, double mass1, double *mass2,
                         float *cflmax, cm1g_state_t *st, int32_t use_graph) {
  (void)nstep; (void)mtime;
  return solve_common(c, dt, mass1, mass2, cflmax, st, 3, use_graph);
}

// ---------------------------------------------------------------------
// Launch shapes and the autotuner.  The choices live on the context's
// DGrid (tile_adv, tile_mom, sound_cfg) and are read by the launchers when
// a step is enqueued, so a change drops the captured graph.
// ---------------------------------------------------------------------
extern "C" int cm1g_tile_shape(int32_t index, int32_t shape[3]) {
  if (!shape || index < 0 || index >= kNumTileShapes) return set_err(CM1G_ERR_ARG, "no tile shape %d", index);
  for (int q = 0; q < 3; q++) shape[q] = kTileShapes[index][q];
  return CM1G_OK;
}

extern "C" int cm1g_scal_tile_shape(int32_t index, int32_t shape[3]) {
  if (!shape || index < 0 || index >= kNumTileShapes) return set_err(CM1G_ERR_ARG, "no tile shape %d", index);
  for (int q = 0; q < 3; q++) shape[q] = kScalShapes[index][q];
  return CM1G_OK;
}

static int apply_tune(cm1g_ctx *c, const cm1g_tune_t *t) {
  if (t->adv_shape < 0 || t->adv_shape >= kNumTileShapes || t->mom_shape < 0 || t->mom_shape >= kNumTileShapes ||
      t->sound_form < -1 || t->sound_form >= kNumSoundCfgs)
    return set_err(CM1G_ERR_ARG, "launch shape out of range (%d %d %d)", t->adv_shape, t->mom_shape, t->sound_form);
  if (c->g.tile_adv != t->adv_shape || c->g.tile_mom != t->mom_shape || c->g.sound_cfg != t->sound_form) {
    drop_graph(c);
    c->gen++;
  }
  c->g.tile_adv = t->adv_shape; c->g.tile_mom = t->mom_shape; c->g.sound_cfg = t->sound_form;
  return CM1G_OK;
}

extern "C" int cm1g_set_tune(cm1g_ctx_t *c, const cm1g_tune_t *t) {
  if (!c || !t) return set_err(CM1G_ERR_ARG, "null argument");
  int rc = apply_tune(c, t);
  if (rc == CM1G_OK) c->tuned_ms = t->step_ms;
  return rc;
}

extern "C" int cm1g_get_tune(cm1g_ctx_t *c, cm1g_tune_t *t) {
  if (!c || !t) return set_err(CM1G_ERR_ARG, "null argument");
  t->adv_shape = c->g.tile_adv; t->mom_shape = c->g.tile_mom; t->sound_form = c->g.sound_cfg;
  t->step_ms = c->tuned_ms;
  return CM1G_OK;
}

// The cache key: device, grid shape and the options that change which
// kernels run (no spaces, so that a cache file line splits on blanks).
static std::string tune_key(const cm1g_ctx *c) {
  cudaDeviceProp prop;
  char name[256] = "gpu";
  int sms = 0;
  if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess) {
    snprintf(name, sizeof name, "%s", prop.name);
    sms = prop.multiProcessorCount;
  } else {
    cudaGetLastError();
  }
  for (char *p = name; *p; p++) if (*p == ' ' || *p == '\t') *p = '_';
  const cm1g_config_t &f = c->cfg;
  char key[512];
  snprintf(key, sizeof key, "%s/sm%d/%dx%dx%d/h%d/q%d/t%d/w%d/pd%d/ns%d/bc%d%d%d%d", name,
           sms, f.ni, f.nj, f.nk, f.ngxy, f.imoist ? f.numq : 0,
           f.iptra ? f.npt : 0, f.advwenos, f.pdtra, f.nsound, f.wbc, f.ebc, f.sbc, f.nbc);
  return key;
}

static std::mutex g_tune_mu;
static std::map<std::string, cm1g_tune_t> g_tune_cache;

static bool tune_file_lookup(const char *path, const std::string &key, cm1g_tune_t *t) {
  FILE *f = fopen(path, "r");
  if (!f) return false;
  char line[1024], k[600];
  bool hit = false;
  while (fgets(line, sizeof line, f)) {
    cm1g_tune_t e{};
    if (sscanf(line, "%599s %d %d %d %f", k, &e.adv_shape, &e.mom_shape, &e.sound_form, &e.step_ms) == 5 &&
        key == k) {
      *t = e;          // the last entry of a key wins
      hit = true;
    }
  }
  fclose(f);
  return hit;
}

static void tune_file_append(const char *path, const std::string &key, const cm1g_tune_t &t) {
  FILE *f = fopen(path, "a");
  if (!f) return;
  fprintf(f, "%s %d %d %d %.6f\n", key.c_str(), t.adv_shape, t.mom_shape, t.sound_form, t.step_ms);
  fclose(f);
}

// Average time of `reps` graph replays of the large step on d with the
// context's current launch shapes (after one untimed replay).
static int time_steps(cm1g_ctx *c, const cm1g_state_t *d, float dt, double mass1, int reps, float *ms) {
  drop_graph(c);
  int rc = graph_step(c, d, dt, mass1);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  CUCHK(cudaEventCreate(&e0));
  CUCHK(cudaEventCreate(&e1));
  cudaEventRecord(e0, c->stream);
  for (int r = 0; r < reps; r++) {
    cudaGraphLaunch(c->gexec, c->stream);
    c->nlaunch += c->graph_nodes;
  }
  cudaEventRecord(e1, c->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "autotune timing: %s", cudaGetErrorString(e));
  *ms = t / (float)reps;
  return CM1G_OK;
}

extern "C" int cm1g_autotune(cm1g_ctx_t *c, float dt, double mass1, const cm1g_state_t *st, int32_t reps,
                             const char *cache_path, cm1g_tune_t *out) {
  if (!c || !st) return set_err(CM1G_ERR_ARG, "null argument");
  int rc = check_state(c, st);
  if (rc) return rc;
  if (!(dt > 0.0f) || !std::isfinite(dt)) return set_err(CM1G_ERR_ARG, "dt must be positive");
  if (c->cfg.apmasscon == 1 && !(mass1 > 0.0)) return set_err(CM1G_ERR_ARG, "mass1 must be positive");
  if (reps < 1) return set_err(CM1G_ERR_ARG, "reps must be at least 1");
  const std::string key = tune_key(c);
  cm1g_tune_t best{};
  bool hit = false;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) { best = it->second; hit = true; }
  }
  if (!hit && cache_path) hit = tune_file_lookup(cache_path, key, &best);
  if (hit) {
    rc = apply_tune(c, &best);
    if (rc) return rc;
    c->tuned_ms = best.step_ms;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = best;
    if (out) *out = best;
    return CM1G_OK;
  }

  // scratch copy of the state (device or host source), so that the timed
  // steps leave the caller's arrays as they were
  const DGrid &g = c->g;
  const size_t ns = nS(g), nu = nU(g), nv = nV(g), nw = nW(g);
  const size_t nq = (c->cfg.imoist ? c->cfg.numq : 0) * ns, npt = (c->cfg.iptra ? c->cfg.npt : 0) * ns;
  const size_t nrw = (size_t)g.NJ * g.NK, nrs = (size_t)g.NI * g.NK;
  cm1g_state_t d = *st;
  struct F { float **dst; size_t n; } fields[] = {
      {&d.ua, nu}, {&d.u3d, nu}, {&d.uten1, nu}, {&d.va, nv}, {&d.v3d, nv}, {&d.vten1, nv},
      {&d.wa, nw}, {&d.w3d, nw}, {&d.wten1, nw}, {&d.ppi, ns}, {&d.pp3d, ns}, {&d.ppx, ns}, {&d.ppten, ns},
      {&d.tha, ns}, {&d.th3d, ns}, {&d.thten1, ns}, {&d.rho, ns}, {&d.prs, ns}, {&d.qa, nq}, {&d.q3d, nq},
      {&d.qten, nq}, {&d.pta, npt}, {&d.pt3d, npt}, {&d.ptten, npt}, {&d.radbcw, nrw}, {&d.radbce, nrw},
      {&d.radbcs, nrs}, {&d.radbcn, nrs},
      {&d.rain, c->cfg.ptype == 1 ? (size_t)g.NI * g.NJ : 0}, {&d.prate, c->cfg.ptype == 1 ? (size_t)g.NI * g.NJ : 0}};
  std::vector<void *> scratch;
  auto release = [&]() {
    cudaStreamSynchronize(c->stream);
    for (void *p : scratch) cudaFree(p);
  };
  for (auto &f : fields) {
    if (!*f.dst || f.n == 0) { *f.dst = nullptr; continue; }
    void *p = nullptr;
    if (cudaMalloc(&p, f.n * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      release();
      return set_err(CM1G_ERR_NOMEM, "autotune scratch state");
    }
    scratch.push_back(p);
    if (cudaMemcpyAsync(p, *f.dst, f.n * sizeof(float), cudaMemcpyDefault, c->stream) != cudaSuccess) {
      release();
      return set_err(CM1G_ERR_CUDA, "autotune state copy: %s", cudaGetErrorString(cudaGetLastError()));
    }
    *f.dst = (float *)p;
  }

  const cm1g_tune_t saved{c->g.tile_adv, c->g.tile_mom, c->g.sound_cfg, c->tuned_ms};
  cm1g_tune_t cur{0, 0, -1, 0.0f};
  float best_ms = 0.0f;
  auto trial = [&](const cm1g_tune_t &t, float *ms) -> int {
    int r = apply_tune(c, &t);
    if (r) return r;
    return time_steps(c, &d, dt, mass1, reps, ms);
  };
  // acoustic form first (the largest single kernel), then the scalar tile,
  // then the momentum tile, each with the others held at the best so far
  const int ncand[3] = {kNumSoundCfgs, kNumTileShapes, kNumTileShapes};
  for (int knob = 0; knob < 3 && rc == CM1G_OK; knob++) {
    int best_v = knob == 0 ? 0 : knob == 1 ? cur.adv_shape : cur.mom_shape;
    float knob_best = 0.0f;
    bool have = false;
    for (int v = 0; v < ncand[knob] && rc == CM1G_OK; v++) {
      if (knob == 0 && v < 2 && c->g.nk > sound_max_nk()) continue;   // tile forms: too many levels
      cm1g_tune_t t = cur;
      if (knob == 0) t.sound_form = v;
      else if (knob == 1) t.adv_shape = v;
      else t.mom_shape = v;
      float ms = 0.0f;
      rc = trial(t, &ms);
      if (rc == CM1G_OK && (!have || ms < knob_best)) { knob_best = ms; best_v = v; have = true; }
    }
    if (knob == 0) cur.sound_form = best_v;
    else if (knob == 1) cur.adv_shape = best_v;
    else cur.mom_shape = best_v;
    best_ms = knob_best;
  }
  drop_graph(c);
  release();
  if (rc) {
    apply_tune(c, &saved);
    return rc;
  }
  cur.step_ms = best_ms;
  rc = apply_tune(c, &cur);
  if (rc) return rc;
  c->tuned_ms = best_ms;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = cur;
  }
  if (cache_path) tune_file_append(cache_path, key, cur);
  if (out) *out = cur;
  return CM1G_OK;
}

// ---------------------------------------------------------------------
// Ensembles of independent members (uneven grids).  Each member keeps its
// own context and stream; one ensemble step forks from the ensemble's
// stream onto every member's stream, runs each member's large step there,
// and joins back, so the members' kernels run side by side and the small
// grids fill the GPU together.  With use_graph the whole fork/join is
// captured once into one CUDA graph (cached on the member states, dt and
// mass1) and replayed with a single launch per step.
// ---------------------------------------------------------------------
struct cm1g_ens {
  std::vector<cm1g_ctx *> m;
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<cm1g_state_t> gstate;
  std::vector<float> gdt;
  std::vector<double> gmass1;
  std::vector<uint64_t> ggen;                 // the members' gen at capture
  int64_t graph_nodes = 0;
};

static void ens_drop_graph(cm1g_ens *e) {
  if (e->exec) cudaGraphExecDestroy(e->exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  e->exec = nullptr; e->graph = nullptr;
}

extern "C" int cm1g_ensemble_create(cm1g_ctx_t **members, int32_t n, cm1g_ens_t **out) {
  if (!members || n < 1 || !out) return set_err(CM1G_ERR_ARG, "null argument or empty ensemble");
  int dev0 = members[0] ? members[0]->device : -1;
  for (int q = 0; q < n; q++) {
    if (!members[q]) return set_err(CM1G_ERR_ARG, "member %d is null", q);
    if (members[q]->device != dev0) return set_err(CM1G_ERR_ARG, "members must share one device");
    for (int r = 0; r < q; r++)
      if (members[r] == members[q] || members[r]->stream == members[q]->stream)
        return set_err(CM1G_ERR_ARG, "members %d and %d share a context or stream", r, q);
  }
  cm1g_ens *e = new cm1g_ens();
  e->m.assign(members, members + n);
  e->join.resize(n);
  bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int q = 0; q < n && ok; q++) ok = cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) { cm1g_ensemble_destroy(e); return set_err(CM1G_ERR_CUDA, "ensemble stream/event creation failed"); }
  *out = e;
  return CM1G_OK;
}

extern "C" int cm1g_ensemble_destroy(cm1g_ens_t *e) {
  if (!e) return CM1G_OK;
  if (e->stream) cudaStreamSynchronize(e->stream);
  ens_drop_graph(e);
  for (cudaEvent_t ev : e->join) if (ev) cudaEventDestroy(ev);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
  return CM1G_OK;
}

// fork onto the members' streams, one large step each, join
static void ens_enqueue(cm1g_ens *e, const cm1g_state_t *st, const float *dt, const double *mass1) {
  cudaEventRecord(e->fork, e->stream);
  for (size_t q = 0; q < e->m.size(); q++) {
    cm1g_ctx *c = e->m[q];
    cudaStreamWaitEvent(c->stream, e->fork, 0);
    run_step(c, &st[q], dt[q], mass1[q]);
    cudaEventRecord(e->join[q], c->stream);
    cudaStreamWaitEvent(e->stream, e->join[q], 0);
  }
}

extern "C" int cm1g_ensemble_step(cm1g_ens_t *e, cm1g_state_t *states, const float *dt, const double *mass1,
                                  double *mass2, float *cflmax, int32_t use_graph) {
  if (!e || !states || !dt || !mass1) return set_err(CM1G_ERR_ARG, "null argument");
  const size_t n = e->m.size();
  for (size_t q = 0; q < n; q++) {
    cm1g_ctx *c = e->m[q];
    int rc = check_state(c, &states[q]);
    if (rc) return rc;
    if (!(dt[q] > 0.0f) || !std::isfinite(dt[q])) return set_err(CM1G_ERR_ARG, "member %zu: dt must be positive", q);
    if (c->cfg.apmasscon == 1 && !(mass1[q] > 0.0)) return set_err(CM1G_ERR_ARG, "member %zu: mass1 must be positive", q);
    const float *req[] = {states[q].ua, states[q].u3d, states[q].va, states[q].v3d, states[q].wa, states[q].w3d,
                          states[q].pp3d, states[q].th3d, states[q].rho};
    for (const float *p : req)
      if (p && !is_device_ptr(p)) return set_err(CM1G_ERR_ARG, "member %zu: ensemble states must be device arrays", q);
  }
  if (use_graph) {
    bool same = e->exec && e->gstate.size() == n &&
                memcmp(e->gstate.data(), states, n * sizeof(cm1g_state_t)) == 0 &&
                memcmp(e->gdt.data(), dt, n * sizeof(float)) == 0 && memcmp(e->gmass1.data(), mass1, n * sizeof(double)) == 0;
    for (size_t q = 0; same && q < n; q++) same = e->ggen[q] == e->m[q]->gen;
    if (!same) {
      ens_drop_graph(e);
      int64_t before = 0;
      for (cm1g_ctx *c : e->m) before += c->nlaunch;
      CUCHK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      ens_enqueue(e, states, dt, mass1);
      cudaGraph_t gr;
      CUCHK(cudaStreamEndCapture(e->stream, &gr));
      e->graph = gr;
      CUCHK(cudaGraphInstantiate(&e->exec, gr, 0));
      int64_t after = 0;
      for (cm1g_ctx *c : e->m) after += c->nlaunch;
      e->graph_nodes = after - before;
      e->gstate.assign(states, states + n);
      e->gdt.assign(dt, dt + n);
      e->gmass1.assign(mass1, mass1 + n);
      e->ggen.resize(n);
      for (size_t q = 0; q < n; q++) e->ggen[q] = e->m[q]->gen;
    }
    CUCHK(cudaGraphLaunch(e->exec, e->stream));
  } else {
    ens_enqueue(e, states, dt, mass1);
  }
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) return set_err(CM1G_ERR_CUDA, "ensemble launch: %s", cudaGetErrorString(err));
  // the members' mass sums and CFL maxima, read back in one synchronisation
  std::vector<double> dv(2 * n);
  std::vector<int> bits(2 * n);
  for (size_t q = 0; q < n; q++) {
    CUCHK(cudaMemcpyAsync(&dv[2 * q], e->m[q]->dscal, 2 * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    CUCHK(cudaMemcpyAsync(&bits[2 * q], e->m[q]->cflbits, 2 * sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  }
  CUCHK(cudaStreamSynchronize(e->stream));
  int rc = CM1G_OK;
  for (size_t q = 0; q < n; q++) {
    float f;
    memcpy(&f, &bits[2 * q], 4);
    if (mass2) mass2[q] = e->m[q]->cfg.apmasscon == 1 ? dv[2 * q] : 0.0;
    if (cflmax) cflmax[q] = f;
    if (bits[2 * q + 1] && rc == CM1G_OK) {
      CUCHK(cudaMemsetAsync(e->m[q]->cflbits + 1, 0, sizeof(int), e->stream));
      rc = set_err(CM1G_ERR_CUDA, "member %zu: scalar pass staged data did not arrive (bulk-copy wait gave up)", q);
    }
    if (!std::isfinite(f) && rc == CM1G_OK)
      rc = set_err(CM1G_ERR_NONFINITE, "member %zu: non-finite velocity after the large step", q);
  }
  return rc;
}

extern "C" int cm1g_ensemble_launch_count(cm1g_ens_t *e, int64_t *count) {
  if (!e || !count) return set_err(CM1G_ERR_ARG, "null argument");
  *count = e->graph_nodes;
  return CM1G_OK;
}

extern "C" int cm1g_closure_set(cm1g_ctx_t *c, const float *params, int32_t enable) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  drop_graph(c);
  c->gen++;
  if (!enable) { c->cl_on = false; return CM1G_OK; }
  if (!params) return set_err(CM1G_ERR_ARG, "null parameters");
  const DGrid &g = c->g;
  if (!c->cl_params) {
    c->cl_params = (float *)dalloc(c, (size_t)mlp_param_count() * sizeof(float));
    for (int dir = 0; dir < 2; dir++) {
      const long nf = (long)(dir ? g.ni : g.ni + 1) * (dir ? g.nj + 1 : g.nj) * g.nk;
      c->cl_nf[dir] = nf;
      c->cl_phi[dir] = (float *)dalloc(c, nf * sizeof(float));
      if (!c->cl_phi[dir]) return set_err(CM1G_ERR_NOMEM, "closure buffers");
    }
    if (!c->cl_params) return set_err(CM1G_ERR_NOMEM, "closure parameters");
  }
  CUCHK(cudaMemcpyAsync(c->cl_params, params, (size_t)mlp_param_count() * sizeof(float), cudaMemcpyDefault,
                        c->stream));
  CUCHK(cudaStreamSynchronize(c->stream));
  c->cl_on = true;
  return CM1G_OK;
}

extern "C" int cm1g_closure_bounds(cm1g_ctx_t *c, float widen) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (!(widen >= 0.0f) || !std::isfinite(widen)) return set_err(CM1G_ERR_ARG, "widen must be finite and >= 0");
  if (widen != c->cl_widen) {
    drop_graph(c);
    c->gen++;
  }
  c->cl_widen = widen;
  return CM1G_OK;
}

extern "C" int cm1g_capture_fluxes(cm1g_ctx_t *c, float *fx, float *fy, float *rx, float *ry) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  drop_graph(c);
  c->gen++;
  if (!fx && !fy && !rx && !ry) { c->cap_fx = c->cap_fy = c->cap_rx = c->cap_ry = nullptr; return CM1G_OK; }
  if (!fx || !fy || !rx || !ry) return set_err(CM1G_ERR_ARG, "give all four capture arrays or none");
  for (const float *p : {fx, fy, rx, ry})
    if (!is_device_ptr(p)) return set_err(CM1G_ERR_ARG, "capture arrays must be device arrays");
  c->cap_fx = fx; c->cap_fy = fy; c->cap_rx = rx; c->cap_ry = ry;
  return CM1G_OK;
}

extern "C" int cm1g_pdefq(cm1g_ctx_t *c, float rmax, double *asq, const float *rho, float *q3d) {
  if (!c || !rho || !q3d) return set_err(CM1G_ERR_ARG, "null argument");
  ProfActive pa(c);
  Stager S(c);
  size_t ns = nS(c->g);
  const float *drho = S.in(rho, ns, false);
  float *dq = S.in(q3d, ns, true);
  CUCHK(cudaMemsetAsync(c->dscal + 8, 0, sizeof(double), c->stream));
  launch_pdefq(c->g, rmax, drho, dq, c->bud, c->dscal + 8, c->stream, &c->nlaunch);
  double a = 0.0;
  CUCHK(cudaMemcpyAsync(&a, c->dscal + 8, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  int rc = S.finish();
  if (asq) *asq += a;
  return rc;
}

static int bc_entry(cm1g_ctx_t *c, float *a, int which, int flag) {
  if (!c || !a) return set_err(CM1G_ERR_ARG, "null argument");
  ProfActive pa(c);
  Stager S(c);
  size_t n = which == 3 ? nU(c->g) : which == 4 ? nV(c->g) : which == 5 ? nW(c->g) : nS(c->g);
  float *d = S.in(a, n, true);
  launch_bc(c->g, d, which, flag, c->stream, &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}
extern "C" int cm1g_bcs(cm1g_ctx_t *c, float *s) { return bc_entry(c, s, 1, 0); }
extern "C" int cm1g_bcp(cm1g_ctx_t *c, float *p) { return bc_entry(c, p, 2, 0); }
extern "C" int cm1g_bcu(cm1g_ctx_t *c, float *u) { return bc_entry(c, u, 3, 0); }
extern "C" int cm1g_bcv(cm1g_ctx_t *c, float *v) { return bc_entry(c, v, 4, 0); }
extern "C" int cm1g_bcw(cm1g_ctx_t *c, float *w, int32_t flag) { return bc_entry(c, w, 5, flag); }

extern "C" int cm1g_advs(cm1g_ctx_t *c, int32_t nrk, int32_t wflag, const float *divx, const float *rru,
                         const float *rrv, const float *rrw, const float *s0, const float *s, float *sten,
                         int32_t pdef, int32_t pdefweno, float dt, double weps) {
  if (!c || !rru || !rrv || !rrw || !divx || !s || !sten || (pdef && !s0)) return set_err(CM1G_ERR_ARG, "null argument");
  if (nrk < 1 || nrk > 3) return set_err(CM1G_ERR_ARG, "nrk must be 1..3");
  ProfActive pa(c);
  Stager S(c);
  const DGrid &g = c->g;
  const float *dru = S.in(rru, nU(g), false), *drv = S.in(rrv, nV(g), false), *drw = S.in(rrw, nW(g), false);
  const float *ddx = S.in(divx, nS(g), false), *ds = S.in(s, nS(g), false);
  const float *ds0 = s0 ? S.in(s0, nS(g), false) : nullptr;
  float *dten = S.in(sten, nS(g), true);
  const int weno = (wflag == 1) && (c->cfg.advwenos == 1 || (c->cfg.advwenos == 2 && nrk == 3));
  if (!pdef) {
    launch_advs(g, dru, drv, drw, 0, ddx, ds, ds0 ? ds0 : ds, 0, dten, nullptr, dten, nullptr, weno, 0, pdefweno,
                weps, dt, 0, c->pdefscr, c->stream, &c->nlaunch);
  } else {
    launch_advs(g, dru, drv, drw, 0, ddx, ds, ds0, 0, dten, nullptr, dten, nullptr, weno, 1, pdefweno, weps, dt,
                0, c->pdefscr, c->stream, &c->nlaunch);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

// Momentum advection of the components selected by `which` (bit 0 u, 1 v,
// 2 w); null tendencies are allowed for the components not selected.
static int adv_momentum_entry(cm1g_ctx_t *c, int which, const float *u3d, const float *v3d, const float *w3d,
                              float *uten, float *vten, float *wten) {
  if (!c || !u3d || !v3d || !w3d) return set_err(CM1G_ERR_ARG, "null argument");
  if (((which & 1) && !uten) || ((which & 2) && !vten) || ((which & 4) && !wten))
    return set_err(CM1G_ERR_ARG, "null argument");
  ProfActive pa(c);
  Stager S(c);
  const DGrid &g = c->g;
  const float *du = S.in(u3d, nU(g), false), *dv = S.in(v3d, nV(g), false), *dw = S.in(w3d, nW(g), false);
  float *tu = (which & 1) ? S.in(uten, nU(g), true) : nullptr;
  float *tv = (which & 2) ? S.in(vten, nV(g), true) : nullptr;
  float *tw = (which & 4) ? S.in(wten, nW(g), true) : nullptr;
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging");
  launch_adv_momentum(g, du, dv, dw, tu, tv, tw, tu, tv, tw, nullptr, nullptr, c->mdivx, c->stream, &c->nlaunch,
                      nullptr, nullptr, which);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

extern "C" int cm1g_advuvw(cm1g_ctx_t *c, int32_t nrk, const float *u3d, const float *v3d, const float *w3d,
                           float *uten, float *vten, float *wten) {
  (void)nrk;
  return adv_momentum_entry(c, 7, u3d, v3d, w3d, uten, vten, wten);
}
extern "C" int cm1g_advu(cm1g_ctx_t *c, int32_t nrk, const float *u3d, float *uten, const float *v3d,
                         const float *w3d) {
  (void)nrk;
  return adv_momentum_entry(c, 1, u3d, v3d, w3d, uten, nullptr, nullptr);
}
extern "C" int cm1g_advv(cm1g_ctx_t *c, int32_t nrk, const float *v3d, float *vten, const float *u3d,
                         const float *w3d) {
  (void)nrk;
  return adv_momentum_entry(c, 2, u3d, v3d, w3d, nullptr, vten, nullptr);
}
extern "C" int cm1g_advw(cm1g_ctx_t *c, int32_t nrk, const float *w3d, float *wten, const float *u3d,
                         const float *v3d) {
  (void)nrk;
  return adv_momentum_entry(c, 4, u3d, v3d, w3d, nullptr, nullptr, wten);
}

extern "C" int cm1g_sound(cm1g_ctx_t *c, float dt, float *radbcw, float *radbce, float *radbcs, float *radbcn,
                          float *rru, float *ua, float *u3d, const float *uten,
                          float *rrv, float *va, float *v3d, const float *vten,
                          float *rrw, float *wa, float *w3d, const float *wten,
                          float *ppi, float *pp3d, const float *piadv, const float *ppten, float *ppx,
                          const float *thv, const float *ppterm, int32_t nrk, float dttmp) {
  (void)dttmp;
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (nrk < 1 || nrk > 3) return set_err(CM1G_ERR_ARG, "nrk must be 1..3");
  const void *req[] = {ua, u3d, uten, va, v3d, vten, wa, w3d, wten, ppi, pp3d, piadv, ppten, ppx, thv, ppterm,
                       rru, rrv, rrw, radbcw, radbce, radbcs, radbcn};
  for (const void *p : req) if (!p) return set_err(CM1G_ERR_ARG, "null argument");
  ProfActive pa(c);
  Stager S(c);
  const DGrid &g = c->g;
  size_t ns = nS(g), nu = nU(g), nv = nV(g), nw = nW(g), nrw = (size_t)g.NJ * g.NK, nrs = (size_t)g.NI * g.NK;
  float *dua = S.in(ua, nu, false), *du3 = S.in(u3d, nu, true);
  const float *dut = S.in(uten, nu, false);
  float *dva = S.in(va, nv, false), *dv3 = S.in(v3d, nv, true);
  const float *dvt = S.in(vten, nv, false);
  float *dwa = S.in(wa, nw, false), *dw3 = S.in(w3d, nw, true);
  const float *dwt = S.in(wten, nw, false);
  float *dppi = S.in(ppi, ns, false), *dpp = S.in(pp3d, ns, true);
  const float *dpia = S.in(piadv, ns, false), *dppt = S.in(ppten, ns, false);
  float *dppx = S.in(ppx, ns, true);
  const float *dthv = S.in(thv, ns, false), *dppterm = S.in(ppterm, ns, false);
  float *dru = S.in(rru, nu, true), *drv = S.in(rrv, nv, true), *drw = S.in(rrw, nw, true);
  // irbc = 2 rewrites the phase speeds each small step (sound.F:261-267)
  const bool rad_out = c->g.irbc == 2;
  float *rw = S.in(radbcw, nrw, rad_out), *re = S.in(radbce, nrw, rad_out), *rs = S.in(radbcs, nrs, rad_out),
        *rn = S.in(radbcn, nrs, rad_out);
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging");
  launch_sound(g, c->cfg.nsound, nrk, dt, dua, du3, dut, dva, dv3, dvt, dwa, dw3, dwt, dppi, dpp, dpia, dppt, dppx,
               dthv, dppterm, dru, drv, drw, rw, re, rs, rn, c->su, c->sv, c->su2, c->sv2, c->d1, c->d2, c->lu, c->rbnd, c->stream,
               &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

extern "C" int cm1g_calcmass(cm1g_ctx_t *c, const float *rho, double *tmass) {
  if (!c || !rho || !tmass) return set_err(CM1G_ERR_ARG, "null argument");
  Stager S(c);
  const float *dr = S.in(rho, nS(c->g), false);
  launch_level_mass(c->g, dr, c->lev, c->stream, &c->nlaunch);
  std::vector<double> lev(c->g.nk + 2);
  CUCHK(cudaMemcpyAsync(lev.data(), c->lev, lev.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  int rc = S.finish();
  if (rc) return rc;
  double tm = 0.0;
  for (int k = 1; k <= c->g.nk; k++) tm = tm + lev[k];
  *tmass = tm * (double)(c->g.dx * c->g.dy * c->g.dz);
  return CM1G_OK;
}

extern "C" int cm1g_dtsmall(int32_t psolver, int32_t nx, int32_t ny, float min_dx, float min_dy, float min_dz,
                            int32_t adapt_dt, float *dt, double *dbldt, int32_t *nsound) {
  if (!dt || !dbldt || !nsound) return set_err(CM1G_ERR_ARG, "null argument");
  const int max_nsound = 192;
  float dtsm;
  if (psolver == 1 || psolver == 4 || psolver == 5) { *nsound = 1; return CM1G_OK; }
  if (psolver == 2) {
    if (ny == 1) dtsm = 0.60f * fminf(min_dx, min_dz) / 360.0f;
    else if (nx == 1) dtsm = 0.60f * fminf(min_dy, min_dz) / 360.0f;
    else dtsm = 0.50f * fminf(fminf(min_dx, min_dy), min_dz) / 360.0f;
  } else if (psolver == 3) {
    if (ny == 1) dtsm = 0.60f * min_dx / 360.0f;
    else if (nx == 1) dtsm = 0.60f * min_dy / 360.0f;
    else dtsm = 0.60f * fminf(min_dx, min_dy) / 360.0f;
  } else {
    return set_err(CM1G_ERR_UNSUPPORTED, "dtsmall: psolver=%d is not built", psolver);
  }
  const double x = *dbldt / (double)dtsm;
  int ns = (int)(x >= 0.0 ? floor(x + 0.5) : ceil(x - 0.5));   // Fortran nint
  if (ns < 4) ns = 4;
  if (ns % 2 != 0) ns = ns + 1;
  if (*dbldt / (double)(float)ns > (double)dtsm) ns = ns + 2;
  if (ns > max_nsound) {
    if (adapt_dt != 1)
      return set_err(CM1G_ERR_ARG, "limit for number of small steps exceeded: nsound=%d > %d; dtl needs to be smaller",
                     ns, max_nsound);
    ns = max_nsound;
    *dbldt = (double)((float)ns * dtsm);
    *dt = (float)*dbldt;
  }
  *nsound = ns;
  return CM1G_OK;
}

extern "C" int cm1g_tendency_init(cm1g_ctx_t *c, int32_t irdamp, float rdalpha, const float *tauh, const float *taus,
                                  const float *tauf, const float *uavg, const float *vavg, const float *thavg,
                                  const float *ua, const float *va, const float *wa, const float *tha, float *uten1,
                                  float *vten1, float *wten1, float *thten1, float *qten, float *ptten) {
  if (!c || !uten1 || !vten1 || !wten1 || !thten1) return set_err(CM1G_ERR_ARG, "null argument");
  if (irdamp < 0 || irdamp > 2) return set_err(CM1G_ERR_ARG, "irdamp must be 0, 1 or 2");
  const DGrid &g = c->g;
  const int numq = c->cfg.imoist ? c->cfg.numq : 0, npt = c->cfg.iptra ? c->cfg.npt : 0;
  if ((numq && !qten) || (npt && !ptten)) return set_err(CM1G_ERR_ARG, "qten/ptten missing");
  if (irdamp && (!tauh || !taus || !tauf || !ua || !va || !wa || !tha))
    return set_err(CM1G_ERR_ARG, "Rayleigh damping needs tauh, taus, tauf, ua, va, wa, tha");
  if (irdamp == 1 && (!g.u0 || !g.v0)) return set_err(CM1G_ERR_ARG, "grid u0/v0 were not given to cm1g_init");
  if (irdamp == 2 && (!uavg || !vavg || !thavg)) return set_err(CM1G_ERR_ARG, "irdamp=2 needs uavg, vavg, thavg");
  ProfActive pa(c);
  Stager S(c);
  const size_t ns = nS(g), nk2 = (size_t)g.NK;
  TendIn t{};
  t.irdamp = irdamp; t.rdalpha = rdalpha;
  if (irdamp) {
    t.tauh = S.in(tauh, ns, false); t.taus = S.in(taus, ns, false); t.tauf = S.in(tauf, nW(g), false);
    t.ua = S.in(ua, nU(g), false); t.va = S.in(va, nV(g), false); t.wa = S.in(wa, nW(g), false);
    t.tha = S.in(tha, ns, false);
    if (irdamp == 2) { t.uavg = S.in(uavg, nk2, false); t.vavg = S.in(vavg, nk2, false); t.thavg = S.in(thavg, nk2, false); }
  }
  t.uten1 = S.in(uten1, nU(g), true); t.vten1 = S.in(vten1, nV(g), true);
  t.wten1 = S.in(wten1, nW(g), true); t.thten1 = S.in(thten1, ns, true);
  t.qten = numq ? S.in(qten, numq * ns, true) : nullptr;
  t.ptten = npt ? S.in(ptten, npt * ns, true) : nullptr;
  t.numq = numq; t.nq = numq + npt;
  launch_tend_init(g, t, c->stream, &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

extern "C" int cm1g_calcener(cm1g_ctx_t *c, const float *zh, const float *rho, const float *ua, const float *va,
                             const float *wa, const float *ppi, const float *tha, const float *qv, const float *ql,
                             const float *qi, const float *vr, double energy[5]) {
  if (!c || !zh || !rho || !ua || !va || !wa || !ppi || !tha || !energy) return set_err(CM1G_ERR_ARG, "null argument");
  ProfActive pa(c);
  Stager S(c);
  const DGrid &g = c->g;
  const size_t ns = nS(g);
  EnerIn e{};
  e.zh = S.in(zh, ns, false); e.rho = S.in(rho, ns, false); e.ua = S.in(ua, nU(g), false);
  e.va = S.in(va, nV(g), false); e.wa = S.in(wa, nW(g), false); e.ppi = S.in(ppi, ns, false);
  e.tha = S.in(tha, ns, false);
  e.qv = qv ? S.in(qv, ns, false) : nullptr; e.ql = ql ? S.in(ql, ns, false) : nullptr;
  e.qi = qi ? S.in(qi, ns, false) : nullptr; e.vr = vr ? S.in(vr, ns, false) : nullptr;
  // constants.F:85-150: latent heats at the reference temperature to = 273.15
  const int tc = c->cfg.testcase;
  const float xlv = tc == 4 ? 2.47e6f : tc == 5 ? 2.50e6f : 2501000.0f, xls = 2834000.0f, to = 273.15f;
  e.lv1 = (tc == 4 || tc == 5) ? xlv : xlv + (g.c.cpl - g.c.cpv) * to;   // constants.F:156-159
  e.ls1 = xls + (g.c.cpi - g.c.cpv) * to;
  double *part = c->ener + 8;
  launch_calcener(g, e, part, c->ener, c->stream, &c->nlaunch);
  double h[4];
  CUCHK(cudaMemcpyAsync(h, c->ener, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  int rc = S.finish();
  if (rc) return rc;
  for (int q = 0; q < 4; q++) energy[q] = h[q];
  energy[4] = ((h[0] + h[1]) + h[2]) + h[3];
  return CM1G_OK;
}

extern "C" int cm1g_maxmin(cm1g_ctx_t *c, const float *a, int32_t stag, float *amax, float *amin, int32_t loc[6]) {
  if (!c || !a || !amax || !amin || !loc) return set_err(CM1G_ERR_ARG, "null argument");
  if (stag < 1 || stag > 4) return set_err(CM1G_ERR_ARG, "stag must be 1..4");
  Stager S(c);
  const DGrid &g = c->g;
  size_t n = stag == 2 ? nU(g) : stag == 3 ? nV(g) : stag == 4 ? nW(g) : nS(g);
  const float *d = S.in(a, n, false);
  launch_maxmin(g, d, stag, c->mm, c->stream, &c->nlaunch);
  unsigned long long h[2];
  CUCHK(cudaMemcpyAsync(h, c->mm, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  int rc = S.finish();
  if (rc) return rc;
  auto dec = [](unsigned int key) {
    unsigned int b = (key & 0x80000000u) ? (key & 0x7fffffffu) : ~key;
    float f; memcpy(&f, &b, 4); return f;
  };
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3);
  unsigned int imax = 0xffffffffu - (unsigned int)(h[0] & 0xffffffffu), imin = (unsigned int)(h[1] & 0xffffffffu);
  *amax = dec((unsigned int)(h[0] >> 32));
  *amin = dec((unsigned int)(h[1] >> 32));
  loc[0] = 1 + (int)(imax % ie); loc[1] = 1 + (int)((imax / ie) % je); loc[2] = 1 + (int)(imax / ((unsigned)ie * je));
  loc[3] = 1 + (int)(imin % ie); loc[4] = 1 + (int)((imin / ie) % je); loc[5] = 1 + (int)(imin / ((unsigned)ie * je));
  return CM1G_OK;
}

// ---------------------------------------------------------------------
// Statistics package (statpack.F:10-658).  cm1g_stat_setup turns the
// switches into a job list (one per reduced quantity) and an output program
// (one operation per rstat entry) in the order of setup_stat_vars
// (statpack.F:666-1458) and statpack (statpack.F:122-600); cm1g_statpack
// launches k_stat_levels and k_stat_finish and copies rstat back once.
// ---------------------------------------------------------------------
namespace {
enum HostSlot { HS_MTIME = 0, HS_QBUDGET, HS_ASQ, HS_BSQ };

std::string trim_name(const char *p, int n) {
  std::string t(p, strnlen(p, n));
  while (!t.empty() && t.back() == ' ') t.pop_back();
  while (!t.empty() && t.front() == ' ') t.erase(t.begin());
  return t;
}
}  // namespace

extern "C" int cm1g_stat_setup(cm1g_ctx_t *c, const cm1g_stat_opts_t *o, int32_t *stat_out) {
  if (!c || !o || !stat_out) return set_err(CM1G_ERR_ARG, "null argument");
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const bool moist = cf.imoist == 1;
  if (o->adapt_dt) return set_err(CM1G_ERR_UNSUPPORTED, "statpack: adapt_dt is not built");
  if (o->stat_rmw) return set_err(CM1G_ERR_UNSUPPORTED, "statpack: stat_rmw (axisymmetric runs) is not built");
  if (o->stat_km || o->stat_kh)
    return set_err(CM1G_ERR_UNSUPPORTED, "statpack: stat_km/stat_kh need the subgrid turbulence, not built");
  if (moist && (o->stat_rhi || o->iice))
    return set_err(CM1G_ERR_UNSUPPORTED, "statpack: ice species (iice, stat_rhi) are not built");
  if (o->bbc == 3) return set_err(CM1G_ERR_UNSUPPORTED, "statpack: bbc=3 (surface layer) is not built");
  if (!o->zh || !o->zf) return set_err(CM1G_ERR_ARG, "statpack: zh and zf are required");
  const int numq = moist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0, nk = g.nk, ni = g.ni, nj = g.nj;
  if (moist && (o->nql1 < 0 || o->nql2 > numq || (o->nql1 > 0 && o->nql2 < o->nql1)))
    return set_err(CM1G_ERR_ARG, "statpack: nql1..nql2 outside 1..numq");
  if (moist && o->stat_pcn && (o->nbudget < 0 || (o->nbudget > 0 && !o->budname)))
    return set_err(CM1G_ERR_ARG, "statpack: stat_pcn needs nbudget names");
  const float *zh = o->zh - 0, *zf = o->zf;   // index k = 0 .. nk+1 (nk+2 for zf)

  std::vector<StatJob> jobs;
  std::vector<StatOp> ops;
  std::vector<std::string> names;
  auto job = [&](int kind, int src, int stag, int klo, int nlev, int ie, int je) {
    StatJob j{};
    j.kind = kind; j.src = src; j.stag = stag; j.qn = 0; j.klo = klo; j.nlev = nlev;
    j.i0 = 1; j.ie = ie; j.j0 = 1; j.je = je; j.k0 = 0; j.r1 = j.r2 = 0.0f;
    jobs.push_back(j);
    return (int)jobs.size() - 1;
  };
  auto op = [&](int kind, int jx, int k, int arg, const std::string &name) {
    ops.push_back(StatOp{kind, jx, k, arg});
    names.push_back(name);
  };
  auto mm = [&](int jx, const std::string &a, const std::string &b) {   // maxmin
    op(SO_MAX, jx, 0, 0, a); op(SO_MIN, jx, 0, 0, b);
  };
  auto mm1 = [&](int jx, const std::string &a, const std::string &b) {  // maxmin2d of level 1
    op(SO_LEVMAX, jx, 1, 0, a); op(SO_LEVMIN, jx, 1, 0, b);
  };
  auto qn = [&](int n) { return trim_name(o->qname[n], 4); };

  op(SO_HOST, -1, 0, HS_MTIME, "mtime");
  if (o->stat_w) {
    int w = job(SK_FIELD, SF_W, 4, 1, nk + 1, ni, nj);
    mm(w, "wmax", "wmin");
    op(SO_ZF_KMAX, w, 0, 0, "zwmax"); op(SO_ZF_KMIN, w, 0, 0, "zwmin");
  }
  if (o->stat_wlevs && o->maxz >= 10000.0f) {   // statpack.F:146-212
    const float zl[5] = {500.0f, 1000.0f, 2500.0f, 5000.0f, 10000.0f};
    const char *nm[5] = {"500", "1000", "2500", "5000", "10k"};
    for (int n = 0; n < 5; n++) {
      if (zl[n] < zf[nk + 1]) {
        int nkm = nk + 1;
        while (zf[nkm] > zl[n] && nkm > 1) nkm--;
        const float r2 = (zl[n] - zf[nkm]) / (zf[nkm + 1] - zf[nkm]);
        int jx = job(SK_WLEV, 0, 1, 1, 1, ni, nj);
        jobs[jx].k0 = nkm; jobs[jx].r1 = 1.0f - r2; jobs[jx].r2 = r2;
        mm1(jx, std::string("wmax") + nm[n], std::string("wmin") + nm[n]);
      } else {
        op(SO_ZERO, -1, 0, 0, std::string("wmax") + nm[n]);
        op(SO_ZERO, -1, 0, 0, std::string("wmin") + nm[n]);
      }
    }
  }
  if (o->stat_u) {
    int u = job(SK_FIELD, SF_U, 2, 1, nk, ni + 1, nj);
    mm(u, "umax", "umin"); mm1(u, "sumax", "sumin");
  }
  if (o->stat_v) {
    int v = job(SK_FIELD, SF_V, 3, 1, nk, ni, nj + 1);
    mm(v, "vmax", "vmin"); mm1(v, "svmax", "svmin");
  }
  if (o->stat_pipert) mm(job(SK_FIELD, SF_PPI, 1, 1, nk, ni, nj), "ppimax", "ppimin");
  if (o->stat_prspert) mm(job(SK_PP, 0, 1, 1, nk, ni, nj), "ppmax", "ppmin");
  if (o->stat_thpert) {
    int t = job(SK_FIELD, SF_THA, 1, 1, nk, ni, nj);
    mm(t, "thpmax", "thpmin"); mm1(t, "sthpmax", "sthpmin");
  }
  if (moist && o->stat_q) {
    for (int n = 0; n < numq; n++) {
      int q = job(SK_FIELD, SF_Q, 1, 1, nk, ni, nj);
      jobs[q].qn = n;
      mm(q, "max" + qn(n), "min" + qn(n));
    }
    mm1(job(SK_PRATE, 0, 1, 1, 1, ni, nj), "pratemax", "pratemin");
  }
  if (o->stat_div) mm(job(SK_DIV, 0, 1, 1, nk, ni, nj), "divmax", "divmin");
  if (moist && o->stat_rh) mm(job(SK_RH, 0, 1, 1, nk, ni, nj), "rhmax", "rhmin");
  for (int n = 0; n < npt; n++) {
    int p = job(SK_FIELD, SF_PT, 1, 1, nk, ni, nj);
    jobs[p].qn = n;
    mm(p, "maxpt" + std::to_string(n + 1), "minpt" + std::to_string(n + 1));
  }
  if (moist && o->stat_the) {
    // calcthe copies the level below above 10 km: those levels repeat values
    int nl = 0;
    while (nl < nk && zh[nl + 1] <= 10000.0f) nl++;
    if (nl < 1) nl = 1;
    int t = job(SK_THE, 0, 1, 1, nl, ni, nj);
    mm(t, "themax", "themin"); mm1(t, "sthemax", "sthemin");
  }
  if (moist && o->stat_cloud) {
    int cl = job(SK_CLOUD, 0, 1, 1, nk, ni, nj);
    op(SO_QCTOP, cl, 0, 0, "qctop"); op(SO_QCBOT, cl, 0, 0, "qcbot");
  }
  if (o->stat_sfcprs) {
    mm1(job(SK_FIELD, SF_PRS, 1, 1, 1, ni, nj), "sprsmax", "sprsmin");
    mm1(job(SK_PSFC, 0, 1, 1, 1, ni, nj), "psfcmax", "psfcmin");
  }
  if (o->stat_wsp) {
    int w = job(SK_WSP, 0, 1, 1, nk, ni, nj);
    mm(w, "wspmax", "wspmin");
    op(SO_ZH_KMAX, w, 0, 0, "zwspmax"); op(SO_ZH_KMIN, w, 0, 0, "zwspmin");
    mm1(w, "swspmax", "swspmin");
  }
  if (o->stat_cfl) op(SO_CFL, job(SK_CFL, 0, 1, 1, nk, ni, nj), 0, 0, "cflmax");
  if (o->stat_vort) {   // vertvort: levels of 1-5 km from zh (misclibs.F:2455-2466)
    int kv[6] = {1, nk + 1, nk + 1, nk + 1, nk + 1, nk + 1};
    for (int k = nk; k >= 1; k--)
      for (int n = 1; n <= 5; n++)
        if (zh[k] >= 1000.0f * n) kv[n] = k;
    const char *nm[6] = {"vortsfc", "vort1km", "vort2km", "vort3km", "vort4km", "vort5km"};
    for (int n = 0; n < 6; n++) {
      if (kv[n] <= nk) {
        int v = job(SK_VORT, 0, 1, 1, 1, ni + 1 - g.ibe, nj + 1 - g.ibn);
        jobs[v].i0 = 1 + g.ibw; jobs[v].j0 = 1 + g.ibs; jobs[v].k0 = kv[n];
        op(SO_VORT, v, kv[n], 0, nm[n]);
      } else {
        op(SO_ZERO, -1, 0, 0, nm[n]);
      }
    }
  }
  if (o->stat_tmass) op(SO_SUM, job(SK_MASS, 0, 1, 1, nk, ni, nj), 0, 1, "tmass");
  if (moist && o->stat_tmois) op(SO_SUM, job(SK_TMOIS, 0, 1, 1, nk, ni, nj), 0, 1, "tmois");
  if (moist && o->stat_qmass)
    for (int n = 0; n < numq; n++) {
      const bool liq = o->nql1 > 0 && n + 1 >= o->nql1 && n + 1 <= o->nql2;
      if (n + 1 == cf.nqv || liq) {
        int q = job(SK_QMAS, 0, 1, 1, nk, ni, nj);
        jobs[q].qn = n;
        op(SO_SUM, q, 0, 1, "mass" + qn(n));
      }
    }
  if (o->stat_tenerg) {
    int e = job(SK_ENER, 0, 1, 1, nk, ni, nj);
    op(SO_SUM, e, 0, 1, "ek"); op(SO_SUM, e, 1, 1, "ei"); op(SO_SUM, e, 2, 1, "ep"); op(SO_SUM, e, 3, 1, "le");
    op(SO_ENER_TOTAL, e, 0, 0, "et");
  }
  if (o->stat_mo) {
    int m = job(SK_MOE, 0, 1, 1, nk, ni, nj);
    op(SO_SUM, m, 0, 1, "tmu"); op(SO_SUM, m, 1, 1, "tmv"); op(SO_SUM, m, 2, 1, "tmw");
  }
  if (o->stat_tmf) {
    int m = job(SK_TMF, 0, 1, 1, nk, ni, nj);
    op(SO_SUM, m, 0, 2, "tmfu"); op(SO_SUM, m, 1, 2, "tmfd");
  }
  if (moist && o->stat_pcn)
    for (int n = 0; n < o->nbudget; n++) {
      ops.push_back(StatOp{SO_HOST, -1, n, HS_QBUDGET});
      names.push_back(trim_name(o->budname + 6 * n, 6));
    }
  if (moist && o->stat_qsrc) {
    for (int n = 0; n < numq; n++) { ops.push_back(StatOp{SO_HOST, -1, n, HS_ASQ}); names.push_back("as" + qn(n)); }
    for (int n = 0; n < numq; n++) { ops.push_back(StatOp{SO_HOST, -1, n, HS_BSQ}); names.push_back("bs" + qn(n)); }
  }
  if (jobs.empty()) job(SK_MASS, 0, 1, 1, 0, ni, nj);   // keeps the job table non-empty (no levels)

  // device tables (grown, never shrunk); chunk records [job][level][chunk]
  const int maxlev = nk + 1;
  int npl = 1;
  for (const StatJob &j : jobs) npl = std::max(npl, (j.ie - j.i0 + 1) * (j.je - j.j0 + 1));
  const int nch = stat_chunks(npl);
  if ((int)jobs.size() > c->st_cap_jobs) {
    if (c->d_st_jobs) { cudaFree(c->d_st_jobs); cudaFree(c->d_st_lev); c->d_st_jobs = nullptr; c->d_st_lev = nullptr; }
    c->st_cap_jobs = (int)jobs.size() + 16;
    CUCHK(cudaMalloc(&c->d_st_jobs, c->st_cap_jobs * sizeof(StatJob)));
    CUCHK(cudaMalloc(&c->d_st_lev, (size_t)c->st_cap_jobs * maxlev * stat_chunks((g.ni + 1) * (g.nj + 1)) *
                                       sizeof(StatLev)));
  }
  if ((int)ops.size() > c->st_cap_ops) {
    if (c->d_st_ops) { cudaFree(c->d_st_ops); cudaFree(c->d_rstat); c->d_st_ops = nullptr; c->d_rstat = nullptr; }
    c->st_cap_ops = (int)ops.size() + 32;
    CUCHK(cudaMalloc(&c->d_st_ops, c->st_cap_ops * sizeof(StatOp)));
    CUCHK(cudaMalloc(&c->d_rstat, c->st_cap_ops * sizeof(float)));
  }
  if (!c->d_st_zh) {
    CUCHK(cudaMalloc(&c->d_st_zh, (size_t)(nk + 2) * sizeof(float)));
    CUCHK(cudaMalloc(&c->d_st_zf, (size_t)(nk + 3) * sizeof(float)));
  }
  CUCHK(cudaMemcpyAsync(c->d_st_jobs, jobs.data(), jobs.size() * sizeof(StatJob), cudaMemcpyHostToDevice, c->stream));
  CUCHK(cudaMemcpyAsync(c->d_st_ops, ops.data(), ops.size() * sizeof(StatOp), cudaMemcpyHostToDevice, c->stream));
  CUCHK(cudaMemcpyAsync(c->d_st_zh, zh, (size_t)(nk + 2) * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CUCHK(cudaMemcpyAsync(c->d_st_zf, zf, (size_t)(nk + 3) * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  CUCHK(cudaStreamSynchronize(c->stream));
  c->st_opts = *o;
  c->st_opts.zh = c->st_opts.zf = nullptr;
  c->st_opts.budname = nullptr;
  c->st_jobs = jobs; c->st_ops = ops; c->st_names = names;
  c->st_nch = nch;
  c->st_ready = true;
  *stat_out = (int32_t)ops.size();
  return CM1G_OK;
}

extern "C" int cm1g_stat_name(cm1g_ctx_t *c, int32_t n, char *name, int32_t len) {
  if (!c || !name || len < 1) return set_err(CM1G_ERR_ARG, "null argument");
  if (!c->st_ready) return set_err(CM1G_ERR_STATE, "cm1g_stat_setup has not been called");
  if (n < 1 || n > (int)c->st_names.size()) return set_err(CM1G_ERR_ARG, "statistic %d out of range", n);
  snprintf(name, (size_t)len, "%s", c->st_names[n - 1].c_str());
  return CM1G_OK;
}

extern "C" int cm1g_statpack(cm1g_ctx_t *c, double mtime, float dt, const float *ua, const float *va,
                             const float *wa, const float *ppi, const float *tha, const float *prs, const float *rho,
                             const float *qa, const float *pta, const float *prate, const double *qbudget,
                             const double *asq, const double *bsq, float *rstat) {
  if (!c || !rstat) return set_err(CM1G_ERR_ARG, "null argument");
  if (!c->st_ready) return set_err(CM1G_ERR_STATE, "cm1g_stat_setup has not been called");
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const bool moist = cf.imoist == 1;
  const int numq = moist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  // the fields the job list reads
  bool need_u = false, need_v = false, need_w = false, need_ppi = false, need_tha = false, need_prs = false;
  bool need_rho = false, need_q = false, need_pt = false;
  for (const StatJob &j : c->st_jobs) {
    if (j.nlev == 0) continue;
    switch (j.kind) {
      case SK_FIELD:
        need_u |= j.src == SF_U; need_v |= j.src == SF_V; need_w |= j.src == SF_W; need_ppi |= j.src == SF_PPI;
        need_tha |= j.src == SF_THA; need_prs |= j.src == SF_PRS; need_q |= j.src == SF_Q; need_pt |= j.src == SF_PT;
        break;
      case SK_PP: case SK_PSFC: need_prs = true; break;
      case SK_DIV: case SK_CFL: need_u = need_v = need_w = true; break;
      case SK_RH: case SK_THE: need_prs = need_tha = need_ppi = need_q = true; break;
      case SK_WSP: case SK_VORT: need_u = need_v = true; break;
      case SK_WLEV: need_w = true; break;
      case SK_CLOUD: need_q = true; break;
      case SK_MASS: need_rho = true; break;
      case SK_TMOIS: case SK_QMAS: need_rho = need_q = true; break;
      case SK_TMF: need_rho = need_w = true; break;
      case SK_MOE: need_rho = need_u = need_v = need_w = true; need_q |= moist; break;
      case SK_ENER: need_rho = need_u = need_v = need_w = need_ppi = need_tha = true; need_q |= moist; break;
      default: break;
    }
  }
  if ((need_u && !ua) || (need_v && !va) || (need_w && !wa) || (need_ppi && !ppi) || (need_tha && !tha) ||
      (need_prs && !prs) || (need_rho && !rho) || (need_q && numq && !qa) || (need_pt && npt && !pta))
    return set_err(CM1G_ERR_ARG, "statpack: a field the statistics need is NULL");
  for (const StatOp &p : c->st_ops) {
    if (p.op != SO_HOST) continue;
    if ((p.arg == HS_QBUDGET && !qbudget) || (p.arg == HS_ASQ && !asq) || (p.arg == HS_BSQ && !bsq))
      return set_err(CM1G_ERR_ARG, "statpack: qbudget/asq/bsq are needed by stat_pcn/stat_qsrc");
  }
  ProfActive pa(c);
  Stager S(c);
  const size_t ns = nS(g);
  StatFields f{};
  f.ua = need_u ? S.in(ua, nU(g), false) : nullptr;
  f.va = need_v ? S.in(va, nV(g), false) : nullptr;
  f.wa = need_w ? S.in(wa, nW(g), false) : nullptr;
  f.ppi = need_ppi ? S.in(ppi, ns, false) : nullptr;
  f.tha = need_tha ? S.in(tha, ns, false) : nullptr;
  f.prs = need_prs ? S.in(prs, ns, false) : nullptr;
  f.rho = need_rho ? S.in(rho, ns, false) : nullptr;
  f.qa = (need_q && numq) ? S.in(qa, (size_t)numq * ns, false) : nullptr;
  f.pta = (need_pt && npt) ? S.in(pta, (size_t)npt * ns, false) : nullptr;
  f.prate = prate ? S.in(prate, (size_t)g.NI * g.NJ, false) : nullptr;
  f.qstride = (long)ns;
  const cm1g_stat_opts_t &o = c->st_opts;
  StatConsts k{};
  const Consts &cc = g.c;
  k.p00 = 1.0e5f; k.eps = cc.rd / cc.rv; k.reps = cc.reps; k.rd = cc.rd; k.rv = cc.rv; k.cp = cc.cp;
  k.cv = cc.cv; k.cvv = cc.cvv; k.cpl = cc.cpl; k.cpi = cc.cpi; k.cpdrd = cc.cpdrd; k.g = cc.g;
  // constants.F:85-160: latent heats at to = 273.15 (testcases 4 and 5 use lv1 = xlv)
  const int tc = cf.testcase;
  const float xlv = tc == 4 ? 2.47e6f : tc == 5 ? 2.50e6f : 2501000.0f, xls = 2834000.0f, to = 273.15f;
  k.lv1 = (tc == 4 || tc == 5) ? xlv : xlv + (cc.cpl - cc.cpv) * to;
  k.ls1 = xls + (cc.cpi - cc.cpv) * to;
  k.dtdx = 0.5f * dt * g.rdx; k.dtdy = 0.5f * dt * g.rdy; k.dtdz = 0.5f * dt * g.rdz;
  k.cgs1 = o.cgs1; k.cgs2 = o.cgs2; k.cgs3 = o.cgs3; k.maxz = o.maxz;
  k.ptype = o.ptype; k.imoist = moist; k.numq = numq; k.nqv = moist ? cf.nqv - 1 : 0;
  k.nql1 = o.nql1 > 0 ? o.nql1 - 1 : -1; k.nql2 = o.nql1 > 0 ? o.nql2 - 1 : -1;
  k.nx = g.ni; k.ny = g.nj;
  k.cloudmask = 0;
  for (int n = 0; n < numq && n < CM1G_MAXQ; n++) if (o.cloudvar[n]) k.cloudmask |= 1u << n;
  k.zh = c->d_st_zh; k.zf = c->d_st_zf;
  const int nops = (int)c->st_ops.size();
  launch_stat(g, f, k, c->d_st_jobs, (int)c->st_jobs.size(), c->d_st_lev, g.nk + 1, c->st_nch, c->d_st_ops, nops,
              c->d_rstat, c->stream, &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  CUCHK(cudaMemcpyAsync(rstat, c->d_rstat, (size_t)nops * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  int rc = S.finish();
  if (rc) return rc;
  for (int p = 0; p < nops; p++) {
    const StatOp &q = c->st_ops[p];
    if (q.op != SO_HOST) continue;
    rstat[p] = q.arg == HS_MTIME ? (float)mtime : q.arg == HS_QBUDGET ? (float)qbudget[q.k]
             : q.arg == HS_ASQ ? (float)asq[q.k] : (float)bsq[q.k];
  }
  return CM1G_OK;
}

extern "C" int cm1g_stat_write(const char *path, int32_t nrec, const float *rstat, int32_t nstat) {
  if (!path || !rstat || nrec < 1 || nstat < 1) return set_err(CM1G_ERR_ARG, "bad argument");
  FILE *fp = fopen(path, "r+b");
  if (!fp) fp = fopen(path, "w+b");
  if (!fp) return set_err(CM1G_ERR_ARG, "cannot open %s", path);
  const long off = (long)(nrec - 1) * 4L * nstat;
  int ok = fseek(fp, off, SEEK_SET) == 0 && fwrite(rstat, sizeof(float), (size_t)nstat, fp) == (size_t)nstat;
  ok = (fclose(fp) == 0) && ok;
  return ok ? CM1G_OK : set_err(CM1G_ERR_ARG, "write to %s failed", path);
}

// ---------------------------------------------------------------------
// Records of output and restart files (k_io.cu) and the restart of the
// state this library advances.
// ---------------------------------------------------------------------
extern "C" int cm1g_records_size(cm1g_ctx_t *c, int32_t n, const int32_t *stag, const int32_t *k1, const int32_t *k2,
                                 int64_t *nvals) {
  if (!c || !stag || !k1 || !k2 || !nvals || n < 0) return set_err(CM1G_ERR_ARG, "bad argument");
  int64_t tot = 0;
  for (int f = 0; f < n; f++) {
    if (stag[f] < 1 || stag[f] > 4) return set_err(CM1G_ERR_ARG, "field %d: stag must be 1..4", f);
    const int kmax = c->g.nk + 1 + (stag[f] == 4);
    if (k1[f] < 0 || k2[f] > kmax || k2[f] < k1[f]) return set_err(CM1G_ERR_ARG, "field %d: levels out of range", f);
    tot += record_count(c->g, stag[f], k1[f], k2[f]);
  }
  *nvals = tot;
  return CM1G_OK;
}

// elements of a field up to level k2 (a 2-D array is levels 0..0)
static size_t field_elems(const DGrid &g, int stag, int k2) {
  const size_t plane = stag == 2 ? (size_t)(g.NI + 1) * g.NJ : stag == 3 ? (size_t)g.NI * (g.NJ + 1)
                                                                         : (size_t)g.NI * g.NJ;
  return plane * (size_t)(k2 + 1);
}

static int records_common(cm1g_ctx_t *c, int32_t n, float *const *fields, const int32_t *stag, const int32_t *k1,
                          const int32_t *k2, float *buf, bool unpack) {
  if (!c || !fields || !buf) return set_err(CM1G_ERR_ARG, "null argument");
  int64_t tot = 0;
  int rc = cm1g_records_size(c, n, stag, k1, k2, &tot);
  if (rc) return rc;
  for (int f = 0; f < n; f++) if (!fields[f]) return set_err(CM1G_ERR_ARG, "field %d is NULL", f);
  ProfActive pa(c);
  Stager S(c);
  float *dbuf = S.in(buf, (size_t)tot, !unpack);
  if (!dbuf) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  int64_t off = 0;
  for (int f = 0; f < n; f++) {
    float *d = S.in(fields[f], field_elems(c->g, stag[f], k2[f]), unpack);
    if (!d) return set_err(CM1G_ERR_NOMEM, "staging alloc");
    launch_pack_records(c->g, d, stag[f], k1[f], k2[f], dbuf + off, unpack, c->stream, &c->nlaunch);
    off += record_count(c->g, stag[f], k1[f], k2[f]);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

extern "C" int cm1g_pack_records(cm1g_ctx_t *c, int32_t n, const float *const *fields, const int32_t *stag,
                                 const int32_t *k1, const int32_t *k2, float *out) {
  return records_common(c, n, const_cast<float *const *>(fields), stag, k1, k2, out, false);
}

extern "C" int cm1g_unpack_records(cm1g_ctx_t *c, int32_t n, float *const *fields, const int32_t *stag,
                                   const int32_t *k1, const int32_t *k2, const float *in) {
  return records_common(c, n, fields, stag, k1, k2, const_cast<float *>(in), true);
}

namespace {
struct RField { std::string name; float *a; int stag, k1, k2; };
const char kRstMagic[8] = {'C', 'M', '1', 'G', 'R', 'S', 'T', '1'};

// restart_write's order of the fields this library advances
// (restart_write.F:692-839): rain, rho, prs, ua, va, wa, ppi, tha, ppx,
// the q arrays, the tracers; the radiative boundary speeds follow
std::vector<RField> restart_fields(cm1g_ctx *c, const cm1g_state_t *d) {
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const long ns = nS(g);
  const int nk = g.nk, numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  std::vector<RField> f;
  if (cf.ptype == 1) f.push_back({"rain", d->rain, 1, 0, 0});
  f.push_back({"rho", d->rho, 1, 1, nk});
  f.push_back({"prs", d->prs, 1, 1, nk});
  f.push_back({"ua", d->ua, 2, 1, nk});
  f.push_back({"va", d->va, 3, 1, nk});
  f.push_back({"wa", d->wa, 4, 1, nk + 1});
  f.push_back({"ppi", d->ppi, 1, 1, nk});
  f.push_back({"tha", d->tha, 1, 1, nk});
  f.push_back({"ppx", d->ppx, 1, 1, nk});
  for (int q = 0; q < numq; q++) f.push_back({"q" + std::to_string(q + 1), d->qa + q * ns, 1, 1, nk});
  for (int q = 0; q < npt; q++) f.push_back({"pt" + std::to_string(q + 1), d->pta + q * ns, 1, 1, nk});
  return f;
}

template <class T> bool put(FILE *fp, const T &v) { return fwrite(&v, sizeof v, 1, fp) == 1; }
template <class T> bool get(FILE *fp, T &v) { return fread(&v, sizeof v, 1, fp) == 1; }
}  // namespace

static int restart_check_state(cm1g_ctx *c, const cm1g_state_t *st) {
  const cm1g_config_t &cf = c->cfg;
  const float *req[] = {st->ua, st->va, st->wa, st->ppi, st->tha, st->ppx, st->rho, st->prs,
                        st->radbcw, st->radbce, st->radbcs, st->radbcn};
  for (const float *p : req) if (!p) return set_err(CM1G_ERR_ARG, "restart: state array missing");
  if (cf.imoist && !st->qa) return set_err(CM1G_ERR_ARG, "restart: qa missing");
  if (cf.iptra && cf.npt > 0 && !st->pta) return set_err(CM1G_ERR_ARG, "restart: pta missing");
  if (cf.ptype == 1 && !st->rain) return set_err(CM1G_ERR_ARG, "restart: rain missing");
  return CM1G_OK;
}

extern "C" int cm1g_restart_write(cm1g_ctx_t *c, const char *path, const cm1g_restart_t *hdr,
                                  const cm1g_state_t *st) {
  if (!c || !path || !hdr || !st) return set_err(CM1G_ERR_ARG, "null argument");
  int rc = restart_check_state(c, st);
  if (rc) return rc;
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const int numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  ProfActive pa(c);
  Stager S(c);
  cm1g_state_t d{};
  const size_t ns = nS(g), n2 = (size_t)g.NI * g.NJ;
  d.ua = S.in(st->ua, nU(g), false); d.va = S.in(st->va, nV(g), false); d.wa = S.in(st->wa, nW(g), false);
  d.ppi = S.in(st->ppi, ns, false); d.tha = S.in(st->tha, ns, false); d.ppx = S.in(st->ppx, ns, false);
  d.rho = S.in(st->rho, ns, false); d.prs = S.in(st->prs, ns, false);
  d.qa = numq ? S.in(st->qa, numq * ns, false) : nullptr;
  d.pta = npt ? S.in(st->pta, npt * ns, false) : nullptr;
  d.rain = cf.ptype == 1 ? S.in(st->rain, n2, false) : nullptr;
  std::vector<RField> flds = restart_fields(c, &d);
  int64_t tot = 0;
  for (auto &f : flds) tot += record_count(g, f.stag, f.k1, f.k2);
  float *dbuf = S.dev_buffer((size_t)tot);
  if (!dbuf || S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  int64_t off = 0;
  for (auto &f : flds) {
    launch_pack_records(g, f.a, f.stag, f.k1, f.k2, dbuf + off, false, c->stream, &c->nlaunch);
    off += record_count(g, f.stag, f.k1, f.k2);
  }
  std::vector<float> h((size_t)tot);
  CUCHK(cudaMemcpyAsync(h.data(), dbuf, (size_t)tot * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  // radiative boundary speeds: (jb:je,kb:ke) and (ib:ie,kb:ke) arrays, their j (i) = 1..n, k = 1..nk
  const size_t nrw = (size_t)g.NJ * g.NK, nrs = (size_t)g.NI * g.NK;
  std::vector<float> rb[4] = {std::vector<float>(nrw), std::vector<float>(nrw), std::vector<float>(nrs),
                              std::vector<float>(nrs)};
  const float *rsrc[4] = {st->radbcw, st->radbce, st->radbcs, st->radbcn};
  for (int s = 0; s < 4; s++)
    CUCHK(cudaMemcpyAsync(rb[s].data(), rsrc[s], rb[s].size() * sizeof(float), cudaMemcpyDefault, c->stream));
  rc = S.finish();
  if (rc) return rc;
  FILE *fp = fopen(path, "wb");
  if (!fp) return set_err(CM1G_ERR_ARG, "cannot create %s", path);
  bool ok = fwrite(kRstMagic, 1, 8, fp) == 8;
  const int32_t ver = 1, nf = (int32_t)flds.size() + 4;
  const int32_t dims[8] = {g.ni, g.nj, g.nk, g.ngxy, numq, npt, cf.ptype, nf};
  ok = ok && put(fp, ver) && fwrite(dims, sizeof(int32_t), 8, fp) == 8;
  ok = ok && put(fp, hdr->nstep) && put(fp, (int32_t)0) && put(fp, hdr->mtime) && put(fp, hdr->dt) &&
       put(fp, hdr->dtlast) && put(fp, hdr->mass1);
  auto put_desc = [&](const std::string &name, int stag, int k1, int k2) {
    char nm[8] = {0};
    memcpy(nm, name.c_str(), std::min<size_t>(8, name.size()));
    const int32_t v[4] = {stag, k1, k2, 0};
    return fwrite(nm, 1, 8, fp) == 8 && fwrite(v, sizeof(int32_t), 4, fp) == 4;
  };
  for (auto &f : flds) ok = ok && put_desc(f.name, f.stag, f.k1, f.k2);
  const char *rbn[4] = {"radbcw", "radbce", "radbcs", "radbcn"};
  for (int s = 0; s < 4; s++) ok = ok && put_desc(rbn[s], 0, 1, g.nk);
  ok = ok && fwrite(h.data(), sizeof(float), h.size(), fp) == h.size();
  for (int s = 0; s < 4; s++) {   // writerbcwe / writerbcsn (restart_write.F:2164-2286): per level, j (i) = 1..n
    const bool we = s < 2;
    const int n = we ? g.nj : g.ni, L = we ? g.NJ : g.NI, lb = we ? g.jb : g.ib;
    for (int k = 1; k <= g.nk && ok; k++)
      ok = fwrite(rb[s].data() + (size_t)k * L + (1 - lb), sizeof(float), (size_t)n, fp) == (size_t)n;
  }
  ok = (fclose(fp) == 0) && ok;
  return ok ? CM1G_OK : set_err(CM1G_ERR_ARG, "write to %s failed", path);
}

extern "C" int cm1g_restart_read(cm1g_ctx_t *c, const char *path, cm1g_restart_t *hdr, cm1g_state_t *st) {
  if (!c || !path || !hdr || !st) return set_err(CM1G_ERR_ARG, "null argument");
  int rc = restart_check_state(c, st);
  if (rc) return rc;
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const int numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  FILE *fp = fopen(path, "rb");
  if (!fp) return set_err(CM1G_ERR_ARG, "cannot open %s", path);
  struct Closer { FILE *f; ~Closer() { fclose(f); } } closer{fp};
  char magic[8];
  int32_t ver = 0, dims[8], pad;
  cm1g_restart_t h{};
  bool ok = fread(magic, 1, 8, fp) == 8 && memcmp(magic, kRstMagic, 8) == 0 && get(fp, ver) && ver == 1 &&
            fread(dims, sizeof(int32_t), 8, fp) == 8;
  if (!ok) return set_err(CM1G_ERR_ARG, "%s is not a restart file of this library", path);
  if (dims[0] != g.ni || dims[1] != g.nj || dims[2] != g.nk || dims[3] != g.ngxy || dims[4] != numq ||
      dims[5] != npt || dims[6] != cf.ptype)
    return set_err(CM1G_ERR_ARG, "restart %s: grid or options differ from the context", path);
  ok = get(fp, h.nstep) && get(fp, pad) && get(fp, h.mtime) && get(fp, h.dt) && get(fp, h.dtlast) && get(fp, h.mass1);
  cm1g_state_t d{};
  ProfActive pa(c);
  Stager S(c);
  const size_t ns = nS(g), n2 = (size_t)g.NI * g.NJ;
  d.ua = S.in(st->ua, nU(g), true); d.va = S.in(st->va, nV(g), true); d.wa = S.in(st->wa, nW(g), true);
  d.ppi = S.in(st->ppi, ns, true); d.tha = S.in(st->tha, ns, true); d.ppx = S.in(st->ppx, ns, true);
  d.rho = S.in(st->rho, ns, true); d.prs = S.in(st->prs, ns, true);
  d.qa = numq ? S.in(st->qa, numq * ns, true) : nullptr;
  d.pta = npt ? S.in(st->pta, npt * ns, true) : nullptr;
  d.rain = cf.ptype == 1 ? S.in(st->rain, n2, true) : nullptr;
  d.u3d = st->u3d ? S.in(st->u3d, nU(g), true) : nullptr;
  d.v3d = st->v3d ? S.in(st->v3d, nV(g), true) : nullptr;
  d.w3d = st->w3d ? S.in(st->w3d, nW(g), true) : nullptr;
  d.pp3d = st->pp3d ? S.in(st->pp3d, ns, true) : nullptr;
  d.th3d = st->th3d ? S.in(st->th3d, ns, true) : nullptr;
  d.q3d = (numq && st->q3d) ? S.in(st->q3d, numq * ns, true) : nullptr;
  d.pt3d = (npt && st->pt3d) ? S.in(st->pt3d, npt * ns, true) : nullptr;
  std::vector<RField> flds = restart_fields(c, &d);
  if (dims[7] != (int32_t)flds.size() + 4) return set_err(CM1G_ERR_ARG, "restart %s: field list differs", path);
  for (size_t q = 0; q < flds.size() + 4 && ok; q++) {
    char nm[8];
    int32_t v[4];
    ok = fread(nm, 1, 8, fp) == 8 && fread(v, sizeof(int32_t), 4, fp) == 4;
    if (ok && q < flds.size()) {
      const RField &f = flds[q];
      if (strncmp(nm, f.name.c_str(), 8) != 0 || v[0] != f.stag || v[1] != f.k1 || v[2] != f.k2)
        return set_err(CM1G_ERR_ARG, "restart %s: field %zu is not %s", path, q, f.name.c_str());
    }
  }
  int64_t tot = 0;
  for (auto &f : flds) tot += record_count(g, f.stag, f.k1, f.k2);
  std::vector<float> hbuf((size_t)tot);
  ok = ok && fread(hbuf.data(), sizeof(float), hbuf.size(), fp) == hbuf.size();
  const size_t nrw = (size_t)g.NJ * g.NK, nrs = (size_t)g.NI * g.NK;
  float *rdst[4] = {st->radbcw, st->radbce, st->radbcs, st->radbcn};
  std::vector<float> rb[4] = {std::vector<float>(nrw), std::vector<float>(nrw), std::vector<float>(nrs),
                              std::vector<float>(nrs)};
  // the arrays' halo values are kept: fetch them on the context's stream,
  // after any work already queued there
  for (int s = 0; s < 4; s++)
    CUCHK(cudaMemcpyAsync(rb[s].data(), rdst[s], rb[s].size() * sizeof(float), cudaMemcpyDefault, c->stream));
  CUCHK(cudaStreamSynchronize(c->stream));
  for (int s = 0; s < 4 && ok; s++) {
    const bool we = s < 2;
    const int n = we ? g.nj : g.ni, L = we ? g.NJ : g.NI, lb = we ? g.jb : g.ib;
    for (int k = 1; k <= g.nk && ok; k++)
      ok = fread(rb[s].data() + (size_t)k * L + (1 - lb), sizeof(float), (size_t)n, fp) == (size_t)n;
  }
  if (!ok) return set_err(CM1G_ERR_ARG, "restart %s: truncated", path);
  float *dbuf = S.dev_buffer((size_t)tot);
  if (!dbuf || S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  CUCHK(cudaMemcpyAsync(dbuf, hbuf.data(), (size_t)tot * sizeof(float), cudaMemcpyHostToDevice, c->stream));
  int64_t off = 0;
  for (auto &f : flds) {
    launch_pack_records(g, f.a, f.stag, f.k1, f.k2, dbuf + off, true, c->stream, &c->nlaunch);
    off += record_count(g, f.stag, f.k1, f.k2);
  }
  for (int s = 0; s < 4; s++)
    CUCHK(cudaMemcpyAsync(rdst[s], rb[s].data(), rb[s].size() * sizeof(float), cudaMemcpyDefault, c->stream));
  // halos as the end of a step leaves them (the stage-3 fills of solve2 and
  // solve3's fills), then the time-t+dt copies equal the time-t arrays
  {
    std::vector<float *> arr{d.ua, d.va, d.wa, d.ppi, d.tha, d.rho, d.ppx};
    std::vector<int> which{3, 4, 5, 2, 1, 2, 2}, flag{0, 0, 1, 0, 0, 0, 0};
    for (int q = 0; q < numq; q++) { arr.push_back(d.qa + q * ns); which.push_back(1); flag.push_back(0); }
    for (int q = 0; q < npt; q++) { arr.push_back(d.pta + q * ns); which.push_back(1); flag.push_back(0); }
    launch_bc_batch(g, arr.data(), which.data(), flag.data(), (int)arr.size(), c->stream, &c->nlaunch);
  }
  auto cp = [&](float *dst, const float *src, size_t n) {
    if (dst && src) cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyDeviceToDevice, c->stream);
  };
  cp(d.u3d, d.ua, nU(g)); cp(d.v3d, d.va, nV(g)); cp(d.w3d, d.wa, nW(g));
  cp(d.pp3d, d.ppi, ns); cp(d.th3d, d.tha, ns);
  if (numq) cp(d.q3d, d.qa, numq * ns);
  if (npt) cp(d.pt3d, d.pta, npt * ns);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  rc = S.finish();
  if (rc) return rc;
  *hdr = h;
  return CM1G_OK;
}

extern "C" int cm1g_diff2(cm1g_ctx_t *c, float kdiff2, int32_t idiff, int32_t bbc, int32_t tbc, const float cgs[3],
                          const float cgt[3], const float *ua, const float *va, const float *wa, const float *rho,
                          const float *tha, const float *qa, const float *pta, float *uten1, float *vten1,
                          float *wten1, float *thten1, float *qten, float *ptten) {
  if (!c || !cgs || !cgt || !ua || !va || !wa || !rho) return set_err(CM1G_ERR_ARG, "null argument");
  if (idiff < 1) return CM1G_OK;                       // solve1.F:689: nothing to add
  if (!(kdiff2 >= 0.0f)) return set_err(CM1G_ERR_ARG, "kdiff2 must be >= 0");
  if ((bbc != 1 && bbc != 2) || (tbc != 1 && tbc != 2))
    return set_err(CM1G_ERR_UNSUPPORTED, "diff2: bbc/tbc 1 (free slip) or 2 (no slip) only (bbc=3 needs the surface layer)");
  if (!uten1 || !vten1 || !wten1) return set_err(CM1G_ERR_ARG, "uten1/vten1/wten1 missing");
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const int numq = cf.imoist ? cf.numq : 0, npt = cf.iptra ? cf.npt : 0;
  const bool scal = idiff == 1;
  if (scal && (!tha || !thten1 || (numq && (!qa || !qten)) || (npt && (!pta || !ptten))))
    return set_err(CM1G_ERR_ARG, "diff2 with idiff=1 needs tha/thten1, qa/qten, pta/ptten");
  if (!c->d2s) {
    const size_t bS = nS(g) * sizeof(float), bW = nW(g) * sizeof(float);
    c->d2s = (float *)dalloc(c, 6 * bS + 3 * bW);
    if (!c->d2s) return set_err(CM1G_ERR_NOMEM, "diff2 scratch");
  }
  ProfActive pa(c);
  Stager S(c);
  const size_t ns = nS(g);
  Diff2Args a{};
  a.kdiff2 = kdiff2; a.bbc = bbc; a.tbc = tbc; a.momentum = 1;
  a.cgs1 = cgs[0]; a.cgs2 = cgs[1]; a.cgs3 = cgs[2]; a.cgt1 = cgt[0]; a.cgt2 = cgt[1]; a.cgt3 = cgt[2];
  a.ua = S.in(ua, nU(g), false); a.va = S.in(va, nV(g), false); a.wa = S.in(wa, nW(g), false);
  a.rho = S.in(rho, ns, false);
  a.uten = S.in(uten1, nU(g), true); a.vten = S.in(vten1, nV(g), true); a.wten = S.in(wten1, nW(g), true);
  float *p = c->d2s;
  a.rr = p; p += ns; a.divx = p; p += ns; a.t11 = p; p += ns; a.t22 = p; p += ns; a.t33 = p; p += ns;
  a.t12 = p; p += ns; a.rf = p; p += nW(g); a.t13 = p; p += nW(g); a.t23 = p;
  a.nsc = 0;
  if (scal) {   // solve1.F:706-733: theta, every q, every tracer
    a.s[a.nsc] = S.in(tha, ns, false); a.sten[a.nsc++] = S.in(thten1, ns, true);
    const float *dq = numq ? S.in(qa, numq * ns, false) : nullptr;
    float *dqt = numq ? S.in(qten, numq * ns, true) : nullptr;
    for (int n = 0; n < numq; n++) { a.s[a.nsc] = dq + n * ns; a.sten[a.nsc++] = dqt + n * ns; }
    const float *dp = npt ? S.in(pta, npt * ns, false) : nullptr;
    float *dpt = npt ? S.in(ptten, npt * ns, true) : nullptr;
    for (int n = 0; n < npt; n++) { a.s[a.nsc] = dp + n * ns; a.sten[a.nsc++] = dpt + n * ns; }
  }
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  launch_diff2(g, a, c->stream, &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

// Smagorinsky LES (sgsmodel=2): deformation, N^2, kmh/kmv, stresses and the
// tendencies solve1 adds (turb.F:1327-1340, 1405-1415, 1629-1640; solve1.F:
// 1113-1240).  kmh/kmv, when given, receive the eddy viscosities (w-arrays).
extern "C" int cm1g_turbsmag(cm1g_ctx_t *c, float csm, int32_t tconfig, int32_t bcturbs, int32_t bbc, int32_t tbc,
                             const float cgs[3], const float cgt[3], const float *ua, const float *va,
                             const float *wa, const float *rho, const float *tha, const float *qa, const float *pta,
                             float *uten1, float *vten1, float *wten1, float *thten1, float *qten, float *ptten,
                             float *kmh, float *kmv) {
  if (!c || !cgs || !cgt || !ua || !va || !wa || !rho || !tha) return set_err(CM1G_ERR_ARG, "null argument");
  if (!uten1 || !vten1 || !wten1) return set_err(CM1G_ERR_ARG, "uten1/vten1/wten1 missing");
  if (!(csm >= 0.0f)) return set_err(CM1G_ERR_ARG, "csm must be >= 0");
  if (tconfig != 1 && tconfig != 2) return set_err(CM1G_ERR_ARG, "tconfig must be 1 or 2");
  if (bcturbs != 1 && bcturbs != 2) return set_err(CM1G_ERR_ARG, "bcturbs must be 1 or 2");
  if ((bbc != 1 && bbc != 2) || (tbc != 1 && tbc != 2))
    return set_err(CM1G_ERR_UNSUPPORTED, "turbsmag: bbc/tbc 1 (free slip) or 2 (no slip) only (bbc=3 needs the surface layer)");
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  if (g.wbc != 1 || g.ebc != 1 || g.sbc != 1 || g.nbc != 1)
    return set_err(CM1G_ERR_UNSUPPORTED, "turbsmag: periodic lateral boundaries only");
  if (cf.imoist) return set_err(CM1G_ERR_UNSUPPORTED, "turbsmag: the moist N^2 of calcnm is not built (imoist=0 only)");
  const int npt = cf.iptra ? cf.npt : 0;
  if (thten1 && npt && (!pta || !ptten)) return set_err(CM1G_ERR_ARG, "turbsmag with tracers needs pta/ptten");
  const size_t ns = nS(g), nw = nW(g);
  if (!c->les) {
    c->les = (float *)dalloc(c, (6 * ns + 6 * nw) * sizeof(float));
    if (!c->les) return set_err(CM1G_ERR_NOMEM, "turbsmag scratch");
  }
  ProfActive pa(c);
  Stager S(c);
  TurbArgs a{};
  a.csm = csm;
  const float prandtl = 1.0f / 3.00f;
  a.prinv = 1.0f / prandtl;
  a.cgs1 = cgs[0]; a.cgs2 = cgs[1]; a.cgs3 = cgs[2]; a.cgt1 = cgt[0]; a.cgt2 = cgt[1]; a.cgt3 = cgt[2];
  a.tconfig = tconfig; a.bcturbs = bcturbs; a.bbc = bbc; a.tbc = tbc;
  a.ua = S.in(ua, nU(g), false); a.va = S.in(va, nV(g), false); a.wa = S.in(wa, nW(g), false);
  a.rho = S.in(rho, ns, false); a.tha = S.in(tha, ns, false);
  a.uten = S.in(uten1, nU(g), true); a.vten = S.in(vten1, nV(g), true); a.wten = S.in(wten1, nW(g), true);
  if (thten1) {
    a.thten = S.in(thten1, ns, true);
    a.numq = 0;
    a.npt = npt;
    a.pta = npt ? S.in(pta, npt * ns, false) : nullptr;
    a.ptten = npt ? S.in(ptten, npt * ns, true) : nullptr;
  }
  float *p = c->les;
  a.t11 = p; p += ns; a.t22 = p; p += ns; a.t33 = p; p += ns; a.t12 = p; p += ns;
  a.cx = p; p += ns; a.cy = p; p += ns;
  a.s13 = p; p += nw; a.s23 = p; p += nw; a.t13 = p; p += nw; a.t23 = p; p += nw;
  a.kmh = kmh ? S.in(kmh, nw, true) : p; p += nw;
  a.kmv = kmv ? S.in(kmv, nw, true) : p;
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  launch_turbsmag(g, a, c->stream, &c->nlaunch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  return S.finish();
}

// writeout (output_format=1): the GrADS records of the fields this library
// advances, in writeout's order, and their descriptors.
namespace {
struct WVar { std::string name; const float *src; int stag, k1, k2, mode; const float *base; };
}

extern "C" int cm1g_writeout(cm1g_ctx_t *c, const char *prefix, int32_t nwrite, double mtime,
                             const cm1g_writeout_opts_t *o, const cm1g_state_t *st) {
  if (!c || !prefix || !o || !st || nwrite < 1) return set_err(CM1G_ERR_ARG, "bad argument");
  const DGrid &g = c->g;
  const cm1g_config_t &cf = c->cfg;
  const int nk = g.nk, numq = cf.imoist ? cf.numq : 0;
  enum { PLAIN = 0, ADDP, SUBP, SUBF, EXNER, EXNERP };
  if ((o->output_prspert) && !g.prs0) return set_err(CM1G_ERR_ARG, "writeout: prspert needs the grid's prs0");
  auto need = [&](const void *p, const char *what) -> int {
    return p ? CM1G_OK : set_err(CM1G_ERR_ARG, "writeout: %s is NULL", what);
  };
  int rc = CM1G_OK;
  if (o->output_th || o->output_thpert) rc = rc ? rc : need(st->tha, "tha");
  if (o->output_prs || o->output_prspert || o->output_pi || o->output_pipert) rc = rc ? rc : need(st->prs, "prs");
  if (o->output_rho || o->output_rhopert) rc = rc ? rc : need(st->rho, "rho");
  if (numq && (o->output_qv || o->output_qvpert || o->output_q)) rc = rc ? rc : need(st->qa, "qa");
  if (o->output_u || o->output_upert) rc = rc ? rc : need(st->ua, "ua");
  if (o->output_v || o->output_vpert) rc = rc ? rc : need(st->va, "va");
  if (o->output_w) rc = rc ? rc : need(st->wa, "wa");
  if (cf.ptype == 1 && (o->output_rain || o->output_prate)) rc = rc ? rc : need(st->rain && st->prate ? st : nullptr, "rain/prate");
  if (rc) return rc;
  ProfActive pa(c);
  Stager S(c);
  const size_t ns = nS(g), n2 = (size_t)g.NI * g.NJ;
  auto dv = [&](const float *p, size_t n) { return p ? (const float *)S.in(p, n, false) : nullptr; };
  const float *tha = dv(st->tha, ns), *prs = dv(st->prs, ns), *rho = dv(st->rho, ns);
  const float *qa = numq ? dv(st->qa, numq * ns) : nullptr;
  const float *ua = dv(st->ua, nU(g)), *va = dv(st->va, nV(g)), *wa = dv(st->wa, nW(g));
  const float *rain = cf.ptype == 1 ? dv(st->rain, n2) : nullptr, *prate = cf.ptype == 1 ? dv(st->prate, n2) : nullptr;
  if (S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
  // writeout.F's order for these variables (writeout.F:2300-7000)
  std::vector<WVar> fs, fu, fv, fw;
  if (cf.ptype == 1 && o->output_rain) fs.push_back({"rain", rain, 1, 0, 0, PLAIN, nullptr});
  if (cf.ptype == 1 && o->output_prate) fs.push_back({"prate", prate, 1, 0, 0, PLAIN, nullptr});
  if (o->output_th) fs.push_back({"th", tha, 1, 1, nk, ADDP, g.th0});
  if (o->output_thpert) fs.push_back({"thpert", tha, 1, 1, nk, PLAIN, nullptr});
  if (o->output_prs) fs.push_back({"prs", prs, 1, 1, nk, PLAIN, nullptr});
  if (o->output_prspert) fs.push_back({"prspert", prs, 1, 1, nk, SUBP, g.prs0});
  if (o->output_pi) fs.push_back({"pi", prs, 1, 1, nk, EXNER, nullptr});
  if (o->output_pipert) fs.push_back({"pipert", prs, 1, 1, nk, EXNERP, nullptr});
  if (o->output_rho) fs.push_back({"rho", rho, 1, 1, nk, PLAIN, nullptr});
  if (o->output_rhopert) fs.push_back({"rhopert", rho, 1, 1, nk, SUBP, g.rho0});
  if (numq) {
    const float *qv = qa + (long)(cf.nqv - 1) * ns;
    if (o->output_qv) fs.push_back({"qv", qv, 1, 1, nk, PLAIN, nullptr});
    if (o->output_qvpert) fs.push_back({"qvpert", qv, 1, 1, nk, SUBP, g.qv0});
    if (o->output_q)
      for (int n = 0; n < numq; n++)
        if (n + 1 != cf.nqv) {
          std::string nm(o->qname[n], strnlen(o->qname[n], 4));
          while (!nm.empty() && nm.back() == ' ') nm.pop_back();
          fs.push_back({nm.empty() ? "q" + std::to_string(n + 1) : nm, qa + (long)n * ns, 1, 1, nk, PLAIN, nullptr});
        }
  }
  if (o->output_u) fu.push_back({"u", ua, 2, 1, nk, PLAIN, nullptr});
  if (o->output_upert) fu.push_back({"upert", ua, 2, 1, nk, SUBF, g.u0});
  if (o->output_v) fv.push_back({"v", va, 3, 1, nk, PLAIN, nullptr});
  if (o->output_vpert) fv.push_back({"vpert", va, 3, 1, nk, SUBF, g.v0});
  if (o->output_w) fw.push_back({"w", wa, 4, 1, nk + 1, PLAIN, nullptr});
  if ((o->output_upert && !g.u0) || (o->output_vpert && !g.v0))
    return set_err(CM1G_ERR_ARG, "writeout: upert/vpert need the grid's u0/v0");
  // level heights for the descriptors (zf(1) = 0, dz/mh between w-levels)
  std::vector<float> mh(g.NK + 2);
  CUCHK(cudaMemcpyAsync(mh.data(), g.mh, mh.size() * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  struct File { const char *tag; std::vector<WVar> *v; int stag; } files[] = {
      {"s", &fs, 1}, {"u", &fu, 2}, {"v", &fv, 3}, {"w", &fw, 4}};
  std::vector<std::vector<float>> host(4);
  for (int f = 0; f < 4; f++) {
    auto &vars = *files[f].v;
    if (vars.empty()) continue;
    int64_t tot = 0;
    for (auto &w : vars) tot += record_count(g, w.stag, w.k1, w.k2);
    float *dbuf = S.dev_buffer((size_t)tot);
    if (!dbuf || S.err) return set_err(CM1G_ERR_NOMEM, "staging alloc");
    int64_t off = 0;
    for (auto &w : vars) {
      launch_pack_records(g, w.src, w.stag, w.k1, w.k2, dbuf + off, false, c->stream, &c->nlaunch, w.mode, w.base);
      off += record_count(g, w.stag, w.k1, w.k2);
    }
    host[f].resize((size_t)tot);
    CUCHK(cudaMemcpyAsync(host[f].data(), dbuf, (size_t)tot * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(CM1G_ERR_CUDA, "%s", cudaGetErrorString(e));
  rc = S.finish();
  if (rc) return rc;
  std::vector<double> zf(nk + 2, 0.0), zh(nk + 1, 0.0);
  for (int k = 1; k <= nk; k++) {
    zf[k + 1] = zf[k] + (double)g.dz / (double)mh[k];
    zh[k] = 0.5 * (zf[k] + zf[k + 1]);
  }
  for (int f = 0; f < 4; f++) {
    auto &vars = *files[f].v;
    if (vars.empty()) continue;
    const std::string base = std::string(prefix) + "_" + files[f].tag;
    const std::string dat = base + ".dat";
    FILE *fp = fopen(dat.c_str(), "r+b");
    if (!fp) fp = fopen(dat.c_str(), "w+b");
    if (!fp) return set_err(CM1G_ERR_ARG, "cannot open %s", dat.c_str());
    const long off = (long)(nwrite - 1) * (long)host[f].size() * 4L;
    bool ok = fseek(fp, off, SEEK_SET) == 0 && fwrite(host[f].data(), 4, host[f].size(), fp) == host[f].size();
    ok = (fclose(fp) == 0) && ok;
    if (!ok) return set_err(CM1G_ERR_ARG, "write to %s failed", dat.c_str());
    // GrADS descriptor of the file (kilometres; one time per call)
    const int nx = g.ni + (files[f].stag == 2), ny = g.nj + (files[f].stag == 3);
    const bool wlev = files[f].stag == 4;
    FILE *cp = fopen((base + ".ctl").c_str(), "w");
    if (!cp) return set_err(CM1G_ERR_ARG, "cannot create %s.ctl", base.c_str());
    const char *slash = strrchr(dat.c_str(), '/');
    fprintf(cp, "dset ^%s\n", slash ? slash + 1 : dat.c_str());
    fprintf(cp, "title CM1 output (%s points), time %.6f s\nundef -999999.9\n", files[f].tag, mtime);
    fprintf(cp, "xdef %d linear %.6f %.6f\n", nx, files[f].stag == 2 ? 0.0 : 0.5e-3 * g.dx, 1.0e-3 * g.dx);
    fprintf(cp, "ydef %d linear %.6f %.6f\n", ny, files[f].stag == 3 ? 0.0 : 0.5e-3 * g.dy, 1.0e-3 * g.dy);
    fprintf(cp, "zdef %d levels\n", wlev ? nk + 1 : nk);
    for (int k = 1; k <= (wlev ? nk + 1 : nk); k++) fprintf(cp, "%.6f\n", 1.0e-3 * (wlev ? zf[k] : zh[k]));
    fprintf(cp, "tdef %d linear 00:00Z03JUL0001 1YR\nvars %zu\n", nwrite, vars.size());
    for (auto &w : vars) fprintf(cp, "%-8s %d 99 %s\n", w.name.c_str(), w.k2 == 0 ? 0 : w.k2 - w.k1 + 1, w.name.c_str());
    fprintf(cp, "endvars\n");
    fclose(cp);
  }
  return CM1G_OK;
}

extern "C" int cm1g_profile(cm1g_ctx_t *c, int32_t enable) {
  if (!c) return set_err(CM1G_ERR_STATE, "null context");
  if (c->prof) { c->prof->drain(); delete c->prof; c->prof = nullptr; }
  if (enable) c->prof = new Profile();
  return CM1G_OK;
}

extern "C" int cm1g_profile_read(cm1g_ctx_t *c, int32_t index, char *name, int32_t name_len, int64_t *launches,
                                 double *total_ms) {
  if (!c || !name || name_len < 2) return set_err(CM1G_ERR_ARG, "null argument");
  if (!c->prof) return set_err(CM1G_ERR_STATE, "profiling is off");
  c->prof->drain();
  if (index < 0 || index >= (int32_t)c->prof->names.size()) return set_err(CM1G_ERR_ARG, "no such entry");
  snprintf(name, (size_t)name_len, "%s", c->prof->names[index].c_str());
  if (launches) *launches = c->prof->count[index];
  if (total_ms) *total_ms = c->prof->ms[index];
  return CM1G_OK;
}
