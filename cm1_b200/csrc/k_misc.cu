// k_misc.cu -- the remaining pieces of the large step: per-stage thermodynamic
// set-up, pressure/density with the dry-air mass fix (FP64 reductions),
// open-boundary phase speeds, CFL, the positive-definite column fix, the
// end-of-step rollover and the domain diagnostics.
#include "cm1g_common.cuh"

namespace cm1g {

// ---------------------------------------------------------------------
// stage set-up: theta_rho (t11), ppterm (t22), thterm (solve2.F:313-446)
// on the interior and piadv = pi0+pp' on 0..ni+1 x 0..nj+1 (solve2.F:1027-1038)
// ---------------------------------------------------------------------
__global__ void k_stage_prep(DGrid g, const float *__restrict__ th3d, const float *__restrict__ pp3d,
                             const float *__restrict__ qv, LiquidIn liq, int imoist, int eqtset,
                             float *__restrict__ t11, float *__restrict__ t22, float *__restrict__ thterm,
                             float *__restrict__ piadv) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);       // 0..ni+1
  const int j = (int)blockIdx.y;                                     // 0..nj+1
  const int k = 1 + (int)blockIdx.z;
  if (i > g.ni + 1) return;
  const long o = iS(g, i, j, k);
  const float pp = LDG(&pp3d[o]);
  piadv[o] = LDG(&g.pi0[k]) + pp;
  if (i < 1 || i > g.ni || j < 1 || j > g.nj) return;
  const Consts &c = g.c;
  const float th3 = LDG(&th3d[o]), th0 = LDG(&g.th0[k]), pi0 = LDG(&g.pi0[k]);
  if (imoist) {
    const float q = fmaxf(LDG(&qv[o]), 0.0f);
    // dum2: the liquid species in index order (solve2.F:315-345); no ice
    float d2 = 0.0f;
    if (liq.n > 0) {
      d2 = LDG(&liq.q[0][o]);
      for (int n = 1; n < liq.n; n++) d2 = d2 + LDG(&liq.q[n][o]);
    }
    const float d3 = 0.0f;
    const float qli = fmaxf(0.0f, d2 + d3);
    // buoyancy dum8 at s-points (solve2.F:395-396) when liquid is present;
    // without it k_mom_tile forms the same expression from theta and qv
    if (liq.b8)
      liq.b8[o] = c.g * ((th3 * LDG(&g.rth0[k]) + c.repsm1 * (q - LDG(&g.qv0[k]))) -
                         ((qli - LDG(&g.qc0[k])) - LDG(&g.qi0[k])));
    t11[o] = (th0 + th3) * (1.0f + c.reps * q) / ((1.0f + q) + qli);
    if (eqtset == 2) {
      const float cpli = c.cpl * fmaxf(0.0f, d2) + c.cpi * fmaxf(0.0f, d3);
      const float cpm = (c.cp + c.cpv * q) + cpli;
      const float cvm = 1.0f / ((c.cv + c.cvv * q) + cpli);
      thterm[o] = (th0 + th3) * ((c.rd + c.rv * q) - c.rovcp * cpm) * cvm;
      t22[o] = (pi0 + pp) * c.rovcp * cpm * cvm;
    } else {
      t22[o] = (pi0 + pp) * c.rddcv;
    }
  } else {
    t11[o] = th0 + th3;
    t22[o] = (pi0 + pp) * c.rddcv;
  }
}

void launch_stage_prep(const DGrid &g, const float *th3d, const float *pp3d, const float *qv, const LiquidIn &liq,
                       int imoist, int eqtset, float *t11, float *t22, float *thterm, float *piadv, cudaStream_t st,
                       int64_t *nl) {
  dim3 grid((g.ni + 2 + 127) / 128, g.nj + 2, g.nk);
  // j index offset: blockIdx.y = j directly (0..nj+1)
  { ProfScope _ps("k_stage_prep", st); k_stage_prep<<<grid, 128, 0, st>>>(g, th3d, pp3d, qv, liq, imoist, eqtset, t11, t22, thterm, piadv); }
  if (nl) *nl += 1;
}

// ---------------------------------------------------------------------
// radbcew4 / radbcns4 (bc.F:2054-2178): column-averaged phase speeds
// ---------------------------------------------------------------------
// One warp per boundary column: the lanes form the phase speeds of 32
// levels at a time, every lane adds them (exchanged by shuffles) in the
// reference's order k = 1..nk, and the lanes write the column average back.
__global__ void k_radbc4(DGrid g, const float *__restrict__ ua, const float *__restrict__ u3d,
                         const float *__restrict__ va, const float *__restrict__ v3d,
                         float *radbcw, float *radbce, float *radbcs, float *radbcn, float dt) {
  const int wib = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
  const int t = (int)blockIdx.x * 4 + wib;     // column along the side
  const int side = (int)blockIdx.y;            // 0 w, 1 e, 2 s, 3 n
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const float umax = 350.0f;                   // csmax, constants.F:45
  const bool ew = side <= 1;
  const int n = ew ? nj : ni;
  bool on = (1 + t <= n);
  if (side == 0) on = on && g.ibw && g.wbc == 2;
  if (side == 1) on = on && g.ibe && g.ebc == 2;
  if (side == 2) on = on && g.ibs && g.sbc == 2;
  if (side == 3) on = on && g.ibn && g.nbc == 2;
  if (!on) return;                             // whole warp leaves together
  // phase speed of level k (0 outside 1..nk)
  auto speed = [&](int k) -> float {
    if (k > nk) return 0.0f;
    if (ew) {
      const int j = 1 + t;
      const int ia = (side == 0) ? 2 : ni, ib2 = (side == 0) ? 3 : ni - 1;
      const float ruf = LDG(&g.ruf[ia - g.ib]);
      float foo = (side == 0) ? (ua[iU(g, ib2, j, k)] - ua[iU(g, ia, j, k)]) : (ua[iU(g, ia, j, k)] - ua[iU(g, ib2, j, k)]);
      float c = g.dx * ruf * (ua[iU(g, ia, j, k)] - u3d[iU(g, ia, j, k)]) / (dt * (copysignf(1.e-10f, foo) + foo));
      return (side == 0) ? fmaxf(fminf(c, 0.0f), -umax) : fminf(fmaxf(c, 0.0f), umax);
    }
    const int i = 1 + t;
    const int ja = (side == 2) ? 2 : nj, jb2 = (side == 2) ? 3 : nj - 1;
    const float rvf = LDG(&g.rvf[ja - g.jb]);
    float foo = (side == 2) ? (va[iV(g, i, jb2, k)] - va[iV(g, i, ja, k)]) : (va[iV(g, i, ja, k)] - va[iV(g, i, jb2, k)]);
    float c = g.dy * rvf * (va[iV(g, i, ja, k)] - v3d[iV(g, i, ja, k)]) / (dt * (copysignf(1.e-10f, foo) + foo));
    return (side == 2) ? fmaxf(fminf(c, 0.0f), -umax) : fminf(fmaxf(c, 0.0f), umax);
  };
  float avg = 0.0f;
  for (int k0 = 1; k0 <= nk; k0 += 32) {
    const float c = speed(k0 + lane);
#pragma unroll
    for (int m = 0; m < 32; m++) {
      const float cm = __shfl_sync(0xffffffffu, c, m);
      if (k0 + m <= nk) avg = avg + cm;
    }
  }
  avg = avg / (float)nk;
  float *r = (side == 0) ? radbcw : (side == 1) ? radbce : (side == 2) ? radbcs : radbcn;
  for (int k = 1 + lane; k <= nk; k += 32) {
    if (ew) r[(1 + t - g.jb) + (long)g.NJ * k] = avg;
    else r[(1 + t - g.ib) + (long)g.NI * k] = avg;
  }
}

void launch_radbc4(const DGrid &g, const float *ua, const float *u3d, const float *va, const float *v3d,
                   float *rw, float *re, float *rs, float *rn, float dt, cudaStream_t st, int64_t *nl) {
  int n = g.ni > g.nj ? g.ni : g.nj;
  dim3 grid((n + 3) / 4, 4);
  { ProfScope _ps("k_radbc4", st); k_radbc4<<<grid, 128, 0, st>>>(g, ua, u3d, va, v3d, rw, re, rs, rn, dt); }
  if (nl) *nl += 1;
}

// radbcew / radbcns with irbc = 1 (bc.F:1948-2046, called by solve1.F:403-409
// before the RK loop): the Klemp-Wilhelmson phase speeds of the step from ua
// and va, u - cstar where negative (west, south), u + cstar where positive
// (east, north), else 0.  One thread per boundary column and level.
__global__ void k_radbc_kw(DGrid g, const float *__restrict__ ua, const float *__restrict__ va, float *rw, float *re,
                           float *rs, float *rn) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x), k = 1 + (int)blockIdx.y;
  if (t < g.nj) {
    const int j = 1 + t;
    const long o = (j - g.jb) + (long)g.NJ * k;
    if (g.ibw && g.wbc == 2) { const float c = LDG(&ua[iU(g, 1, j, k)]) - g.cstar; rw[o] = (c < 0.0f) ? c : 0.0f; }
    if (g.ibe && g.ebc == 2) { const float c = LDG(&ua[iU(g, g.ni + 1, j, k)]) + g.cstar; re[o] = (c > 0.0f) ? c : 0.0f; }
  }
  if (t < g.ni) {
    const int i = 1 + t;
    const long o = (i - g.ib) + (long)g.NI * k;
    if (g.ibs && g.sbc == 2) { const float c = LDG(&va[iV(g, i, 1, k)]) - g.cstar; rs[o] = (c < 0.0f) ? c : 0.0f; }
    if (g.ibn && g.nbc == 2) { const float c = LDG(&va[iV(g, i, g.nj + 1, k)]) + g.cstar; rn[o] = (c > 0.0f) ? c : 0.0f; }
  }
}

void launch_radbc_kw(const DGrid &g, const float *ua, const float *va, float *rw, float *re, float *rs, float *rn,
                     cudaStream_t st, int64_t *nl) {
  const int n = g.ni > g.nj ? g.ni : g.nj;
  dim3 grid((n + 127) / 128, g.nk);
  { ProfScope _ps("k_radbc_kw", st); k_radbc_kw<<<grid, 128, 0, st>>>(g, ua, va, rw, re, rs, rn); }
  if (nl) *nl += 1;
}

// ---------------------------------------------------------------------
// pressure and density (solve2.F:1580-1606) with the per-level FP64
// sums of apmasscon (solve2.F:1617-1648).  Block (x, k) covers a chunk of
// level k and writes its partial sums; k_masscon_finish adds them in a
// fixed order.
// ---------------------------------------------------------------------
__device__ __forceinline__ void prs_rho(const DGrid &g, float pp, float th3, const float *qv, long o, int k,
                                        int imoist, float *prs, float *rho) {
  const Consts &c = g.c;
  const float pi = LDG(&g.pi0[k]) + pp;
  // pi**(cp/rd) in binary64, rounded once: the correctly rounded binary32
  // power, which is what the reference's powf (glibc) returns for all but
  // rare inputs.  A last-place difference here moves rho, hence the FP64
  // mass sum of apmasscon, hence the uniform pi' shift of the mass fix,
  // which on near-uniform pressure fields (the CBL) is a visible fraction
  // of pi''s range.
  const float pr = 1.0e5f * (float)pow((double)pi, (double)c.cpdrd);
  prs[o] = pr;
  if (imoist) rho[o] = pr / ((LDG(&g.th0[k]) + th3) * pi * (c.rd + fmaxf(0.0f, LDG(&qv[o])) * c.rv));
  else rho[o] = pr / (c.rd * (LDG(&g.th0[k]) + th3) * pi);
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red) {
  const int t = threadIdx.x;
  red[t] = v;
  __syncthreads();
  for (int s = NT / 2; s > 0; s >>= 1) {
    if (t < s) red[t] = red[t] + red[t + s];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

static const int PR_NT = 256, PR_PER = 8;

__global__ void __launch_bounds__(PR_NT) k_prs_rho(DGrid g, const float *__restrict__ pp3d, const float *__restrict__ th3d,
                                                   const float *__restrict__ qv, int imoist, float *prs, float *rho,
                                                   double *part3, double *part4, int nchunk, int do_sums) {
  __shared__ double red[PR_NT];
  const int k = 1 + (int)blockIdx.y;
  const long npl = (long)g.ni * g.nj;
  const long base = (long)blockIdx.x * PR_NT * PR_PER;
  double s3 = 0.0, s4 = 0.0;
  for (int r = 0; r < PR_PER; r++) {
    long t = base + (long)r * PR_NT + threadIdx.x;
    if (t >= npl) break;
    int i = 1 + (int)(t % g.ni), j = 1 + (int)(t / g.ni);
    long o = iS(g, i, j, k);
    float pp = LDG(&pp3d[o]);
    prs_rho(g, pp, LDG(&th3d[o]), qv, o, k, imoist, prs, rho);
    if (do_sums) {
      s3 = s3 + (double)(rho[o] * LDG(&g.ruh[i - g.ib]) * LDG(&g.rvh[j - g.jb]) * LDG(&g.rmh[k]));
      s4 = s4 + (double)(LDG(&g.pi0[k]) + pp);
    }
  }
  if (!do_sums) return;
  s3 = block_sum<PR_NT>(s3, red);
  s4 = block_sum<PR_NT>(s4, red);
  if (threadIdx.x == 0) {
    part3[(long)k * nchunk + blockIdx.x] = s3;
    part4[(long)k * nchunk + blockIdx.x] = s4;
  }
}

// mass2, tem (solve2.F:1985-2000); dev[0] = mass2, dev[1] = p2, devf[0] = tem
__global__ void k_masscon_finish(DGrid g, const double *part3, const double *part4, int nchunk, double mass1,
                                 double *dev, float *devf) {
  __shared__ double red[128];
  double t3 = 0.0, t4 = 0.0;
  for (int k = 1 + (int)threadIdx.x; k <= g.nk; k += blockDim.x) {
    double a = 0.0, b = 0.0;
    for (int c = 0; c < nchunk; c++) { a = a + part3[(long)k * nchunk + c]; b = b + part4[(long)k * nchunk + c]; }
    t3 = t3 + a; t4 = t4 + b;
  }
  t3 = block_sum<128>(t3, red);
  t4 = block_sum<128>(t4, red);
  if (threadIdx.x == 0) {
    double mass2 = t3, p2 = t4;
    double n = (double)((long long)g.ni * g.nj * g.nk);
    dev[0] = mass2; dev[1] = p2;
    devf[0] = (float)((pow(mass1 / mass2, (double)g.c.rddcv) - 1.0) * p2 / n);
  }
}

__global__ void k_masscon_apply(DGrid g, float *pp3d, const float *__restrict__ th3d, const float *__restrict__ qv,
                                int imoist, float *prs, float *rho, const float *devf) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni) return;
  const long o = iS(g, i, j, k);
  const float tem = devf[0];
  const float pp = pp3d[o] + tem;
  pp3d[o] = pp;
  prs_rho(g, pp, LDG(&th3d[o]), qv, o, k, imoist, prs, rho);
}

// rr = 1/rho over the physical cells and one halo cell (solve3.F:660-675,
// solve2.F:2036-2046): the reciprocal the scalar form of the 6th-order
// diffusion multiplies by.
__global__ void k_recip_rho(DGrid g, const float *__restrict__ rho, float *rr) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x), j = (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni + 1) return;
  const long o = iS(g, i, j, k);
  rr[o] = 1.0f / LDG(&rho[o]);
}

void launch_recip_rho(const DGrid &g, const float *rho, float *rr, cudaStream_t st, int64_t *nl) {
  dim3 grid((g.ni + 2 + 127) / 128, g.nj + 2, g.nk);
  { ProfScope _ps("k_recip_rho", st); k_recip_rho<<<grid, 128, 0, st>>>(g, rho, rr); }
  if (nl) *nl += 1;
}

int prs_nchunk(const DGrid &g) { return (int)(((long)g.ni * g.nj + PR_NT * PR_PER - 1) / (PR_NT * PR_PER)); }

void launch_prs_rho(const DGrid &g, const float *pp3d, const float *th3d, const float *qv, int imoist,
                    float *prs, float *rho, double *part3, double *part4, int do_sums, cudaStream_t st, int64_t *nl) {
  int nchunk = prs_nchunk(g);
  dim3 grid(nchunk, g.nk);
  { ProfScope _ps("k_prs_rho", st); k_prs_rho<<<grid, PR_NT, 0, st>>>(g, pp3d, th3d, qv, imoist, prs, rho, part3, part4, nchunk, do_sums); }
  if (nl) *nl += 1;
}

void launch_masscon(const DGrid &g, float *pp3d, const float *th3d, const float *qv, int imoist, float *prs,
                    float *rho, const double *part3, const double *part4, double mass1, double *dev, float *devf,
                    cudaStream_t st, int64_t *nl) {
  { ProfScope _ps("k_masscon_finish", st); k_masscon_finish<<<1, 128, 0, st>>>(g, part3, part4, prs_nchunk(g), mass1, dev, devf); }
  dim3 grid((g.ni + 127) / 128, g.nj, g.nk);
  { ProfScope _ps("k_masscon_apply", st); k_masscon_apply<<<grid, 128, 0, st>>>(g, pp3d, th3d, qv, imoist, prs, rho, devf); }
  if (nl) *nl += 2;
}

// ---------------------------------------------------------------------
// calccflquick (misclibs.F:2726-2814): max Courant number, stored as the
// bits of a non-negative float so atomicMax on int orders it correctly.
// ---------------------------------------------------------------------
// Each block walks all levels of a 128-column strip of one row and reduces
// in registers, shuffles and shared memory, so one atomic per block
// (instead of one per warp) reaches the result.
__global__ void k_cfl(DGrid g, const float *__restrict__ u, const float *__restrict__ v, const float *__restrict__ w,
                      float dt, int *out) {
  __shared__ float red[4];
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y;
  float wmax = 0.0f;
  if (i <= g.ni) {
    const float dtdx = 0.5f * dt * g.rdx, dtdy = 0.5f * dt * g.rdy, dtdz = 0.5f * dt * g.rdz;
    const float uh = LDG(&g.uh[i - g.ib]), vh = LDG(&g.vh[j - g.jb]);
    for (int k = 1; k <= g.nk; k++) {
      float a1 = (LDG(&u[iU(g, i, j, k)]) + LDG(&u[iU(g, i + 1, j, k)])) * dtdx * uh;
      float a2 = (LDG(&v[iV(g, i, j, k)]) + LDG(&v[iV(g, i, j + 1, k)])) * dtdy * vh;
      float a3 = (LDG(&w[iW(g, i, j, k)]) + LDG(&w[iW(g, i, j, k + 1)])) * dtdz * LDG(&g.mh[k]);
      float wsp = sqrtf((a1 * a1 + a2 * a2) + a3 * a3);
      if (!(wsp <= 3.0e38f)) wsp = INFINITY;   // NaN/Inf velocity: reported as an error by the host
      wmax = fmaxf(wmax, wsp);
    }
  }
  for (int s = 16; s > 0; s >>= 1) wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, s));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = wmax;
  __syncthreads();
  if (threadIdx.x == 0) atomicMax(out, __float_as_int(fmaxf(fmaxf(red[0], red[1]), fmaxf(red[2], red[3]))));
}

void launch_cfl(const DGrid &g, const float *u, const float *v, const float *w, float dt, int *out,
                cudaStream_t st, int64_t *nl) {
  cudaMemsetAsync(out, 0, sizeof(int), st);
  dim3 grid((g.ni + 127) / 128, g.nj);
  { ProfScope _ps("k_cfl", st); k_cfl<<<grid, 128, 0, st>>>(g, u, v, w, dt, out); }
  if (nl) *nl += 1;
}

// ---------------------------------------------------------------------
// pdefq (misclibs.F:1037-1117), pdscheme=1: per-column mass-conserving
// clipping.  bud[j*ni+i-1] receives a2-a1 of the column.
// ---------------------------------------------------------------------
// The column is walked in chunks of PQ levels whose loads are issued
// together; the sums still run k = 1..nk in order.
__global__ void k_pdefq(DGrid g, float rmax, const float *__restrict__ rho, float *__restrict__ q, double *bud) {
  constexpr int PQ = 12;   // levels of a column loaded together (latency: one thread per column)
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y;
  if (i > g.ni) return;
  const float ruh = LDG(&g.ruh[i - g.ib]), rvh = LDG(&g.rvh[j - g.jb]);
  const long plane = (long)g.NI * g.NJ, oc = iS(g, i, j, 0);
  const int nk = g.nk;
  double t1 = 0.0, t2 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int k0 = 1; k0 <= nk; k0 += PQ) {
    float rr[PQ], qq[PQ];
#pragma unroll
    for (int m = 0; m < PQ; m++) {
      const int k = k0 + m;
      rr[m] = (k <= nk) ? LDG(&rho[oc + k * plane]) : 0.0f;
      qq[m] = (k <= nk) ? q[oc + k * plane] : 0.0f;
    }
#pragma unroll
    for (int m = 0; m < PQ; m++) {
      const int k = k0 + m;
      if (k > nk) break;
      const float r = rr[m], rmh = LDG(&g.rmh[k]);
      float v = qq[m];
      t1 = t1 + (double)(r * v);
      a1 = a1 + (double)(r * v * ruh * rvh * rmh);
      if (v < rmax) { v = 0.0f; q[oc + k * plane] = v; }
      t2 = t2 + (double)(r * v);
    }
  }
  double t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20);
  if (t3 < 0.0) t3 = 1.0;
  for (int k0 = 1; k0 <= nk; k0 += PQ) {
    float rr[PQ], qq[PQ];
#pragma unroll
    for (int m = 0; m < PQ; m++) {
      const int k = k0 + m;
      rr[m] = (k <= nk) ? LDG(&rho[oc + k * plane]) : 0.0f;
      qq[m] = (k <= nk) ? q[oc + k * plane] : 0.0f;
    }
#pragma unroll
    for (int m = 0; m < PQ; m++) {
      const int k = k0 + m;
      if (k > nk) break;
      const float v = (float)(t3 * (double)qq[m]);
      q[oc + k * plane] = v;
      a2 = a2 + (double)(rr[m] * v * ruh * rvh * LDG(&g.rmh[k]));
    }
  }
  if (bud) bud[(long)(j - 1) * g.ni + (i - 1)] = a2 - a1;
}

// budget: asq += sum_j (sum_i bud) * dx*dy*dz, fixed order
__global__ void k_pdefq_budget(DGrid g, const double *bud, double *asq) {
  __shared__ double red[128];
  double s = 0.0;
  for (int j = 1 + (int)threadIdx.x; j <= g.nj; j += blockDim.x) {
    double bj = 0.0;
    for (int i = 0; i < g.ni; i++) bj = bj + bud[(long)(j - 1) * g.ni + i];
    s = s + bj * (double)(g.dx * g.dy * g.dz);
  }
  s = block_sum<128>(s, red);
  if (threadIdx.x == 0) asq[0] = asq[0] + s;
}

void launch_pdefq(const DGrid &g, float rmax, const float *rho, float *q, double *bud, double *asq,
                  cudaStream_t st, int64_t *nl) {
  dim3 grid((g.ni + 127) / 128, g.nj);
  { ProfScope _ps("k_pdefq", st); k_pdefq<<<grid, 128, 0, st>>>(g, rmax, rho, q, bud); }
  if (asq) { ProfScope _ps("k_pdefq_budget", st); k_pdefq_budget<<<1, 128, 0, st>>>(g, bud, asq); }
  if (nl) *nl += 2;
}

// ---------------------------------------------------------------------
// solve3 pieces: ppx = pp3d + ppx (solve3.F:276-283) and the rollover
// copies over the reference's ranges (solve3.F:546-640).
// ---------------------------------------------------------------------
__global__ void k_ppx_update(DGrid g, const float *__restrict__ pp3d, float *ppx) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni) return;
  const long o = iS(g, i, j, k);
  ppx[o] = LDG(&pp3d[o]) + ppx[o];
}

// Rollover copies dst = src over i = ilo..ihi, j = jlo..jhi, k = 1..nk
// (solve3.F:546-640) for up to CP_MAXB arrays in one launch: blockIdx.y
// picks the array, each warp copies one row segment (coalesced along i).
static const int CP_MAXB = 16;
struct CopyItem {
  const float *src;
  float *dst;
  long pitch, plane;
  int ilo, ihi, jlo, jhi;
};
struct CopyBatch {
  CopyItem it[CP_MAXB];
  int n, nk, ib, jb;
};

__global__ void k_copy_batch(CopyBatch b) {
  const CopyItem c = b.it[blockIdx.y];
  const int warp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = (int)(threadIdx.x & 31);
  const int nrow = c.jhi - c.jlo + 1;
  if (warp >= nrow * b.nk) return;
  const int k = 1 + warp / nrow, j = c.jlo + warp % nrow;
  const long base = (long)(j - b.jb) * c.pitch + (long)k * c.plane - b.ib;
  for (int i = c.ilo + lane; i <= c.ihi; i += 32) c.dst[base + i] = LDG(&c.src[base + i]);
}

void launch_ppx_update(const DGrid &g, const float *pp3d, float *ppx, cudaStream_t st, int64_t *nl) {
  dim3 grid((g.ni + 127) / 128, g.nj, g.nk);
  { ProfScope _ps("k_ppx_update", st); k_ppx_update<<<grid, 128, 0, st>>>(g, pp3d, ppx); }
  if (nl) *nl += 1;
}

// stag: 1 s, 2 u, 3 v, 4 w layout of each array
void launch_copy_batch(const DGrid &g, const float *const *src, float *const *dst, const int *stag, const int *ilo,
                       const int *ihi, const int *jlo, const int *jhi, int n, cudaStream_t st, int64_t *nl) {
  for (int base = 0; base < n; base += CP_MAXB) {
    CopyBatch b{};
    b.n = (n - base < CP_MAXB) ? n - base : CP_MAXB;
    b.nk = g.nk; b.ib = g.ib; b.jb = g.jb;
    int maxrows = 0;
    for (int q = 0; q < b.n; q++) {
      const int t = base + q;
      const long pitch = (stag[t] == 2) ? g.NI + 1 : g.NI, rows = (stag[t] == 3) ? g.NJ + 1 : g.NJ;
      b.it[q] = CopyItem{src[t], dst[t], pitch, pitch * rows, ilo[t], ihi[t], jlo[t], jhi[t]};
      const int r = (jhi[t] - jlo[t] + 1) * g.nk;
      if (r > maxrows) maxrows = r;
    }
    dim3 grid((maxrows + 7) / 8, b.n);
    { ProfScope _ps("k_copy_batch", st); k_copy_batch<<<grid, 256, 0, st>>>(b); }
    if (nl) *nl += 1;
  }
}

// ---------------------------------------------------------------------
// pre-RK tendencies of solve1 (solve1.F:414-486): Rayleigh damping of u, v,
// w, theta (irdamp=1: toward the base state; irdamp=2: toward the mean
// profiles uavg/vavg/thavg), else zero, on i = 1..ni+1, j = 1..nj+1,
// k = 1..nk; the moisture and tracer tendencies are zeroed on the interior.
// ---------------------------------------------------------------------

__global__ void k_tend_init(DGrid g, TendIn t) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni + 1) return;
  const long o = iS(g, i, j, k), ou = iU(g, i, j, k), ov = iV(g, i, j, k);
  const float ra = t.rdalpha;
  if (t.irdamp == 1 || t.irdamp == 2) {
    const float tu = LDG(&t.tauh[o - 1]) + LDG(&t.tauh[o]);
    const float tv = LDG(&t.tauh[o - g.NI]) + LDG(&t.tauh[o]);
    const float ur = (t.irdamp == 1) ? LDG(&g.u0[ou]) : LDG(&t.uavg[k]);
    const float vr = (t.irdamp == 1) ? LDG(&g.v0[ov]) : LDG(&t.vavg[k]);
    t.uten1[ou] = -(ra * 0.5f * tu * (LDG(&t.ua[ou]) - ur));
    t.vten1[ov] = -(ra * 0.5f * tv * (LDG(&t.va[ov]) - vr));
    t.wten1[o] = -(ra * LDG(&t.tauf[o]) * LDG(&t.wa[o]));
    const float th = (t.irdamp == 1) ? LDG(&t.tha[o]) : (LDG(&g.th0[k]) - LDG(&t.thavg[k])) + LDG(&t.tha[o]);
    t.thten1[o] = -(ra * LDG(&t.taus[o]) * th);
  } else {
    t.uten1[ou] = 0.0f; t.vten1[ov] = 0.0f; t.wten1[o] = 0.0f; t.thten1[o] = 0.0f;
  }
  if (i <= g.ni && j <= g.nj)
    for (int n = 0; n < t.nq; n++) {
      float *q = (n < t.numq) ? t.qten + (long)n * nS(g) : t.ptten + (long)(n - t.numq) * nS(g);
      q[o] = 0.0f;
    }
}

void launch_tend_init(const DGrid &g, const TendIn &t, cudaStream_t st, int64_t *nl) {
  dim3 grid((g.ni + 1 + 127) / 128, g.nj + 1, g.nk);
  { ProfScope _ps("k_tend_init", st); k_tend_init<<<grid, 128, 0, st>>>(g, t); }
  if (nl) *nl += 1;
}

// ---------------------------------------------------------------------
// calcener (misclibs.F:3343-3454, umove = vmove = 0): FP64 kinetic,
// internal, potential and latent energy.  Per-cell terms keep the
// reference's operand kinds (binary32 factors promoted where a binary64
// operand meets them); block (x, k) adds its chunk of level k, and
// k_ener_finish adds the chunks and then the levels in a fixed order.
// ---------------------------------------------------------------------
static const int EN_NT = 256, EN_PER = 8;

__global__ void __launch_bounds__(EN_NT) k_ener_part(DGrid g, EnerIn e, double *part, int nchunk) {
  __shared__ double red[EN_NT];
  const int k = 1 + (int)blockIdx.y;
  const long npl = (long)g.ni * g.nj;
  const long base = (long)blockIdx.x * EN_NT * EN_PER;
  const Consts &c = g.c;
  double f1 = 0.0, f2 = 0.0, f3 = 0.0, f4 = 0.0;
  for (int r = 0; r < EN_PER; r++) {
    const long t = base + (long)r * EN_NT + threadIdx.x;
    if (t >= npl) break;
    const int i = 1 + (int)(t % g.ni), j = 1 + (int)(t / g.ni);
    const long o = iS(g, i, j, k), ou = iU(g, i, j, k), ov = iV(g, i, j, k);
    const double tem = (double)(LDG(&g.ruh[i - g.ib]) * LDG(&g.rvh[j - g.jb]) * LDG(&g.rmh[k]));
    const float u1 = LDG(&e.ua[ou]), u2 = LDG(&e.ua[ou + 1]), v1 = LDG(&e.va[ov]), v2 = LDG(&e.va[ov + g.NI]);
    const float w1 = LDG(&e.wa[o]), w2 = LDG(&e.wa[o + (long)g.NI * g.NJ]);
    const double ww = (double)(0.5f * (w1 + w2));
    const float q_v = e.qv ? LDG(&e.qv[o]) : 0.0f, q_l = e.ql ? LDG(&e.ql[o]) : 0.0f;
    const float q_i = e.qi ? LDG(&e.qi[o]) : 0.0f, v_r = e.vr ? LDG(&e.vr[o]) : 0.0f;
    const double qtot = (double)((q_v + q_l) + q_i);
    const float rr = LDG(&e.rho[o]);
    const float ke = (0.5f * (u1 * u1 + u2 * u2) + 0.5f * (v1 * v1 + v2 * v2)) + 0.5f * (w1 * w1 + w2 * w2);
    f1 = (f1 + (double)rr * tem * (1.0 + qtot) * 0.5 * (double)ke) +
         (double)(q_l * rr) * tem * 0.5 * ((double)(v_r * v_r) - 2.0 * ww * (double)v_r);
    const double tmp = (double)((LDG(&g.th0[k]) + LDG(&e.tha[o])) * (LDG(&g.pi0[k]) + LDG(&e.ppi[o])));
    f2 = f2 + (double)rr * tem * (double)(c.cv + c.cvv * q_v) * tmp;
    f3 = f3 + (double)rr * tem * (1.0 + qtot) * (double)c.g * (double)LDG(&e.zh[o]);
    f4 = (f4 + (double)rr * tem * (double)q_l * ((double)c.cpl * tmp - (double)e.lv1)) +
         (double)rr * tem * (double)q_i * ((double)c.cpi * tmp - (double)e.ls1);
  }
  double s[4] = {f1, f2, f3, f4};
  for (int q = 0; q < 4; q++) {
    red[threadIdx.x] = s[q];
    __syncthreads();
    for (int h = EN_NT / 2; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[((long)q * g.nk + (k - 1)) * nchunk + blockIdx.x] = red[0];
    __syncthreads();
  }
}

__global__ void k_ener_finish(DGrid g, const double *part, int nchunk, double *out) {
  const int q = (int)threadIdx.x;   // 0 ek, 1 ei, 2 ep, 3 le
  if (q >= 4) return;
  double tot = 0.0;
  for (int k = 0; k < g.nk; k++) {
    double f = 0.0;
    for (int c = 0; c < nchunk; c++) f = f + part[((long)q * g.nk + k) * nchunk + c];
    tot = tot + f;
  }
  out[q] = tot * (double)(g.dx * g.dy * g.dz);
}

int ener_chunks(const DGrid &g) { return (int)(((long)g.ni * g.nj + EN_NT * EN_PER - 1) / (EN_NT * EN_PER)); }

void launch_calcener(const DGrid &g, const EnerIn &e, double *part, double *out, cudaStream_t st, int64_t *nl) {
  const int nchunk = ener_chunks(g);
  dim3 grid(nchunk, g.nk);
  { ProfScope _ps("k_ener_part", st); k_ener_part<<<grid, EN_NT, 0, st>>>(g, e, part, nchunk); }
  { ProfScope _ps("k_ener_finish", st); k_ener_finish<<<1, 32, 0, st>>>(g, part, nchunk, out); }
  if (nl) *nl += 2;
}

// ---------------------------------------------------------------------
// calcmass (misclibs.F:3134-3191) and maxmin (maxmin.F:5-119)
// ---------------------------------------------------------------------
__global__ void k_level_mass(DGrid g, const float *__restrict__ rho, double *lev) {
  __shared__ double red[256];
  const int k = 1 + (int)blockIdx.x;
  double s = 0.0;
  for (long t = threadIdx.x; t < (long)g.ni * g.nj; t += blockDim.x) {
    int i = 1 + (int)(t % g.ni), j = 1 + (int)(t / g.ni);
    s = s + (double)(LDG(&rho[iS(g, i, j, k)]) * LDG(&g.ruh[i - g.ib]) * LDG(&g.rvh[j - g.jb]) * LDG(&g.rmh[k]));
  }
  s = block_sum<256>(s, red);
  if (threadIdx.x == 0) lev[k] = s;
}

void launch_level_mass(const DGrid &g, const float *rho, double *lev, cudaStream_t st, int64_t *nl) {
  { ProfScope _ps("k_level_mass", st); k_level_mass<<<g.nk, 256, 0, st>>>(g, rho, lev); }
  if (nl) *nl += 1;
}

// max and min with the first (i fastest, then j, then k) location of each;
// ties resolve to the lowest linear index as the serial loop does.
__global__ void k_maxmin(DGrid g, const float *__restrict__ a, int stag, unsigned long long *omax,
                         unsigned long long *omin) {
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3), ke = g.nk + (stag == 4);
  const long n = (long)ie * je * ke;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int i = 1 + (int)(t % ie), j = 1 + (int)((t / ie) % je), k = 1 + (int)(t / ((long)ie * je));
  const long o = stag == 2 ? iU(g, i, j, k) : stag == 3 ? iV(g, i, j, k) : iS(g, i, j, k);
  float v = LDG(&a[o]);
  // order-preserving key: float bits mapped to unsigned, index in the low word
  unsigned int b = __float_as_uint(v);
  unsigned int key = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  unsigned int idx = (unsigned int)t;
  atomicMax(omax, ((unsigned long long)key << 32) | (unsigned long long)(0xffffffffu - idx));
  atomicMin(omin, ((unsigned long long)key << 32) | (unsigned long long)idx);
}

void launch_maxmin(const DGrid &g, const float *a, int stag, unsigned long long *om, cudaStream_t st, int64_t *nl) {
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3), ke = g.nk + (stag == 4);
  long n = (long)ie * je * ke;
  cudaMemsetAsync(om, 0, sizeof(unsigned long long), st);
  cudaMemsetAsync(om + 1, 0xff, sizeof(unsigned long long), st);
  { ProfScope _ps("k_maxmin", st); k_maxmin<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, a, stag, om, om + 1); }
  if (nl) *nl += 1;
}

}  // namespace cm1g
