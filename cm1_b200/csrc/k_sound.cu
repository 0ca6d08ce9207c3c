// k_sound.cu -- acoustic substeps of sound.F (psolver=3, no terrain).
//
// One kernel per small step.  A thread owns one (i,j) column and walks it
// twice: upward it forms the new u, v (pressure-gradient update, sound.F:
// 321-341, with the open-boundary updates of bc.F:2392-2686 folded in), the
// explicit pi' forcing fpk (sound.F:479-502) and the forward elimination of
// the vertically implicit w equation (sound.F:659-716); downward it
// back-substitutes w (sound.F:718-733), updates pi' with divergence damping
// (sound.F:746-760) and accumulates the small-step-averaged velocities
// (sound.F:806-835).  The column recursion lives in shared memory.
//
// Neighbour columns read u, v and ppd from the previous small step, so u, v
// and ppd are double-buffered; w and pi' are only read by their own column
// and are updated in place.  The east/north face velocity of a cell is
// recomputed from the same old values by the neighbour that needs it, which
// reproduces the stored value exactly.
#include "cm1g_common.cuh"

namespace cm1g {

struct SoundIO {
  const float *u_in, *v_in;       // u, v before this small step (full halo)
  float *u_out, *v_out;           // u, v after it
  const float *w_in;              // w before (== w_out after the first step)
  float *w_out;
  const float *pp_in;             // pi' before (== pp_out after the first step)
  float *pp_out;
  const float *ppd_in;            // damped pi' (1-point halo)
  float *ppd_out;
  float *rru, *rrv, *rrw;         // running sums / averages
  const float *wa;                // start-of-stage w (first step: rrw = wa*beta)
  const float *uten, *vten, *wten, *ppten;
  const float *thv, *ppterm, *piadv;
  const float *radbcw, *radbce, *radbcs, *radbcn;
  float *ppx;                     // last step of the final stage: kdiv*(pi'_new - pi'_old)
};

struct SoundStep {
  float dts, tavg;
  int first, last, write_ppx;
};

#define RJK(g, a, j, k) ((a)[((j) - (g).jb) + (long)(g).NJ * (k)])
#define RIK(g, a, i, k) ((a)[((i) - (g).ib) + (long)(g).NI * (k)])

template <int NT>
__global__ void __launch_bounds__(NT) k_sound_step(DGrid g, SoundIO io, SoundStep p) {
  extern __shared__ float sm[];
  const int tid = threadIdx.x + blockDim.x * threadIdx.y;
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const bool active = (i <= ni && j <= nj);
  if (!active) return;
  float *s_pf = sm;                 // pi'_old + fpk       [k*NT + tid]
  float *s_d1 = sm + (nk + 2) * NT; // LU factor dum1
  float *s_d2 = sm + 2 * (nk + 2) * NT;
#define SM(a, k) a[(k) * NT + tid]

  const float dts = p.dts, alph = g.alph, beta = 1.0f - alph, asq = alph * alph;
  const float cp = g.c.cp, rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
  const float tem1pg = rdx * cp * 0.5f, tem2pg = rdy * cp * 0.5f;      // sound.F:321-322
  const float temx = dts * 0.5f * rdx, temy = dts * 0.5f * rdy;        // sound.F:479-480
  const float uh_i = LDG(&g.uh[i - g.ib]), vh_j = LDG(&g.vh[j - g.jb]);
  const float uf_i = LDG(&g.uf[i - g.ib]), uf_ip = LDG(&g.uf[i + 1 - g.ib]);
  const float vf_j = LDG(&g.vf[j - g.jb]), vf_jp = LDG(&g.vf[j + 1 - g.jb]);
  const float dtu_i = dts * LDG(&g.dtu0[i2(g, i, j)]), dtu_ip = dts * LDG(&g.dtu0[i2(g, i + 1, j)]);
  const float dtv_j = dts * LDG(&g.dtv0[i2(g, i, j)]), dtv_jp = dts * LDG(&g.dtv0[i2(g, i, j + 1)]);
  const bool openw = (g.wbc == 2 && g.ibw && i == 1), opene = (g.ebc == 2 && g.ibe && i == ni);
  const bool opens = (g.sbc == 2 && g.ibs && j == 1), openn = (g.nbc == 2 && g.ibn && j == nj);

  // ---------------- upward pass ----------------
  float pk1p = 0.f, pk2p = 0.f, qkp = 0.f, ppp = 0.f, pfp = 0.f, d1p = 0.f, d2p = 0.f, wlast = 0.f;
  for (int k = 1; k <= nk; k++) {
    // stage coefficients (sound.F:117-135, 188-189)
    const float mhk = LDG(&g.mh[k]), rr0k = LDG(&g.rr0[k]);
    const float temq = dts * rdz * mhk;
    const float r2 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k + 1]);
    const float r1 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k]);
    const float temm = dts * rdz * cp * LDG(&g.mf[k]);
    const float c1a = LDG(&g.c1[k]), c1b = LDG(&g.c1[k + 1]), c2a = LDG(&g.c2[k]), c2b = LDG(&g.c2[k + 1]);
    const long o = iS(g, i, j, k);
    const float pia = LDG(&io.piadv[o]);
    const float qk = temq * LDG(&io.ppterm[o]);
    const float pk2 = (k == nk) ? 0.0f : r2 * (-c2b * LDG(&io.piadv[iS(g, i, j, k + 1)]) + (1.0f - c1b) * pia);
    const float pk1 = (k == 1) ? 0.0f : r1 * (+c1a * LDG(&io.piadv[iS(g, i, j, k - 1)]) + (c2a - 1.0f) * pia);

    // new u at faces i and i+1, v at faces j and j+1
    const float thc = LDG(&io.thv[o]);
    const float ppc = LDG(&io.ppd_in[o]);
    float un0, unp, vn0, vnp;
    {
      const long ou = iU(g, i, j, k), oup = iU(g, i + 1, j, k);
      float uo = io.u_in[ou];
      if (openw)
        uo = uo + dts * (-RJK(g, io.radbcw, j, k) * (io.u_in[oup] - io.u_in[ou]) * rdx * LDG(&g.uh[1 - g.ib]) + LDG(&io.uten[ou]));
      un0 = uo + dtu_i * (LDG(&io.uten[ou]) - tem1pg * (ppc - LDG(&io.ppd_in[iS(g, i - 1, j, k)])) * uf_i *
                                                  (thc + LDG(&io.thv[iS(g, i - 1, j, k)])));
      float uop = io.u_in[oup];
      if (opene)
        uop = uop + dts * (-RJK(g, io.radbce, j, k) * (io.u_in[oup] - io.u_in[ou]) * rdx * LDG(&g.uh[ni - g.ib]) + LDG(&io.uten[oup]));
      unp = uop + dtu_ip * (LDG(&io.uten[oup]) - tem1pg * (LDG(&io.ppd_in[iS(g, i + 1, j, k)]) - ppc) * uf_ip *
                                                     (LDG(&io.thv[iS(g, i + 1, j, k)]) + thc));
      io.u_out[ou] = un0;
      if (i == ni) io.u_out[oup] = unp;
      const long ov = iV(g, i, j, k), ovp = iV(g, i, j + 1, k);
      float vo = io.v_in[ov];
      if (opens)
        vo = vo + dts * (-RIK(g, io.radbcs, i, k) * (io.v_in[ovp] - io.v_in[ov]) * rdy * LDG(&g.vh[1 - g.jb]) + LDG(&io.vten[ov]));
      vn0 = vo + dtv_j * (LDG(&io.vten[ov]) - tem2pg * (ppc - LDG(&io.ppd_in[iS(g, i, j - 1, k)])) * vf_j *
                                                  (thc + LDG(&io.thv[iS(g, i, j - 1, k)])));
      float vop = io.v_in[ovp];
      if (openn)
        vop = vop + dts * (-RIK(g, io.radbcn, i, k) * (io.v_in[ovp] - io.v_in[ov]) * rdy * LDG(&g.vh[nj - g.jb]) + LDG(&io.vten[ovp]));
      vnp = vop + dtv_jp * (LDG(&io.vten[ovp]) - tem2pg * (LDG(&io.ppd_in[iS(g, i, j + 1, k)]) - ppc) * vf_jp *
                                                     (LDG(&io.thv[iS(g, i, j + 1, k)]) + thc));
      io.v_out[ov] = vn0;
      if (j == nj) io.v_out[ovp] = vnp;
      // running sums of u, v (sound.F:806-835)
      if (p.last) {
        io.rru[ou] = ((p.first ? 0.0f : io.rru[ou]) + un0) * p.tavg;
        if (i == ni) io.rru[oup] = ((p.first ? 0.0f : io.rru[oup]) + unp) * p.tavg;
        io.rrv[ov] = ((p.first ? 0.0f : io.rrv[ov]) + vn0) * p.tavg;
        if (j == nj) io.rrv[ovp] = ((p.first ? 0.0f : io.rrv[ovp]) + vnp) * p.tavg;
      } else {
        io.rru[ou] = (p.first ? 0.0f : io.rru[ou]) + un0;
        if (i == ni) io.rru[oup] = (p.first ? 0.0f : io.rru[oup]) + unp;
        io.rrv[ov] = (p.first ? 0.0f : io.rrv[ov]) + vn0;
        if (j == nj) io.rrv[ovp] = (p.first ? 0.0f : io.rrv[ovp]) + vnp;
      }
    }
    // fpk (sound.F:486-498)
    const float wk = io.w_in[iW(g, i, j, k)];
    const float wkp = (k == nk) ? 0.0f : io.w_in[iW(g, i, j, k + 1)];
    float div = (unp - un0) * rdx * uh_i + (vnp - vn0) * rdy * vh_j;
    if (fabsf(div) < g.smeps) div = 0.0f;
    const float X = un0 * (pia - LDG(&io.piadv[iS(g, i - 1, j, k)])) + unp * (LDG(&io.piadv[iS(g, i + 1, j, k)]) - pia);
    const float Y = vn0 * (pia - LDG(&io.piadv[iS(g, i, j - 1, k)])) + vnp * (LDG(&io.piadv[iS(g, i, j + 1, k)]) - pia);
    const float A = dts * (LDG(&io.ppten[o]) - LDG(&io.ppterm[o]) * div);
    const float B = -(X * temx * uh_i) - Y * temy * vh_j;
    const float C = beta * (wk * (pk1 + qk) + wkp * (pk2 - qk));
    const float fpk = (A + B) + C;
    const float pp = io.pp_in[o];
    const float pf = pp + fpk;
    SM(s_pf, k) = pf;
    // forward elimination (sound.F:659-716)
    if (k >= 2) {
      const float mm = temm * (c2a * thc + c1a * LDG(&io.thv[iS(g, i, j, k - 1)]));
      const float cc = -asq * (-mm * (pk2 - qk));
      const float bb = 1.0f - asq * (+mm * (-(pk1 + qk) + (pk2p - qkp)));
      const float fwk = dts * LDG(&io.wten[iW(g, i, j, k)]) + beta * (-mm * (pp - ppp));
      const float dd = wk + fwk + alph * (-mm * (pf - pfp));
      if (k == 2) {
        const float rr = 1.0f / bb;
        d1p = -cc * rr;
        d2p = dd * rr;
        SM(s_d1, k) = d1p; SM(s_d2, k) = d2p;
      } else {
        const float aa = -asq * (+mm * (pk1p + qkp));
        const float rr = 1.0f / (aa * d1p + bb);
        if (k < nk) {
          d1p = -cc * rr;
          d2p = (dd - aa * d2p) * rr;
          SM(s_d1, k) = d1p; SM(s_d2, k) = d2p;
        } else {
          wlast = (dd - aa * d2p) * rr;
        }
      }
    }
    pk1p = pk1; pk2p = pk2; qkp = qk; ppp = pp; pfp = pf;
  }

  // ---------------- downward pass ----------------
  float wup = 0.0f;   // w at k+1 (w(nk+1) = 0)
  for (int k = nk; k >= 1; k--) {
    const long o = iS(g, i, j, k);
    float wk;
    if (k == nk) wk = wlast;
    else if (k >= 2) wk = SM(s_d1, k) * wup + SM(s_d2, k);
    else wk = io.w_in[iW(g, i, j, 1)];
    const float mhk = LDG(&g.mh[k]), rr0k = LDG(&g.rr0[k]);
    const float temq = dts * rdz * mhk;
    const float r2 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k + 1]);
    const float r1 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k]);
    const float pia = LDG(&io.piadv[o]);
    const float qk = temq * LDG(&io.ppterm[o]);
    const float pk2 = (k == nk) ? 0.0f : r2 * (-LDG(&g.c2[k + 1]) * LDG(&io.piadv[iS(g, i, j, k + 1)]) + (1.0f - LDG(&g.c1[k + 1])) * pia);
    const float pk1 = (k == 1) ? 0.0f : r1 * (+LDG(&g.c1[k]) * LDG(&io.piadv[iS(g, i, j, k - 1)]) + (LDG(&g.c2[k]) - 1.0f) * pia);
    const float ppold = io.pp_in[o];
    float pn = SM(s_pf, k) + alph * (wk * (pk1 + qk) + wup * (pk2 - qk));
    if (fabsf(pn) < g.smeps) pn = 0.0f;
    const float d1 = g.kdiv * (pn - ppold);
    io.pp_out[o] = pn;
    io.ppd_out[o] = pn + d1;
    if (p.write_ppx) io.ppx[o] = d1;
    const long ow = iW(g, i, j, k);
    if (k >= 2) io.w_out[ow] = wk;
    const float acc0 = p.first ? LDG(&io.wa[ow]) * beta : io.rrw[ow];
    io.rrw[ow] = p.last ? (acc0 + wk * alph) * p.tavg : acc0 + wk;
    wup = wk;
  }
#undef SM
}

void launch_bc(const DGrid &g, float *a, int which, int wflag, cudaStream_t st, int64_t *nlaunch);

// Number of small steps and their length for RK stage nrk (sound.F:79-101).
void sound_nloop(int nsound, int nrk, float dt, int *nloop_out, float *dts_out) {
  int nloop;
  float dts;
  if (nrk == 1) {
    float f = (float)nsound / 3.0f;
    nloop = (int)(f >= 0.0f ? floorf(f + 0.5f) : ceilf(f - 0.5f));   // Fortran nint
    dts = dt / ((float)nloop * 3.0f);
    if (dts > (dt / (float)nsound)) { nloop = nloop + 1; dts = dt / ((float)nloop * 3.0f); }
  } else if (nrk == 2) {
    nloop = (int)(0.5f * (float)nsound);
    dts = dt / (float)nsound;
  } else {
    nloop = nsound;
    dts = dt / (float)nsound;
  }
  *nloop_out = nloop;
  *dts_out = dts;
}

static const int SOUND_BX = 32, SOUND_BY = 2;

size_t sound_smem_bytes(const DGrid &g) { return (size_t)3 * (g.nk + 2) * SOUND_BX * SOUND_BY * sizeof(float); }

// One RK stage of acoustic steps.  Buffers: ua/va/wa/ppi/ppx are the stage
// start values; u3d/v3d/w3d/pp3d receive the result; su/sv are scratch for
// the u/v double buffer, d1/d2 for ppd.  rru/rrv/rrw receive the averages.
void launch_sound(const DGrid &g, int nsound, int nrk, float dt,
                  const float *ua, float *u3d, const float *uten, const float *va, float *v3d, const float *vten,
                  const float *wa, float *w3d, const float *wten, const float *ppi, float *pp3d,
                  const float *piadv, const float *ppten, float *ppx, const float *thv, const float *ppterm,
                  float *rru, float *rrv, float *rrw, const float *radbcw, const float *radbce,
                  const float *radbcs, const float *radbcn, float *su, float *sv, float *d1, float *d2,
                  cudaStream_t st, int64_t *nl) {
  int nloop;
  float dts;
  sound_nloop(nsound, nrk, dt, &nloop, &dts);
  dim3 blk(SOUND_BX, SOUND_BY);
  dim3 grid((g.ni + SOUND_BX - 1) / SOUND_BX, (g.nj + SOUND_BY - 1) / SOUND_BY);
  size_t smem = sound_smem_bytes(g);
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(k_sound_step<SOUND_BX * SOUND_BY>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_set = true;
  }
  const float *uin = ua, *vin = va, *ppdin = ppx;
  for (int n = 1; n <= nloop; n++) {
    SoundIO io;
    const bool to3d = ((nloop - n) % 2) == 0;
    io.u_in = uin; io.v_in = vin;
    io.u_out = to3d ? u3d : su; io.v_out = to3d ? v3d : sv;
    io.w_in = (n == 1) ? wa : w3d; io.w_out = w3d;
    io.pp_in = (n == 1) ? ppi : pp3d; io.pp_out = pp3d;
    io.ppd_in = ppdin; io.ppd_out = (n % 2) ? d1 : d2;
    io.rru = rru; io.rrv = rrv; io.rrw = rrw; io.wa = wa;
    io.uten = uten; io.vten = vten; io.wten = wten; io.ppten = ppten;
    io.thv = thv; io.ppterm = ppterm; io.piadv = piadv;
    io.radbcw = radbcw; io.radbce = radbce; io.radbcs = radbcs; io.radbcn = radbcn;
    io.ppx = ppx;
    SoundStep sp;
    sp.dts = dts; sp.tavg = 1.0f / (float)nloop;
    sp.first = (n == 1); sp.last = (n == nloop); sp.write_ppx = (nrk == 3 && n == nloop);
    { ProfScope _ps("k_sound_step", st); k_sound_step<SOUND_BX * SOUND_BY><<<grid, blk, smem, st>>>(g, io, sp); }
    if (nl) *nl += 1;
    if (n < nloop) launch_bc(g, io.ppd_out, 2, 0, st, nl);
    uin = io.u_out; vin = io.v_out; ppdin = io.ppd_out;
  }
}

}  // namespace cm1g
