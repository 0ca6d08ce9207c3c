// k_sound.cu -- acoustic substeps of sound.F (psolver=3, no terrain).
//
// One kernel launch per small step.  A block owns a tile of TX consecutive
// columns (i) of one row (j), all levels, and works in three phases:
//
//  1. point-parallel (warp w takes levels w+1, w+1+NW, ...; lanes run along
//     i so every global access is a coalesced row segment): new u and v by
//     the pressure-gradient update (sound.F:321-341) with the open-boundary
//     updates of bc.F:2392-2686 folded in, the running sums of u and v
//     (sound.F:806-835), the explicit pi' forcing fpk (sound.F:479-502), and
//     the per-level pieces of the implicit w equation, kept in shared memory;
//  2. column-sequential (one thread per column): the Thomas forward
//     elimination and back substitution of sound.F:659-733, entirely in
//     shared memory, with the reference's operation order;
//  3. point-parallel again: pi' update with divergence damping
//     (sound.F:746-760), new w and the averaged w.
//
// Neighbour columns read u, v and ppd from the previous small step, so u, v
// and ppd are double-buffered; w and pi' are read only by their own column
// and are updated in place.  The east/north face velocity of a cell is
// recomputed from the same old values by the neighbour that needs it, which
// reproduces the stored value exactly.
#include <cstdlib>
#include <cstring>
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
  float *radbcw, *radbce, *radbcs, *radbcn;   // phase speeds (irbc = 2: formed and stored here)
  float *ppx;                     // last step of the final stage: kdiv*(pi'_new - pi'_old)
  float *lu;                      // column sweep: LU factors (a scalar-shaped scratch array)
  const float *ubw, *ube, *vbs, *vbn;   // roflux = 1: this step's restricted boundary u/v (k_openbc_restrict)
};

struct SoundStep {
  float dts, tavg;
  int first, last, write_ppx;
  int ppd_mapped;   // ppd_in's halo is not filled: read bcp's source points instead
};

// Offsets of the west/east/south/north neighbours of ppd at (i,j).  From the
// second small step on, ppd_in comes from the previous step of this kernel
// and its 1-point halo is not filled; the value bcp would put there
// (bc.F:380-518: periodic wrap, else the adjacent interior point) is read
// from the point bcp copies it from.
struct PpdNbr { long w, e, s, n; };
__device__ __forceinline__ PpdNbr ppd_nbr(const DGrid &g, int mapped, int i, int j) {
  PpdNbr d{-1L, 1L, -(long)g.NI, (long)g.NI};
  if (mapped) {
    if (i == 1) d.w = (g.wbc == 1) ? (long)(g.ni - 1) : 0L;
    if (i == g.ni) d.e = (g.ebc == 1) ? -(long)(g.ni - 1) : 0L;
    if (j == 1) d.s = (g.sbc == 1) ? (long)(g.nj - 1) * g.NI : 0L;
    if (j == g.nj) d.n = (g.nbc == 1) ? -(long)(g.nj - 1) * g.NI : 0L;
  }
  return d;
}

#define RJK(g, a, j, k) ((a)[((j) - (g).jb) + (long)(g).NJ * (k)])
#define RIK(g, a, i, k) ((a)[((i) - (g).ib) + (long)(g).NI * (k)])

// Phase speed of an open-boundary point for this small step.  With irbc = 2
// the Klemp-Wilhelmson speed is formed from the current velocity at every
// small step (sound.F:261-267; radbcew/radbcns, bc.F:1948-2046): u - cstar
// where negative at the west and south boundaries, u + cstar where positive
// at the east and north ones, else 0; it is stored for the state.  Otherwise
// the stored speed (irbc = 4 from radbcew4/ns4, irbc = 1 from the start of
// the step) is used.
__device__ __forceinline__ float radbc_in(const DGrid &g, float &slot, float ub) {
  if (g.irbc != 2) return slot;
  const float c = ub - g.cstar;
  const float r = (c < 0.0f) ? c : 0.0f;
  slot = r;
  return r;
}
__device__ __forceinline__ float radbc_out(const DGrid &g, float &slot, float ub) {
  if (g.irbc != 2) return slot;
  const float c = ub + g.cstar;
  const float r = (c > 0.0f) ? c : 0.0f;
  slot = r;
  return r;
}

// roflux = 1: the open-boundary velocities of one acoustic step, restricted
// so that the inflow through the open boundaries balances the outflow
// (restrict_openbc_we/sn, bc.F:2180-2384, called by sound.F:283-285 and
// 299-301 after the boundary tendency of ssopenbcw/e/s/n).  One block: the
// thread of level k forms the level's boundary values and its binary64
// outflow and inflow sums (over j, resp. i, west/south before east/north,
// as the reference's loops run), one thread adds the levels in order, and
// the outflow points are scaled by inflow/outflow.  The acoustic kernels
// then read the values instead of forming them.  Shared memory: 4 (nk+1)
// doubles.
__global__ void k_openbc_restrict(DGrid g, SoundIO io, float dts, float *ubw, float *ube, float *vbs, float *vbn) {
  extern __shared__ double rsum[];   // out/in sums of the we and sn boundaries by level
  const int ni = g.ni, nj = g.nj, nk = g.nk, L = nk + 1;
  double *tow = rsum, *tiw = rsum + L, *tos = rsum + 2 * L, *tis = rsum + 3 * L;
  __shared__ double t3[2];
  const bool w = g.wbc == 2 && g.ibw, e = g.ebc == 2 && g.ibe, s = g.sbc == 2 && g.ibs, n = g.nbc == 2 && g.ibn;
  const float rdx = g.rdx, rdy = g.rdy;
  for (int k = 1 + (int)threadIdx.x; k <= nk; k += blockDim.x) {
    const float r0 = LDG(&g.rho0[k]), rm = LDG(&g.rmh[k]);
    double to = 0.0, ti = 0.0;
    if (w)
      for (int j = 1; j <= nj; j++) {
        const long o = iU(g, 1, j, k);
        const float u0v = io.u_in[o], u1v = io.u_in[o + 1];
        const float uo = u0v + dts * (-radbc_in(g, RJK(g, io.radbcw, j, k), u0v) * (u1v - u0v) * rdx *
                                      LDG(&g.uh[1 - g.ib]) + LDG(&io.uten[o]));
        RJK(g, ubw, j, k) = uo;
        const float f = r0 * uo * LDG(&g.rvh[j - g.jb]) * rm;
        to = to - (double)fminf(0.0f, f);
        ti = ti + (double)fmaxf(0.0f, f);
      }
    if (e)
      for (int j = 1; j <= nj; j++) {
        const long o = iU(g, ni + 1, j, k);
        const float u1v = io.u_in[o], u0v = io.u_in[o - 1];
        const float uo = u1v + dts * (-radbc_out(g, RJK(g, io.radbce, j, k), u1v) * (u1v - u0v) * rdx *
                                      LDG(&g.uh[ni - g.ib]) + LDG(&io.uten[o]));
        RJK(g, ube, j, k) = uo;
        const float f = r0 * uo * LDG(&g.rvh[j - g.jb]) * rm;
        to = to + (double)fmaxf(0.0f, f);
        ti = ti - (double)fminf(0.0f, f);
      }
    tow[k] = to; tiw[k] = ti;
    to = 0.0; ti = 0.0;
    if (s)
      for (int i = 1; i <= ni; i++) {
        const long o = iV(g, i, 1, k);
        const float v0v = io.v_in[o], v1v = io.v_in[o + g.NI];
        const float vo = v0v + dts * (-radbc_in(g, RIK(g, io.radbcs, i, k), v0v) * (v1v - v0v) * rdy *
                                      LDG(&g.vh[1 - g.jb]) + LDG(&io.vten[o]));
        RIK(g, vbs, i, k) = vo;
        const float f = r0 * vo * LDG(&g.ruh[i - g.ib]) * rm;
        to = to - (double)fminf(0.0f, f);
        ti = ti + (double)fmaxf(0.0f, f);
      }
    if (n)
      for (int i = 1; i <= ni; i++) {
        const long o = iV(g, i, nj + 1, k);
        const float v1v = io.v_in[o], v0v = io.v_in[o - g.NI];
        const float vo = v1v + dts * (-radbc_out(g, RIK(g, io.radbcn, i, k), v1v) * (v1v - v0v) * rdy *
                                      LDG(&g.vh[nj - g.jb]) + LDG(&io.vten[o]));
        RIK(g, vbn, i, k) = vo;
        const float f = r0 * vo * LDG(&g.ruh[i - g.ib]) * rm;
        to = to + (double)fmaxf(0.0f, f);
        ti = ti - (double)fminf(0.0f, f);
      }
    tos[k] = to; tis[k] = ti;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    const double *to = threadIdx.x == 0 ? tow : tos, *ti = threadIdx.x == 0 ? tiw : tis;
    double fo = 0.0, fi = 0.0;
    for (int k = 1; k <= nk; k++) { fo = fo + to[k]; fi = fi + ti[k]; }
    t3[threadIdx.x] = (fi + 1.0e-20) / (fo + 1.0e-20);
  }
  __syncthreads();
  const double tw = t3[0], ts = t3[1];
  for (int k = 1 + (int)threadIdx.x; k <= nk; k += blockDim.x) {
    const float r0 = LDG(&g.rho0[k]);
    const double r0d = (double)r0;
    for (int j = 1; j <= nj && (w || e); j++) {
      if (w) {
        const double u1 = (double)(r0 * RJK(g, ubw, j, k));
        if (u1 < 0.0) RJK(g, ubw, j, k) = (float)(u1 * tw / r0d);
      }
      if (e) {
        const double u1 = (double)(r0 * RJK(g, ube, j, k));
        if (u1 > 0.0) RJK(g, ube, j, k) = (float)(u1 * tw / r0d);
      }
    }
    for (int i = 1; i <= ni && (s || n); i++) {
      if (s) {
        const double u1 = (double)(r0 * RIK(g, vbs, i, k));
        if (u1 < 0.0) RIK(g, vbs, i, k) = (float)(u1 * ts / r0d);
      }
      if (n) {
        const double u1 = (double)(r0 * RIK(g, vbn, i, k));
        if (u1 > 0.0) RIK(g, vbn, i, k) = (float)(u1 * ts / r0d);
      }
    }
  }
}

static const int SND_TX = 32;     // columns per tile (one warp wide)
static const int SND_NW = 8;      // warps per block
static const int SND_KPT = 16;    // max levels per thread: nk <= SND_NW*SND_KPT

#ifndef CM1G_SND_MINB
#define CM1G_SND_MINB 3      // resident blocks per SM the tile kernel is compiled for
#endif
#ifndef CM1G_SND_UNROLL
#define CM1G_SND_UNROLL 1    // phase-1 levels a warp keeps in flight
#endif
constexpr int kSndUnroll = CM1G_SND_UNROLL;

template <int TX, int NW, int KPT>
__global__ void __launch_bounds__(TX * NW, CM1G_SND_MINB) k_sound_tile(DGrid g, SoundIO io, SoundStep p) {
  extern __shared__ float sm[];
  const int lane = threadIdx.x, w = threadIdx.y;
  const int i = 1 + (int)blockIdx.x * TX + lane;
  const int j = 1 + (int)blockIdx.y;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const bool active = (i <= ni);
  const int L = nk + 2;
  float *PF = sm;               // pi'_old + fpk
  float *P1 = sm + 1 * L * TX;  // pk1 + qk
  float *P2 = sm + 2 * L * TX;  // pk2 - qk
  float *MM = sm + 3 * L * TX;  // mm, then the LU factor dum1
  float *DD = sm + 4 * L * TX;  // w_old + fwk, then dum2, then the new w (DD(1) = w(1))
#define S(a, k) a[(k) * TX + lane]

  const float dts = p.dts, alph = g.alph, beta = 1.0f - alph, asq = alph * alph;
  const float cp = g.c.cp, rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;

  // ---------------- phase 1 ----------------
  if (active) {
    const float tem1pg = rdx * cp * 0.5f, tem2pg = rdy * cp * 0.5f;      // sound.F:321-322
    const float temx = dts * 0.5f * rdx, temy = dts * 0.5f * rdy;        // sound.F:479-480
    const float uh_i = LDG(&g.uh[i - g.ib]), vh_j = LDG(&g.vh[j - g.jb]);
    const float uf_i = LDG(&g.uf[i - g.ib]), uf_ip = LDG(&g.uf[i + 1 - g.ib]);
    const float vf_j = LDG(&g.vf[j - g.jb]), vf_jp = LDG(&g.vf[j + 1 - g.jb]);
    const float dtu_i = dts * LDG(&g.dtu0[i2(g, i, j)]), dtu_ip = dts * LDG(&g.dtu0[i2(g, i + 1, j)]);
    const float dtv_j = dts * LDG(&g.dtv0[i2(g, i, j)]), dtv_jp = dts * LDG(&g.dtv0[i2(g, i, j + 1)]);
    const bool openw = (g.wbc == 2 && g.ibw && i == 1), opene = (g.ebc == 2 && g.ibe && i == ni);
    const bool opens = (g.sbc == 2 && g.ibs && j == 1), openn = (g.nbc == 2 && g.ibn && j == nj);
    const PpdNbr pn_ = ppd_nbr(g, p.ppd_mapped, i, j);
    // warps take interleaved levels (w+1, w+1+NW, ...): at any time the
    // block's warps work on adjacent levels and share their vertical
    // neighbours through L1
    const long plane = (long)g.NI * g.NJ;
#pragma unroll kSndUnroll
    for (int m = 0; m < KPT; m++) {
      const int k = 1 + w + m * NW;
      if (k > nk) break;
      const long o = iS(g, i, j, k);
      const long ou = iU(g, i, j, k), oup = ou + 1;
      const long ov = iV(g, i, j, k), ovp = ov + g.NI;
      // ---- loads (all independent)
      const float pia = LDG(&io.piadv[o]);
      const float pid = (k > 1) ? LDG(&io.piadv[o - plane]) : 0.0f;
      const float thd = (k > 1) ? LDG(&io.thv[o - plane]) : 0.0f;
      const float ppm = (k > 1) ? io.pp_in[o - plane] : 0.0f;
      const float wk = io.w_in[o];
      const float piw = LDG(&io.piadv[o - 1]), pie = LDG(&io.piadv[o + 1]);
      const float pis = LDG(&io.piadv[o - g.NI]), pin = LDG(&io.piadv[o + g.NI]);
      const float piu = (k < nk) ? LDG(&io.piadv[o + plane]) : 0.0f;
      const float thc = LDG(&io.thv[o]), thw = LDG(&io.thv[o - 1]), the = LDG(&io.thv[o + 1]);
      const float ths = LDG(&io.thv[o - g.NI]), thn = LDG(&io.thv[o + g.NI]);
      const float ppc = LDG(&io.ppd_in[o]), ppw = LDG(&io.ppd_in[o + pn_.w]), ppe = LDG(&io.ppd_in[o + pn_.e]);
      const float pps = LDG(&io.ppd_in[o + pn_.s]), ppn = LDG(&io.ppd_in[o + pn_.n]);
      const float u0v = LDG(&io.u_in[ou]), u1v = LDG(&io.u_in[oup]);
      const float v0v = LDG(&io.v_in[ov]), v1v = LDG(&io.v_in[ovp]);
      const float ut0 = LDG(&io.uten[ou]), ut1 = LDG(&io.uten[oup]);
      const float vt0 = LDG(&io.vten[ov]), vt1 = LDG(&io.vten[ovp]);
      const float pptn = LDG(&io.ppten[o]), pptm = LDG(&io.ppterm[o]);
      const float wkp = (k < nk) ? io.w_in[o + plane] : 0.0f;
      const float pp = io.pp_in[o];
      const float wtn = LDG(&io.wten[o]);
      const float accu0 = p.first ? 0.0f : io.rru[ou];
      const float accv0 = p.first ? 0.0f : io.rrv[ov];
      // ---- u at faces i, i+1 and v at faces j, j+1
      float uo = u0v;
      if (openw) uo = g.roflux ? RJK(g, io.ubw, j, k) : uo + dts * (-radbc_in(g, RJK(g, io.radbcw, j, k), u0v) * (u1v - u0v) * rdx * LDG(&g.uh[1 - g.ib]) + ut0);
      const float un0 = uo + dtu_i * (ut0 - tem1pg * (ppc - ppw) * uf_i * (thc + thw));
      float uop = u1v;
      if (opene) uop = g.roflux ? RJK(g, io.ube, j, k) : uop + dts * (-radbc_out(g, RJK(g, io.radbce, j, k), u1v) * (u1v - u0v) * rdx * LDG(&g.uh[ni - g.ib]) + ut1);
      const float unp = uop + dtu_ip * (ut1 - tem1pg * (ppe - ppc) * uf_ip * (the + thc));
      float vo = v0v;
      if (opens) vo = g.roflux ? RIK(g, io.vbs, i, k) : vo + dts * (-radbc_in(g, RIK(g, io.radbcs, i, k), v0v) * (v1v - v0v) * rdy * LDG(&g.vh[1 - g.jb]) + vt0);
      const float vn0 = vo + dtv_j * (vt0 - tem2pg * (ppc - pps) * vf_j * (thc + ths));
      float vop = v1v;
      if (openn) vop = g.roflux ? RIK(g, io.vbn, i, k) : vop + dts * (-radbc_out(g, RIK(g, io.radbcn, i, k), v1v) * (v1v - v0v) * rdy * LDG(&g.vh[nj - g.jb]) + vt1);
      const float vnp = vop + dtv_jp * (vt1 - tem2pg * (ppn - ppc) * vf_jp * (thn + thc));
      io.u_out[ou] = un0;
      io.v_out[ov] = vn0;
      if (p.last) {
        io.rru[ou] = (accu0 + un0) * p.tavg;
        io.rrv[ov] = (accv0 + vn0) * p.tavg;
      } else {
        io.rru[ou] = accu0 + un0;
        io.rrv[ov] = accv0 + vn0;
      }
      if (i == ni) {
        io.u_out[oup] = unp;
        const float a1 = p.first ? 0.0f : io.rru[oup];
        io.rru[oup] = p.last ? (a1 + unp) * p.tavg : a1 + unp;
      }
      if (j == nj) {
        io.v_out[ovp] = vnp;
        const float a1 = p.first ? 0.0f : io.rrv[ovp];
        io.rrv[ovp] = p.last ? (a1 + vnp) * p.tavg : a1 + vnp;
      }
      // ---- stage coefficients (sound.F:117-135, 188-189)
      const float mhk = LDG(&g.mh[k]), rr0k = LDG(&g.rr0[k]);
      const float temq = dts * rdz * mhk;
      const float r2 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k + 1]);
      const float r1 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k]);
      const float temm = dts * rdz * cp * LDG(&g.mf[k]);
      const float c1a = LDG(&g.c1[k]), c1b = LDG(&g.c1[k + 1]), c2a = LDG(&g.c2[k]), c2b = LDG(&g.c2[k + 1]);
      const float qk = temq * pptm;
      const float pk2 = (k == nk) ? 0.0f : r2 * (-c2b * piu + (1.0f - c1b) * pia);
      const float pk1 = (k == 1) ? 0.0f : r1 * (+c1a * pid + (c2a - 1.0f) * pia);
      const float p1 = pk1 + qk, p2 = pk2 - qk;
      // ---- fpk (sound.F:486-498)
      float div = (unp - un0) * rdx * uh_i + (vnp - vn0) * rdy * vh_j;
      if (fabsf(div) < g.smeps) div = 0.0f;
      const float X = un0 * (pia - piw) + unp * (pie - pia);
      const float Y = vn0 * (pia - pis) + vnp * (pin - pia);
      const float A = dts * (pptn - pptm * div);
      const float B = -(X * temx * uh_i) - Y * temy * vh_j;
      const float C = beta * (wk * p1 + wkp * p2);
      const float fpk = (A + B) + C;
      S(PF, k) = pp + fpk;
      S(P1, k) = p1;
      S(P2, k) = p2;
      if (k >= 2) {
        const float mm = temm * (c2a * thc + c1a * thd);
        const float fwk = dts * wtn + beta * (-mm * (pp - ppm));
        S(MM, k) = mm;
        S(DD, k) = wk + fwk;
      }
      if (k == 1) S(DD, 1) = wk;
    }
  }
  __syncthreads();

  // phase 3's global inputs of this warp's levels (pi' before the step and
  // the running sum of w; the column's own points), loaded now so that they
  // arrive while warp 0 runs the Thomas solve
  float ppo[KPT], acs[KPT];
  if (active) {
#pragma unroll
    for (int m = 0; m < KPT; m++) {
      const int k = 1 + w + m * NW;
      ppo[m] = 0.0f; acs[m] = 0.0f;
      if (k <= nk) {
        const long o = iS(g, i, j, k);
        ppo[m] = io.pp_in[o];
        acs[m] = p.first ? LDG(&io.wa[o]) * beta : io.rrw[o];
      }
    }
  }

  // ---------------- phase 2: Thomas solve for w, k = 2..nk ----------------
  // The first and last levels are peeled off so that the loop body has no
  // branches and its shared-memory reads (independent of the recurrence)
  // can be issued ahead of the dependent chain; nk >= 6 (cm1g_init).
  if (w == 0 && active) {
    float d1p, d2p;
    {
      const int k = 2;
      const float mm = S(MM, k);
      const float bb = 1.0f - asq * (+mm * (-S(P1, k) + S(P2, k - 1)));
      const float dd = S(DD, k) + alph * (-mm * (S(PF, k) - S(PF, k - 1)));
      const float cc = -asq * (-mm * S(P2, k));
      // __frcp_rn is the correctly rounded 1/x, the same value as 1.0f/x
      const float rr = __frcp_rn(bb);
      d1p = -cc * rr;
      d2p = dd * rr;
      S(MM, k) = d1p; S(DD, k) = d2p;
    }
#pragma unroll 4
    for (int k = 3; k < nk; k++) {
      const float mm = S(MM, k);
      const float bb = 1.0f - asq * (+mm * (-S(P1, k) + S(P2, k - 1)));
      const float dd = S(DD, k) + alph * (-mm * (S(PF, k) - S(PF, k - 1)));
      const float aa = -asq * (+mm * S(P1, k - 1));
      const float cc = -asq * (-mm * S(P2, k));
      const float rr = __frcp_rn(aa * d1p + bb);
      d1p = -cc * rr;
      d2p = (dd - aa * d2p) * rr;
      S(MM, k) = d1p; S(DD, k) = d2p;
    }
    {
      const int k = nk;
      const float mm = S(MM, k);
      const float bb = 1.0f - asq * (+mm * (-S(P1, k) + S(P2, k - 1)));
      const float dd = S(DD, k) + alph * (-mm * (S(PF, k) - S(PF, k - 1)));
      const float aa = -asq * (+mm * S(P1, k - 1));
      const float rr = __frcp_rn(aa * d1p + bb);
      S(DD, k) = (dd - aa * d2p) * rr;   // w(nk)
    }
    float wup = S(DD, nk);
#pragma unroll 4
    for (int k = nk - 1; k >= 2; k--) {
      wup = S(MM, k) * wup + S(DD, k);
      S(DD, k) = wup;
    }
  }
  __syncthreads();

  // ---------------- phase 3 ----------------
  if (active) {
#pragma unroll
    for (int m = 0; m < KPT; m++) {
      const int k = 1 + w + m * NW;
      if (k > nk) break;
      const long o = iS(g, i, j, k);
      const float wk = S(DD, k);
      const float wkp = (k < nk) ? S(DD, k + 1) : 0.0f;
      float pn = S(PF, k) + alph * (wk * S(P1, k) + wkp * S(P2, k));
      if (fabsf(pn) < g.smeps) pn = 0.0f;
      const float d1 = g.kdiv * (pn - ppo[m]);
      const float ac = acs[m];
      io.pp_out[o] = pn;
      io.ppd_out[o] = pn + d1;
      if (p.write_ppx) io.ppx[o] = d1;
      if (k >= 2) io.w_out[o] = wk;
      io.rrw[o] = p.last ? (ac + wk * alph) * p.tavg : ac + wk;
    }
  }
#undef S
}

// ---------------------------------------------------------------------
// Column-sweep form of one small step.  Each thread owns one column (i,j)
// and walks it twice, with no block-wide barrier:
//
//  up   (k = 1..nk): the explicit updates of phase 1 above, then at once the
//       Thomas forward elimination of level k (it needs only level k and the
//       previous level, whose coefficients are carried in registers, as are
//       the vertical neighbours pi_adv(k-1), theta_v(k-1), pi'(k-1), w(k+1));
//  down (k = nk..1): back substitution fused with the pi' update, divergence
//       damping and the w average of phase 3.
//
// Between the sweeps the column keeps: the LU factor dum1(k) in the scratch
// array lu (private to the thread; in global memory rather than shared
// memory so that the block's column count does not depend on nk and more
// columns are resident per SM: 20 warps at 96 registers against 12 with a
// shared array at nk = 128, 51 against 76 ms per CBL step), dum2(k) in
// w_out(k) and pi'_old+fpk in
// ppd_out(k) -- both arrays are this column's own and are overwritten with
// their final values on the way down; w(k) is no longer needed by the up
// sweep once level k is done, and ppd_out is not the buffer neighbours read.
// pk1+qk and pk2-qk are recomputed on the way down from the same inputs.
// The arithmetic and its order are those of the tile form.
// ---------------------------------------------------------------------
static const int SNC_TX = 32;
// grids with at least this many columns (ni*nj) use the column-sweep form
#ifndef CM1G_SOUND_COL_MIN_COLUMNS
#define CM1G_SOUND_COL_MIN_COLUMNS (1L << 20)
#endif

template <int TX, int TY>
__global__ void __launch_bounds__(TX * TY, 5) k_sound_col(DGrid g, SoundIO io, SoundStep p) {
  const int lane = threadIdx.x;
  const int i = 1 + (int)blockIdx.x * TX + lane;
  const int j = 1 + (int)blockIdx.y * TY + (int)threadIdx.y;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  if (i > ni || j > nj) return;     // no barriers below
  const float dts = p.dts, alph = g.alph, beta = 1.0f - alph, asq = alph * alph;
  const float cp = g.c.cp, rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
  const long plane = (long)g.NI * g.NJ;
  const long oc = iS(g, i, j, 0), ocu = iU(g, i, j, 0), ocv = iV(g, i, j, 0);
  const long planeU = (long)(g.NI + 1) * g.NJ, planeV = (long)g.NI * (g.NJ + 1);
  // the LU factor dum1 of level k (the column's own point of io.lu)
  auto D1 = [&](int k) -> float & { return io.lu[oc + k * plane]; };

  // pk1+qk and pk2-qk of level k (sound.F:117-135, 188-189)
  auto coef = [&](int k, float pid, float pia, float piu, float pptm, float *p1, float *p2) {
    const float mhk = LDG(&g.mh[k]), rr0k = LDG(&g.rr0[k]);
    const float temq = dts * rdz * mhk;
    const float r2 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k + 1]);
    const float r1 = dts * rdz * mhk * rr0k * LDG(&g.rf0[k]);
    const float c1a = LDG(&g.c1[k]), c1b = LDG(&g.c1[k + 1]), c2a = LDG(&g.c2[k]), c2b = LDG(&g.c2[k + 1]);
    const float qk = temq * pptm;
    const float pk2 = (k == nk) ? 0.0f : r2 * (-c2b * piu + (1.0f - c1b) * pia);
    const float pk1 = (k == 1) ? 0.0f : r1 * (+c1a * pid + (c2a - 1.0f) * pia);
    *p1 = pk1 + qk;
    *p2 = pk2 - qk;
  };

  // ---------------- up ----------------
  {
    const float tem1pg = rdx * cp * 0.5f, tem2pg = rdy * cp * 0.5f;      // sound.F:321-322
    const float temx = dts * 0.5f * rdx, temy = dts * 0.5f * rdy;        // sound.F:479-480
    const float uh_i = LDG(&g.uh[i - g.ib]), vh_j = LDG(&g.vh[j - g.jb]);
    const float uf_i = LDG(&g.uf[i - g.ib]), uf_ip = LDG(&g.uf[i + 1 - g.ib]);
    const float vf_j = LDG(&g.vf[j - g.jb]), vf_jp = LDG(&g.vf[j + 1 - g.jb]);
    const float dtu_i = dts * LDG(&g.dtu0[i2(g, i, j)]), dtu_ip = dts * LDG(&g.dtu0[i2(g, i + 1, j)]);
    const float dtv_j = dts * LDG(&g.dtv0[i2(g, i, j)]), dtv_jp = dts * LDG(&g.dtv0[i2(g, i, j + 1)]);
    const bool openw = (g.wbc == 2 && g.ibw && i == 1), opene = (g.ebc == 2 && g.ibe && i == ni);
    const bool opens = (g.sbc == 2 && g.ibs && j == 1), openn = (g.nbc == 2 && g.ibn && j == nj);
    const PpdNbr pn_ = ppd_nbr(g, p.ppd_mapped, i, j);
    // carried from the level below: pi_adv(k-1), pi_adv(k), theta_v(k-1), pi'(k-1), w(k)
    float pid = 0.0f, pia = LDG(&io.piadv[oc + plane]), thd = 0.0f, ppm = 0.0f, wk = io.w_in[oc + plane];
    // carried Thomas state: coefficients of level k-1 and the running factors
    float p1m = 0.0f, p2m = 0.0f, pfm = 0.0f, d1p = 0.0f, d2p = 0.0f;
    // the loads of level k+1 are issued before level k is computed, so each
    // thread keeps two levels of reads in flight (none of them is written by
    // this sweep before it is read)
    struct LvIn {
      float piw, pie, pis, pin, piu, thc, thw, the, ths, thn, ppc, ppw, ppe, pps, ppn;
      float u0v, u1v, v0v, v1v, ut0, ut1, vt0, vt1, pptn, pptm, wkp, pp, wtn, accu0, accv0;
    };
    auto load = [&](int k, LvIn &L) {
      const long o = oc + k * plane, ou = ocu + k * planeU, oup = ou + 1, ov = ocv + k * planeV, ovp = ov + g.NI;
      L.piw = LDG(&io.piadv[o - 1]); L.pie = LDG(&io.piadv[o + 1]);
      L.pis = LDG(&io.piadv[o - g.NI]); L.pin = LDG(&io.piadv[o + g.NI]);
      L.piu = (k < nk) ? LDG(&io.piadv[o + plane]) : 0.0f;
      L.thc = LDG(&io.thv[o]); L.thw = LDG(&io.thv[o - 1]); L.the = LDG(&io.thv[o + 1]);
      L.ths = LDG(&io.thv[o - g.NI]); L.thn = LDG(&io.thv[o + g.NI]);
      L.ppc = LDG(&io.ppd_in[o]); L.ppw = LDG(&io.ppd_in[o + pn_.w]); L.ppe = LDG(&io.ppd_in[o + pn_.e]);
      L.pps = LDG(&io.ppd_in[o + pn_.s]); L.ppn = LDG(&io.ppd_in[o + pn_.n]);
      L.u0v = LDG(&io.u_in[ou]); L.u1v = LDG(&io.u_in[oup]);
      L.v0v = LDG(&io.v_in[ov]); L.v1v = LDG(&io.v_in[ovp]);
      L.ut0 = LDG(&io.uten[ou]); L.ut1 = LDG(&io.uten[oup]);
      L.vt0 = LDG(&io.vten[ov]); L.vt1 = LDG(&io.vten[ovp]);
      L.pptn = LDG(&io.ppten[o]); L.pptm = LDG(&io.ppterm[o]);
      L.wkp = (k < nk) ? io.w_in[o + plane] : 0.0f;
      L.pp = io.pp_in[o];
      L.wtn = LDG(&io.wten[o]);
      L.accu0 = p.first ? 0.0f : io.rru[ou];
      L.accv0 = p.first ? 0.0f : io.rrv[ov];
    };
    LvIn cur, nxt;
    load(1, cur);
#pragma unroll 1
    for (int k = 1; k <= nk; k++) {
      if (k < nk) load(k + 1, nxt);
      const long o = oc + k * plane, ou = ocu + k * planeU, oup = ou + 1, ov = ocv + k * planeV, ovp = ov + g.NI;
      const float piw = cur.piw, pie = cur.pie, pis = cur.pis, pin = cur.pin, piu = cur.piu;
      const float thc = cur.thc, thw = cur.thw, the = cur.the, ths = cur.ths, thn = cur.thn;
      const float ppc = cur.ppc, ppw = cur.ppw, ppe = cur.ppe, pps = cur.pps, ppn = cur.ppn;
      const float u0v = cur.u0v, u1v = cur.u1v, v0v = cur.v0v, v1v = cur.v1v;
      const float ut0 = cur.ut0, ut1 = cur.ut1, vt0 = cur.vt0, vt1 = cur.vt1;
      const float pptn = cur.pptn, pptm = cur.pptm, wkp = cur.wkp, pp = cur.pp, wtn = cur.wtn;
      const float accu0 = cur.accu0, accv0 = cur.accv0;
      // ---- u at faces i, i+1 and v at faces j, j+1 (sound.F:321-341, bc.F:2392-2686)
      float uo = u0v;
      if (openw) uo = g.roflux ? RJK(g, io.ubw, j, k) : uo + dts * (-radbc_in(g, RJK(g, io.radbcw, j, k), u0v) * (u1v - u0v) * rdx * LDG(&g.uh[1 - g.ib]) + ut0);
      const float un0 = uo + dtu_i * (ut0 - tem1pg * (ppc - ppw) * uf_i * (thc + thw));
      float uop = u1v;
      if (opene) uop = g.roflux ? RJK(g, io.ube, j, k) : uop + dts * (-radbc_out(g, RJK(g, io.radbce, j, k), u1v) * (u1v - u0v) * rdx * LDG(&g.uh[ni - g.ib]) + ut1);
      const float unp = uop + dtu_ip * (ut1 - tem1pg * (ppe - ppc) * uf_ip * (the + thc));
      float vo = v0v;
      if (opens) vo = g.roflux ? RIK(g, io.vbs, i, k) : vo + dts * (-radbc_in(g, RIK(g, io.radbcs, i, k), v0v) * (v1v - v0v) * rdy * LDG(&g.vh[1 - g.jb]) + vt0);
      const float vn0 = vo + dtv_j * (vt0 - tem2pg * (ppc - pps) * vf_j * (thc + ths));
      float vop = v1v;
      if (openn) vop = g.roflux ? RIK(g, io.vbn, i, k) : vop + dts * (-radbc_out(g, RIK(g, io.radbcn, i, k), v1v) * (v1v - v0v) * rdy * LDG(&g.vh[nj - g.jb]) + vt1);
      const float vnp = vop + dtv_jp * (vt1 - tem2pg * (ppn - ppc) * vf_jp * (thn + thc));
      io.u_out[ou] = un0;
      io.v_out[ov] = vn0;
      if (p.last) {
        io.rru[ou] = (accu0 + un0) * p.tavg;
        io.rrv[ov] = (accv0 + vn0) * p.tavg;
      } else {
        io.rru[ou] = accu0 + un0;
        io.rrv[ov] = accv0 + vn0;
      }
      if (i == ni) {
        io.u_out[oup] = unp;
        const float a1 = p.first ? 0.0f : io.rru[oup];
        io.rru[oup] = p.last ? (a1 + unp) * p.tavg : a1 + unp;
      }
      if (j == nj) {
        io.v_out[ovp] = vnp;
        const float a1 = p.first ? 0.0f : io.rrv[ovp];
        io.rrv[ovp] = p.last ? (a1 + vnp) * p.tavg : a1 + vnp;
      }
      float p1, p2;
      coef(k, pid, pia, piu, pptm, &p1, &p2);
      // ---- fpk (sound.F:486-498)
      float div = (unp - un0) * rdx * uh_i + (vnp - vn0) * rdy * vh_j;
      if (fabsf(div) < g.smeps) div = 0.0f;
      const float X = un0 * (pia - piw) + unp * (pie - pia);
      const float Y = vn0 * (pia - pis) + vnp * (pin - pia);
      const float A = dts * (pptn - pptm * div);
      const float B = -(X * temx * uh_i) - Y * temy * vh_j;
      const float C = beta * (wk * p1 + wkp * p2);
      const float fpk = (A + B) + C;
      const float pf = pp + fpk;
      io.ppd_out[o] = pf;                               // kept for the down sweep
      if (k >= 2) {
        // ---- Thomas forward elimination of level k (sound.F:659-733)
        const float temm = dts * rdz * cp * LDG(&g.mf[k]);
        const float mm = temm * (LDG(&g.c2[k]) * thc + LDG(&g.c1[k]) * thd);
        const float fwk = dts * wtn + beta * (-mm * (pp - ppm));
        const float ddk = wk + fwk;
        const float bb = 1.0f - asq * (+mm * (-p1 + p2m));
        const float dd = ddk + alph * (-mm * (pf - pfm));
        // __frcp_rn is the correctly rounded 1/x, the same value as 1.0f/x
        if (k == 2) {
          const float cc = -asq * (-mm * p2);
          const float rr = __frcp_rn(bb);
          d1p = -cc * rr;
          d2p = dd * rr;
          D1(k) = d1p;
          io.w_out[o] = d2p;
        } else {
          const float aa = -asq * (+mm * p1m);
          const float rr = __frcp_rn(aa * d1p + bb);
          if (k < nk) {
            const float cc = -asq * (-mm * p2);
            d1p = -cc * rr;
            d2p = (dd - aa * d2p) * rr;
            D1(k) = d1p;
            io.w_out[o] = d2p;
          } else {
            io.w_out[o] = (dd - aa * d2p) * rr;       // w(nk)
          }
        }
      }
      // carry to level k+1
      pid = pia; pia = piu; thd = thc; ppm = pp; wk = wkp;
      p1m = p1; p2m = p2; pfm = pf;
      cur = nxt;
    }
  }

  // ---------------- down ----------------
  {
    // the loads of level k-1 are issued before level k is computed; none of
    // them is written at level k (each level writes only its own points)
    struct DnIn { float pid, pptm, pf, po, ac, wo, d1; };
    auto dload = [&](int k, DnIn &L) {
      const long o = oc + k * plane;
      L.pid = (k > 1) ? LDG(&io.piadv[o - plane]) : 0.0f;
      L.pptm = LDG(&io.ppterm[o]);
      L.pf = io.ppd_out[o];
      L.po = io.pp_in[o];
      L.ac = p.first ? LDG(&io.wa[o]) * beta : io.rrw[o];
      L.wo = (k >= 2) ? io.w_out[o] : io.w_in[o];
      L.d1 = (k >= 2 && k < nk) ? D1(k) : 0.0f;
    };
    float wup = 0.0f;                                   // w(k+1); w(nk+1) = 0
    float pia = LDG(&io.piadv[oc + nk * plane]), piu = 0.0f;
    DnIn dc, dn;
    dload(nk, dc);
#pragma unroll 1
    for (int k = nk; k >= 1; k--) {
      if (k > 1) dload(k - 1, dn);
      const long o = oc + k * plane;
      const float pid = dc.pid, pptm = dc.pptm, pf = dc.pf, po = dc.po, ac = dc.ac;
      float wk;
      if (k == nk) wk = dc.wo;
      else if (k >= 2) wk = dc.d1 * wup + dc.wo;
      else wk = dc.wo;
      float p1, p2;
      coef(k, pid, pia, piu, pptm, &p1, &p2);
      float pn = pf + alph * (wk * p1 + wup * p2);
      if (fabsf(pn) < g.smeps) pn = 0.0f;
      const float d1 = g.kdiv * (pn - po);
      io.pp_out[o] = pn;
      io.ppd_out[o] = pn + d1;
      if (p.write_ppx) io.ppx[o] = d1;
      if (k >= 2) io.w_out[o] = wk;
      io.rrw[o] = p.last ? (ac + wk * alph) * p.tavg : ac + wk;
      wup = wk; piu = pia; pia = pid;
      dc = dn;
    }
  }
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

size_t sound_smem_bytes(const DGrid &g) { return (size_t)5 * (g.nk + 2) * SND_TX * sizeof(float); }
int sound_max_nk() { return SND_NW * SND_KPT; }
// grids with more levels run the column sweep
static bool sound_tall(const DGrid &g) { return g.nk > SND_NW * SND_KPT; }

// The acoustic kernel's forms (kNumSoundCfgs): the tile form with 8 or 4
// warps over the levels of 32 columns, and the column sweep with 32 x 4 or
// 32 x 2 columns per block.  Both tile forms cover SND_NW * SND_KPT levels.
static_assert(SND_NW * SND_KPT == (SND_NW / 2) * (SND_KPT * 2), "both tile forms cover the same levels");

static void sound_set_attributes() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_sound_tile<SND_TX, SND_NW, SND_KPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       200 * 1024);
  cudaFuncSetAttribute(k_openbc_restrict, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaFuncSetAttribute(k_sound_tile<SND_TX, SND_NW / 2, SND_KPT * 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       200 * 1024);
  // three blocks of 5 column arrays each; the rest of the unified L1 stays
  // cache for the neighbour reads of phase 1
  cudaFuncSetAttribute(k_sound_tile<SND_TX, SND_NW, SND_KPT>, cudaFuncAttributePreferredSharedMemoryCarveout, 70);
  cudaFuncSetAttribute(k_sound_tile<SND_TX, SND_NW / 2, SND_KPT * 2>, cudaFuncAttributePreferredSharedMemoryCarveout,
                       70);
  done = true;
}

// One RK stage of acoustic steps.  At the first stage the reference starts
// from the current u3d/v3d/w3d/pp3d (sound.F:192-208); at later stages it
// first resets them to the start-of-step ua/va/wa/ppi (sound.F:212-230).
// u3d/v3d/w3d/pp3d receive the result; su/sv/su2/sv2 are scratch for the
// u/v double buffer, d1/d2 for ppd, lu (scalar-shaped) for the column
// sweep's LU factors, rbnd (2 NJ*NK + 2 NI*NK floats; roflux = 1 only) for
// the restricted boundary velocities.  rru/rrv/rrw receive the averages.
void launch_sound(const DGrid &g, int nsound, int nrk, float dt,
                  const float *ua, float *u3d, const float *uten, const float *va, float *v3d, const float *vten,
                  const float *wa, float *w3d, const float *wten, const float *ppi, float *pp3d,
                  const float *piadv, const float *ppten, float *ppx, const float *thv, const float *ppterm,
                  float *rru, float *rrv, float *rrw, float *radbcw, float *radbce,
                  float *radbcs, float *radbcn, float *su, float *sv, float *su2, float *sv2,
                  float *d1, float *d2, float *lu, float *rbnd, cudaStream_t st, int64_t *nl) {
  int nloop;
  float dts;
  sound_nloop(nsound, nrk, dt, &nloop, &dts);
  // The column-sweep form keeps one thread per column, so it needs many
  // columns to fill the GPU; smaller grids use the tile form, whose warps
  // split the levels of a column.  g.sound_cfg (set by the autotuner or
  // cm1g_set_tune) overrides the choice, and CM1G_SOUND_FORM=col|tile
  // (read at each call) overrides both.
  int cfg = g.sound_cfg;
  if (cfg < 0 || cfg >= kNumSoundCfgs) cfg = ((long)g.ni * g.nj >= (long)CM1G_SOUND_COL_MIN_COLUMNS) ? 2 : 0;
  if (const char *f = getenv("CM1G_SOUND_FORM")) {
    if (!strcmp(f, "col")) cfg = 2;
    else if (!strcmp(f, "tile")) cfg = 0;
  }
  // the tile forms hold at most sound_max_nk() levels of a column
  const bool tall = sound_tall(g);
  if (tall && cfg < 2) cfg = 2;
  const bool restrict_open = g.roflux && ((g.wbc == 2 && g.ibw) || (g.ebc == 2 && g.ibe) ||
                                          (g.sbc == 2 && g.ibs) || (g.nbc == 2 && g.ibn));
  const int cty = (cfg == 3) ? 2 : 4, nw = (cfg == 1) ? SND_NW / 2 : SND_NW;
  const bool col = cfg >= 2;
  dim3 blk = col ? dim3(SNC_TX, cty) : dim3(SND_TX, nw);
  dim3 grid = col ? dim3((g.ni + SNC_TX - 1) / SNC_TX, (g.nj + cty - 1) / cty)
                  : dim3((g.ni + SND_TX - 1) / SND_TX, g.nj);
  const size_t smem = col ? 0 : sound_smem_bytes(g);
  sound_set_attributes();
  const float *uin = (nrk == 1) ? u3d : ua, *vin = (nrk == 1) ? v3d : va, *ppdin = ppx;
  for (int n = 1; n <= nloop; n++) {
    SoundIO io;
    const bool to3d = ((nloop - n) % 2) == 0;
    io.u_in = uin; io.v_in = vin;
    io.u_out = to3d ? u3d : su; io.v_out = to3d ? v3d : sv;
    if (io.u_out == io.u_in) { io.u_out = su2; io.v_out = sv2; }
    io.w_in = (n == 1 && nrk != 1) ? wa : w3d; io.w_out = w3d;
    io.pp_in = (n == 1 && nrk != 1) ? ppi : pp3d; io.pp_out = pp3d;
    io.ppd_in = ppdin; io.ppd_out = (n % 2) ? d1 : d2;
    io.rru = rru; io.rrv = rrv; io.rrw = rrw; io.wa = wa;
    io.uten = uten; io.vten = vten; io.wten = wten; io.ppten = ppten;
    io.thv = thv; io.ppterm = ppterm; io.piadv = piadv;
    io.radbcw = radbcw; io.radbce = radbce; io.radbcs = radbcs; io.radbcn = radbcn;
    io.ppx = ppx;
    io.lu = lu;
    float *ubw = rbnd, *ube = rbnd ? rbnd + (size_t)g.NJ * g.NK : nullptr;
    float *vbs = rbnd ? ube + (size_t)g.NJ * g.NK : nullptr, *vbn = rbnd ? vbs + (size_t)g.NI * g.NK : nullptr;
    io.ubw = ubw; io.ube = ube; io.vbs = vbs; io.vbn = vbn;
    SoundStep sp;
    sp.dts = dts; sp.tavg = 1.0f / (float)nloop;
    sp.first = (n == 1); sp.last = (n == nloop); sp.write_ppx = (nrk == 3 && n == nloop);
    sp.ppd_mapped = (n > 1);
    if (restrict_open) {
      ProfScope _ps("k_openbc_restrict", st);
      k_openbc_restrict<<<1, 256, (size_t)4 * (g.nk + 1) * sizeof(double), st>>>(g, io, dts, ubw, ube, vbs, vbn);
      if (nl) *nl += 1;
    }
    {
      ProfScope _ps("k_sound_step", st);
      switch (cfg) {
        case 1: k_sound_tile<SND_TX, SND_NW / 2, SND_KPT * 2><<<grid, blk, smem, st>>>(g, io, sp); break;
        case 2: k_sound_col<SNC_TX, 4><<<grid, blk, 0, st>>>(g, io, sp); break;
        case 3: k_sound_col<SNC_TX, 2><<<grid, blk, 0, st>>>(g, io, sp); break;
        default: k_sound_tile<SND_TX, SND_NW, SND_KPT><<<grid, blk, smem, st>>>(g, io, sp); break;
      }
    }
    if (nl) *nl += 1;
    uin = io.u_out; vin = io.v_out; ppdin = io.ppd_out;
  }
}

}  // namespace cm1g
