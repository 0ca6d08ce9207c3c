// k_adv.cu -- flux-form advection tendencies (adv.F, adv_routines.F).
//
// The production passes are k-marching tiles (k_mom_tile for u, v, w;
// k_advs_tile for the scalars): each face flux is evaluated once, from a
// level staged in shared memory with its 3-point halo, instead of being
// stored in dumx/dumy/dumz; the rho0-weighted fluxes rru/rrv/rrw and their
// divergence are formed on the fly, so a momentum pass reads u, v, w (and
// theta/qv for buoyancy) and writes only the tendency.  The per-point
// scalar kernels (k_advs, k_advs_pdef1/2) serve the per-routine entry
// cm1g_advs.  Every expression keeps the reference's operand order.
#include "cm1g_common.cuh"
#include "k_face.cuh"

namespace cm1g {

// ---------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------
struct Vel {  // momentum-pass view of u,v,w and the mass-flux weights
  const float *__restrict__ u, *__restrict__ v, *__restrict__ w;
};

__device__ __forceinline__ float RRU(const DGrid &g, const Vel &q, int i, int j, int k) {
  return LDG(&g.rho0[k]) * LDG(&q.u[iU(g, i, j, k)]);             // solve2.F:499
}
__device__ __forceinline__ float RRV(const DGrid &g, const Vel &q, int i, int j, int k) {
  return LDG(&g.rho0[k]) * LDG(&q.v[iV(g, i, j, k)]);             // solve2.F:504
}
__device__ __forceinline__ float RRW(const DGrid &g, const Vel &q, int i, int j, int k) {
  if (k <= 1 || k >= g.nk + 1) return 0.0f;                       // solve2.F:509-511
  return LDG(&g.rf0[k]) * LDG(&q.w[iW(g, i, j, k)]);              // solve2.F:516
}
// divx of the momentum pass (solve2.F:590-596)
__device__ __forceinline__ float DIVX(const DGrid &g, const Vel &q, int i, int j, int k) {
  float d = ((RRU(g, q, i + 1, j, k) - RRU(g, q, i, j, k)) * g.rdx * LDG(&g.uh[i - g.ib]) +
             (RRV(g, q, i, j + 1, k) - RRV(g, q, i, j, k)) * g.rdy * LDG(&g.vh[j - g.jb])) +
            (RRW(g, q, i, j, k + 1) - RRW(g, q, i, j, k)) * g.rdz * LDG(&g.mh[k]);
  if (fabsf(d) < g.smeps) d = 0.0f;
  return d;
}

// buoyancy of a w level from th3d(i,j,kk) and qv(i,j,kk) (solve2.F:313-446, dum8 of the moist and dry forms)
__device__ __forceinline__ float buoy_v(const DGrid &g, float th3, float qvv, bool moist, int kk) {
  if (moist) {
    float q = fmaxf(qvv, 0.0f);
    float qli = fmaxf(0.0f, 0.0f + 0.0f);
    return g.c.g * ((th3 * LDG(&g.rth0[kk]) + g.c.repsm1 * (q - LDG(&g.qv0[kk]))) - ((qli - LDG(&g.qc0[kk])) - LDG(&g.qi0[kk])));
  }
  return g.c.g * th3 * LDG(&g.rth0[kk]);
}


// ---------------------------------------------------------------------
// Tiled momentum advection (the production path of advu/advv/advw).
//
// divx of the momentum pass (solve2.F:590-596) is formed once per stage at
// the s-points i = 0..ni+1, j = 0..nj+1 by k_mom_divx.  k_mom_tile then
// works like the scalar tile: a block owns TX x TY points of one velocity
// component (STAG 2 u, 3 v, 4 w) and marches upward; at each level the
// component is staged with a 3-point lateral halo in shared memory, every
// x- and y-face flux (hadv_flx5 stag=2/3/4) is evaluated once, and the
// vertical face flux (vadv_flx5 with the lower-order pieces at the column
// ends) comes from a per-thread register window and is carried to the next
// level.  The face velocities are formed exactly as the reference forms
// them (ubar/vbar/wbar of adv_routines.F:1388-1460, 3299-3384) and the
// open-boundary fixes of adv.F are applied to the cells they concern.
// ---------------------------------------------------------------------
__global__ void k_mom_divx(DGrid g, Vel q, float *__restrict__ divx) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni + 1) return;
  divx[iS(g, i, j, k)] = DIVX(g, q, i, j, k);
}

// vertical face flux of a u/v column at w-level kk; wv[d+3] = a(kk+d), d = -3..2
__device__ __forceinline__ float zflux_uv(const DGrid &g, const float *wv, float wbar, int kk) {
  const int nk = g.nk;
  auto A = [&](int d) { return wv[d + 3]; };
  if (kk >= 4 && kk <= nk - 2) {
    const bool up = (wbar >= 0.0f);
    return wbar * flx5(up ? A(-3) : A(2), up ? A(-2) : A(1), up ? A(-1) : A(0), up ? A(0) : A(-1), up ? A(1) : A(-2));
  }
  const float c2k = LDG(&g.c2[kk]);
  if (kk == 2) {
    if (wbar >= 0.0f) { float cc2 = 0.5f * (c2k + c2k), cc1 = 1.0f - cc2; return wbar * (cc1 * A(-1) + cc2 * A(0)); }
    return wbar * flx3(A(1), A(0), A(-1));
  }
  if (kk == nk) {
    if (wbar >= 0.0f) return wbar * flx3(A(-2), A(-1), A(0));
    float cc2 = 0.5f * (c2k + c2k), cc1 = 1.0f - cc2; return wbar * (cc1 * A(-1) + cc2 * A(0));
  }
  if (kk == 3) {
    if (wbar >= 0.0f) return wbar * flx3(A(-2), A(-1), A(0));
    return wbar * flx5(A(2), A(1), A(0), A(-1), A(-2));
  }
  if (wbar >= 0.0f) return wbar * flx5(A(-3), A(-2), A(-1), A(0), A(1));
  return wbar * flx3(A(1), A(0), A(-1));
}

// vertical face flux of a w column at s-level kk; wv[d+2] = w(kk+d), d = -2..3
__device__ __forceinline__ float zflux_w(const DGrid &g, const float *wv, float wbar, int kk) {
  const int nk = g.nk;
  auto A = [&](int d) { return wv[d + 2]; };
  if (kk >= 3 && kk <= nk - 2) {
    const bool up = (wbar >= 0.0f);
    return wbar * flx5(up ? A(-2) : A(3), up ? A(-1) : A(2), up ? A(0) : A(1), up ? A(1) : A(0), up ? A(2) : A(-1));
  }
  if (kk == 1) {
    if (wbar >= 0.0f) return wbar * 0.5f * (A(0) + A(1));
    return wbar * flx3(A(2), A(1), A(0));
  }
  if (kk == nk) {
    if (wbar >= 0.0f) return wbar * flx3(A(-1), A(0), A(1));
    return wbar * 0.5f * (A(0) + A(1));
  }
  if (kk == 2) {
    if (wbar >= 0.0f) return wbar * flx3(A(-1), A(0), A(1));
    return wbar * flx5(A(3), A(2), A(1), A(0), A(-1));
  }
  if (wbar >= 0.0f) return wbar * flx5(A(-2), A(-1), A(0), A(1), A(2));
  return wbar * flx3(A(2), A(1), A(0));
}

__device__ __forceinline__ float hflux_mom(float r, const float *p, int stride) {
  const float a0 = p[0], a1 = p[stride], a2 = p[2 * stride], a3 = p[3 * stride], a4 = p[4 * stride], a5 = p[5 * stride];
  const bool up = (r >= 0.0f);
  return r * flx5(up ? a0 : a5, up ? a1 : a4, up ? a2 : a3, up ? a3 : a2, up ? a4 : a1);
}

template <int TX, int TY, int KC, int STAG, int DIFF>
__global__ void __launch_bounds__(TX * TY, 3) k_mom_tile(DGrid g, Vel q, const float *__restrict__ divx,
                                                      const float *ten1, float *ten,
                                                      const float *__restrict__ th3d, const float *__restrict__ qv,
                                                      const float *__restrict__ b8, Diff6 df) {
  constexpr int NT = TX * TY;
  constexpr int SW = TX + 6, SH = TY + 6, SP = SW + 1;
  constexpr int NST = (SW * SH + NT - 1) / NT;
  constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
  __shared__ float ss[SH * SP];
  __shared__ float fx[NFX], fxv[NFX], fy[NFY], fyv[NFY];
  __shared__ float dfx[NFX], dfy[NFY];     // 6th-order diffusion fluxes
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int i0 = 1 + (int)blockIdx.x * TX, j0 = 1 + (int)blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const int pitch = (STAG == 2) ? g.NI + 1 : g.NI;      // x extent of the component's array
  const int rows = (STAG == 3) ? g.NJ + 1 : g.NJ;
  const int plane = pitch * rows;   // < 2^31 points (cm1g_init)
  const float *__restrict__ A = (STAG == 2) ? q.u : (STAG == 3) ? q.v : q.w;
  const int ilo = (STAG == 2) ? (g.ibw ? 2 : 1) : 1, ihi = (STAG == 2) ? (g.ibe ? ni : ni + 1) : ni;
  const int jlo = (STAG == 3) ? (g.ibs ? 2 : 1) : 1, jhi = (STAG == 3) ? (g.ibn ? nj : nj + 1) : nj;
  const bool active = (i >= ilo && i <= ihi && j >= jlo && j <= jhi);
  const int iea = ni + g.ngxy + (STAG == 2 ? 1 : 0), jea = nj + g.ngxy + (STAG == 3 ? 1 : 0);
  const bool doitw = (g.wbc == 2 && g.ibw), doite = (g.ebc == 2 && g.ibe);
  const bool doits = (g.sbc == 2 && g.ibs), doitn = (g.nbc == 2 && g.ibn);
  const int oc = active ? (i - g.ib) + pitch * (j - g.jb) : 0;

  int soff[NST], sidx[NST];
#pragma unroll
  for (int s = 0; s < NST; s++) {
    const int t = tid + s * NT;
    soff[s] = -1; sidx[s] = -1;
    if (t < SW * SH) {
      const int yy = t / SW, xx = t - yy * SW;
      const int ii = i0 - 3 + xx, jj = j0 - 3 + yy;
      sidx[s] = yy * SP + xx;
      if (ii <= iea && jj <= jea) soff[s] = (ii - g.ib) + pitch * (jj - g.jb);
    }
  }
  // faces owned by this thread: index-space position (-1 in fxi: none)
  using FS = FaceSlots<NT, NFX, NFY>;
  int fxi[2], fxj[2], fyi[2], fyj[2];
#pragma unroll
  for (int s = 0; s < 2; s++) {
    fxi[s] = -1; fxj[s] = 0; fyi[s] = -1; fyj[s] = 0;
    const int f = FS::x(tid, s), fy_ = FS::y(tid, s);
    if (f < NFX) {
      const int row = f / (TX + 1), col = f - row * (TX + 1);
      const int ii = (STAG == 2) ? i0 - 1 + col : i0 + col, jj = j0 + row;   // s-point (u) or u-point (v, w)
      if (ii >= 0 && ii <= ni + 1 && jj <= nj + 1) { fxi[s] = ii; fxj[s] = jj; }
    }
    if (fy_ < NFY) {
      const int row = fy_ / TX, col = fy_ - row * TX;
      const int ii = i0 + col, jj = (STAG == 3) ? j0 - 1 + row : j0 + row;    // s-point (v) or v-point (u, w)
      if (jj >= 0 && jj <= nj + 1 && ii <= ni + 1) { fyi[s] = ii; fyj[s] = jj; }
    }
  }

  // vertical window: wv[d] = a(kb0 + d), kb0 = upper face - 3 (u, v) or - 2 (w)
  const int kfirst = (STAG == 4) ? 2 : 1;
  const int kc0 = kfirst + (int)blockIdx.z * KC, kc1 = min(nk, kc0 + KC - 1);
  const int koff = (STAG == 4) ? -2 : -3;
  const int kmaxA = (STAG == 4) ? nk + 2 : nk + 1;
  auto AV = [&](int kk) -> float { return (kk >= 0 && kk <= kmaxA) ? LDG(&A[kk * plane + oc]) : 0.0f; };
  auto RRWc = [&](int ii, int jj, int kk) -> float {
    if (kk <= 1 || kk >= nk + 1) return 0.0f;
    return LDG(&g.rf0[kk]) * LDG(&q.w[iW(g, ii, jj, kk)]);
  };
  auto WBAR = [&](int kk) -> float {
    if (STAG == 2) return 0.5f * (RRWc(i, j, kk) + RRWc(i - 1, j, kk));
    if (STAG == 3) return 0.5f * (RRWc(i, j, kk) + RRWc(i, j - 1, kk));
    return 0.5f * (RRWc(i, j, kk) + RRWc(i, j, kk + 1));
  };
  auto ZF = [&](const float *win, int kk) -> float {
    return (STAG == 4) ? zflux_w(g, win, WBAR(kk), kk) : zflux_uv(g, win, WBAR(kk), kk);
  };
  // faces of level k: upper ku, lower ku-1; u/v faces exist for kk = 2..nk, w faces for kk = 1..nk
  const int kfmin = (STAG == 4) ? 1 : 2;
  float wv[6];
  float fzlo = 0.0f;
  {
    const int ku = (STAG == 4) ? kc0 : kc0 + 1;
#pragma unroll
    for (int d = 0; d < 6; d++) wv[d] = active ? AV(ku + koff + d) : 0.0f;
    if (active && ku - 1 >= kfmin) {
      float w0[6];
#pragma unroll
      for (int d = 0; d < 6; d++) w0[d] = AV(ku - 1 + koff + d);
      fzlo = ZF(w0, ku - 1);
    }
  }

  // Every global read of a level is issued one level ahead (into the p*
  // registers), so it is in flight while the previous level computes; the
  // component arrays and the other inputs are not written by this kernel
  // (ten may alias ten1 only point by point).
  float pst[NST], pxa[2], pxb[2], pya[2], pyb[2], pw0 = 0.0f, pw1 = 0.0f, pt1 = 0.0f, pd0 = 0.0f, pd1 = 0.0f;
  float pb0 = 0.0f, pb1 = 0.0f, pb2 = 0.0f, pb3 = 0.0f, pwtop = 0.0f;
  auto fetch = [&](int kf) {
    const float *Ak = A + kf * plane;
#pragma unroll
    for (int s = 0; s < NST; s++) pst[s] = (soff[s] >= 0) ? LDG(&Ak[soff[s]]) : 0.0f;
#pragma unroll
    for (int s = 0; s < 2; s++) {
      pxa[s] = pxb[s] = pya[s] = pyb[s] = 0.0f;
      if (fxi[s] >= 0) {
        const int ii = fxi[s], jj = fxj[s];
        if (STAG == 3) { pxa[s] = LDG(&q.u[iU(g, ii, jj, kf)]); pxb[s] = LDG(&q.u[iU(g, ii, jj - 1, kf)]); }
        if (STAG == 4) { pxa[s] = LDG(&q.u[iU(g, ii, jj, kf)]); pxb[s] = LDG(&q.u[iU(g, ii, jj, kf - 1)]); }
      }
      if (fyi[s] >= 0) {
        const int ii = fyi[s], jj = fyj[s];
        if (STAG == 2) { pya[s] = LDG(&q.v[iV(g, ii, jj, kf)]); pyb[s] = LDG(&q.v[iV(g, ii - 1, jj, kf)]); }
        if (STAG == 4) { pya[s] = LDG(&q.v[iV(g, ii, jj, kf)]); pyb[s] = LDG(&q.v[iV(g, ii, jj, kf - 1)]); }
      }
    }
    if (active) {
      const int ku = (STAG == 4) ? kf : kf + 1;       // upper face of level kf
      if (ku <= nk) {
        const int ia = (STAG == 2) ? i - 1 : i, ja = (STAG == 3) ? j - 1 : j, ka = (STAG == 4) ? ku + 1 : ku;
        pw0 = (ku <= 1 || ku >= nk + 1) ? 0.0f : LDG(&q.w[iW(g, i, j, ku)]);
        pw1 = (ka <= 1 || ka >= nk + 1) ? 0.0f : LDG(&q.w[iW(g, ia, ja, ka)]);
      }
      const int oS = (int)iS(g, i, j, kf);
      pt1 = ten1[kf * plane + oc];
      pd0 = LDG(&divx[oS]);
      pd1 = LDG(&divx[oS - ((STAG == 2) ? 1 : (STAG == 3) ? g.NI : g.NI * g.NJ)]);
      if (STAG == 4 && b8) {          // buoyancy of the stage set-up (liquid water present)
        pb0 = LDG(&b8[oS - g.NI * g.NJ]); pb1 = LDG(&b8[oS]);
      } else if (STAG == 4 && th3d) {
        pb0 = LDG(&th3d[oS - g.NI * g.NJ]); pb1 = LDG(&th3d[oS]);
        if (qv) { pb2 = LDG(&qv[oS - g.NI * g.NJ]); pb3 = LDG(&qv[oS]); }
      }
      pwtop = AV(ku + koff + 5);
    }
  };
  // wbar of face kk from its two averaged w values (RRW of solve2.F:509-516)
  auto WBARp = [&](int kk, float w0, float w1) -> float {
    const int ka = (STAG == 4) ? kk + 1 : kk;
    const float r0 = (kk <= 1 || kk >= nk + 1) ? 0.0f : LDG(&g.rf0[kk]) * w0;
    const float r1 = (ka <= 1 || ka >= nk + 1) ? 0.0f : LDG(&g.rf0[ka]) * w1;
    return 0.5f * (r0 + r1);
  };
  fetch(kc0);

  for (int k = kc0; k <= kc1; k++) {
    const float r0k = LDG(&g.rho0[k]);
#pragma unroll
    for (int s = 0; s < NST; s++)
      if (sidx[s] >= 0) ss[sidx[s]] = pst[s];
    // face velocities that come from the other components
    float ubar[2] = {0.0f, 0.0f}, vbar[2] = {0.0f, 0.0f};
    float c1k = 0.0f, c2k = 0.0f, cc1 = 0.0f, cc2 = 0.0f;
    if (STAG == 4) {
      c1k = LDG(&g.c1[k]); c2k = LDG(&g.c2[k]);
      cc2 = 0.5f * (c2k + c2k); cc1 = 1.0f - cc2;
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
      if (STAG == 3) ubar[s] = 0.5f * (r0k * pxa[s] + r0k * pxb[s]);
      if (STAG == 4) ubar[s] = cc2 * (r0k * pxa[s]) + cc1 * (LDG(&g.rho0[k - 1]) * pxb[s]);
      if (STAG == 2) vbar[s] = 0.5f * (r0k * pya[s] + r0k * pyb[s]);
      if (STAG == 4) vbar[s] = cc2 * (r0k * pya[s]) + cc1 * (LDG(&g.rho0[k - 1]) * pyb[s]);
    }
    const float w0 = pw0, w1 = pw1, t1 = pt1, dv0 = pd0, dv1 = pd1, b0 = pb0, b1 = pb1, b2 = pb2, b3 = pb3;
    if (k < kc1) fetch(k + 1);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const int f = FS::x(tid, s);
      if (fxi[s] >= 0) {
        const int row = f / (TX + 1), col = f - row * (TX + 1);
        const float *p = &ss[(row + 3) * SP + col];
        float r = ubar[s];
        if (STAG == 2) r = 0.5f * (r0k * p[2] + r0k * p[3]);
        fx[f] = hflux_mom(r, p, 1);
        fxv[f] = r;
        if (DIFF) {
          // the face between p[2] and p[3]: s-point fxi (u: adv.F:1190-1193),
          // u-point fxi (v: adv.F:2128-2132; w: adv.F:3124-3130)
          const int ii = fxi[s], jj = fxj[s];
          const float d = diff6_stencil(p[0], p[1], p[2], p[3], p[4], p[5]);
          float fd;
          if (STAG == 2) {
            fd = d * LDG(&df.rho[iS(g, ii, jj, k)]);
          } else if (STAG == 3) {
            fd = d * 0.25f * ((LDG(&df.rho[iS(g, ii - 1, jj - 1, k)]) + LDG(&df.rho[iS(g, ii, jj, k)])) +
                              (LDG(&df.rho[iS(g, ii - 1, jj, k)]) + LDG(&df.rho[iS(g, ii, jj - 1, k)])));
          } else {
            fd = d * 0.5f * (cc2 * (LDG(&df.rho[iS(g, ii - 1, jj, k)]) + LDG(&df.rho[iS(g, ii, jj, k)])) +
                             cc1 * (LDG(&df.rho[iS(g, ii - 1, jj, k - 1)]) + LDG(&df.rho[iS(g, ii, jj, k - 1)])));
          }
          dfx[f] = diff6_limit(fd, p[3], p[2], df.mdiff);
        }
      }
      if (fyi[s] >= 0) {
        const int fy_ = FS::y(tid, s);
        const int row = fy_ / TX, col = fy_ - row * TX;
        const float *p = &ss[row * SP + col + 3];
        float r = vbar[s];
        if (STAG == 3) r = 0.5f * (r0k * p[2 * SP] + r0k * p[3 * SP]);
        fy[fy_] = hflux_mom(r, p, SP);
        fyv[fy_] = r;
        if (DIFF) {
          // the face between p[2 SP] and p[3 SP]: v-point fyj (u: adv.F:1210-1215;
          // w: adv.F:3146-3152), s-point fyj (v: adv.F:2151-2153)
          const int ii = fyi[s], jj = fyj[s];
          const float d = diff6_stencil(p[0], p[SP], p[2 * SP], p[3 * SP], p[4 * SP], p[5 * SP]);
          float fd;
          if (STAG == 2) {
            fd = d * 0.25f * ((LDG(&df.rho[iS(g, ii - 1, jj - 1, k)]) + LDG(&df.rho[iS(g, ii, jj, k)])) +
                              (LDG(&df.rho[iS(g, ii - 1, jj, k)]) + LDG(&df.rho[iS(g, ii, jj - 1, k)])));
          } else if (STAG == 3) {
            fd = d * LDG(&df.rho[iS(g, ii, jj, k)]);
          } else {
            fd = d * 0.5f * (cc2 * (LDG(&df.rho[iS(g, ii, jj - 1, k)]) + LDG(&df.rho[iS(g, ii, jj, k)])) +
                             cc1 * (LDG(&df.rho[iS(g, ii, jj - 1, k - 1)]) + LDG(&df.rho[iS(g, ii, jj, k - 1)])));
          }
          dfy[fy_] = diff6_limit(fd, p[3 * SP], p[2 * SP], df.mdiff);
        }
      }
    }
    const int ku = (STAG == 4) ? k : k + 1;
    float fzhi = 0.0f, ac = 0.0f;
    if (active) {
      ac = ss[(ty + 3) * SP + tx + 3];
      if (ku <= nk) {
        const float wb = WBARp(ku, w0, w1);
        fzhi = (STAG == 4) ? zflux_w(g, wv, wb, ku) : zflux_uv(g, wv, wb, ku);
      }
    }
    __syncthreads();
    if (active) {
      const int xi = ty * (TX + 1) + tx, yi = ty * TX + tx;
      float fx0 = fx[xi], fxp = fx[xi + 1], fy0 = fy[yi], fyp = fy[yi + TX];
      float advx, advy, advz;
      const int oS = (int)iS(g, i, j, k);
      if (STAG == 2) {
        auto RRV2 = [&](int ii, int jj) { return LDG(&g.rho0[k]) * LDG(&q.v[iV(g, ii, jj, k)]); };
        advx = -(fxp - fx0) * g.rdx * LDG(&g.uf[i - g.ib]);
        const bool fs = doits && j == 1 && (RRV2(i, 1) + RRV2(i - 1, 1)) >= 0.0f;
        const bool fn = doitn && j == nj && (RRV2(i, nj + 1) + RRV2(i - 1, nj + 1)) <= 0.0f;
        if (fs) fy0 = fyp;
        if (fn) fyp = fy0;
        advy = -(fyp - fy0) * g.rdy * LDG(&g.vh[j - g.jb]);
        if (fs)
          advy = advy - LDG(&q.u[iU(g, i, 1, k)]) * 0.5f *
                            ((RRV2(i - 1, 2) - RRV2(i - 1, 1)) + (RRV2(i, 2) - RRV2(i, 1))) * g.rdy * LDG(&g.vh[1 - g.jb]);
        if (fn)
          advy = advy - LDG(&q.u[iU(g, i, nj, k)]) * 0.5f *
                            ((RRV2(i - 1, nj + 1) - RRV2(i - 1, nj)) + (RRV2(i, nj + 1) - RRV2(i, nj))) * g.rdy *
                            LDG(&g.vh[nj - g.jb]);
      } else if (STAG == 3) {
        auto RRU2 = [&](int ii, int jj) { return LDG(&g.rho0[k]) * LDG(&q.u[iU(g, ii, jj, k)]); };
        const bool fw = doitw && i == 1 && (RRU2(1, j) + RRU2(1, j - 1)) >= 0.0f;
        const bool fe = doite && i == ni && (RRU2(ni + 1, j) + RRU2(ni + 1, j - 1)) <= 0.0f;
        if (fw) fx0 = fxp;
        if (fe) fxp = fx0;
        advx = -(fxp - fx0) * g.rdx * LDG(&g.uh[i - g.ib]);
        advy = -(fyp - fy0) * g.rdy * LDG(&g.vf[j - g.jb]);
        if (fw)
          advx = advx - LDG(&q.v[iV(g, 1, j, k)]) * 0.5f *
                            ((RRU2(2, j - 1) - RRU2(1, j - 1)) + (RRU2(2, j) - RRU2(1, j))) * g.rdx * LDG(&g.uh[1 - g.ib]);
        if (fe)
          advx = advx - LDG(&q.v[iV(g, ni, j, k)]) * 0.5f *
                            ((RRU2(ni + 1, j - 1) - RRU2(ni, j - 1)) + (RRU2(ni + 1, j) - RRU2(ni, j))) * g.rdx *
                            LDG(&g.uh[ni - g.ib]);
      } else {
        const float ub0 = fxv[xi], ubp = fxv[xi + 1], vb0 = fyv[yi], vbp = fyv[yi + TX];
        const bool fw = doitw && i == 1 && ub0 >= 0.0f, fe = doite && i == ni && ubp <= 0.0f;
        const bool fs = doits && j == 1 && vb0 >= 0.0f, fn = doitn && j == nj && vbp <= 0.0f;
        if (fw) fx0 = fxp;
        if (fe) fxp = fx0;
        if (fs) fy0 = fyp;
        if (fn) fyp = fy0;
        advx = -(fxp - fx0) * g.rdx * LDG(&g.uh[i - g.ib]);
        advy = -(fyp - fy0) * g.rdy * LDG(&g.vh[j - g.jb]);
        auto RRUk = [&](int ii, int kk) { return LDG(&g.rho0[kk]) * LDG(&q.u[iU(g, ii, j, kk)]); };
        auto RRVk = [&](int jj, int kk) { return LDG(&g.rho0[kk]) * LDG(&q.v[iV(g, i, jj, kk)]); };
        const float ww = ac;
        if (fw)
          advx = advx - ww * (c1k * (RRUk(2, k - 1) - RRUk(1, k - 1)) + c2k * (RRUk(2, k) - RRUk(1, k))) * g.rdx *
                            LDG(&g.uh[1 - g.ib]);
        if (fe)
          advx = advx - ww * (c1k * (RRUk(ni + 1, k - 1) - RRUk(ni, k - 1)) + c2k * (RRUk(ni + 1, k) - RRUk(ni, k))) *
                            g.rdx * LDG(&g.uh[ni - g.ib]);
        if (fs)
          advy = advy - ww * (c1k * (RRVk(2, k - 1) - RRVk(1, k - 1)) + c2k * (RRVk(2, k) - RRVk(1, k))) * g.rdy *
                            LDG(&g.vh[1 - g.jb]);
        if (fn)
          advy = advy - ww * (c1k * (RRVk(nj + 1, k - 1) - RRVk(nj, k - 1)) + c2k * (RRVk(nj + 1, k) - RRVk(nj, k))) *
                            g.rdy * LDG(&g.vh[nj - g.jb]);
      }
      if (DIFF) {   // adv.F:1199-1201, 1220-1222; 2139-2141, 2160-2162; 3135-3137, 3160-3162
        const float ddx = df.coef * (dfx[xi + 1] - dfx[xi]), ddy = df.coef * (dfy[yi + TX] - dfy[yi]);
        if (STAG == 2) {
          const float rs = LDG(&df.rho[iS(g, i - 1, j, k)]) + LDG(&df.rho[iS(g, i, j, k)]);
          advx = advx + ddx * (r0k + r0k) / rs;
          advy = advy + ddy * (r0k + r0k) / rs;
        } else if (STAG == 3) {
          const float rs = LDG(&df.rho[iS(g, i, j - 1, k)]) + LDG(&df.rho[iS(g, i, j, k)]);
          advx = advx + ddx * (r0k + r0k) / rs;
          advy = advy + ddy * (r0k + r0k) / rs;
        } else {
          const float rf = LDG(&g.rf0[k]);
          const float rs = 0.5f * (LDG(&df.rho[iS(g, i, j, k - 1)]) + LDG(&df.rho[iS(g, i, j, k)]));
          advx = advx + ddx * rf / rs;
          advy = advy + ddy * rf / rs;
        }
      }
      if (STAG == 4) {
        advz = -(fzhi - fzlo) * g.rdz * LDG(&g.mf[k]);
      } else {
        const float mhk = LDG(&g.mh[k]);
        if (k == 1) advz = -fzhi * g.rdz * mhk;
        else if (k == nk) advz = +fzlo * g.rdz * mhk;
        else advz = -(fzhi - fzlo) * g.rdz * mhk;
      }
      const int o = k * plane + oc;
      if (STAG == 2) {
        ten[o] = t1 + (((advx + advy) + advz) + ac * 0.5f * (dv0 + dv1)) * LDG(&g.rr0[k]);
      } else if (STAG == 3) {
        ten[o] = t1 + (((advx + advy) + advz) + ac * 0.5f * (dv0 + dv1)) * LDG(&g.rr0[k]);
      } else {
        float t = t1 + (((advx + advy) + advz) + ac * (c2k * dv0 + c1k * dv1)) * LDG(&g.rrf0[k]);
        if (b8) t = t + (c1k * b0 + c2k * b1);
        else if (th3d) t = t + (c1k * buoy_v(g, b0, b2, qv != nullptr, k - 1) + c2k * buoy_v(g, b1, b3, qv != nullptr, k));
        ten[o] = t;
      }
#pragma unroll
      for (int d = 0; d < 5; d++) wv[d] = wv[d + 1];
      wv[5] = pwtop;            // top of the window of level k+1 (fetched above)
      fzlo = fzhi;
    }
  }
}

template <int TX, int TY, int KC>
static void mom_tiles_shape(const DGrid &g, const Vel &q, const float *uten1, const float *vten1,
                            const float *wten1, float *uten, float *vten, float *wten, const float *th3d,
                            const float *qv, const float *b8, const float *divx, const Diff6 &df,
                            cudaStream_t st, int which) {
  dim3 blk(TX, TY);
  const int kch = (g.nk + KC - 1) / KC, kchw = (g.nk - 1 + KC - 1) / KC;
  if (which & 1) {
    dim3 grid((g.ni + 1 + TX - 1) / TX, (g.nj + TY - 1) / TY, kch);
    ProfScope _ps("k_advu", st);
    if (df.rho) k_mom_tile<TX, TY, KC, 2, 1><<<grid, blk, 0, st>>>(g, q, divx, uten1, uten, nullptr, nullptr, nullptr, df);
    else k_mom_tile<TX, TY, KC, 2, 0><<<grid, blk, 0, st>>>(g, q, divx, uten1, uten, nullptr, nullptr, nullptr, df);
  }
  if (which & 2) {
    dim3 grid((g.ni + TX - 1) / TX, (g.nj + 1 + TY - 1) / TY, kch);
    ProfScope _ps("k_advv", st);
    if (df.rho) k_mom_tile<TX, TY, KC, 3, 1><<<grid, blk, 0, st>>>(g, q, divx, vten1, vten, nullptr, nullptr, nullptr, df);
    else k_mom_tile<TX, TY, KC, 3, 0><<<grid, blk, 0, st>>>(g, q, divx, vten1, vten, nullptr, nullptr, nullptr, df);
  }
  if (which & 4) {
    dim3 grid((g.ni + TX - 1) / TX, (g.nj + TY - 1) / TY, kchw);
    ProfScope _ps("k_advw", st);
    if (df.rho) k_mom_tile<TX, TY, KC, 4, 1><<<grid, blk, 0, st>>>(g, q, divx, wten1, wten, th3d, qv, b8, df);
    else k_mom_tile<TX, TY, KC, 4, 0><<<grid, blk, 0, st>>>(g, q, divx, wten1, wten, th3d, qv, b8, df);
  }
}

void launch_adv_momentum(const DGrid &g, const float *u, const float *v, const float *w,
                         const float *uten1, const float *vten1, const float *wten1,
                         float *uten, float *vten, float *wten, const float *th3d, const float *qv,
                         float *divx, cudaStream_t st, int64_t *nl, const Diff6 *diff, const float *b8,
                         int which) {
  // which: bit 0 u (advu), bit 1 v (advv), bit 2 w (advw)
  Vel q{u, v, w};
  const Diff6 df = diff ? *diff : Diff6{};
  {
    dim3 grid((g.ni + 2 + 127) / 128, g.nj + 2, g.nk);
    ProfScope _ps("k_mom_divx", st);
    k_mom_divx<<<grid, 128, 0, st>>>(g, q, divx);
  }
#define CM1G_MOM_SHAPE(n)                                                                                     \
  case n:                                                                                                     \
    mom_tiles_shape<kTileShapes[n][0], kTileShapes[n][1], kTileShapes[n][2]>(g, q, uten1, vten1, wten1, uten, \
                                                                             vten, wten, th3d, qv, b8, divx, df, st, \
                                                                             which);                                \
    break;
  switch (g.tile_mom) {
    CM1G_MOM_SHAPE(1)
    CM1G_MOM_SHAPE(2)
    CM1G_MOM_SHAPE(3)
    CM1G_MOM_SHAPE(4)
    default: CM1G_MOM_SHAPE(0)
  }
#undef CM1G_MOM_SHAPE
  if (nl) *nl += 1 + ((which & 1) != 0) + ((which & 2) != 0) + ((which & 4) != 0);
}

// ---------------------------------------------------------------------
// advs: adv.F:14-903 for one scalar.
//
// The fluxes use the small-step-averaged velocities rru/rrv/rrw as sound
// leaves them; getdivx's rho0/rf0 weighting (misclibs.F:251-276) and divx
// (misclibs.F:330-340) are applied on the fly.  `sadd` (the theta offset
// th0-300, solve2.F:1365-1372) is added to s when given.
// ---------------------------------------------------------------------
struct SAdv {
  const float *__restrict__ rru, *__restrict__ rrv, *__restrict__ rrw;  // averaged velocities or fluxes
  const float *__restrict__ s;      // advected field (full halo)
  const float *__restrict__ s0;     // RK base value (pdef only)
  const float *__restrict__ divx;   // caller's divx (adv.F argument) or null: formed here
  const float *__restrict__ thterm; // moist theta: thten -= div(u_avg)*thterm (solve2.F:1320-1329)
  int weighted;                     // 1: rru/rrv/rrw are velocities to be weighted here
  int sadd;                         // add th0(k)-th0r to s (theta)
  Diff6 df{};                       // 6th-order diffusion (df.rho null: none)
};

__device__ __forceinline__ float sval(const DGrid &g, const SAdv &a, int i, int j, int k) {
  float v = LDG(&a.s[iS(g, i, j, k)]);
  if (a.sadd) v = (LDG(&g.th0[k]) - 300.0f) + v;
  return v;
}
__device__ __forceinline__ float FU(const DGrid &g, const SAdv &a, int i, int j, int k) {
  float v = LDG(&a.rru[iU(g, i, j, k)]);
  return a.weighted ? v * LDG(&g.rho0[k]) : v;
}
__device__ __forceinline__ float FV(const DGrid &g, const SAdv &a, int i, int j, int k) {
  float v = LDG(&a.rrv[iV(g, i, j, k)]);
  return a.weighted ? v * LDG(&g.rho0[k]) : v;
}
__device__ __forceinline__ float FW(const DGrid &g, const SAdv &a, int i, int j, int k) {
  if (a.weighted && (k <= 1 || k >= g.nk + 1)) return 0.0f;
  float v = LDG(&a.rrw[iW(g, i, j, k)]);
  return a.weighted ? v * LDG(&g.rf0[k]) : v;
}
// getdiv of the averaged velocities (misclibs.F:127-136), for the moist theta term
__device__ __forceinline__ float RAWDIV(const DGrid &g, const SAdv &a, int i, int j, int k) {
  auto W = [&](int kk) { return (kk <= 1 || kk >= g.nk + 1) ? 0.0f : LDG(&a.rrw[iW(g, i, j, kk)]); };
  float d = ((LDG(&a.rru[iU(g, i + 1, j, k)]) - LDG(&a.rru[iU(g, i, j, k)])) * g.rdx * LDG(&g.uh[i - g.ib]) +
             (LDG(&a.rrv[iV(g, i, j + 1, k)]) - LDG(&a.rrv[iV(g, i, j, k)])) * g.rdy * LDG(&g.vh[j - g.jb])) +
            (W(k + 1) - W(k)) * g.rdz * LDG(&g.mh[k]);
  if (fabsf(d) < g.smeps) d = 0.0f;
  return d;
}
__device__ __forceinline__ float SDIV(const DGrid &g, const SAdv &a, int i, int j, int k) {
  if (a.divx) return LDG(&a.divx[iS(g, i, j, k)]);
  float d = ((FU(g, a, i + 1, j, k) - FU(g, a, i, j, k)) * g.rdx * LDG(&g.uh[i - g.ib]) +
             (FV(g, a, i, j + 1, k) - FV(g, a, i, j, k)) * g.rdy * LDG(&g.vh[j - g.jb])) +
            (FW(g, a, i, j, k + 1) - FW(g, a, i, j, k)) * g.rdz * LDG(&g.mh[k]);
  if (fabsf(d) < g.smeps) d = 0.0f;
  return d;
}

// x-face flux dumx(i,j,k) (hadv_flx5/hadv_weno5 stag=1)
__device__ __forceinline__ float sflux_x(const DGrid &g, const SAdv &a, int i, int j, int k, int weno, int pdef, double weps) {
  float r = FU(g, a, i, j, k), s1, s2, s3, s4, s5;
  if (r >= 0.0f) { s1 = sval(g, a, i - 3, j, k); s2 = sval(g, a, i - 2, j, k); s3 = sval(g, a, i - 1, j, k); s4 = sval(g, a, i, j, k); s5 = sval(g, a, i + 1, j, k); }
  else { s1 = sval(g, a, i + 2, j, k); s2 = sval(g, a, i + 1, j, k); s3 = sval(g, a, i, j, k); s4 = sval(g, a, i - 1, j, k); s5 = sval(g, a, i - 2, j, k); }
  if (!weno) return r * flx5(s1, s2, s3, s4, s5);
  if (pdef == 1 && !(absmax5(s1, s2, s3, s4, s5) > (float)weps)) return 0.0f;
  return r * weno5(s1, s2, s3, s4, s5, weps);
}
__device__ __forceinline__ float sflux_y(const DGrid &g, const SAdv &a, int i, int j, int k, int weno, int pdef, double weps) {
  float r = FV(g, a, i, j, k), s1, s2, s3, s4, s5;
  if (r >= 0.0f) { s1 = sval(g, a, i, j - 3, k); s2 = sval(g, a, i, j - 2, k); s3 = sval(g, a, i, j - 1, k); s4 = sval(g, a, i, j, k); s5 = sval(g, a, i, j + 1, k); }
  else { s1 = sval(g, a, i, j + 2, k); s2 = sval(g, a, i, j + 1, k); s3 = sval(g, a, i, j, k); s4 = sval(g, a, i, j - 1, k); s5 = sval(g, a, i, j - 2, k); }
  if (!weno) return r * flx5(s1, s2, s3, s4, s5);
  if (pdef == 1 && !(absmax5(s1, s2, s3, s4, s5) > (float)weps)) return 0.0f;
  return r * weno5(s1, s2, s3, s4, s5, weps);
}
// vertical flux dumz(i,j,kk), kk=2..nk (vadv_flx5 / vadv_weno5 stag=1)
__device__ __forceinline__ float sflux_z(const DGrid &g, const SAdv &a, int i, int j, int kk, int weno, int pdefweno, double weps) {
  const int nk = g.nk;
  auto A = [&](int k) { return sval(g, a, i, j, k); };
  float r = FW(g, a, i, j, kk);
  const float c1k = LDG(&g.c1[kk]), c2k = LDG(&g.c2[kk]);
  if (!weno) {
    if (kk >= 4 && kk <= nk - 2) {
      if (r >= 0.0f) return r * flx5(A(kk - 3), A(kk - 2), A(kk - 1), A(kk), A(kk + 1));
      return r * flx5(A(kk + 2), A(kk + 1), A(kk), A(kk - 1), A(kk - 2));
    }
    if (kk == 2) {
      if (r >= 0.0f) return r * (c1k * A(kk - 1) + c2k * A(kk));
      return r * flx3(A(kk + 1), A(kk), A(kk - 1));
    }
    if (kk == nk) {
      if (r >= 0.0f) return r * flx3(A(kk - 2), A(kk - 1), A(kk));
      return r * (c1k * A(kk - 1) + c2k * A(kk));
    }
    if (kk == 3) {
      if (r >= 0.0f) return r * flx3(A(kk - 2), A(kk - 1), A(kk));
      return r * flx5(A(kk + 2), A(kk + 1), A(kk), A(kk - 1), A(kk - 2));
    }
    if (r >= 0.0f) return r * flx5(A(kk - 3), A(kk - 2), A(kk - 1), A(kk), A(kk + 1));
    return r * flx3(A(kk + 1), A(kk), A(kk - 1));
  }
  // WENO: lower-order pieces at 2 and nk are common to both forms
  if (kk == 2) {
    if (r >= 0.0f) return r * (c1k * A(kk - 1) + c2k * A(kk));
    return r * upstrpd(A(kk + 1), A(kk), A(kk - 1), weps);
  }
  if (kk == nk) {
    if (r > 0.0f) return r * upstrpd(A(kk - 2), A(kk - 1), A(kk), weps);
    return r * (c1k * A(kk - 1) + c2k * A(kk));
  }
  if (pdefweno == 1) {
    // vadv_weno5 pdef form (adv_routines.F:2386-2421) then vadv_lwr_weno_35_b
    if (kk == 3 && r > 0.0f) return r * upstrpd(A(kk - 2), A(kk - 1), A(kk), weps);
    if (kk == nk - 1 && r < 0.0f) return r * upstrpd(A(kk + 1), A(kk), A(kk - 1), weps);
    float s1, s2, s3, s4, s5;
    if (r >= 0.0f) { s1 = A(kk - 3); s2 = A(kk - 2); s3 = A(kk - 1); s4 = A(kk); s5 = A(kk + 1); }
    else { s1 = A(kk + 2); s2 = A(kk + 1); s3 = A(kk); s4 = A(kk - 1); s5 = A(kk - 2); }
    bool doit = absmax5(s1, s2, s3, s4, s5) > (float)weps;
    return doit ? r * weno5(s1, s2, s3, s4, s5, weps) : 0.0f;
  }
  if (kk >= 4 && kk <= nk - 2) {
    if (r >= 0.0f) return r * weno5(A(kk - 3), A(kk - 2), A(kk - 1), A(kk), A(kk + 1), weps);
    return r * weno5(A(kk + 2), A(kk + 1), A(kk), A(kk - 1), A(kk - 2), weps);
  }
  if (kk == 3) {
    if (r >= 0.0f) return r * upstrpd(A(kk - 2), A(kk - 1), A(kk), weps);
    return r * weno5(A(kk + 2), A(kk + 1), A(kk), A(kk - 1), A(kk - 2), weps);
  }
  if (r >= 0.0f) return r * weno5(A(kk - 3), A(kk - 2), A(kk - 1), A(kk), A(kk + 1), weps);
  return r * upstrpd(A(kk + 1), A(kk), A(kk - 1), weps);
}

struct AdvParts { float advx, advy, advz; };

// advx/advy/advz of one cell with the open-bc inflow fix-ups (adv.F:129-335, 451-577)
__device__ __forceinline__ AdvParts advs_parts(const DGrid &g, const SAdv &a, int i, int j, int k,
                                               int weno, int pdef, int pdefweno, double weps) {
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const bool doitw = (g.wbc == 2 && g.ibw), doite = (g.ebc == 2 && g.ibe);
  const bool doits = (g.sbc == 2 && g.ibs), doitn = (g.nbc == 2 && g.ibn);
  float fx0 = sflux_x(g, a, i, j, k, weno, pdef, weps), fxp = sflux_x(g, a, i + 1, j, k, weno, pdef, weps);
  if (doitw && i == 1 && FU(g, a, 1, j, k) >= 0.0f) fx0 = fxp;
  if (doite && i == ni && FU(g, a, ni + 1, j, k) <= 0.0f) fxp = fx0;
  float fy0 = sflux_y(g, a, i, j, k, weno, pdef, weps), fyp = sflux_y(g, a, i, j + 1, k, weno, pdef, weps);
  if (doits && j == 1 && FV(g, a, i, 1, k) >= 0.0f) fy0 = fyp;
  if (doitn && j == nj && FV(g, a, i, nj + 1, k) <= 0.0f) fyp = fy0;
  AdvParts p;
  p.advx = -(fxp - fx0) * g.rdx * LDG(&g.uh[i - g.ib]);
  p.advy = -(fyp - fy0) * g.rdy * LDG(&g.vh[j - g.jb]);
  float sc = sval(g, a, i, j, k);
  if (doitw && i == 1 && FU(g, a, 1, j, k) >= 0.0f)
    p.advx = p.advx - sc * (FU(g, a, 2, j, k) - FU(g, a, 1, j, k)) * g.rdx * LDG(&g.uh[1 - g.ib]);
  if (doite && i == ni && FU(g, a, ni + 1, j, k) <= 0.0f)
    p.advx = p.advx - sc * (FU(g, a, ni + 1, j, k) - FU(g, a, ni, j, k)) * g.rdx * LDG(&g.uh[ni - g.ib]);
  if (doits && j == 1 && FV(g, a, i, 1, k) >= 0.0f)
    p.advy = p.advy - sc * (FV(g, a, i, 2, k) - FV(g, a, i, 1, k)) * g.rdy * LDG(&g.vh[1 - g.jb]);
  if (doitn && j == nj && FV(g, a, i, nj + 1, k) <= 0.0f)
    p.advy = p.advy - sc * (FV(g, a, i, nj + 1, k) - FV(g, a, i, nj, k)) * g.rdy * LDG(&g.vh[nj - g.jb]);
  const float mhk = LDG(&g.mh[k]);
  if (k == 1) p.advz = -sflux_z(g, a, i, j, 2, weno, pdefweno, weps) * g.rdz * mhk;
  else if (k == nk) p.advz = +sflux_z(g, a, i, j, nk, weno, pdefweno, weps) * g.rdz * mhk;
  else p.advz = -(sflux_z(g, a, i, j, k + 1, weno, pdefweno, weps) - sflux_z(g, a, i, j, k, weno, pdefweno, weps)) * g.rdz * mhk;
  return p;
}

// Non-pdef scalar pass: sten_out = sten_in + (adv + s*divx)*rr0, and when
// snew is given, snew = s0 + dt*sten_out with the smeps flush (solve2.F:1419-1425).
__global__ void k_advs(DGrid g, SAdv a, const float *sten_in,
                       float *sten_out, float *__restrict__ snew, const float *__restrict__ sbase,
                       int weno, int pdefweno, double weps, float dt, int flush) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni) return;
  AdvParts p = advs_parts(g, a, i, j, k, weno, 0, pdefweno, weps);
  long o = iS(g, i, j, k);
  float ten = sten_in[o];
  if (a.thterm) ten = ten - RAWDIV(g, a, i, j, k) * LDG(&a.thterm[o]);
  ten = ten + (((p.advx + p.advy) + p.advz) + sval(g, a, i, j, k) * SDIV(g, a, i, j, k)) * LDG(&g.rr0[k]);
  if (sten_out) sten_out[o] = ten;
  if (snew) {
    float v = LDG(&sbase[o]) + dt * ten;
    if (flush && fabsf(v) < g.smeps) v = 0.0f;
    snew[o] = v;
  }
}

// pdef pass 1: advx/advy/advz and the provisional masses of pdefx1/y1/z
// (pdef.F:35-102, 289-340, 478-496).
__global__ void k_advs_pdef1(DGrid g, SAdv a, float *__restrict__ advx, float *__restrict__ advy, float *__restrict__ advz,
                             float *__restrict__ dumx, float *__restrict__ dumy, float *__restrict__ dumz,
                             int weno, int pdefweno, double weps, float dt) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni) return;
  const int ni = g.ni, nj = g.nj;
  AdvParts p = advs_parts(g, a, i, j, k, weno, 1, pdefweno, weps);
  long o = iS(g, i, j, k);
  advx[o] = p.advx; advy[o] = p.advy; advz[o] = p.advz;
  const float s = sval(g, a, i, j, k), s0 = LDG(&a.s0[o]), r0k = LDG(&g.rho0[k]);
  float dx = r0k * s0 + dt * (p.advx + s * (FU(g, a, i + 1, j, k) - FU(g, a, i, j, k)) * g.rdx * LDG(&g.uh[i - g.ib]));
  if (g.wbc == 2 && g.ibw && i == 1 && FU(g, a, 1, j, k) >= 0.0f) dx = r0k * s0;
  if (g.ebc == 2 && g.ibe && i == ni && FU(g, a, ni + 1, j, k) <= 0.0f) dx = r0k * s0;
  float dy = r0k * s0 + dt * (p.advy + s * (FV(g, a, i, j + 1, k) - FV(g, a, i, j, k)) * g.rdy * LDG(&g.vh[j - g.jb]));
  if (g.sbc == 2 && g.ibs && j == 1 && FV(g, a, i, 1, k) >= 0.0f) dy = r0k * s0;
  if (g.nbc == 2 && g.ibn && j == nj && FV(g, a, i, nj + 1, k) <= 0.0f) dy = r0k * s0;
  float dz = r0k * s0 + dt * (p.advz + s * (FW(g, a, i, j, k + 1) - FW(g, a, i, j, k)) * g.rdz * LDG(&g.mh[k]));
  dumx[o] = dx; dumy[o] = dy; dumz[o] = dz;
}

// Mass moved into point c by the pdef scatter of pdefx2/pdefy2/pdefz
// (pdef.F:158-174), gathered in the scatter's loop order: contribution from
// the lower neighbour, then the point itself, then the upper neighbour.
__device__ __forceinline__ void pdef_gather(float dm2, float dm1, float d0, float dp1, float dp2, float smeps,
                                            float *mass, bool *flag) {
  float m = 0.0f;
  bool f = false;
  if (dm1 < 0.0f) {  // the point below scatters: we are its upper neighbour
    float foo1 = fmaxf(0.0f, dm2), foo2 = fmaxf(0.0f, d0);
    if (foo1 + foo2 > smeps) {
      float foo3 = fmaxf(dm1, -(foo1 + foo2)) / (foo1 + foo2);
      m = m + foo2 * foo3;
      if (d0 > smeps) f = true;
    }
  }
  if (d0 < 0.0f) {
    float foo1 = fmaxf(0.0f, dm1), foo2 = fmaxf(0.0f, dp1);
    if (foo1 + foo2 > smeps) {
      float foo3 = fmaxf(d0, -(foo1 + foo2)) / (foo1 + foo2);
      m = m - (foo1 + foo2) * foo3;
      f = true;
    }
  }
  if (dp1 < 0.0f) {
    float foo1 = fmaxf(0.0f, d0), foo2 = fmaxf(0.0f, dp2);
    if (foo1 + foo2 > smeps) {
      float foo3 = fmaxf(dp1, -(foo1 + foo2)) / (foo1 + foo2);
      m = m + foo1 * foo3;
      if (d0 > smeps) f = true;
    }
  }
  *mass = m; *flag = f;
}

// pdef pass 2: pdefz, pdefx2, pdefy2 fixes (pdef.F:117-264, 358-454,
// 459-581) and the tendency/update of adv.F:650-659 + solve2.F:1513-1520.
// dumx/dumy carry halo values filled by the lateral bc (pdef.F:102, 338).
__global__ void k_advs_pdef2(DGrid g, SAdv a, const float *__restrict__ advx, const float *__restrict__ advy,
                             const float *__restrict__ advz, const float *__restrict__ dumx,
                             const float *__restrict__ dumy, const float *__restrict__ dumz,
                             const float *sten_in, float *sten_out, float *__restrict__ snew,
                             const float *__restrict__ sbase, float dt, int flush) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = 1 + (int)blockIdx.z;
  if (i > g.ni) return;
  const int nk = g.nk;
  const float smeps = g.smeps, rdt = 1.0f / dt;
  long o = iS(g, i, j, k);
  const float s = sval(g, a, i, j, k), s0 = LDG(&a.s0[o]), r0k = LDG(&g.rho0[k]);
  float m; bool f;
  // z (pdefz): dum(0)=dum(nk+1)=0
  auto DZ = [&](int kk) { return (kk < 1 || kk > nk) ? 0.0f : LDG(&dumz[iS(g, i, j, kk)]); };
  float az = LDG(&advz[o]);
  pdef_gather(DZ(k - 2), DZ(k - 1), DZ(k), DZ(k + 1), DZ(k + 2), smeps, &m, &f);
  if (f) az = (DZ(k) + m - r0k * s0) * rdt - s * (FW(g, a, i, j, k + 1) - FW(g, a, i, j, k)) * g.rdz * LDG(&g.mh[k]);
  // x (pdefx2)
  auto DX = [&](int ii) { return LDG(&dumx[iS(g, ii, j, k)]); };
  float ax = LDG(&advx[o]);
  pdef_gather(DX(i - 2), DX(i - 1), DX(i), DX(i + 1), DX(i + 2), smeps, &m, &f);
  if (f) ax = (DX(i) + m - r0k * s0) * rdt - s * (FU(g, a, i + 1, j, k) - FU(g, a, i, j, k)) * g.rdx * LDG(&g.uh[i - g.ib]);
  // y (pdefy2)
  auto DY = [&](int jj) { return LDG(&dumy[iS(g, i, jj, k)]); };
  float ay = LDG(&advy[o]);
  pdef_gather(DY(j - 2), DY(j - 1), DY(j), DY(j + 1), DY(j + 2), smeps, &m, &f);
  if (f) ay = (DY(j) + m - r0k * s0) * rdt - s * (FV(g, a, i, j + 1, k) - FV(g, a, i, j, k)) * g.rdy * LDG(&g.vh[j - g.jb]);
  float ten = sten_in[o] + (((ax + ay) + az) + s * SDIV(g, a, i, j, k)) * LDG(&g.rr0[k]);
  if (sten_out) sten_out[o] = ten;
  if (snew) {
    float v = LDG(&sbase[o]) + dt * ten;
    if (flush && fabsf(v) < g.smeps) v = 0.0f;
    snew[o] = v;
  }
}

// Tiled form of pass 2: a block owns TX x TY columns and marches upward;
// each level's dumx (with its +-2 halo in x) and dumy (+-2 in y) are staged
// in shared memory (double-buffered, one barrier per level), dumz comes
// from a per-column register window, and every read of a level is issued
// one level ahead.  Same arithmetic as k_advs_pdef2.
template <int TX, int TY, int KC>
__global__ void __launch_bounds__(TX * TY) k_advs_pdef2_tile(DGrid g, SAdv a, const float *__restrict__ advx,
                                                             const float *__restrict__ advy, const float *__restrict__ advz,
                                                             const float *__restrict__ dumx, const float *__restrict__ dumy,
                                                             const float *__restrict__ dumz, const float *__restrict__ sten_in,
                                                             float *__restrict__ snew, const float *__restrict__ sbase,
                                                             float dt, int flush) {
  constexpr int NT = TX * TY;
  constexpr int XW = TX + 4, YH = TY + 4;
  constexpr int NSX = (XW * TY + NT - 1) / NT, NSY = (TX * YH + NT - 1) / NT;
  __shared__ float sx[2][TY * XW], sy[2][YH * TX];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int i0 = 1 + (int)blockIdx.x * TX, j0 = 1 + (int)blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int ni = g.ni, nj = g.nj, nk = g.nk, NI = g.NI, NJ = g.NJ;
  const bool active = (i <= ni && j <= nj);
  const int planeS = NI * NJ, planeU = (NI + 1) * NJ, planeV = NI * (NJ + 1);   // < 2^31 points (cm1g_init)
  const float smeps = g.smeps, rdt = 1.0f / dt;
  const float uh_i = active ? LDG(&g.uh[i - g.ib]) : 0.0f, vh_j = active ? LDG(&g.vh[j - g.jb]) : 0.0f;
  const int oc = active ? (i - g.ib) + NI * (j - g.jb) : 0;
  const int ocu = active ? (i - g.ib) + (NI + 1) * (j - g.jb) : 0;
  int xo[NSX], xs[NSX], yo[NSY], ys[NSY];   // staging: source offset in the plane (-1: none), slot
#pragma unroll
  for (int q = 0; q < NSX; q++) {
    const int t = tid + q * NT;
    xo[q] = -1; xs[q] = 0;
    if (t < XW * TY) {
      const int yy = t / XW, xx = t - yy * XW, ii = i0 - 2 + xx, jj = j0 + yy;
      if (ii <= ni + 2 && jj <= nj) { xo[q] = (ii - g.ib) + NI * (jj - g.jb); xs[q] = t; }
    }
  }
#pragma unroll
  for (int q = 0; q < NSY; q++) {
    const int t = tid + q * NT;
    yo[q] = -1; ys[q] = 0;
    if (t < TX * YH) {
      const int yy = t / TX, xx = t - yy * TX, ii = i0 + xx, jj = j0 - 2 + yy;
      if (ii <= ni && jj <= nj + 2) { yo[q] = (ii - g.ib) + NI * (jj - g.jb); ys[q] = t; }
    }
  }
  const int kc0 = 1 + (int)blockIdx.z * KC, kc1 = min(nk, kc0 + KC - 1);
  auto DZ = [&](int kk) { return (kk < 1 || kk > nk) ? 0.0f : LDG(&dumz[kk * planeS + oc]); };
  auto WR = [&](int kk) { return (kk <= 1 || kk >= nk + 1) ? 0.0f : LDG(&a.rrw[kk * planeS + oc]); };
  float zw[5];                                  // dumz(k-2 .. k+2)
#pragma unroll
  for (int d = 0; d < 5; d++) zw[d] = active ? DZ(kc0 - 2 + d) : 0.0f;
  float wlo = active ? WR(kc0) : 0.0f;          // raw averaged w through the bottom face

  float psx[NSX], psy[NSY], pax = 0.f, pay = 0.f, paz = 0.f, ps = 0.f, ps0 = 0.f, pt = 0.f, pb = 0.f;
  float pu0 = 0.f, pu1 = 0.f, pv0 = 0.f, pv1 = 0.f, pwhi = 0.f, pztop = 0.f;
  auto fetch = [&](int kf) {
#pragma unroll
    for (int q = 0; q < NSX; q++) psx[q] = (xo[q] >= 0) ? LDG(&dumx[kf * planeS + xo[q]]) : 0.0f;
#pragma unroll
    for (int q = 0; q < NSY; q++) psy[q] = (yo[q] >= 0) ? LDG(&dumy[kf * planeS + yo[q]]) : 0.0f;
    if (active) {
      const int o = kf * planeS + oc, ou = kf * planeU + ocu, ov = kf * planeV + oc;
      pax = LDG(&advx[o]); pay = LDG(&advy[o]); paz = LDG(&advz[o]);
      ps = LDG(&a.s[o]);
      if (a.sadd) ps = (LDG(&g.th0[kf]) - 300.0f) + ps;
      ps0 = LDG(&a.s0[o]); pt = sten_in[o]; pb = LDG(&sbase[o]);
      pu0 = LDG(&a.rru[ou]); pu1 = LDG(&a.rru[ou + 1]);
      pv0 = LDG(&a.rrv[ov]); pv1 = LDG(&a.rrv[ov + NI]);
      pwhi = WR(kf + 1);
      pztop = DZ(kf + 2);                       // top of the dumz window of level kf
    }
  };
  fetch(kc0);
  for (int k = kc0; k <= kc1; k++) {
    const int b = k & 1;
#pragma unroll
    for (int q = 0; q < NSX; q++) if (xo[q] >= 0) sx[b][xs[q]] = psx[q];
#pragma unroll
    for (int q = 0; q < NSY; q++) if (yo[q] >= 0) sy[b][ys[q]] = psy[q];
    const float ax0 = pax, ay0 = pay, az0 = paz, s = ps, s0 = ps0, t1 = pt, base = pb;
    const float u0r = pu0, u1r = pu1, v0r = pv0, v1r = pv1, whi = pwhi;
    if (k < kc1) fetch(k + 1);
    __syncthreads();
    if (active) {
      const float r0k = LDG(&g.rho0[k]), mhk = LDG(&g.mh[k]);
      const float fu0 = u0r * r0k, fu1 = u1r * r0k, fv0 = v0r * r0k, fv1 = v1r * r0k;
      const float fwlo = wlo * LDG(&g.rf0[k]), fwhi = whi * LDG(&g.rf0[k + 1]);
      float m; bool f;
      // z (pdefz): dum(0)=dum(nk+1)=0
      float az = az0;
      pdef_gather(zw[0], zw[1], zw[2], zw[3], zw[4], smeps, &m, &f);
      if (f) az = (zw[2] + m - r0k * s0) * rdt - s * (fwhi - fwlo) * g.rdz * mhk;
      // x (pdefx2)
      const float *px = &sx[b][ty * XW + tx];
      float ax = ax0;
      pdef_gather(px[0], px[1], px[2], px[3], px[4], smeps, &m, &f);
      if (f) ax = (px[2] + m - r0k * s0) * rdt - s * (fu1 - fu0) * g.rdx * uh_i;
      // y (pdefy2)
      const float *py = &sy[b][ty * TX + tx];
      float ay = ay0;
      pdef_gather(py[0], py[TX], py[2 * TX], py[3 * TX], py[4 * TX], smeps, &m, &f);
      if (f) ay = (py[2 * TX] + m - r0k * s0) * rdt - s * (fv1 - fv0) * g.rdy * vh_j;
      float div = ((fu1 - fu0) * g.rdx * uh_i + (fv1 - fv0) * g.rdy * vh_j) + (fwhi - fwlo) * g.rdz * mhk;
      if (fabsf(div) < g.smeps) div = 0.0f;
      const float ten = t1 + (((ax + ay) + az) + s * div) * LDG(&g.rr0[k]);
      float v = base + dt * ten;
      if (flush && fabsf(v) < g.smeps) v = 0.0f;
      snew[k * planeS + oc] = v;
#pragma unroll
      for (int d = 0; d < 4; d++) zw[d] = zw[d + 1];
      zw[4] = pztop;            // dumz(k+3), fetched with level k+1 above
      wlo = whi;
    }
  }
}

// ---------------------------------------------------------------------
// Tiled scalar advection (the production path of advs).
//
// A block owns TX x TY columns and marches upward through the levels.  At
// each level the advected field is staged with its 3-point lateral halo in
// shared memory; every x- and y-face flux is evaluated once (the WENO5 or
// 5th-order value of hadv_weno5/hadv_flx5) and shared by the two cells it
// separates; the vertical face flux of the level above is evaluated from a
// per-thread register window of the column and carried to the next level as
// its lower face.  Each cell therefore costs three face evaluations instead
// of six.  MODE_UPDATE writes snew = s0 + dt*ten (solve2.F:1419-1425,
// 1513-1520, 1951-1957); MODE_PDEF1 writes advx/advy/advz and the
// provisional masses of pdefx1/pdefy1/pdefz for the second pdef pass.
// ---------------------------------------------------------------------
enum { MODE_UPDATE = 0, MODE_PDEF1 = 1 };

struct STileOut {
  const float *sten_in;       // fixed tendency (thten1, qten, ptten)
  const float *sbase;         // RK base value (tha, qa, pta)
  float *snew;                // MODE_UPDATE output
  float *advx, *advy, *advz, *dumx, *dumy, *dumz;   // MODE_PDEF1 outputs
  TileExtras ex;              // learned face values / flux capture (update mode)
};

// The block has TY rows of cell threads and one more row of TX threads:
// the (TX+1)*TY x-faces and TX*(TY+1) y-faces of a level are spread at most
// one of each per thread, so the cell threads evaluate three faces (x, y and
// the z face above their cell) and the extra row two; staging
// sources, face addresses and the column offset are 32-bit in-plane offsets
// computed once per block; the raw averaged velocities of the faces are kept
// in shared memory for the divergence terms of the cell owners.  All
// arrays must have fewer than 2^31 points per horizontal plane.
template <int TX, int TY, int KC, int MODE, int WENO, int DIFF>
__global__ void __launch_bounds__(TX * (TY + 1), 3) k_advs_tile(DGrid g, SAdv a, STileOut out, int pdef, int pdefweno,
                                                       double weps, float dt, int flush) {
  constexpr int NT = TX * (TY + 1);                        // TY cell rows + the row of the extra faces
  constexpr int SW = TX + 6, SH = TY + 6, SP = SW + 1;     // staged plane, pitch SP
  constexpr int NST = (SW * SH + NT - 1) / NT;              // staging slots per thread
  constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);   // faces of one level
  __shared__ float ss[SH * SP];
  __shared__ float fx[NFX], ux[NFX], fy[NFY], vy[NFY];
  __shared__ float dfx[NFX], dfy[NFY];     // 6th-order diffusion fluxes (adv.F:356-395)
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
  const int i0 = 1 + (int)blockIdx.x * TX, j0 = 1 + (int)blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int ni = g.ni, nj = g.nj, nk = g.nk, NI = g.NI, NJ = g.NJ;
  const bool active = (ty < TY && i <= ni && j <= nj);
  const bool doitw = (g.wbc == 2 && g.ibw), doite = (g.ebc == 2 && g.ibe);
  const bool doits = (g.sbc == 2 && g.ibs), doitn = (g.nbc == 2 && g.ibn);
  const int ie = ni + g.ngxy, je = nj + g.ngxy;
  const int planeS = NI * NJ, planeU = (NI + 1) * NJ, planeV = NI * (NJ + 1);   // < 2^31 points (cm1g_init)
  const float uh_i = active ? LDG(&g.uh[i - g.ib]) : 0.0f, vh_j = active ? LDG(&g.vh[j - g.jb]) : 0.0f;
  const int oc = active ? (i - g.ib) + NI * (j - g.jb) : 0;   // the column's in-plane offset

  int soff[NST], sidx[NST];     // staging: source offset (-1: outside the arrays), slot in ss (-1: none)
#pragma unroll
  for (int q = 0; q < NST; q++) {
    const int t = tid + q * NT;
    soff[q] = -1; sidx[q] = -1;
    if (t < SW * SH) {
      const int yy = t / SW, xx = t - yy * SW;
      const int ii = i0 - 3 + xx, jj = j0 - 3 + yy;
      sidx[q] = yy * SP + xx;
      if (ii <= ie && jj <= je) soff[q] = (ii - g.ib) + NI * (jj - g.jb);
    }
  }
  int fxo[2], fxs[2], fyo[2], fys[2];   // face offsets (-1: no face) and stencil starts in ss
  int fxl[2], fyl[2];                   // in-level index of the face in the learned-value arrays
  int fxr[2];                           // s-plane offset of the cell (i, j) right of an x-face
  using FS = FaceSlots<NT, NFX, NFY>;
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int f = FS::x(tid, q), fy_ = FS::y(tid, q);
    fxo[q] = -1; fxs[q] = 0; fyo[q] = -1; fys[q] = 0; fxl[q] = 0; fyl[q] = 0; fxr[q] = 0;
    if (f < NFX) {
      const int row = f / (TX + 1), col = f - row * (TX + 1);
      const int ii = i0 + col, jj = j0 + row;
      if (ii <= ni + 1 && jj <= nj) {
        fxo[q] = (ii - g.ib) + (NI + 1) * (jj - g.jb); fxs[q] = (row + 3) * SP + col;
        fxl[q] = (jj - 1) * (ni + 1) + (ii - 1);
        fxr[q] = (ii - g.ib) + NI * (jj - g.jb);
      }
    }
    if (fy_ < NFY) {
      const int row = fy_ / TX, col = fy_ - row * TX;
      const int ii = i0 + col, jj = j0 + row;
      if (ii <= ni && jj <= nj + 1) {
        fyo[q] = (ii - g.ib) + NI * (jj - g.jb); fys[q] = row * SP + col + 3;
        fyl[q] = (jj - 1) * ni + (ii - 1);
      }
    }
  }

  auto SV = [&](int kk) -> float {
    float v = LDG(&a.s[kk * planeS + oc]);
    if (a.sadd) v = (LDG(&g.th0[kk]) - 300.0f) + v;
    return v;
  };
  // averaged w of a w-level (zero at the bottom and top boundaries)
  auto WRAW = [&](int kk) -> float { return (kk <= 1 || kk >= nk + 1) ? 0.0f : LDG(&a.rrw[kk * planeS + oc]); };

  // register window of the column: wv[d+3] = s(k+1+d), d = -3..2 (for the top face of level k);
  // the block covers levels kc0..kc1 of its columns (blockIdx.z selects the chunk)
  const int kc0 = 1 + (int)blockIdx.z * KC, kc1 = min(nk, kc0 + KC - 1);
  float wv[6];
#pragma unroll
  for (int d = 0; d < 6; d++) {
    const int kk = kc0 - 2 + d;
    wv[d] = (active && kk >= 0 && kk <= nk + 1) ? SV(kk) : 0.0f;
  }
  float wlo = active ? WRAW(kc0) : 0.0f;       // raw averaged w through the bottom face of the level
  float fwlo = wlo * LDG(&g.rf0[kc0]);
  float fzlo = 0.0f;                            // flux through the bottom face of the level
  if (active && kc0 >= 2) {
    float w0[6];
#pragma unroll
    for (int d = 0; d < 6; d++) {
      const int kk = kc0 - 3 + d;
      w0[d] = (kk >= 0 && kk <= nk + 1) ? SV(kk) : 0.0f;
    }
    fzlo = zflux_win(g, w0, fwlo, kc0, WENO, pdefweno, weps);
  }

  // Every global read of a level (the staged plane, the face velocities, the
  // cell's inputs and the next top of the column window) is issued one level
  // ahead, so it is in flight while the previous level computes.  None of
  // these arrays is written by this kernel.
  float pst[NST], pru[2], prv[2], pwhi = 0.0f, pe0 = 0.0f, pe1 = 0.0f, pe2 = 0.0f, pwtop = 0.0f;
  auto fetch = [&](int kf) {
    const float *sk = a.s + kf * planeS;
#pragma unroll
    for (int q = 0; q < NST; q++) pst[q] = (soff[q] >= 0) ? LDG(&sk[soff[q]]) : 0.0f;
#pragma unroll
    for (int q = 0; q < 2; q++) {
      pru[q] = (fxo[q] >= 0) ? LDG(&a.rru[kf * planeU + fxo[q]]) : 0.0f;
      prv[q] = (fyo[q] >= 0) ? LDG(&a.rrv[kf * planeV + fyo[q]]) : 0.0f;
    }
    if (active) {
      const int o = kf * planeS + oc;
      pwhi = WRAW(kf + 1);
      if (MODE == MODE_UPDATE) {
        pe0 = out.sten_in[o];
        pe1 = LDG(&out.sbase[o]);
        if (a.thterm) pe2 = LDG(&a.thterm[o]);
      } else {
        pe0 = LDG(&a.s0[o]);
      }
      pwtop = (kf + 3 <= nk + 1) ? SV(kf + 3) : 0.0f;   // top of the window of level kf
    }
  };
  fetch(kc0);

  for (int k = kc0; k <= kc1; k++) {
    const float r0k = LDG(&g.rho0[k]);
    const float th0m = a.sadd ? (LDG(&g.th0[k]) - 300.0f) : 0.0f;
    // ---- stage the level with its halo; take the raw face velocities
#pragma unroll
    for (int q = 0; q < NST; q++) {
      if (sidx[q] >= 0) {
        float v = pst[q];
        if (soff[q] >= 0 && a.sadd) v = th0m + v;
        ss[sidx[q]] = v;
      }
    }
    const float ru[2] = {pru[0], pru[1]}, rv[2] = {prv[0], prv[1]};
    const float whi = pwhi, e0 = pe0, e1 = pe1, e2 = pe2;
    if (k < kc1) fetch(k + 1);
    __syncthreads();
    // ---- face values: each x/y face once, each upper z face once per column
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int f = FS::x(tid, q), fy_ = FS::y(tid, q);
      if (fxo[q] >= 0) {
        const float *p = &ss[fxs[q]];
        const float r = ru[q] * r0k;
        float ph = __int_as_float(0x7fc00000);
        if (MODE == MODE_UPDATE && out.ex.phix) ph = out.ex.phix[(k - 1) * (ni + 1) * nj + fxl[q]];
        const float fl = (ph == ph) ? r * ph : hflux5(r, p[0], p[1], p[2], p[3], p[4], p[5], WENO, pdef, weps);
        fx[f] = fl;
        ux[f] = ru[q];
        if (DIFF) {   // face between s(i-1) and s(i): p[2], p[3]
          const int ro = k * planeS + fxr[q];                           // rho(i,j)
          const float fd = diff6_stencil(p[0], p[1], p[2], p[3], p[4], p[5]) * 0.5f *
                           (LDG(&a.df.rho[ro - 1]) + LDG(&a.df.rho[ro]));
          dfx[f] = diff6_limit(fd, p[3], p[2], a.df.mdiff);
        }
        if (MODE == MODE_UPDATE && out.ex.capfx) {
          out.ex.capfx[k * planeU + fxo[q]] = fl;
          out.ex.caprx[k * planeU + fxo[q]] = r;
        }
      }
      if (fyo[q] >= 0) {
        const float *p = &ss[fys[q]];
        const float r = rv[q] * r0k;
        float ph = __int_as_float(0x7fc00000);
        if (MODE == MODE_UPDATE && out.ex.phiy) ph = out.ex.phiy[(k - 1) * ni * (nj + 1) + fyl[q]];
        const float fl = (ph == ph) ? r * ph
                                    : hflux5(r, p[0], p[SP], p[2 * SP], p[3 * SP], p[4 * SP], p[5 * SP], WENO, pdef, weps);
        fy[fy_] = fl;
        vy[fy_] = rv[q];
        if (DIFF) {   // face between s(j-1) and s(j): p[2 SP], p[3 SP]
          const int ro = k * planeS + fyo[q];                           // rho(i,j)
          const float fd = diff6_stencil(p[0], p[SP], p[2 * SP], p[3 * SP], p[4 * SP], p[5 * SP]) * 0.5f *
                           (LDG(&a.df.rho[ro - NI]) + LDG(&a.df.rho[ro]));
          dfy[fy_] = diff6_limit(fd, p[3 * SP], p[2 * SP], a.df.mdiff);
        }
        if (MODE == MODE_UPDATE && out.ex.capfy) {
          out.ex.capfy[k * planeV + fyo[q]] = fl;
          out.ex.capry[k * planeV + fyo[q]] = r;
        }
      }
    }
    const float fwhi = whi * LDG(&g.rf0[k + 1]);
    float fzhi = 0.0f, sc = 0.0f;
    if (active) {
      sc = ss[(ty + 3) * SP + tx + 3];
      if (k + 1 <= nk) fzhi = zflux_win(g, wv, fwhi, k + 1, WENO, pdefweno, weps);
    }
    __syncthreads();
    if (active) {
      const int o = k * planeS + oc;
      const int xi = ty * (TX + 1) + tx, yi = ty * TX + tx;
      float fx0 = fx[xi], fxp = fx[xi + 1], fy0 = fy[yi], fyp = fy[yi + TX];
      const float u0r = ux[xi], u1r = ux[xi + 1], v0r = vy[yi], v1r = vy[yi + TX];
      const float fu0 = u0r * r0k, fu1 = u1r * r0k, fv0 = v0r * r0k, fv1 = v1r * r0k;
      // adv.F:212-268
      if (doitw && i == 1 && fu0 >= 0.0f) fx0 = fxp;
      if (doite && i == ni && fu1 <= 0.0f) fxp = fx0;
      if (doits && j == 1 && fv0 >= 0.0f) fy0 = fyp;
      if (doitn && j == nj && fv1 <= 0.0f) fyp = fy0;
      float advx = -(fxp - fx0) * g.rdx * uh_i;
      float advy = -(fyp - fy0) * g.rdy * vh_j;
      // adv.F:286-335
      if (doitw && i == 1 && fu0 >= 0.0f) advx = advx - sc * (fu1 - fu0) * g.rdx * uh_i;
      if (doite && i == ni && fu1 <= 0.0f) advx = advx - sc * (fu1 - fu0) * g.rdx * uh_i;
      if (doits && j == 1 && fv0 >= 0.0f) advy = advy - sc * (fv1 - fv0) * g.rdy * vh_j;
      if (doitn && j == nj && fv1 <= 0.0f) advy = advy - sc * (fv1 - fv0) * g.rdy * vh_j;
      if (DIFF) {   // adv.F:375-378, 397-400
        const float ri = LDG(&a.df.ri[o]);
        advx = advx + a.df.coef * (dfx[xi + 1] - dfx[xi]) * ri * r0k;
        advy = advy + a.df.coef * (dfy[yi + TX] - dfy[yi]) * ri * r0k;
      }
      const float mhk = LDG(&g.mh[k]);
      float advz;
      if (k == 1) advz = -fzhi * g.rdz * mhk;
      else if (k == nk) advz = +fzlo * g.rdz * mhk;
      else advz = -(fzhi - fzlo) * g.rdz * mhk;
      float div = ((fu1 - fu0) * g.rdx * uh_i + (fv1 - fv0) * g.rdy * vh_j) + (fwhi - fwlo) * g.rdz * mhk;
      if (fabsf(div) < g.smeps) div = 0.0f;
      if (MODE == MODE_UPDATE) {
        float ten = e0;
        if (a.thterm) {   // getdiv of the averaged velocities (misclibs.F:127-136)
          float rd = ((u1r - u0r) * g.rdx * uh_i + (v1r - v0r) * g.rdy * vh_j) + (whi - wlo) * g.rdz * mhk;
          if (fabsf(rd) < g.smeps) rd = 0.0f;
          ten = ten - rd * e2;
        }
        ten = ten + (((advx + advy) + advz) + sc * div) * LDG(&g.rr0[k]);
        float v = e1 + dt * ten;
        if (flush && fabsf(v) < g.smeps) v = 0.0f;
        out.snew[o] = v;
      } else {
        // pdefx1 / pdefy1 / pdefz provisional masses (pdef.F:35-102, 289-340, 478-496)
        out.advx[o] = advx; out.advy[o] = advy; out.advz[o] = advz;
        const float s0 = e0;
        float dx = r0k * s0 + dt * (advx + sc * (fu1 - fu0) * g.rdx * uh_i);
        if (doitw && i == 1 && fu0 >= 0.0f) dx = r0k * s0;
        if (doite && i == ni && fu1 <= 0.0f) dx = r0k * s0;
        float dy = r0k * s0 + dt * (advy + sc * (fv1 - fv0) * g.rdy * vh_j);
        if (doits && j == 1 && fv0 >= 0.0f) dy = r0k * s0;
        if (doitn && j == nj && fv1 <= 0.0f) dy = r0k * s0;
        out.dumx[o] = dx; out.dumy[o] = dy;
        out.dumz[o] = r0k * s0 + dt * (advz + sc * (fwhi - fwlo) * g.rdz * mhk);
      }
      // slide the column window and carry the upper face to the next level
#pragma unroll
      for (int d = 0; d < 5; d++) wv[d] = wv[d + 1];
      wv[5] = pwtop;            // s(k+4), the new top of the window for level k+1
      fzlo = fzhi;
      fwlo = fwhi;
      wlo = whi;
    }
    // no barrier here: the next level's staging writes ss, which nobody reads
    // after the second barrier, and fx/fy/ux/vy are rewritten only after the
    // next level's first barrier, which every thread reaches after this level.
  }
}

void launch_bc(const DGrid &g, float *a, int which, int wflag, cudaStream_t st, int64_t *nlaunch);
void launch_bc_batch(const DGrid &g, float *const *arrays, const int *which, const int *wflag, int n,
                     cudaStream_t st, int64_t *nlaunch);

// One k_advs_tile launch: WENO and the 6th-order diffusion (a.df.rho set)
// select compile-time variants, so the plain pass carries no diffusion code.
template <int TX, int TY, int KC, int MODE>
static void advs_tile_launch(dim3 grid, dim3 blk, cudaStream_t st, int weno, const DGrid &g, const SAdv &a,
                             const STileOut &o, int pdef, int pdefweno, double weps, float dt, int flush) {
  if (a.df.rho) {
    if (weno) k_advs_tile<TX, TY, KC, MODE, 1, 1><<<grid, blk, 0, st>>>(g, a, o, pdef, pdefweno, weps, dt, flush);
    else k_advs_tile<TX, TY, KC, MODE, 0, 1><<<grid, blk, 0, st>>>(g, a, o, pdef, pdefweno, weps, dt, flush);
  } else {
    if (weno) k_advs_tile<TX, TY, KC, MODE, 1, 0><<<grid, blk, 0, st>>>(g, a, o, pdef, pdefweno, weps, dt, flush);
    else k_advs_tile<TX, TY, KC, MODE, 0, 0><<<grid, blk, 0, st>>>(g, a, o, pdef, pdefweno, weps, dt, flush);
  }
}

// Production scalar pass (MODE_UPDATE, or the pdef two-pass form) with the
// tile shape TX x TY x KC.
template <int TX, int TY, int KC>
static void advs_tiled_shape(const DGrid &g, const SAdv &a, STileOut o, int weno, int pdef, int pdefweno,
                             double weps, float dt, int flush, float *scratch, cudaStream_t st, int64_t *nl) {
  // k_advs_tile: TY cell rows and the row of the tile's extra faces; pass 2
  // (no face evaluations) takes TY + 1 cell rows per block
  dim3 blk(TX, TY + 1), grid((g.ni + TX - 1) / TX, (g.nj + TY - 1) / TY, (g.nk + KC - 1) / KC);
  dim3 grid2((g.ni + TX - 1) / TX, (g.nj + TY) / (TY + 1), (g.nk + KC - 1) / KC);
  if (!pdef) {
    ProfScope _ps("k_advs_tile", st);
    advs_tile_launch<TX, TY, KC, MODE_UPDATE>(grid, blk, st, weno, g, a, o, 0, pdefweno, weps, dt, flush);
    if (nl) *nl += 1;
    return;
  }
  long n = nS(g);
  o.advx = scratch; o.advy = scratch + n; o.advz = scratch + 2 * n;
  o.dumx = scratch + 3 * n; o.dumy = scratch + 4 * n; o.dumz = scratch + 5 * n;
  {
    ProfScope _ps("k_advs_tile_pdef1", st);
    advs_tile_launch<TX, TY, KC, MODE_PDEF1>(grid, blk, st, weno, g, a, o, 1, pdefweno, weps, dt, flush);
  }
  {
    float *arr[2] = {o.dumx, o.dumy};
    const int which[2] = {1, 1};
    launch_bc_batch(g, arr, which, nullptr, 2, st, nl);
  }
  {
    ProfScope _ps("k_advs_pdef2", st);
    k_advs_pdef2_tile<TX, TY + 1, KC><<<grid2, blk, 0, st>>>(g, a, o.advx, o.advy, o.advz, o.dumx, o.dumy, o.dumz,
                                                       o.sten_in, o.snew, o.sbase, dt, flush);
  }
  if (nl) *nl += 2;
}

void launch_advs_tiled(const DGrid &g, const float *rru, const float *rrv, const float *rrw, const float *s,
                       const float *s0, int sadd, const float *ten1, const float *thterm, float *snew, int weno,
                       int pdef, int pdefweno, double weps, float dt, int flush, float *scratch, cudaStream_t st,
                       int64_t *nl, const TileExtras *ex, const Diff6 *diff) {
  SAdv a{rru, rrv, rrw, s, s0, nullptr, thterm, 1, sadd};
  if (diff) a.df = *diff;
  STileOut o{};
  o.sten_in = ten1; o.sbase = s0; o.snew = snew;
  if (ex) o.ex = *ex;
  static_assert(kNumTileShapes == 5, "one case per tile shape");
#define CM1G_ADVS_SHAPE(n)                                                                                      \
  case n:                                                                                                      \
    advs_tiled_shape<kScalShapes[n][0], kScalShapes[n][1], kScalShapes[n][2]>(g, a, o, weno, pdef, pdefweno,    \
                                                                              weps, dt, flush, scratch, st, nl); \
    break;
  switch (g.tile_adv) {
    CM1G_ADVS_SHAPE(1)
    CM1G_ADVS_SHAPE(2)
    CM1G_ADVS_SHAPE(3)
    CM1G_ADVS_SHAPE(4)
    default: CM1G_ADVS_SHAPE(0)
  }
#undef CM1G_ADVS_SHAPE
}

// One advs call + RK update.  s = field (full halo), s0 = RK base,
// ten1 = fixed tendency.  pdef selects the two-pass positive-definite form.
// scratch must hold 6 s-arrays when pdef is set.
void launch_advs(const DGrid &g, const float *rru, const float *rrv, const float *rrw, int weighted,
                 const float *divx, const float *s, const float *s0, int sadd, const float *ten1,
                 const float *thterm, float *sten_out, float *snew, int weno, int pdef, int pdefweno,
                 double weps, float dt, int flush, float *scratch, cudaStream_t st, int64_t *nl) {
  SAdv a{rru, rrv, rrw, s, s0, divx, thterm, weighted, sadd};
  const int bx = 128;
  dim3 grid((g.ni + bx - 1) / bx, g.nj, g.nk);
  if (!pdef) {
    { ProfScope _ps("k_advs", st); k_advs<<<grid, bx, 0, st>>>(g, a, ten1, sten_out, snew, s0, weno, pdefweno, weps, dt, flush); }
    if (nl) *nl += 1;
    return;
  }
  long n = nS(g);
  float *advx = scratch, *advy = scratch + n, *advz = scratch + 2 * n;
  float *dumx = scratch + 3 * n, *dumy = scratch + 4 * n, *dumz = scratch + 5 * n;
  { ProfScope _ps("k_advs_pdef1", st); k_advs_pdef1<<<grid, bx, 0, st>>>(g, a, advx, advy, advz, dumx, dumy, dumz, weno, pdefweno, weps, dt); }
  launch_bc(g, dumx, 1, 0, st, nl);
  launch_bc(g, dumy, 1, 0, st, nl);
  { ProfScope _ps("k_advs_pdef2", st); k_advs_pdef2<<<grid, bx, 0, st>>>(g, a, advx, advy, advz, dumx, dumy, dumz, ten1, sten_out, snew, s0, dt, flush); }
  if (nl) *nl += 2;
}

}  // namespace cm1g
