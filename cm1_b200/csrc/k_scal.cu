// k_scal.cu -- scalar advection of one RK stage for every advected field in
// one launch: advs (adv.F:14-903) as solve2 calls it for theta
// (solve2.F:1394), each moisture array (1490/1510) and each passive tracer
// (1941), followed by the RK update of each (solve2.F:1419-1425, 1513-1520,
// 1951-1957).  All fields of a stage are advected by the same averaged
// velocities rru/rrv/rrw, so one block advances every field over its tile:
//
//  * a block owns TX x TY columns and KC levels; it walks the items
//    (field n, level k) field by field, level by level upward;
//  * the level of a field is staged in shared memory with its 3-point halo by
//    one-dimensional bulk copies (cp.async.bulk), one per row, into a ring of
//    RD planes; warp 0 issues the copies of item t+RD as soon as item t's
//    plane has been read, and an mbarrier per ring slot tells the block when
//    they have landed, so each plane is in flight while RD-1 others compute;
//  * the caller's rows are not 16-byte aligned (a row holds NI = ni+6
//    floats), so each row copy takes the aligned superset of its 38 values;
//    the plane's row pitch SP is chosen congruent to NI modulo 4, so that
//    every row lands with element x at plane[c + r*SP + x] for a c that is
//    the same for all rows of the plane;
//  * each x- and y-face flux is evaluated once (hflux5, the WENO5 or
//    5th-order value), the vertical face of the level above comes from a
//    per-thread register window of the column (zflux_win) and is carried to
//    the next level;
//  * one barrier per item: the face fluxes and face velocities are double
//    buffered by item parity.
//
// Every face value and the update use the operations of k_advs_tile in the
// same order, so the result is bit-identical to advancing the fields one
// launch at a time.  Waits on the mbarriers are bounded: a block that gives
// up sets *err and leaves without writing (the host reports the error).
#include <cstdint>
#include "cm1g_common.cuh"
#include "k_face.cuh"

namespace cm1g {

constexpr int SC_MAX = 16;      // fields per launch

struct ScalPass {
  ScalField f[SC_MAX];
  int n;
  const float *rru, *rrv, *rrw; // small-step-averaged velocities (sound.F:806-835)
  const float *thterm;          // moist theta: thten -= div(u_avg) * thterm (solve2.F:1320-1329); null: none
  float dt;
  int *err;                     // set to 1 when a block gives up waiting for its staged data
};

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_arrive(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false if the phase did not complete within the limit
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

}  // namespace

// Row pitch of a staged plane: at least TX + 16 floats (the aligned superset
// of a row's TX + 6 values is at most TX + 12) and congruent to NI modulo 4.
template <int TX>
__host__ __device__ __forceinline__ int scal_pitch(int NI) {
  const int p0 = TX + 16;
  return p0 + (((NI - p0) % 4) + 4) % 4;
}

template <int TX, int TY, int KC, int WENO>
__global__ void __launch_bounds__(TX * (TY + 1), 3) k_scal_tile(DGrid g, ScalPass P) {
  constexpr int NT = TX * (TY + 1);
  constexpr int SW = TX + 6, SH = TY + 6;                  // staged columns and rows
  constexpr int RD = 4;                                     // ring of staged planes
  constexpr int PL = ((8 + (SH - 1) * (TX + 19) + TX + 12) + 3) / 4 * 4;   // floats per plane
  constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
  constexpr int NL = KC + 8;                                // cached profile levels kc0-3 .. kc0+KC+4
  static_assert(SH <= 32, "one lane per staged row");
  __shared__ __align__(128) float ring[RD][PL];
  __shared__ float fx[2][NFX], ux[2][NFX], fy[2][NFY], vy[2][NFY];
  __shared__ float prof[7][NL];   // rho0, rf0, mh, rr0, th0-300, c1, c2 by level
  __shared__ __align__(8) uint64_t bars[RD];

  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty, lane = tid & 31;
  // the first warp of the extra row issues the staging copies
  const bool stager = (tid >= TX * TY && tid < TX * TY + 32);
  const int i0 = 1 + (int)blockIdx.x * TX, j0 = 1 + (int)blockIdx.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int ni = g.ni, nj = g.nj, nk = g.nk, NI = g.NI, NJ = g.NJ;
  const bool active = (ty < TY && i <= ni && j <= nj);
  const bool doitw = (g.wbc == 2 && g.ibw), doite = (g.ebc == 2 && g.ibe);
  const bool doits = (g.sbc == 2 && g.ibs), doitn = (g.nbc == 2 && g.ibn);
  // the open-boundary fix-ups of adv.F touch only the cells next to an open edge
  const bool edge = (doitw && i0 == 1) || (doite && i0 + TX - 1 >= ni) || (doits && j0 == 1) ||
                    (doitn && j0 + TY - 1 >= nj);
  const int je = nj + g.ngxy;
  // 32-bit offsets: cm1g_init refuses arrays of 2^31 points or more
  const int planeS = NI * NJ, planeU = (NI + 1) * NJ, planeV = NI * (NJ + 1);
  const int SP = scal_pitch<TX>(NI);
  const float uh_i = active ? LDG(&g.uh[i - g.ib]) : 0.0f, vh_j = active ? LDG(&g.vh[j - g.jb]) : 0.0f;
  const int oc = active ? (i - g.ib) + NI * (j - g.jb) : 0;   // the column's in-plane offset
  const int orow0 = (i0 - 3 - g.ib) + NI * (j0 - 3 - g.jb);    // first staged element of a plane
  const int kc0 = 1 + (int)blockIdx.z * KC, kc1 = min(nk, kc0 + KC - 1);
  const int nlev = kc1 - kc0 + 1, nitem = P.n * nlev;
  const int kb0 = kc0 - 3;                                     // level of prof[.][0]
  const float rdx = g.rdx, rdy = g.rdy, rdz = g.rdz, smeps = g.smeps, dt = P.dt;

  // faces of this thread: a cell row's thread owns the x face on the west of
  // its cell and the y face on its south; the extra row's threads own the y
  // faces north of the tile and (the first TY of them) the x faces east of it,
  // so that every cell thread evaluates three faces and no thread more
  int fxo = -1, fxs = 0, fyo = -1, fys = 0, fxd = NFX, fyd;
  {
    int xrow = ty, xcol = tx;
    if (ty == TY) { xrow = tx; xcol = TX; }
    if (xrow < TY) {
      fxd = xrow * (TX + 1) + xcol;
      const int ii = i0 + xcol, jj = j0 + xrow;
      if (ii <= ni + 1 && jj <= nj) { fxo = (ii - g.ib) + (NI + 1) * (jj - g.jb); fxs = (xrow + 3) * SP + xcol; }
    }
    fyd = ty * TX + tx;
    const int ii = i0 + tx, jj = j0 + ty;
    if (ii <= ni && jj <= nj + 1) { fyo = (ii - g.ib) + NI * (jj - g.jb); fys = ty * SP + tx + 3; }
  }
  const int csel = (ty + 3) * SP + tx + 3;   // the cell in a staged plane
  const int xi = ty * (TX + 1) + tx, yi = ty * TX + tx;

  // vertical profiles of the block's levels (0 outside 0..nk+1)
  for (int e = tid; e < 7 * NL; e += NT) {
    const int a = e / NL, k = kb0 + e - a * NL;
    float v = 0.0f;
    if (k >= 0 && k <= nk + 1) {
      switch (a) {
        case 0: v = LDG(&g.rho0[k]); break;
        case 1: v = LDG(&g.rf0[k]); break;
        case 2: v = LDG(&g.mh[k]); break;
        case 3: v = LDG(&g.rr0[k]); break;
        case 4: v = LDG(&g.th0[k]) - 300.0f; break;
        case 5: v = LDG(&g.c1[k]); break;
        default: v = LDG(&g.c2[k]); break;
      }
    }
    prof[a][e - a * NL] = v;
  }
  const float *PR0 = prof[0] - kb0, *PRF = prof[1] - kb0, *PMH = prof[2] - kb0, *PRR = prof[3] - kb0,
              *PTH = prof[4] - kb0, *PC1 = prof[5] - kb0, *PC2 = prof[6] - kb0;

  // ---- staging: items in order (field, level) -> ring slot item % RD
  const uint32_t bar0 = smem_u32(&bars[0]);
  if (tid == 0) {
    for (int b = 0; b < RD; b++) mbar_init(bar0 + 8 * b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // warp 0: the row copies of the item (field nf, level kf) into slot `slot`
  // (rows beyond je are never read)
  auto issue = [&](int nf, int kf, int slot) {
    const float *p0 = P.f[nf].s + (kf * planeS + orow0);
    const int l0 = (int)(((uintptr_t)p0 >> 2) & 3);
    uint32_t bytes = 0, dst = 0;
    const float *src = nullptr;
    if (lane < SH && j0 - 3 + lane <= je) {
      const uintptr_t a0 = (uintptr_t)(p0 + lane * NI);
      const uintptr_t as = a0 & ~(uintptr_t)15, ae = (a0 + 4 * SW + 15) & ~(uintptr_t)15;
      const int lr = (int)((a0 >> 2) & 3);
      bytes = (uint32_t)(ae - as);
      src = (const float *)as;
      dst = smem_u32(&ring[slot][l0 + 4 + lane * SP - lr]);
    }
    const uint32_t total = __reduce_add_sync(0xffffffffu, bytes);
    if (lane == 0) mbar_expect_arrive(bar0 + 8 * slot, total);
    __syncwarp();
    if (bytes) bulk_g2s(dst, src, bytes, bar0 + 8 * slot);
  };
  int in_ = 0, ik_ = kc0, it_ = 0;   // next item to issue
  auto issue_next = [&]() {
    issue(in_, ik_, it_ % RD);
    it_++;
    if (++ik_ > kc1) { ik_ = kc0; in_++; }
  };
  if (stager)
    while (it_ < RD && it_ < nitem) issue_next();

  // ---- per-item global reads, issued one item ahead
  float pru = 0.0f, prv = 0.0f, pwhi = 0.0f, pe0 = 0.0f, pe1 = 0.0f, pe2 = 0.0f, pwtop = 0.0f;
  auto fetch = [&](int nf, int kf) {
    const ScalField &F = P.f[nf];
    const float *uk = P.rru + kf * planeU, *vk = P.rrv + kf * planeV;
    pru = (fxo >= 0) ? LDG(&uk[fxo]) : 0.0f;
    prv = (fyo >= 0) ? LDG(&vk[fyo]) : 0.0f;
    if (active) {
      const int o = kf * planeS + oc;
      pwhi = (kf + 1 >= nk + 1) ? 0.0f : LDG(&P.rrw[o + planeS]);
      pe0 = F.ten1[o];
      pe1 = LDG(&F.sbase[o]);
      if (F.sadd && P.thterm) pe2 = LDG(&P.thterm[o]);
      float v = 0.0f;
      if (kf + 3 <= nk + 1) {
        v = LDG(&F.s[o + 3 * planeS]);
        if (F.sadd) v = PTH[kf + 3] + v;
      }
      pwtop = v;
    }
  };

  float wv[6] = {0, 0, 0, 0, 0, 0};   // s(k-2 .. k+3) of the column, for the top face of level k
  int tfail = -1, t = 0;
  fetch(0, kc0);
  for (int n = 0; n < P.n && tfail < 0; n++) {
    const ScalField &F = P.f[n];
    const int sadd = F.sadd, pdw = F.pdefweno, flush = F.flush;
    const double weps = F.weps;
    const bool tht = sadd && P.thterm;
    float *snew = F.snew;
    // the column window and the face below the first level
    float fzlo = 0.0f, fwlo = 0.0f, wlo = 0.0f;
    if (active) {
      const float *sc = F.s + oc;
      auto SV = [&](int kk) -> float {
        float v = LDG(&sc[kk * planeS]);
        if (sadd) v = PTH[kk] + v;
        return v;
      };
#pragma unroll
      for (int d = 0; d < 6; d++) {
        const int kk = kc0 - 2 + d;
        wv[d] = (kk >= 0 && kk <= nk + 1) ? SV(kk) : 0.0f;
      }
      wlo = (kc0 <= 1) ? 0.0f : LDG(&P.rrw[kc0 * planeS + oc]);
      fwlo = wlo * PRF[kc0];
      if (kc0 >= 2) {
        float w0[6];
#pragma unroll
        for (int d = 0; d < 6; d++) {
          const int kk = kc0 - 3 + d;
          w0[d] = (kk >= 0 && kk <= nk + 1) ? SV(kk) : 0.0f;
        }
        fzlo = zflux_core(w0, fwlo, kc0, nk, PC1[kc0], PC2[kc0], WENO, pdw, weps);
      }
    }
    for (int k = kc0; k <= kc1; k++, t++) {
      const float r0k = PR0[k], th0m = sadd ? PTH[k] : 0.0f;
      const float ru0 = pru, rv0 = prv;
      const float whi = pwhi, e0 = pe0, e1 = pe1, e2 = pe2;
      if (k < kc1) fetch(n, k + 1);                 // pwtop becomes s(k+4): the next level's window top
      else if (n + 1 < P.n) fetch(n + 1, kc0);
      const int b = t & 1, slot = t % RD;
      // ---- the staged plane of this item
      const bool ok = mbar_wait(bar0 + 8 * slot, (uint32_t)((t / RD) & 1));
      const float *pl = &ring[slot][(int)((((uintptr_t)(F.s + (k * planeS + orow0))) >> 2) & 3) + 4];
      // ---- face values: each x/y face once, the upper z face once per column
      auto xface = [&](float ru) {
        const float *p = pl + fxs;
        float s0 = p[0], s1 = p[1], s2 = p[2], s3 = p[3], s4 = p[4], s5 = p[5];
        if (sadd) { s0 = th0m + s0; s1 = th0m + s1; s2 = th0m + s2; s3 = th0m + s3; s4 = th0m + s4; s5 = th0m + s5; }
        fx[b][fxd] = hflux5(ru * r0k, s0, s1, s2, s3, s4, s5, WENO, 0, weps);
        ux[b][fxd] = ru;
      };
      auto yface = [&](float rv) {
        const float *p = pl + fys;
        float s0 = p[0], s1 = p[SP], s2 = p[2 * SP], s3 = p[3 * SP], s4 = p[4 * SP], s5 = p[5 * SP];
        if (sadd) { s0 = th0m + s0; s1 = th0m + s1; s2 = th0m + s2; s3 = th0m + s3; s4 = th0m + s4; s5 = th0m + s5; }
        fy[b][fyd] = hflux5(rv * r0k, s0, s1, s2, s3, s4, s5, WENO, 0, weps);
        vy[b][fyd] = rv;
      };
      if (fxo >= 0) xface(ru0);
      if (fyo >= 0) yface(rv0);
      const float fwhi = whi * PRF[k + 1];
      float fzhi = 0.0f, sc = 0.0f;
      if (active) {
        sc = pl[csel];
        if (sadd) sc = th0m + sc;
        const int kk = k + 1;
        if (kk >= 4 && kk <= nk - 2) fzhi = zflux_inner(wv, fwhi, WENO, pdw, weps);
        else if (kk <= nk) fzhi = zflux_core(wv, fwhi, kk, nk, PC1[kk], PC2[kk], WENO, pdw, weps);
      }
      if (__syncthreads_or(!ok)) { tfail = t; break; }
      // the plane of this item has been read: its slot takes the item RD later
      if (stager && it_ < nitem) issue_next();
      if (active) {
        float fx0 = fx[b][xi], fxp = fx[b][xi + 1], fy0 = fy[b][yi], fyp = fy[b][yi + TX];
        const float u0r = ux[b][xi], u1r = ux[b][xi + 1], v0r = vy[b][yi], v1r = vy[b][yi + TX];
        const float fu0 = u0r * r0k, fu1 = u1r * r0k, fv0 = v0r * r0k, fv1 = v1r * r0k;
        float advx, advy;
        if (!edge) {
          advx = -(fxp - fx0) * rdx * uh_i;
          advy = -(fyp - fy0) * rdy * vh_j;
        } else {
          // adv.F:212-268
          if (doitw && i == 1 && fu0 >= 0.0f) fx0 = fxp;
          if (doite && i == ni && fu1 <= 0.0f) fxp = fx0;
          if (doits && j == 1 && fv0 >= 0.0f) fy0 = fyp;
          if (doitn && j == nj && fv1 <= 0.0f) fyp = fy0;
          advx = -(fxp - fx0) * rdx * uh_i;
          advy = -(fyp - fy0) * rdy * vh_j;
          // adv.F:286-335
          if (doitw && i == 1 && fu0 >= 0.0f) advx = advx - sc * (fu1 - fu0) * rdx * uh_i;
          if (doite && i == ni && fu1 <= 0.0f) advx = advx - sc * (fu1 - fu0) * rdx * uh_i;
          if (doits && j == 1 && fv0 >= 0.0f) advy = advy - sc * (fv1 - fv0) * rdy * vh_j;
          if (doitn && j == nj && fv1 <= 0.0f) advy = advy - sc * (fv1 - fv0) * rdy * vh_j;
        }
        const float mhk = PMH[k];
        float advz;
        if (k == 1) advz = -fzhi * rdz * mhk;
        else if (k == nk) advz = +fzlo * rdz * mhk;
        else advz = -(fzhi - fzlo) * rdz * mhk;
        float div = ((fu1 - fu0) * rdx * uh_i + (fv1 - fv0) * rdy * vh_j) + (fwhi - fwlo) * rdz * mhk;
        if (fabsf(div) < smeps) div = 0.0f;
        float ten = e0;
        if (tht) {   // getdiv of the averaged velocities (misclibs.F:127-136)
          float rd = ((u1r - u0r) * rdx * uh_i + (v1r - v0r) * rdy * vh_j) + (whi - wlo) * rdz * mhk;
          if (fabsf(rd) < smeps) rd = 0.0f;
          ten = ten - rd * e2;
        }
        ten = ten + (((advx + advy) + advz) + sc * div) * PRR[k];
        float v = e1 + dt * ten;
        if (flush && fabsf(v) < smeps) v = 0.0f;
        snew[k * planeS + oc] = v;
        // slide the column window and carry the upper face to the next level
#pragma unroll
        for (int d = 0; d < 5; d++) wv[d] = wv[d + 1];
        wv[5] = pwtop;
        fzlo = fzhi;
        fwlo = fwhi;
        wlo = whi;
      }
    }
  }
  if (tfail >= 0) {
    // leave no bulk copy in flight into this block's shared memory: wait (each
    // wait bounded) for the items issued but not consumed
    if (tid == 0) atomicExch(P.err, 1);
    for (int u = tfail; u < nitem && u < tfail + RD; u++) (void)mbar_wait(bar0 + 8 * (u % RD), (uint32_t)((u / RD) & 1));
  }
}

template <int TX, int TY, int KC>
static void scal_shape(const DGrid &g, const ScalPass &P, int weno, cudaStream_t st) {
  dim3 blk(TX, TY + 1), grid((g.ni + TX - 1) / TX, (g.nj + TY - 1) / TY, (g.nk + KC - 1) / KC);
  if (weno) k_scal_tile<TX, TY, KC, 1><<<grid, blk, 0, st>>>(g, P);
  else k_scal_tile<TX, TY, KC, 0><<<grid, blk, 0, st>>>(g, P);
}

// One launch for `n` fields (at most SC_MAX) advanced by the same averaged
// velocities; thterm applies to the field with sadd set.
void launch_scal_pass(const DGrid &g, const ScalField *f, int n, const float *rru, const float *rrv,
                      const float *rrw, const float *thterm, int weno, float dt, int *err, cudaStream_t st,
                      int64_t *nl) {
  for (int a = 0; a < n; a += SC_MAX) {
    ScalPass P{};
    P.n = (n - a < SC_MAX) ? n - a : SC_MAX;
    for (int m = 0; m < P.n; m++) P.f[m] = f[a + m];
    P.rru = rru; P.rrv = rrv; P.rrw = rrw; P.thterm = thterm; P.dt = dt; P.err = err;
    ProfScope _ps("k_scal_tile", st);
    static_assert(kNumTileShapes == 5, "one case per tile shape");
#define CM1G_SCAL_SHAPE(m) \
  case m: scal_shape<kScalShapes[m][0], kScalShapes[m][1], kScalShapes[m][2]>(g, P, weno, st); break;
    switch (g.tile_adv) {
      CM1G_SCAL_SHAPE(1)
      CM1G_SCAL_SHAPE(2)
      CM1G_SCAL_SHAPE(3)
      CM1G_SCAL_SHAPE(4)
      default: CM1G_SCAL_SHAPE(0)
    }
#undef CM1G_SCAL_SHAPE
    if (nl) *nl += 1;
  }
}

}  // namespace cm1g
