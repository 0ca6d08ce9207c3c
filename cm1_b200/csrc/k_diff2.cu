// k_diff2.cu -- 2nd-order diffusion with a fixed viscosity (difforder=2):
// the stress tensor of diff2def (diff2.F:743-1221, Cartesian grid, no
// terrain) and the tendencies diff2u/v/w/s (diff2.F:11-735) that solve1 adds
// to uten1 ... ptten (solve1.F:686-734), with rr = 1/rho and the w-level
// density rf of solve3.F:660-678.
//
// Four launches: k_d2_tensor forms rr, rf, divx and the raw t11..t33 at
// every point; k_d2_lateral applies the wall conditions of the lateral
// boundaries (free slip 3, no slip 4) in the reference's order; k_d2_column
// applies the bottom/top conditions and the rf weighting of t13, t23 column
// by column; k_d2_tend adds the momentum tendencies and the scalar ones.
// Binary32 throughout in the Fortran's evaluation order (--fmad=false).
#include "cm1g_common.cuh"
#include "k_diff2.cuh"

namespace cm1g {

__global__ void k_d2_tensor(DGrid g, Diff2Args a) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 0 .. ni+1
  const int j = (int)blockIdx.y;                                // 0 .. nj+1
  const int k = 1 + (int)blockIdx.z;                            // 1 .. nk+1
  if (i > g.ni + 1) return;
  const int nk = g.nk;
  const float coef = a.kdiff2;
  const long o = iS(g, i, j, k);
  const long pl = (long)g.NI * g.NJ;
  const float *rho = a.rho, *ua = a.ua, *va = a.va, *wa = a.wa;
  // rr and rf (solve3.F:660-678)
  if (k <= nk) a.rr[o] = 1.0f / rho[o];
  if (k == 1) a.rf[o] = a.cgs1 * rho[o] + a.cgs2 * rho[o + pl] + a.cgs3 * rho[o + 2 * pl];
  else if (k == nk + 1) a.rf[o] = a.cgt1 * rho[o - pl] + a.cgt2 * rho[o - 2 * pl] + a.cgt3 * rho[o - 3 * pl];
  else a.rf[o] = LDG(&g.c1[k]) * rho[o - pl] + LDG(&g.c2[k]) * rho[o];
  if (k <= nk) {
    // diff2def.F:773-795: divx and the stress tensor at s-points and t12
    const long ou = iU(g, i, j, k), ov = iV(g, i, j, k);
    const float uh = LDG(&g.uh[i - g.ib]), vh = LDG(&g.vh[j - g.jb]), mh = LDG(&g.mh[k]);
    float dv = (ua[ou + 1] - ua[ou]) * g.rdx * uh + (va[ov + g.NI] - va[ov]) * g.rdy * vh +
               (wa[o + pl] - wa[o]) * g.rdz * mh;
    if (fabsf(dv) < g.smeps) dv = 0.0f;
    a.divx[o] = dv;
    a.t11[o] = coef * rho[o] * (ua[ou + 1] - ua[ou]) * g.rdx * uh;
    a.t22[o] = coef * rho[o] * (va[ov + g.NI] - va[ov]) * g.rdy * vh;
    a.t33[o] = coef * rho[o] * (wa[o + pl] - wa[o]) * g.rdz * mh;
    const float uf = LDG(&g.uf[i - g.ib]), vf = LDG(&g.vf[j - g.jb]);
    a.t12[o] = coef * ((ua[ou] - ua[ou - (g.NI + 1)]) * g.rdy * vf + (va[ov] - va[ov - 1]) * g.rdx * uf) * 0.25f *
               ((rho[o - 1 - g.NI] + rho[o]) + (rho[o - 1] + rho[o - g.NI]));
  }
  // t13, t23 at k = 2..nk (diff2def.F:852-858)
  if (k >= 2 && k <= nk && i >= 1 && j >= 1) {
    const long ou = iU(g, i, j, k), ov = iV(g, i, j, k);
    const float mf = LDG(&g.mf[k]), uf = LDG(&g.uf[i - g.ib]), vf = LDG(&g.vf[j - g.jb]);
    a.t13[o] = coef * ((ua[ou] - ua[ou - (long)(g.NI + 1) * g.NJ]) * g.rdz * mf + (wa[o] - wa[o - 1]) * g.rdx * uf);
    a.t23[o] = coef * ((va[ov] - va[ov - (long)g.NI * (g.NJ + 1)]) * g.rdz * mf + (wa[o] - wa[o - g.NI]) * g.rdy * vf);
  } else if (k == 1 || k == nk + 1) {
    a.t13[o] = 0.0f;   // set by the bottom/top conditions where the tendencies read them
    a.t23[o] = 0.0f;
  }
}

// Lateral walls (diff2def.F:797-917): one warp per level, the four sides in
// the reference's order (west, east, south, north), lanes along a side.
__global__ void k_d2_lateral(DGrid g, Diff2Args a) {
  const int k = 1 + (int)blockIdx.x;
  const int lane = (int)threadIdx.x;
  const int ni = g.ni, nj = g.nj;
  const float coef = a.kdiff2;
  const float *rho = a.rho;
  auto R4 = [&](int i, int j) {   // (rho(i-1,j-1)+rho(i,j))+(rho(i-1,j)+rho(i,j-1)); the 0.25 is applied before it
    return (rho[iS(g, i - 1, j - 1, k)] + rho[iS(g, i, j, k)]) + (rho[iS(g, i - 1, j, k)] + rho[iS(g, i, j - 1, k)]);
  };
  float *t12 = a.t12, *t13 = a.t13, *t23 = a.t23;
  // t12 at every level 1..nk
  if (g.wbc == 3 && g.ibw) for (int j = 1 + lane; j <= nj + 1; j += 32) t12[iS(g, 1, j, k)] = t12[iS(g, 2, j, k)];
  else if (g.wbc == 4 && g.ibw)
    for (int j = 1 + lane; j <= nj + 1; j += 32)
      t12[iS(g, 1, j, k)] = coef * 2.0f * a.va[iV(g, 1, j, k)] * g.rdx * LDG(&g.uf[1 - g.ib]) * 0.25f * R4(1, j);
  __syncwarp();
  if (g.ebc == 3 && g.ibe) for (int j = 1 + lane; j <= nj + 1; j += 32) t12[iS(g, ni + 1, j, k)] = t12[iS(g, ni, j, k)];
  else if (g.ebc == 4 && g.ibe)
    for (int j = 1 + lane; j <= nj + 1; j += 32)
      t12[iS(g, ni + 1, j, k)] = -coef * 2.0f * a.va[iV(g, ni, j, k)] * g.rdx * LDG(&g.uf[ni + 1 - g.ib]) * 0.25f * R4(ni + 1, j);
  __syncwarp();
  if (g.sbc == 3 && g.ibs) for (int i = 1 + lane; i <= ni + 1; i += 32) t12[iS(g, i, 1, k)] = t12[iS(g, i, 2, k)];
  else if (g.sbc == 4 && g.ibs)
    for (int i = 1 + lane; i <= ni + 1; i += 32)
      t12[iS(g, i, 1, k)] = coef * 2.0f * a.ua[iU(g, i, 1, k)] * g.rdy * LDG(&g.vf[1 - g.jb]) * 0.25f * R4(i, 1);
  __syncwarp();
  if (g.nbc == 3 && g.ibn) for (int i = 1 + lane; i <= ni + 1; i += 32) t12[iS(g, i, nj + 1, k)] = t12[iS(g, i, nj, k)];
  else if (g.nbc == 4 && g.ibn)
    for (int i = 1 + lane; i <= ni + 1; i += 32)
      t12[iS(g, i, nj + 1, k)] = -coef * 2.0f * a.ua[iU(g, i, nj, k)] * g.rdy * LDG(&g.vf[nj + 1 - g.jb]) * 0.25f * R4(i, nj + 1);
  __syncwarp();
  if (k == 1) return;   // t13, t23 at k = 2..nk
  if (g.wbc == 3 && g.ibw) for (int j = 1 + lane; j <= nj; j += 32) t13[iS(g, 1, j, k)] = t13[iS(g, 2, j, k)];
  else if (g.wbc == 4 && g.ibw)
    for (int j = 1 + lane; j <= nj; j += 32) t13[iS(g, 1, j, k)] = coef * 2.0f * a.wa[iS(g, 1, j, k)] * g.rdx * LDG(&g.uf[1 - g.ib]);
  __syncwarp();
  if (g.ebc == 3 && g.ibe) for (int j = 1 + lane; j <= nj; j += 32) t13[iS(g, ni + 1, j, k)] = t13[iS(g, ni, j, k)];
  else if (g.ebc == 4 && g.ibe)
    for (int j = 1 + lane; j <= nj; j += 32)
      t13[iS(g, ni + 1, j, k)] = -coef * 2.0f * a.wa[iS(g, ni, j, k)] * g.rdx * LDG(&g.uf[ni + 1 - g.ib]);
  __syncwarp();
  if (g.sbc == 3 && g.ibs) for (int i = 1 + lane; i <= ni; i += 32) t23[iS(g, i, 1, k)] = t23[iS(g, i, 2, k)];
  else if (g.sbc == 4 && g.ibs)
    for (int i = 1 + lane; i <= ni; i += 32) t23[iS(g, i, 1, k)] = coef * 2.0f * a.wa[iS(g, i, 1, k)] * g.rdy * LDG(&g.vf[1 - g.jb]);
  __syncwarp();
  if (g.nbc == 3 && g.ibn) for (int i = 1 + lane; i <= ni; i += 32) t23[iS(g, i, nj + 1, k)] = t23[iS(g, i, nj, k)];
  else if (g.nbc == 4 && g.ibn)
    for (int i = 1 + lane; i <= ni; i += 32)
      t23[iS(g, i, nj + 1, k)] = -coef * 2.0f * a.wa[iS(g, i, nj, k)] * g.rdy * LDG(&g.vf[nj + 1 - g.jb]);
}

// Bottom/top conditions and the rf weighting of t13, t23 (diff2def.F:926-989)
__global__ void k_d2_column(DGrid g, Diff2Args a) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 1 .. ni+1
  const int j = 1 + (int)blockIdx.y;                                // 1 .. nj+1
  if (i > g.ni + 1) return;
  const int nk = g.nk;
  const float coef = a.kdiff2;
  float *t13 = a.t13, *t23 = a.t23;
  const bool in13 = j <= g.nj, in23 = i <= g.ni;   // ranges of the t13 and t23 conditions
  const long o1 = iS(g, i, j, 1), o2 = iS(g, i, j, 2), on = iS(g, i, j, nk), on1 = iS(g, i, j, nk + 1);
  const float mf1 = LDG(&g.mf[1]), mfn = LDG(&g.mf[nk + 1]);
  if (a.bbc == 1) {
    if (in13) t13[o1] = t13[o2];
    if (in23) t23[o1] = t23[o2];
  } else if (a.bbc == 2) {
    if (in13) t13[o1] = coef * 2.0f * (a.ua[iU(g, i, j, 1)] + 0.0f) * g.rdz * mf1;
    if (in23) t23[o1] = coef * 2.0f * (a.va[iV(g, i, j, 1)] + 0.0f) * g.rdz * mf1;
  }
  if (a.tbc == 1) {
    if (in13) t13[on1] = t13[on];
    if (in23) t23[on1] = t23[on];
  } else if (a.tbc == 2) {
    if (in13) t13[on1] = -coef * 2.0f * a.ua[iU(g, i, j, nk)] * g.rdz * mfn;
    if (in23) t23[on1] = -coef * 2.0f * a.va[iV(g, i, j, nk)] * g.rdz * mfn;
  }
  for (int k = 1; k <= nk + 1; k++) {
    const long o = iS(g, i, j, k);
    t13[o] = t13[o] * 0.5f * (a.rf[o - 1] + a.rf[o]);
    t23[o] = t23[o] * 0.5f * (a.rf[o - g.NI] + a.rf[o]);
  }
}

// diff2u/v/w (diff2.F:11-532) and diff2s (diff2.F:540-735) for nsc scalars
__global__ void k_d2_tend(DGrid g, Diff2Args a) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 1 .. ni+1
  const int j = 1 + (int)blockIdx.y;                                // 1 .. nj+1
  const int k = 1 + (int)blockIdx.z;                                // 1 .. nk
  if (i > g.ni + 1) return;
  const int ni = g.ni, nj = g.nj, nk = g.nk;
  const float twdth = 2.0f / 3.0f;
  const long o = iS(g, i, j, k), pl = (long)g.NI * g.NJ;
  const float *rho = a.rho;
  const float rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
  if (a.momentum) {
    if (j <= nj) {   // u at (i, j), i = 1..ni+1
      const float d0 = 2.0f * a.t11[o] - rho[o] * twdth * a.divx[o];
      const float dm = 2.0f * a.t11[o - 1] - rho[o - 1] * twdth * a.divx[o - 1];
      const float fx = (d0 - dm) * rdx * LDG(&g.uf[i - g.ib]);
      const float fy = (a.t12[o + g.NI] - a.t12[o]) * rdy * LDG(&g.vh[j - g.jb]);
      const float fz = (a.t13[o + pl] - a.t13[o]) * rdz * LDG(&g.mh[k]);
      const long ou = iU(g, i, j, k);
      a.uten[ou] = a.uten[ou] + ((fx + fy) + fz) / (0.5f * (rho[o - 1] + rho[o]));
    }
    if (i <= ni) {   // v at (i, j), j = 1..nj+1
      const float fx = (a.t12[o + 1] - a.t12[o]) * rdx * LDG(&g.uh[i - g.ib]);
      const float d0 = 2.0f * a.t22[o] - rho[o] * twdth * a.divx[o];
      const float dm = 2.0f * a.t22[o - g.NI] - rho[o - g.NI] * twdth * a.divx[o - g.NI];
      const float fy = (d0 - dm) * rdy * LDG(&g.vf[j - g.jb]);
      const float fz = (a.t23[o + pl] - a.t23[o]) * rdz * LDG(&g.mh[k]);
      const long ov = iV(g, i, j, k);
      a.vten[ov] = a.vten[ov] + ((fx + fy) + fz) / (0.5f * (rho[o - g.NI] + rho[o]));
    }
    if (i <= ni && j <= nj && k >= 2) {   // w at (i, j, k), k = 2..nk
      const float fx = (a.t13[o + 1] - a.t13[o]) * rdx * LDG(&g.uh[i - g.ib]);
      const float fy = (a.t23[o + g.NI] - a.t23[o]) * rdy * LDG(&g.vh[j - g.jb]);
      const float d0 = 2.0f * a.t33[o] - rho[o] * twdth * a.divx[o];
      const float dm = 2.0f * a.t33[o - pl] - rho[o - pl] * twdth * a.divx[o - pl];
      const float fz = (d0 - dm) * rdz * LDG(&g.mf[k]);
      a.wten[o] = a.wten[o] + ((fx + fy) + fz) / a.rf[o];
    }
  }
  if (i > ni || j > nj) return;
  // scalars (diff2s): x, y and z fluxes of each s, sten += (...)*rr
  const float coef = a.kdiff2;
  const float uf0 = LDG(&g.uf[i - g.ib]), uf1 = LDG(&g.uf[i + 1 - g.ib]);
  const float vf0 = LDG(&g.vf[j - g.jb]), vf1 = LDG(&g.vf[j + 1 - g.jb]);
  const float uh = LDG(&g.uh[i - g.ib]), vh = LDG(&g.vh[j - g.jb]), mh = LDG(&g.mh[k]);
  const float mf0 = LDG(&g.mf[k]), mf1 = LDG(&g.mf[k + 1]);
  for (int n = 0; n < a.nsc; n++) {
    const float *s = a.s[n];
    const float dxl = 0.5f * (rho[o] + rho[o - 1]) * (s[o] - s[o - 1]) * rdx * uf0;
    const float dxr = 0.5f * (rho[o + 1] + rho[o]) * (s[o + 1] - s[o]) * rdx * uf1;
    const float dfx = coef * (dxr - dxl) * rdx * uh;
    const float dyl = 0.5f * (rho[o] + rho[o - g.NI]) * (s[o] - s[o - g.NI]) * rdy * vf0;
    const float dyr = 0.5f * (rho[o + g.NI] + rho[o]) * (s[o + g.NI] - s[o]) * rdy * vf1;
    const float dfy = coef * (dyr - dyl) * rdy * vh;
    const float dzl = (k == 1) ? 0.0f : (s[o] - s[o - pl]) * rdz * mf0;
    const float dzu = (k == nk) ? 0.0f : (s[o + pl] - s[o]) * rdz * mf1;
    const float dfz = coef * (a.rf[o + pl] * dzu - a.rf[o] * dzl) * rdz * mh;
    a.sten[n][o] = a.sten[n][o] + ((dfx + dfy) + dfz) * a.rr[o];
  }
}

void launch_diff2(const DGrid &g, const Diff2Args &a, cudaStream_t st, int64_t *nl) {
  {
    dim3 grid((g.ni + 2 + 127) / 128, g.nj + 2, g.nk + 1);
    ProfScope _ps("k_d2_tensor", st);
    k_d2_tensor<<<grid, 128, 0, st>>>(g, a);
  }
  const bool walls = (g.ibw && (g.wbc == 3 || g.wbc == 4)) || (g.ibe && (g.ebc == 3 || g.ebc == 4)) ||
                     (g.ibs && (g.sbc == 3 || g.sbc == 4)) || (g.ibn && (g.nbc == 3 || g.nbc == 4));
  if (walls) {
    ProfScope _ps("k_d2_lateral", st);
    k_d2_lateral<<<g.nk, 32, 0, st>>>(g, a);
    if (nl) *nl += 1;
  }
  {
    dim3 grid((g.ni + 1 + 127) / 128, g.nj + 1);
    ProfScope _ps("k_d2_column", st);
    k_d2_column<<<grid, 128, 0, st>>>(g, a);
  }
  {
    dim3 grid((g.ni + 1 + 127) / 128, g.nj + 1, g.nk);
    ProfScope _ps("k_d2_tend", st);
    k_d2_tend<<<grid, 128, 0, st>>>(g, a);
  }
  if (nl) *nl += 3;
}

}  // namespace cm1g
