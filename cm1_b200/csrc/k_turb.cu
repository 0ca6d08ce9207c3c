// k_turb.cu -- Smagorinsky subgrid turbulence (sgsmodel=2) of an LES,
// Cartesian grid without terrain, periodic lateral boundaries, dry N^2,
// explicit vertical mixing (doimpl=0):
//   calcdef   rho*S_ij and the deformations defv, defh (turb.F:4711-5423)
//   calcnm    dry squared Brunt-Vaisala frequency (turb.F:5432-5480)
//   turbsmag  kmh, kmv for tconfig 1 and 2, bcw's zero rows and periodic
//             halo, khh = kmh/Pr, khv = kmv/Pr (turb.F:3375-3621)
//   gettau    stresses t_ij = 2 K rho S_ij with sfcstress's bbc 1/2 and the
//             top conditions tbc 1/2 (turb.F:4059-4506, 4515-4582)
//   turbu, turbv, turbw, turbs/turbsz   the tendencies solve1 adds to
//             uten1, vten1, wten1, thten1, qten, ptten (turbtend.F:18-692,
//             1052-1424, 1816-2180, 2473-2885; solve1.F:1113-1240)
//
// Four launches: k_les_strain (rho*S_ij at every point), k_les_km (N^2, the
// deformations and kmh/kmv, the halo ring evaluated at its periodic image),
// k_les_stress (t_ij in place; t13/t23 with the bottom and top rows; the
// scalar fluxes' face coefficients, shared by every scalar) and
// k_les_tend (momentum and all scalars, blockIdx.z over levels and fields).
// Binary32 in the Fortran's evaluation order (--fmad=false); the logarithm
// of calcnm and the cube root of tconfig=1 are evaluated in binary64 and
// rounded once.
#include "cm1g_common.cuh"
#include "k_turb.cuh"

namespace cm1g {

// w-level density rf (solve3.F:660-678)
__device__ __forceinline__ float les_rf(const DGrid &g, const TurbArgs &a, int i, int j, int k) {
  const long pl = (long)g.NI * g.NJ;
  const long o = iS(g, i, j, k);
  if (k == 1) return a.cgs1 * a.rho[o] + a.cgs2 * a.rho[o + pl] + a.cgs3 * a.rho[o + 2 * pl];
  if (k == g.nk + 1) return a.cgt1 * a.rho[o - pl] + a.cgt2 * a.rho[o - 2 * pl] + a.cgt3 * a.rho[o - 3 * pl];
  return LDG(&g.c1[k]) * a.rho[o - pl] + LDG(&g.c2[k]) * a.rho[o];
}

// calcdef, Cartesian without terrain (turb.F:4772-4790, 4880-4893)
__global__ void k_les_strain(DGrid g, TurbArgs a) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 0 .. ni+1
  const int j = (int)blockIdx.y;                                // 0 .. nj+1
  const int k = 1 + (int)blockIdx.z;                            // 1 .. nk
  if (i > g.ni + 1) return;
  const float rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
  const float *rho = a.rho, *ua = a.ua, *va = a.va, *wa = a.wa;
  const long o = iS(g, i, j, k);
  const float uh = LDG(&g.uh[i - g.ib]), vh = LDG(&g.vh[j - g.jb]);
  const float uf = LDG(&g.uf[i - g.ib]), vf = LDG(&g.vf[j - g.jb]);
  const float temz = rdz * LDG(&g.mh[k]);
  a.t11[o] = rho[o] * (ua[iU(g, i + 1, j, k)] - ua[iU(g, i, j, k)]) * rdx * uh;
  a.t22[o] = rho[o] * (va[iV(g, i, j + 1, k)] - va[iV(g, i, j, k)]) * rdy * vh;
  a.t33[o] = rho[o] * (wa[iW(g, i, j, k + 1)] - wa[iW(g, i, j, k)]) * temz;
  a.t12[o] = 0.5f * ((ua[iU(g, i, j, k)] - ua[iU(g, i, j - 1, k)]) * rdy * vf +
                     (va[iV(g, i, j, k)] - va[iV(g, i - 1, j, k)]) * rdx * uf) * 0.25f *
             ((rho[iS(g, i - 1, j - 1, k)] + rho[o]) + (rho[iS(g, i - 1, j, k)] + rho[iS(g, i, j - 1, k)]));
  if (k >= 2 && i >= 1 && j >= 1) {
    const float mfk = LDG(&g.mf[k]);
    a.s13[o] = 0.5f * ((wa[iW(g, i, j, k)] - wa[iW(g, i - 1, j, k)]) * rdx * uf +
                       (ua[iU(g, i, j, k)] - ua[iU(g, i, j, k - 1)]) * rdz * 0.5f * (mfk + mfk)) *
               0.5f * (les_rf(g, a, i - 1, j, k) + les_rf(g, a, i, j, k));
    a.s23[o] = 0.5f * ((wa[iW(g, i, j, k)] - wa[iW(g, i, j - 1, k)]) * rdy * vf +
                       (va[iV(g, i, j, k)] - va[iV(g, i, j, k - 1)]) * rdz * 0.5f * (mfk + mfk)) *
               0.5f * (les_rf(g, a, i, j - 1, k) + les_rf(g, a, i, j, k));
  }
}

__device__ __forceinline__ float sq(float x) { return x * x; }

// calcnm (dry), the deformations of calcdef (turb.F:5366-5390) and kmh/kmv
// of turbsmag; (i, j) on the halo ring takes the value of its periodic image
// (bcw), and the bottom and top rows are zero (bcw flag 1, bc.F:1126-1137).
__global__ void k_les_km(DGrid g, TurbArgs a) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 0 .. ni+1
  const int j = (int)blockIdx.y;                                // 0 .. nj+1
  const int k = 1 + (int)blockIdx.z;                            // 1 .. nk+1
  if (i > g.ni + 1) return;
  const long od = iS(g, i, j, k);
  if (k == 1 || k == g.nk + 1) { a.kmh[od] = 0.0f; a.kmv[od] = 0.0f; return; }
  const int ii = i < 1 ? i + g.ni : (i > g.ni ? i - g.ni : i);
  const int jj = j < 1 ? j + g.nj : (j > g.nj ? j - g.nj : j);
  const long pl = (long)g.NI * g.NJ;
  const long o = iS(g, ii, jj, k), om = o - pl;
  const float c1 = LDG(&g.c1[k]), c2 = LDG(&g.c2[k]);
  const float tmp11 = c1 * sq(a.t11[om]) + c2 * sq(a.t11[o]);
  const float tmp22 = c1 * sq(a.t22[om]) + c2 * sq(a.t22[o]);
  const float tmp33 = c1 * sq(a.t33[om]) + c2 * sq(a.t33[o]);
  const long o11 = iS(g, ii + 1, jj + 1, k), o01 = iS(g, ii, jj + 1, k), o10 = iS(g, ii + 1, jj, k);
  const float tmp12 = 0.25f * (c1 * ((sq(a.t12[om]) + sq(a.t12[o11 - pl])) + (sq(a.t12[o01 - pl]) + sq(a.t12[o10 - pl]))) +
                               c2 * ((sq(a.t12[o]) + sq(a.t12[o11])) + (sq(a.t12[o01]) + sq(a.t12[o10]))));
  const float tmp13 = 0.5f * (sq(a.s13[o]) + sq(a.s13[o10]));
  const float tmp23 = 0.5f * (sq(a.s23[o]) + sq(a.s23[o01]));
  const float rf = les_rf(g, a, ii, jj, k);
  const float rrf = 1.0f / sq(rf);
  const float defv = 4.0f * (tmp13 + tmp23) * rrf;
  const float defh = (2.0f * ((tmp11 + tmp22) + tmp33) + 4.0f * tmp12) * rrf;
  // calcnm, imoist=0 (turb.F:5458-5468)
  const float th0k = LDG(&g.th0[k]), th0m = LDG(&g.th0[k - 1]);
  const float q = (th0k + a.tha[o]) / (th0m + a.tha[om]);
  const float nm = (float)log((double)q) * g.c.g * g.rdz * LDG(&g.mf[k]);
  const float dmin = 1.0e-10f;
  const float rmf = 1.0f / LDG(&g.mf[k]);
  const float dxr = g.dx * LDG(&g.ruh[ii - g.ib]), dyr = g.dy * LDG(&g.rvh[jj - g.jb]);
  float kmh, kmv;
  if (a.tconfig == 1) {
    const float grd = (float)pow((double)((dxr * dyr) * (g.dz * rmf)), (double)0.33333333f);
    kmh = sq(a.csm * grd) * sqrtf(fmaxf(defv + defh - nm * a.prinv, dmin));
    kmv = kmh;
  } else {
    const float lenh = sqrtf(dxr * dyr);
    const float grd = g.dz * rmf;
    kmh = sq(a.csm * lenh) * sqrtf(fmaxf(defh, dmin));
    kmv = sq(a.csm * grd) * sqrtf(fmaxf(defv - nm * a.prinv, dmin));
  }
  a.kmh[od] = kmh;
  a.kmv[od] = kmv;
}

// gettau (Cartesian) with sfcstress's bottom row and the top row
__global__ void k_les_stress(DGrid g, TurbArgs a) {
  const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 0 .. ni+1
  const int j = (int)blockIdx.y;                                // 0 .. nj+1
  const int k = 1 + (int)blockIdx.z;                            // 1 .. nk+1
  if (i > g.ni + 1) return;
  const int nk = g.nk;
  const long pl = (long)g.NI * g.NJ;
  const long o = iS(g, i, j, k);
  const float *kmh = a.kmh, *kmv = a.kmv;
  if (k <= nk) {
    const float tem = kmh[o] + kmh[o + pl];
    a.t11[o] = a.t11[o] * tem;
    a.t22[o] = a.t22[o] * tem;
    a.t33[o] = a.t33[o] * tem;
    if (i >= 1 && j >= 1) {
      const long omm = iS(g, i - 1, j - 1, k), om0 = iS(g, i - 1, j, k), o0m = iS(g, i, j - 1, k);
      a.t12[o] = a.t12[o] * 0.25f *
                 (((kmh[omm] + kmh[o]) + (kmh[om0] + kmh[o0m])) +
                  ((kmh[omm + pl] + kmh[o + pl]) + (kmh[om0 + pl] + kmh[o0m + pl])));
    }
  }
  if (i < 1 || j < 1) return;
  const long ox = iS(g, i - 1, j, k), oy = iS(g, i, j - 1, k);
  if (k <= nk) {
    // turbs' face coefficients (turbtend.F:68-77): khh = kmh * prinv at the
    // four points, summed as the Fortran does, times -0.125 (rho + rho); the
    // Fortran's left-to-right product forms this factor first
    const float pr = a.prinv;
    a.cx[o] = -0.125f * (a.rho[o] + a.rho[ox]) * ((kmh[o] * pr + kmh[ox] * pr) + (kmh[o + pl] * pr + kmh[ox + pl] * pr));
    a.cy[o] = -0.125f * (a.rho[o] + a.rho[oy]) * ((kmh[o] * pr + kmh[oy] * pr) + (kmh[o + pl] * pr + kmh[oy + pl] * pr));
  }
  if (k >= 2 && k <= nk) {
    a.t13[o] = a.s13[o] * (kmv[ox] + kmv[o]);
    a.t23[o] = a.s23[o] * (kmv[oy] + kmv[o]);
  } else if (k == 1) {
    if (a.bbc == 1) {            // free slip: t13(1) = t13(2)
      a.t13[o] = a.s13[o + pl] * (kmv[ox + pl] + kmv[o + pl]);
      a.t23[o] = a.s23[o + pl] * (kmv[oy + pl] + kmv[o + pl]);
    } else {                     // no slip (turb.F:4550-4562), ugr = ua, vgr = va
      const float rdz = g.rdz, mf = LDG(&g.mf[1]);
      a.t13[o] = 2.0f * a.ua[iU(g, i, j, 1)] * rdz * 0.5f * (mf + mf) * 0.5f *
                 (les_rf(g, a, i - 1, j, 1) + les_rf(g, a, i, j, 1)) * 0.5f * (kmv[ox + pl] + kmv[o + pl]);
      a.t23[o] = 2.0f * a.va[iV(g, i, j, 1)] * rdz * 0.5f * (mf + mf) * 0.5f *
                 (les_rf(g, a, i, j - 1, 1) + les_rf(g, a, i, j, 1)) * 0.5f * (kmv[oy + pl] + kmv[o + pl]);
    }
  } else {
    if (a.tbc == 1) {            // free slip: t13(nk+1) = t13(nk)
      a.t13[o] = a.s13[o - pl] * (kmv[ox - pl] + kmv[o - pl]);
      a.t23[o] = a.s23[o - pl] * (kmv[oy - pl] + kmv[o - pl]);
    } else {                     // no slip (turb.F:4407-4419)
      const float rdz = g.rdz, mf = LDG(&g.mf[nk + 1]);
      a.t13[o] = -(2.0f * a.ua[iU(g, i, j, nk)] * rdz * 0.5f * (mf + mf) * 0.5f *
                   (les_rf(g, a, i - 1, j, nk + 1) + les_rf(g, a, i, j, nk + 1)) * 0.5f * (kmv[ox - pl] + kmv[o - pl]));
      a.t23[o] = -(2.0f * a.va[iV(g, i, j, nk)] * rdz * 0.5f * (mf + mf) * 0.5f *
                   (les_rf(g, a, i, j - 1, nk + 1) + les_rf(g, a, i, j, nk + 1)) * 0.5f * (kmv[oy - pl] + kmv[o - pl]));
    }
  }
}

// scalar value as turbs sees it: theta minus th0r plus th0 (solve1.F:1184-1195)
__device__ __forceinline__ float les_s(const DGrid &g, const float *s, bool th, int i, int j, int k) {
  const float v = s[iS(g, i, j, k)];
  return th ? (LDG(&g.th0[k]) - 300.0f) + v : v;
}

// x/y flux dumx, dumy of turbs (turbtend.F:66-78): the face coefficient
// times the difference, rdx and the metric, in the Fortran's order
__device__ __forceinline__ float les_sfx(const DGrid &g, const TurbArgs &a, const float *s, bool th, int i, int j, int k,
                                         bool ydir) {
  const int im = ydir ? i : i - 1, jm = ydir ? j - 1 : j;
  const long o = iS(g, i, j, k);
  const float met = ydir ? LDG(&g.vf[j - g.jb]) : LDG(&g.uf[i - g.ib]);
  return (ydir ? a.cy[o] : a.cx[o]) * (les_s(g, s, th, i, j, k) - les_s(g, s, th, im, jm, k)) * (ydir ? g.rdy : g.rdx) *
         met;
}

// vertical flux dumz of turbsz, explicit (turbtend.F:480-510)
__device__ __forceinline__ float les_sfz(const DGrid &g, const TurbArgs &a, const float *s, bool th, int i, int j, int k) {
  const int nk = g.nk;
  if (k == 1 || k == nk + 1) {
    if (a.bcturbs == 1) return 0.0f;
    k = (k == 1) ? 2 : nk;
  }
  const float khv = a.kmv[iS(g, i, j, k)] * a.prinv;
  return -khv * (les_s(g, s, th, i, j, k) - les_s(g, s, th, i, j, k - 1)) * g.rdz * LDG(&g.mf[k]) *
         les_rf(g, a, i, j, k);
}

// tendencies: blockIdx.z < nk for momentum level k; then one z per (scalar, k)
__global__ void k_les_tend(DGrid g, TurbArgs a) {
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);   // 1 .. ni+1
  const int j = 1 + (int)blockIdx.y;                                // 1 .. nj+1
  const int nk = g.nk;
  const int z = (int)blockIdx.z;
  const int k = 1 + z % nk, f = z / nk;
  if (i > g.ni + 1) return;
  const float rdx = g.rdx, rdy = g.rdy, rdz = g.rdz;
  const long pl = (long)g.NI * g.NJ;
  const long o = iS(g, i, j, k);
  if (f == 0) {
    const float tem = rdz * 0.5f;
    if (j <= g.nj) {   // turbu (turbtend.F:1101-1104, 1290-1296; turbuz 1408-1416)
      const float tx = (a.t11[o] - a.t11[iS(g, i - 1, j, k)]) * rdx * LDG(&g.uf[i - g.ib]);
      const float ty = (a.t12[iS(g, i, j + 1, k)] - a.t12[o]) * rdy * LDG(&g.vh[j - g.jb]);
      const float tz = (a.t13[o + pl] - a.t13[o]) * tem * (LDG(&g.mh[k]) + LDG(&g.mh[k]));
      const float rru0 = 1.0f / (0.5f * (a.rho[iS(g, i - 1, j, k)] + a.rho[o]));
      const long ou = iU(g, i, j, k);
      a.uten[ou] = a.uten[ou] + ((tx + ty) + tz) * rru0;
    }
    if (i <= g.ni) {   // turbv
      const float tx = (a.t12[iS(g, i + 1, j, k)] - a.t12[o]) * rdx * LDG(&g.uh[i - g.ib]);
      const float ty = (a.t22[o] - a.t22[iS(g, i, j - 1, k)]) * rdy * LDG(&g.vf[j - g.jb]);
      const float tz = (a.t23[o + pl] - a.t23[o]) * tem * (LDG(&g.mh[k]) + LDG(&g.mh[k]));
      const float rrv0 = 1.0f / (0.5f * (a.rho[iS(g, i, j - 1, k)] + a.rho[o]));
      const long ov = iV(g, i, j, k);
      a.vten[ov] = a.vten[ov] + ((tx + ty) + tz) * rrv0;
    }
    if (i <= g.ni && j <= g.nj && k >= 2) {   // turbw
      const float tx = (a.t13[iS(g, i + 1, j, k)] - a.t13[o]) * rdx * LDG(&g.uh[i - g.ib]);
      const float ty = (a.t23[iS(g, i, j + 1, k)] - a.t23[o]) * rdy * LDG(&g.vh[j - g.jb]);
      const float tz = (a.t33[o] - a.t33[o - pl]) * rdz * LDG(&g.mf[k]);
      const long ow = iW(g, i, j, k);
      a.wten[ow] = a.wten[ow] + ((tx + ty) + tz) / les_rf(g, a, i, j, k);
    }
    return;
  }
  if (i > g.ni || j > g.nj) return;
  // turbs: field f-1 (theta, then q, then tracers)
  const int n = f - 1;
  const long ns = (long)pl * g.NK;
  const bool th = n == 0;
  const float *s = th ? a.tha : (n <= a.numq ? a.qa + (n - 1) * ns : a.pta + (n - 1 - a.numq) * ns);
  float *sten = th ? a.thten : (n <= a.numq ? a.qten + (n - 1) * ns : a.ptten + (n - 1 - a.numq) * ns);
  const float tx = -(les_sfx(g, a, s, th, i + 1, j, k, false) - les_sfx(g, a, s, th, i, j, k, false)) * rdx *
                   LDG(&g.uh[i - g.ib]);
  const float ty = -(les_sfx(g, a, s, th, i, j + 1, k, true) - les_sfx(g, a, s, th, i, j, k, true)) * rdy *
                   LDG(&g.vh[j - g.jb]);
  const float tz = -(les_sfz(g, a, s, th, i, j, k + 1) - les_sfz(g, a, s, th, i, j, k)) * rdz * LDG(&g.mh[k]);
  const float rr = 1.0f / a.rho[o];
  sten[o] = sten[o] + ((tx + ty) + tz) * rr;
}

void launch_turbsmag(const DGrid &g, const TurbArgs &a, cudaStream_t st, int64_t *nl) {
  // one row of 128 points per block (32 x 8 blocks measured no faster)
  const int bx = 128;
  {
    dim3 grid((g.ni + 2 + bx - 1) / bx, g.nj + 2, g.nk);
    ProfScope _ps("k_les_strain", st);
    k_les_strain<<<grid, bx, 0, st>>>(g, a);
  }
  {
    dim3 grid((g.ni + 2 + bx - 1) / bx, g.nj + 2, g.nk + 1);
    ProfScope _ps("k_les_km", st);
    k_les_km<<<grid, bx, 0, st>>>(g, a);
  }
  {
    dim3 grid((g.ni + 2 + bx - 1) / bx, g.nj + 2, g.nk + 1);
    ProfScope _ps("k_les_stress", st);
    k_les_stress<<<grid, bx, 0, st>>>(g, a);
  }
  {
    const int nf = 1 + (a.thten ? 1 + a.numq + a.npt : 0);
    dim3 grid((g.ni + 1 + bx - 1) / bx, g.nj + 1, g.nk * nf);
    ProfScope _ps("k_les_tend", st);
    k_les_tend<<<grid, bx, 0, st>>>(g, a);
  }
  if (nl) *nl += 4;
}

}  // namespace cm1g
