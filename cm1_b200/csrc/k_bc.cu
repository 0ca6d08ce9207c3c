// k_bc.cu -- lateral halo fills of bc.F run in-domain on the device.
//
// The reference fills west/east halos first and then copies whole
// south/north rows (bcs, bcp, bcu, bcw; bc.F:180-523, 528-717, 942-1146),
// except bcv which does south/north first (bc.F:722-937).  Each direction is
// one kernel phase here so the corner values come out exactly as the serial
// loop order leaves them.  Every phase reads only points the same phase does
// not write, so its threads need no ordering among themselves.
#include "cm1g_common.cuh"

namespace cm1g {

enum Stag { STAG_S = 1, STAG_U = 2, STAG_V = 3, STAG_W = 4 };
static const int BC_MAXB = 16;

__device__ __forceinline__ long idxStag(const DGrid &g, int stag, int i, int j, int k) {
  return stag == STAG_U ? iU(g, i, j, k) : stag == STAG_V ? iV(g, i, j, k) : iS(g, i, j, k);
}

// West/east fills of row j, level k (j over the widest range any branch
// uses, jb..je+1).
__device__ __forceinline__ void bc_x_row(const DGrid &g, float *__restrict__ a, int stag, int pmode, int j, int k) {
  const int ni = g.ni, nj = g.nj, ng = g.ngxy;
  const int jeS = nj + ng + (stag == STAG_V ? 1 : 0);  // je or je+1
  if (j > jeS) return;
  if (pmode) {  // bcp: width 1, rows 0..nj+1 (bc.F:380-440)
    if (j < 0 || j > nj + 1) return;
    if (g.wbc == 1) a[iS(g, 0, j, k)] = a[iS(g, ni, j, k)];
    else if (g.wbc >= 2 && g.wbc <= 4) a[iS(g, 0, j, k)] = a[iS(g, 1, j, k)];
    if (g.ebc == 1) a[iS(g, ni + 1, j, k)] = a[iS(g, 1, j, k)];
    else if (g.ebc >= 2 && g.ebc <= 4) a[iS(g, ni + 1, j, k)] = a[iS(g, ni, j, k)];
    return;
  }
  const int jlo2 = 0, jhi2 = (stag == STAG_V) ? nj + 2 : nj + 1;  // open / wall row range
  // ---- west
  if (g.wbc == 1) {
    for (int h = 1; h <= ng; h++) a[idxStag(g, stag, 1 - h, j, k)] = a[idxStag(g, stag, ni + 1 - h, j, k)];
  } else if (j >= jlo2 && j <= jhi2) {
    if (g.wbc == 2) {
      float v = a[idxStag(g, stag, 1, j, k)];
      for (int i = 1 - ng; i <= 0; i++) a[idxStag(g, stag, i, j, k)] = v;
    } else if (g.wbc == 3 || g.wbc == 4) {
      if (stag == STAG_U) {
        a[iU(g, 1, j, k)] = 0.0f;
        for (int h = 1; h <= ng; h++) a[iU(g, 1 - h, j, k)] = -a[iU(g, 1 + h, j, k)];
      } else {
        for (int h = 1; h <= ng; h++) a[idxStag(g, stag, 1 - h, j, k)] = a[idxStag(g, stag, h, j, k)];
      }
    }
  }
  // ---- east
  if (g.ebc == 1) {
    if (stag == STAG_U)
      for (int h = 1; h <= ng; h++) a[iU(g, ni + 1 + h, j, k)] = a[iU(g, 1 + h, j, k)];
    else
      for (int h = 1; h <= ng; h++) a[idxStag(g, stag, ni + h, j, k)] = a[idxStag(g, stag, h, j, k)];
  } else if (j >= jlo2 && j <= jhi2) {
    if (g.ebc == 2) {
      if (stag == STAG_U) {
        float v = a[iU(g, ni + 1, j, k)];
        for (int i = ni + 2; i <= ni + 1 + ng; i++) a[iU(g, i, j, k)] = v;
      } else {
        float v = a[idxStag(g, stag, ni, j, k)];
        for (int i = ni + 1; i <= ni + ng; i++) a[idxStag(g, stag, i, j, k)] = v;
      }
    } else if (g.ebc == 3 || g.ebc == 4) {
      if (stag == STAG_U) {
        a[iU(g, ni + 1, j, k)] = 0.0f;
        for (int h = 1; h <= ng; h++) a[iU(g, ni + 1 + h, j, k)] = -a[iU(g, ni + 1 - h, j, k)];
      } else {
        for (int h = 1; h <= ng; h++) a[idxStag(g, stag, ni + h, j, k)] = a[idxStag(g, stag, ni + 1 - h, j, k)];
      }
    }
  }
}

// South/north fills of column i, plane kp (and w's top/bottom zeros).  i runs
// over ib..ie+1; kp = 0.. covers k = 1..nk (w: k = 2..nk, then one extra plane
// for the top/bottom zeros of bcw(flag=1)).
__device__ __forceinline__ void bc_y_col(const DGrid &g, float *__restrict__ a, int stag, int pmode, int wflag, int i,
                                         int kp) {
  const int ni = g.ni, nj = g.nj, nk = g.nk, ng = g.ngxy;
  const int ieS = ni + ng + (stag == STAG_U ? 1 : 0);
  if (i > ieS) return;
  if (stag == STAG_W && kp == nk - 1) {  // extra plane: bc.F:1127-1137
    if (wflag == 1 && i >= 0 && i <= ni + 1)
      for (int j = 0; j <= nj + 1; j++) { a[iW(g, i, j, 1)] = 0.0f; a[iW(g, i, j, nk + 1)] = 0.0f; }
    return;
  }
  const int k = kp + (stag == STAG_W ? 2 : 1);
  if (pmode) {  // bcp rows (bc.F:458-518)
    if (i < 0 || i > ni + 1) return;
    if (g.sbc == 1) a[iS(g, i, 0, k)] = a[iS(g, i, nj, k)];
    else if (g.sbc >= 2 && g.sbc <= 4) a[iS(g, i, 0, k)] = a[iS(g, i, 1, k)];
    if (g.nbc == 1) a[iS(g, i, nj + 1, k)] = a[iS(g, i, 1, k)];
    else if (g.nbc >= 2 && g.nbc <= 4) a[iS(g, i, nj + 1, k)] = a[iS(g, i, nj, k)];
    return;
  }
  const int ilo2 = 0, ihi2 = (stag == STAG_U) ? ni + 2 : ni + 1;
  // ---- south
  if (g.sbc == 1) {
    if (stag == STAG_V)
      for (int h = 1; h <= ng; h++) a[iV(g, i, 1 - h, k)] = a[iV(g, i, nj + 1 - h, k)];
    else
      for (int h = 1; h <= ng; h++) a[idxStag(g, stag, i, 1 - h, k)] = a[idxStag(g, stag, i, nj + 1 - h, k)];
  } else if (i >= ilo2 && i <= ihi2) {
    if (g.sbc == 2) {
      float v = a[idxStag(g, stag, i, 1, k)];
      for (int j = 1 - ng; j <= 0; j++) a[idxStag(g, stag, i, j, k)] = v;
    } else if (g.sbc == 3 || g.sbc == 4) {
      if (stag == STAG_V) {
        for (int h = 1; h <= ng; h++) a[iV(g, i, 1 - h, k)] = -a[iV(g, i, h + 1, k)];
        a[iV(g, i, 1, k)] = 0.0f;
      } else {
        for (int h = 1; h <= ng; h++) a[idxStag(g, stag, i, 1 - h, k)] = a[idxStag(g, stag, i, h, k)];
      }
    }
  }
  // ---- north
  if (g.nbc == 1) {
    if (stag == STAG_V)
      for (int h = 1; h <= ng; h++) a[iV(g, i, nj + 1 + h, k)] = a[iV(g, i, 1 + h, k)];
    else
      for (int h = 1; h <= ng; h++) a[idxStag(g, stag, i, nj + h, k)] = a[idxStag(g, stag, i, h, k)];
  } else if (i >= ilo2 && i <= ihi2) {
    if (g.nbc == 2) {
      if (stag == STAG_V) {
        float v = a[iV(g, i, nj + 1, k)];
        for (int j = nj + 2; j <= nj + 1 + ng; j++) a[iV(g, i, j, k)] = v;
      } else {
        float v = a[idxStag(g, stag, i, nj, k)];
        for (int j = nj + 1; j <= nj + ng; j++) a[idxStag(g, stag, i, j, k)] = v;
      }
    } else if (g.nbc == 3 || g.nbc == 4) {
      if (stag == STAG_V) {
        for (int h = 1; h <= ng; h++) a[iV(g, i, nj + 1 + h, k)] = -a[iV(g, i, nj + 1 - h, k)];
        a[iV(g, i, nj + 1, k)] = 0.0f;
      } else {
        for (int h = 1; h <= ng; h++) a[idxStag(g, stag, i, nj + h, k)] = a[idxStag(g, stag, i, nj + 1 - h, k)];
      }
    }
  }
}

// One launch runs one phase for up to BC_MAXB arrays: blockIdx.z picks the
// array, and the array's own order decides whether this phase is its x or y
// fill (bcv fills south/north first).  Arrays in a batch must be distinct.
struct BcBatch {
  float *a[BC_MAXB];
  int stag[BC_MAXB], pmode[BC_MAXB], wflag[BC_MAXB];
  int n;
};

__global__ void k_bc_phase(DGrid g, BcBatch b, int phase) {
  const int n = (int)blockIdx.z;
  const int stag = b.stag[n];
  const bool yfirst = (stag == STAG_V);
  const bool doy = (phase == 0) ? yfirst : !yfirst;
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x), kp = (int)blockIdx.y;
  const int nkk = (stag == STAG_W) ? g.nk - 1 : g.nk;
  if (doy) {
    if (kp > nkk - (stag == STAG_W ? 0 : 1)) return;
    bc_y_col(g, b.a[n], stag, b.pmode[n], b.wflag[n], g.ib + t, kp);
  } else {
    if (kp >= nkk) return;
    bc_x_row(g, b.a[n], stag, b.pmode[n], g.jb + t, kp + (stag == STAG_W ? 2 : 1));
  }
}

static int bc_stag(int which) { return which == 3 ? STAG_U : which == 4 ? STAG_V : which == 5 ? STAG_W : STAG_S; }

// which = 1 bcs, 2 bcp, 3 bcu, 4 bcv, 5 bcw, for each array of the list.
void launch_bc_batch(const DGrid &g, float *const *arrays, const int *which, const int *wflag, int n,
                     cudaStream_t st, int64_t *nlaunch) {
  for (int base = 0; base < n; base += BC_MAXB) {
    BcBatch b{};
    b.n = (n - base < BC_MAXB) ? n - base : BC_MAXB;
    for (int q = 0; q < b.n; q++) {
      b.a[q] = arrays[base + q];
      b.stag[q] = bc_stag(which[base + q]);
      b.pmode[q] = (which[base + q] == 2);
      b.wflag[q] = wflag ? wflag[base + q] : 0;
    }
    dim3 blk(128);
    const int span = (g.NI > g.NJ ? g.NI : g.NJ) + 1;
    dim3 grid((span + 127) / 128, g.nk, b.n);
    { ProfScope _ps("k_bc_phase", st); k_bc_phase<<<grid, blk, 0, st>>>(g, b, 0); }
    { ProfScope _ps("k_bc_phase", st); k_bc_phase<<<grid, blk, 0, st>>>(g, b, 1); }
    if (nlaunch) *nlaunch += 2;
  }
}

void launch_bc(const DGrid &g, float *a, int which, int wflag, cudaStream_t st, int64_t *nlaunch) {
  launch_bc_batch(g, &a, &which, &wflag, 1, st, nlaunch);
}

}  // namespace cm1g
