// cm1g_common.cuh -- device-side grid descriptor, Fortran-layout indexing and
// the face-value functions shared by the large-step kernels.
//
// All fields use the reference's Fortran layout (i fastest) with lower
// bounds ib=1-ngxy, jb=1-ngxy, kb=0.  Without terrain the base state and the
// vertical metrics are horizontally uniform, so the kernels read them as
// 1-D profiles indexed by k (checked when the context is created).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cm1g {

struct Consts {
  float g, rd, rv, cp, cv, cpv, cvv, cpl, cpi;
  float rovcp, rddcv, cpdrd, reps, repsm1;
};

// Everything a kernel needs to know about the grid; passed by value.
struct DGrid {
  int ni, nj, nk, ngxy;
  int ib, jb;                 // kb = 0
  int NI, NJ, NK;             // extents of s-arrays
  float dx, dy, dz, rdx, rdy, rdz;
  int wbc, ebc, sbc, nbc;
  int ibw, ibe, ibs, ibn;
  float smeps, alph, kdiv;
  int irbc;                   // open-boundary phase speeds: 1 and 2 Klemp-Wilhelmson, 4 Durran-Klemp
  float cstar;                // the Klemp-Wilhelmson gravity-wave speed of irbc 1 and 2
  int roflux;                 // 1: the open boundaries' outflow is restricted to the inflow at every acoustic step
  Consts c;
  // vertical profiles (index k, k = 0..nk+1; w-profiles to nk+2)
  const float *mh, *rmh, *mf, *rho0, *rr0, *rf0, *rrf0, *c1, *c2, *pi0, *th0, *rth0, *qv0, *qc0, *qi0;
  const float *prs0;          // base-state pressure profile (output only; null when not given)
  // horizontal metrics (index i-ib / j-jb)
  const float *uh, *ruh, *uf, *ruf, *vh, *rvh, *vf, *rvf;
  const float *dtu0, *dtv0;   // (ib:ie, jb:je)
  const float *u0, *v0;       // base-state winds, full u-/v-arrays (Rayleigh damping)
  // launch shapes (cm1g_set_tune / cm1g_autotune): index into the tile-shape
  // table of the scalar and momentum passes, and the acoustic kernel's form
  // (-1: chosen by the number of columns)
  int tile_adv, tile_mom, sound_cfg;
};

// Tile shapes of the scalar and momentum passes: x and y extent of a block
// (threads) and the levels one block marches through (z).  Entry 0 is the
// default; the others are the autotuner's candidates.
constexpr int kNumTileShapes = 5;
constexpr int kTileShapes[kNumTileShapes][3] = {{32, 8, 16}, {32, 8, 8}, {32, 4, 16}, {64, 4, 16}, {32, 8, 32}};
// Tile shapes of the scalar passes (k_scal_tile, k_advs_tile), indexed like
// kTileShapes: TX x TY cells and KC levels per block; the block has one more
// row of TX threads than the tile has cell rows (the row that evaluates the
// tile's north and east faces), so a block is TX x (TY + 1) threads.
constexpr int kScalShapes[kNumTileShapes][3] = {{32, 7, 16}, {32, 7, 8}, {32, 3, 16}, {64, 3, 16}, {32, 7, 32}};
// Forms of the acoustic kernel: 0 tile (32 columns x 8 warps over the
// levels), 1 tile with 4 warps, 2 column sweep 32 x 4 columns, 3 column
// sweep 32 x 2 columns.
constexpr int kNumSoundCfgs = 4;

// Fortran-layout offsets.  s and w arrays share the plane (NI*NJ); u arrays
// have NI+1 points in x, v arrays NJ+1 rows.
__host__ __device__ __forceinline__ long iS(const DGrid &g, int i, int j, int k) {
  return (long)(i - g.ib) + (long)g.NI * ((long)(j - g.jb) + (long)g.NJ * (long)k);
}
__host__ __device__ __forceinline__ long iW(const DGrid &g, int i, int j, int k) { return iS(g, i, j, k); }
__host__ __device__ __forceinline__ long iU(const DGrid &g, int i, int j, int k) {
  return (long)(i - g.ib) + (long)(g.NI + 1) * ((long)(j - g.jb) + (long)g.NJ * (long)k);
}
__host__ __device__ __forceinline__ long iV(const DGrid &g, int i, int j, int k) {
  return (long)(i - g.ib) + (long)g.NI * ((long)(j - g.jb) + (long)(g.NJ + 1) * (long)k);
}
__host__ __device__ __forceinline__ long i2(const DGrid &g, int i, int j) {
  return (long)(i - g.ib) + (long)g.NI * (long)(j - g.jb);
}
__host__ __device__ __forceinline__ long nS(const DGrid &g) { return (long)g.NI * g.NJ * g.NK; }
__host__ __device__ __forceinline__ long nU(const DGrid &g) { return (long)(g.NI + 1) * g.NJ * g.NK; }
__host__ __device__ __forceinline__ long nV(const DGrid &g) { return (long)g.NI * (g.NJ + 1) * g.NK; }
__host__ __device__ __forceinline__ long nW(const DGrid &g) { return (long)g.NI * g.NJ * (g.NK + 1); }

#define LDG(p) __ldg(p)

// ---------------------------------------------------------------------
// Face values (binary32 arithmetic in the reference's evaluation order;
// adv_routines.F:5971-6205, 6331-6355).  The library is compiled with
// --fmad=false so that each product and sum rounds as the Fortran does.
// ---------------------------------------------------------------------
__device__ __forceinline__ float flx3(float s1, float s2, float s3) {
  return ((-1.0f / 6.0f) * s1 + (5.0f / 6.0f) * s2) + (2.0f / 6.0f) * s3;
}
__device__ __forceinline__ float flx5(float s1, float s2, float s3, float s4, float s5) {
  return ((((2.0f / 60.0f) * s1 + (-13.0f / 60.0f) * s2) + (47.0f / 60.0f) * s3) +
          (27.0f / 60.0f) * s4) + (-3.0f / 60.0f) * s5;
}

// WENO5 with Borges et al. (2008) weights.  Smoothness indicators in
// binary32 (as the Fortran evaluates them), weights and quotient in binary64.
//
// The reference (adv_routines.F:6166-6205) forms each weight with its own
// binary64 division, w_i = c_i (1 + min(1e30, tau/(b_i+weps))^2), and the
// face value as (w1 q1 + w2 q2 + w3 q3)/(w1 + w2 + w3) rounded to binary32.
// The fast path folds the three divisions into one over the common
// denominator d1^2 d2^2 d3^2.  Both binary64 results lie within 17 units of
// the last binary64 place, times max|q_i|, of the exact weighted average, so
// they differ by less than 2^-46 max|q_i|; when the folded value is farther
// than that from both ends of the rounding interval of its binary32 result,
// the reference's value rounds to the same binary32 number.  Otherwise (about
// one face in a million) the face is evaluated exactly as the reference
// does, so the result is always the reference's binary32 value.
static __device__ __noinline__ float weno5_ref(double b1, double b2, double b3, float q1, float q2, float q3,
                                               double weps) {
  const double tau = fabs(b1 - b3);
  double r;
  r = fmin(1.0e30, tau / (b1 + weps)); double w1 = (double)0.1f * (1.0 + r * r);
  r = fmin(1.0e30, tau / (b2 + weps)); double w2 = (double)0.6f * (1.0 + r * r);
  r = fmin(1.0e30, tau / (b3 + weps)); double w3 = (double)0.3f * (1.0 + r * r);
  double num = (w1 * (double)q1 + w2 * (double)q2) + w3 * (double)q3;
  double den = (w1 + w2) + w3;
  return (float)(num / den);
}
__device__ __forceinline__ float weno5(float s1, float s2, float s3, float s4, float s5, double weps) {
  const float c1312 = 13.0f / 12.0f;
  float t, u;
  t = (s1 - 2.0f * s2) + s3; u = (s1 - 4.0f * s2) + 3.0f * s3;
  double b1 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  t = (s2 - 2.0f * s3) + s4; u = s2 - s4;
  double b2 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  t = (s3 - 2.0f * s4) + s5; u = (3.0f * s3 - 4.0f * s4) + s5;
  double b3 = (double)(c1312 * (t * t) + 0.25f * (u * u));
  float q1 = ((2.0f / 6.0f) * s1 + (-7.0f / 6.0f) * s2) + (11.0f / 6.0f) * s3;
  float q2 = ((-1.0f / 6.0f) * s2 + (5.0f / 6.0f) * s3) + (2.0f / 6.0f) * s4;
  float q3 = ((2.0f / 6.0f) * s3 + (5.0f / 6.0f) * s4) + (-1.0f / 6.0f) * s5;
  double tau = fabs(b1 - b3);
  double d1 = b1 + weps, d2 = b2 + weps, d3 = b3 + weps;
  double tt = tau * tau;
  if (tau < 1.0e30 * d1 && tau < 1.0e30 * d2 && tau < 1.0e30 * d3) {
    double e1 = d1 * d1, e2 = d2 * d2, e3 = d3 * d3;
    double a1 = (double)0.1f * (e1 + tt) * (e2 * e3);
    double a2 = (double)0.6f * (e2 + tt) * (e1 * e3);
    double a3 = (double)0.3f * (e3 + tt) * (e1 * e2);
    double num = (a1 * (double)q1 + a2 * (double)q2) + a3 * (double)q3;
    double den = (a1 + a2) + a3;
    const double v = num / den;
    const float f = (float)v;
    const float qm = fmaxf(fmaxf(fabsf(q1), fabsf(q2)), fabsf(q3));
    if (qm == 0.0f) return 0.0f;   // q1 = q2 = q3 = 0: both forms give exactly 0
    // e = v - f is exact (Sterbenz); f's rounding interval reaches h = 2^(E-24)
    // on each side (E = the binary exponent of f), h/2 toward zero when f is a
    // power of two; v's binary32 rounding is safe when |e| + delta < h.
    const double fd = (double)f;
    const double e = v - fd;
    double h = __hiloint2double(__double2hiint(fd) & 0x7ff00000, 0) * 5.9604644775390625e-08;   // 2^-24
    if ((__float_as_int(f) & 0x7fffff) == 0) h = 0.5 * h;
    const double delta = (double)qm * 1.4210854715202004e-14;   // 2^-46
    if (fabs(e) + delta < h) return f;
  }
  return weno5_ref(b1, b2, b3, q1, q2, q3, weps);
}

__device__ __forceinline__ float upstrpd(float s1, float s2, float s3, double weps) {
  float dd = s2 - s1;
  float rr = (s3 - s2) / (copysignf((float)weps, dd) + dd);
  float phi = fmaxf(0.0f, fminf(rr, fminf((1.0f / 6.0f) + (2.0f / 6.0f) * rr, 1.0f)));
  return s2 + phi * (s2 - s1);
}

__device__ __forceinline__ float absmax5(float a, float b, float c, float d, float e) {
  return fmaxf(fmaxf(fmaxf(fmaxf(fabsf(a), fabsf(b)), fabsf(c)), fabsf(d)), fabsf(e));
}

// Optional extras of the scalar tile (k_advs_tile, update mode):
//  phix/phiy  learned face values of the horizontal faces (NaN: use WENO5),
//             indexed f = (k-1)*nfx*nfy + (j-1)*nfx + (i-1) with
//             nfx x nfy = (ni+1) x nj for x-faces and ni x (nj+1) for y-faces;
//  cap*       capture of the x/y face fluxes and face mass fluxes the
//             kernel used (u-/v-array layout), for building training targets.
struct TileExtras {
  const float *phix = nullptr, *phiy = nullptr;
  float *capfx = nullptr, *capfy = nullptr, *caprx = nullptr, *capry = nullptr;
};

// 6th-order horizontal diffusion inside the advection passes (idiff=1,
// difforder=6; adv.F:342-406, 1177-1236, 2115-2174, 3109-3170).  rho null:
// no diffusion.  ri is 1/rho as the scalar form uses it (rr of solve2; it
// may lag rho by one stage), coef = kdiff6/64/dt, mdiff the limiter.
struct Diff6 {
  const float *rho = nullptr, *ri = nullptr;
  float coef = 0.0f;
  int mdiff = 0;
};

// The difference stencil of a face between a(-1) and a(0), as the Fortran
// evaluates it: (10 (a0 - am1) - 5 (ap1 - am2)) + (ap2 - am3).
__device__ __forceinline__ float diff6_stencil(float am3, float am2, float am1, float a0, float ap1, float ap2) {
  return (10.0f * (a0 - am1) - 5.0f * (ap1 - am2)) + (ap2 - am3);
}
// the mdiff limiter: no flux against the local gradient
__device__ __forceinline__ float diff6_limit(float f, float a0, float am1, int mdiff) {
  return (mdiff == 1 && f * (a0 - am1) <= 0.0f) ? 0.0f : f;
}

// One advected field of the fused scalar pass of an RK stage (k_scal.cu).
struct ScalField {
  const float *s;               // stage input (full halo)
  const float *sbase;           // RK base value (tha, qa, pta)
  const float *ten1;            // fixed tendency (thten1, qten, ptten)
  float *snew;                  // stage output
  double weps;                  // WENO epsilon of the field (solve2.F:1391, 1472-1514, 1941)
  int sadd;                     // theta: advect th0(k) - 300 + s (solve2.F:1365-1372)
  int flush;                    // |snew| < smeps -> 0 (theta and moisture)
  int pdefweno;                 // pdef form of the vertical WENO (adv_routines.F:2386-2421)
};

// Liquid water of the stage set-up (ptype=1): the RK-stage input of each
// liquid species (at most two: Kessler's qc, qr) and the buoyancy array
// that the stage set-up writes for the w tendency (null without liquid).
struct LiquidIn {
  const float *q[2] = {nullptr, nullptr};
  int n = 0;
  float *b8 = nullptr;
};

// Inputs of the solve1 tendency initialisation and of calcener (k_misc.cu).
struct TendIn {
  int irdamp;
  float rdalpha;
  const float *tauh, *taus, *tauf, *uavg, *vavg, *thavg, *ua, *va, *wa, *tha;
  float *uten1, *vten1, *wten1, *thten1, *qten, *ptten;
  int nq;     // moisture + tracer arrays to zero (qten first, then ptten)
  int numq;
};
struct EnerIn {
  const float *zh, *rho, *ua, *va, *wa, *ppi, *tha, *qv, *ql, *qi, *vr;
  float lv1, ls1;
};

// Records a message for cm1g_last_error() and returns code (C++ linkage,
// not part of the C-ABI).
int report_error(int code, const char *msg);

// Per-kernel device timing (the library's counterpart of the reference's
// timestats, input.F:359-387).  When a profile is active every kernel launch
// site brackets its launch with a pair of CUDA events on the launch stream;
// the elapsed times are summed per kernel name when the profile is read.
struct Profile;
extern thread_local Profile *g_profile;
void prof_record(const char *name, cudaStream_t st, bool begin);

struct ProfScope {
  const char *name;
  cudaStream_t st;
  ProfScope(const char *n, cudaStream_t s) : name(n), st(s) { if (g_profile) prof_record(name, st, true); }
  ~ProfScope() { if (g_profile) prof_record(name, st, false); }
};

}  // namespace cm1g
