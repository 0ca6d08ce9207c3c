// k_face.cuh -- face values of the scalar passes (hflux5, zflux_win) and the
// spread of a tile's faces over its threads (FaceSlots), shared by the
// per-scalar tile (k_adv.cu) and the fused multi-scalar pass (k_scal.cu) so
// that both evaluate every face with the same binary32/binary64 operations.
#pragma once
#include "cm1g_common.cuh"

namespace cm1g {

// Face loop of the tiles: each thread owns face `tid` of each direction
// (none where tid is past the level's faces), and the faces past one per
// thread (NFX - NT x-faces, NFY - NT y-faces, when a level has more faces
// than the block has threads) go to the threads from warp 1 (x) and the
// warps after those (y), so that the second pass of the loop is spread over
// other warps than the first.  A block with one thread row more than the
// tile has cell rows has at most one face of each direction per thread.
template <int NT, int NFX, int NFY>
struct FaceSlots {
  static constexpr int EX = NFX > NT ? NFX - NT : 0, EY = NFY > NT ? NFY - NT : 0;
  static constexpr int X1 = 32;
  static constexpr int Y1 = 32 * (1 + (EX + 31) / 32);
  static_assert(X1 + EX <= NT && Y1 + EY <= NT, "the extra faces fit the block");
  // face index of slot q (0 or 1) of thread tid; >= NFX / NFY: none
  __device__ static __forceinline__ int x(int tid, int q) {
    return q == 0 ? (tid < NFX ? tid : NFX) : ((tid >= X1 && tid < X1 + EX) ? NT + tid - X1 : NFX);
  }
  __device__ static __forceinline__ int y(int tid, int q) {
    return q == 0 ? (tid < NFY ? tid : NFY) : ((tid >= Y1 && tid < Y1 + EY) ? NT + tid - Y1 : NFY);
  }
};

// vertical face flux at level kk from wv[d+3] = s(kk+d), d = -3..2, with the
// interpolation weights c1(kk), c2(kk) of the 2nd-order pieces given
__device__ __forceinline__ float zflux_core(const float *wv, float r, int kk, int nk, float c1k, float c2k, int weno,
                                            int pdefweno, double weps) {
  auto A = [&](int d) { return wv[d + 3]; };
  if (!weno) {
    if (kk >= 4 && kk <= nk - 2) {
      const bool up = (r >= 0.0f);
      return r * flx5(up ? A(-3) : A(2), up ? A(-2) : A(1), up ? A(-1) : A(0), up ? A(0) : A(-1), up ? A(1) : A(-2));
    }
    if (kk == 2) {
      if (r >= 0.0f) return r * (c1k * A(-1) + c2k * A(0));
      return r * flx3(A(1), A(0), A(-1));
    }
    if (kk == nk) {
      if (r >= 0.0f) return r * flx3(A(-2), A(-1), A(0));
      return r * (c1k * A(-1) + c2k * A(0));
    }
    if (kk == 3) {
      if (r >= 0.0f) return r * flx3(A(-2), A(-1), A(0));
      return r * flx5(A(2), A(1), A(0), A(-1), A(-2));
    }
    if (r >= 0.0f) return r * flx5(A(-3), A(-2), A(-1), A(0), A(1));
    return r * flx3(A(1), A(0), A(-1));
  }
  if (kk == 2) {
    if (r >= 0.0f) return r * (c1k * A(-1) + c2k * A(0));
    return r * upstrpd(A(1), A(0), A(-1), weps);
  }
  if (kk == nk) {
    if (r > 0.0f) return r * upstrpd(A(-2), A(-1), A(0), weps);
    return r * (c1k * A(-1) + c2k * A(0));
  }
  if (pdefweno == 1) {
    if (kk == 3 && r > 0.0f) return r * upstrpd(A(-2), A(-1), A(0), weps);
    if (kk == nk - 1 && r < 0.0f) return r * upstrpd(A(1), A(0), A(-1), weps);
    float s1, s2, s3, s4, s5;
    if (r >= 0.0f) { s1 = A(-3); s2 = A(-2); s3 = A(-1); s4 = A(0); s5 = A(1); }
    else { s1 = A(2); s2 = A(1); s3 = A(0); s4 = A(-1); s5 = A(-2); }
    return (absmax5(s1, s2, s3, s4, s5) > (float)weps) ? r * weno5(s1, s2, s3, s4, s5, weps) : 0.0f;
  }
  if (kk >= 4 && kk <= nk - 2) {
    // upwind-ordered stencil first, so a warp with both signs evaluates one WENO
    const bool up = (r >= 0.0f);
    return r * weno5(up ? A(-3) : A(2), up ? A(-2) : A(1), up ? A(-1) : A(0), up ? A(0) : A(-1), up ? A(1) : A(-2),
                     weps);
  }
  if (kk == 3) {
    if (r >= 0.0f) return r * upstrpd(A(-2), A(-1), A(0), weps);
    return r * weno5(A(2), A(1), A(0), A(-1), A(-2), weps);
  }
  if (r >= 0.0f) return r * weno5(A(-3), A(-2), A(-1), A(0), A(1), weps);
  return r * upstrpd(A(1), A(0), A(-1), weps);
}
__device__ __forceinline__ float zflux_win(const DGrid &g, const float *wv, float r, int kk, int weno, int pdefweno,
                                           double weps) {
  return zflux_core(wv, r, kk, g.nk, LDG(&g.c1[kk]), LDG(&g.c2[kk]), weno, pdefweno, weps);
}
// The same face where 4 <= kk <= nk-2 (full 5-point stencils on both sides),
// the case of every level but the two lowest and two highest faces.
__device__ __forceinline__ float zflux_inner(const float *wv, float r, int weno, int pdefweno, double weps) {
  auto A = [&](int d) { return wv[d + 3]; };
  const bool up = (r >= 0.0f);
  const float s1 = up ? A(-3) : A(2), s2 = up ? A(-2) : A(1), s3 = up ? A(-1) : A(0), s4 = up ? A(0) : A(-1),
              s5 = up ? A(1) : A(-2);
  if (!weno) return r * flx5(s1, s2, s3, s4, s5);
  if (pdefweno == 1) return (absmax5(s1, s2, s3, s4, s5) > (float)weps) ? r * weno5(s1, s2, s3, s4, s5, weps) : 0.0f;
  return r * weno5(s1, s2, s3, s4, s5, weps);
}

// horizontal face flux from five upwind-ordered values
__device__ __forceinline__ float hflux5(float r, float sm3, float sm2, float sm1, float s0, float sp1, float sp2,
                                        int weno, int pdef, double weps) {
  float s1, s2, s3, s4, s5;
  if (r >= 0.0f) { s1 = sm3; s2 = sm2; s3 = sm1; s4 = s0; s5 = sp1; }
  else { s1 = sp2; s2 = sp1; s3 = s0; s4 = sm1; s5 = sm2; }
  if (!weno) return r * flx5(s1, s2, s3, s4, s5);
  if (pdef == 1 && !(absmax5(s1, s2, s3, s4, s5) > (float)weps)) return 0.0f;
  return r * weno5(s1, s2, s3, s4, s5, weps);
}

}  // namespace cm1g
