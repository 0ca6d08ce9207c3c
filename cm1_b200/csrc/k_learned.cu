// k_learned.cu -- learned coarse-grid advection closure.
//
// A small MLP (7 inputs -> 64 -> 64 -> 6, ReLU or GELU, BF16 weights, FP32
// accumulation) predicts, for one horizontal face of a coarse grid, the six
// coefficients of a linear reconstruction of the advected scalar from the
// face's six-point upwind-ordered stencil.  The coefficients are projected
// to sum to 1, so the face value phi = sum_k c_k s_k reproduces constants;
// where phi leaves the range of the four stencil cells nearest the face
// (two on each side), the scalar kernel falls back to the WENO5 face value:
// the face value then creates no new extremum in its neighbourhood, and a
// positive field stays positive.
//
// Features of a face (k_face_features): the stencil s_1..s_6 ordered from
// the far upwind cell to the far downwind cell, normalised as
// (s_k - mean) / (max - min + 1e-6), plus the face Courant number |u| dt/dx;
// the mean m and the scale d = max - min + 1e-6 are kept so that
// phi = m + d * sum_k c_k x_k.
//
// Parameters are one FP32 array (the master copy the optimiser updates):
//   W1 [8][64] (input k, hidden n; row 7 is padding), b1[64],
//   W2 [64][64], b2[64], W3 [64][8] (columns 6, 7 unused), b3[8].
// The forward kernel rounds the weights and activations to BF16 and runs
// the three layers as warp-level tensor-core MMAs (mma.sync m16n8k16,
// BF16 x BF16 -> FP32); the backward kernel uses the same BF16-rounded
// operands so its gradient is the gradient of the computed forward.
#include <algorithm>
#include <cstdint>
#include <cuda_bf16.h>
#include "cm1g_common.cuh"

namespace cm1g {

constexpr int MLP_IN = 8, MLP_H = 64, MLP_OUT = 8, MLP_NC = 6;
constexpr int P_W1 = 0, P_B1 = P_W1 + MLP_IN * MLP_H, P_W2 = P_B1 + MLP_H, P_B2 = P_W2 + MLP_H * MLP_H;
constexpr int P_W3 = P_B2 + MLP_H, P_B3 = P_W3 + MLP_H * MLP_OUT, P_TOTAL = P_B3 + MLP_OUT;

// The hidden activation: ReLU (gelu = 0; one instruction, exact on the host
// and the device) or GELU (gelu = 1; z Phi(z) with CUDA's erff, the
// activation the closure's specification names), selected by cm1g_mlp_set_activation.
__device__ __forceinline__ float act(float z, int gelu) {
  return gelu ? 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)) : fmaxf(z, 0.0f);
}
// d act / dz: Phi(z) + z phi(z) for GELU
__device__ __forceinline__ float act_grad(float z, int gelu) {
  if (!gelu) return z > 0.0f ? 1.0f : 0.0f;
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  return cdf + z * (0.39894228040143268f * expf(-0.5f * z * z));
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

// D = A(16x16, row) * B(16x8, col) + D, BF16 inputs, FP32 accumulators
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared copy of the weights, transposed (n-major) so that the two
// consecutive k of a B fragment are adjacent.
struct MlpSmem {
  __nv_bfloat16 w1t[MLP_H][16];       // k 8..15 zero
  __nv_bfloat16 w2t[MLP_H][MLP_H];
  __nv_bfloat16 w3t[MLP_OUT][MLP_H];
  float b1[MLP_H], b2[MLP_H], b3[MLP_OUT];
};

__device__ void load_weights(MlpSmem &S, const float *__restrict__ p) {
  for (int t = threadIdx.x; t < MLP_H * 16; t += blockDim.x) {
    const int n = t / 16, k = t % 16;
    S.w1t[n][k] = __float2bfloat16_rn(k < MLP_IN ? p[P_W1 + k * MLP_H + n] : 0.0f);
  }
  for (int t = threadIdx.x; t < MLP_H * MLP_H; t += blockDim.x) {
    const int n = t / MLP_H, k = t % MLP_H;
    S.w2t[n][k] = __float2bfloat16_rn(p[P_W2 + k * MLP_H + n]);
  }
  for (int t = threadIdx.x; t < MLP_OUT * MLP_H; t += blockDim.x) {
    const int n = t / MLP_H, k = t % MLP_H;
    S.w3t[n][k] = __float2bfloat16_rn(p[P_W3 + k * MLP_OUT + n]);
  }
  for (int t = threadIdx.x; t < MLP_H; t += blockDim.x) { S.b1[t] = p[P_B1 + t]; S.b2[t] = p[P_B2 + t]; }
  for (int t = threadIdx.x; t < MLP_OUT; t += blockDim.x) S.b3[t] = p[P_B3 + t];
}

// B fragment of a transposed weight tile: rows n0+g, k0+2t..+1 and k0+2t+8..+9
template <int KS>
__device__ __forceinline__ void bfrag(const __nv_bfloat16 (*wt)[KS], int n0, int k0, int g, int t, uint32_t &b0,
                                      uint32_t &b1) {
  b0 = *reinterpret_cast<const uint32_t *>(&wt[n0 + g][k0 + 2 * t]);
  b1 = *reinterpret_cast<const uint32_t *>(&wt[n0 + g][k0 + 2 * t + 8]);
}

// The three layers for the 16 rows of one warp.  a: the layer-1 A
// fragment (rows g and g+8 of the tile, inputs 2t, 2t+1).  On return d holds
// the outputs before the projection (row g: columns 2t, 2t+1 in d[0..1];
// row g+8 in d[2..3]; zero for t = 3, the unused columns 6 and 7) and ca/cb
// the projection's shift (1 - sum y)/6 of rows g and g+8.  z1/z2 (may be
// null) receive the pre-activations of rows ra, rb (< n).
__device__ __forceinline__ void mlp_tile(const MlpSmem &S, const uint32_t a[4], int ra, int rb, int n, float *z1,
                                         float *z2, float d[4], float &ca, float &cb, int gelu) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  (void)g;
  float h[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    float e[4] = {0.f, 0.f, 0.f, 0.f};
    uint32_t b0, b1;
    bfrag<16>(S.w1t, nt * 8, 0, lane >> 2, t, b0, b1);
    mma_bf16(e, a, b0, b1);
    const int c0 = nt * 8 + 2 * t;
    e[0] += S.b1[c0]; e[1] += S.b1[c0 + 1]; e[2] += S.b1[c0]; e[3] += S.b1[c0 + 1];
    if (z1) {
      if (ra < n) { z1[(long)ra * MLP_H + c0] = e[0]; z1[(long)ra * MLP_H + c0 + 1] = e[1]; }
      if (rb < n) { z1[(long)rb * MLP_H + c0] = e[2]; z1[(long)rb * MLP_H + c0 + 1] = e[3]; }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) h[nt][q] = act(e[q], gelu);
  }
  // layer 2: the accumulator tiles of layer 1 are the A fragments of layer 2
  uint32_t A[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    A[kt][0] = pack_bf16(h[2 * kt][0], h[2 * kt][1]);
    A[kt][1] = pack_bf16(h[2 * kt][2], h[2 * kt][3]);
    A[kt][2] = pack_bf16(h[2 * kt + 1][0], h[2 * kt + 1][1]);
    A[kt][3] = pack_bf16(h[2 * kt + 1][2], h[2 * kt + 1][3]);
  }
#pragma unroll
  for (int nt = 0; nt < 8; nt++) {
    float e[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int kt = 0; kt < 4; kt++) {
      uint32_t b0, b1;
      bfrag<MLP_H>(S.w2t, nt * 8, kt * 16, lane >> 2, t, b0, b1);
      mma_bf16(e, A[kt], b0, b1);
    }
    const int c0 = nt * 8 + 2 * t;
    e[0] += S.b2[c0]; e[1] += S.b2[c0 + 1]; e[2] += S.b2[c0]; e[3] += S.b2[c0 + 1];
    if (z2) {
      if (ra < n) { z2[(long)ra * MLP_H + c0] = e[0]; z2[(long)ra * MLP_H + c0 + 1] = e[1]; }
      if (rb < n) { z2[(long)rb * MLP_H + c0] = e[2]; z2[(long)rb * MLP_H + c0 + 1] = e[3]; }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) h[nt][q] = act(e[q], gelu);
  }
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    A[kt][0] = pack_bf16(h[2 * kt][0], h[2 * kt][1]);
    A[kt][1] = pack_bf16(h[2 * kt][2], h[2 * kt][3]);
    A[kt][2] = pack_bf16(h[2 * kt + 1][0], h[2 * kt + 1][1]);
    A[kt][3] = pack_bf16(h[2 * kt + 1][2], h[2 * kt + 1][3]);
  }
  // layer 3 (N = 8, columns 6 and 7 unused)
  d[0] = d[1] = d[2] = d[3] = 0.f;
#pragma unroll
  for (int kt = 0; kt < 4; kt++) {
    uint32_t b0, b1;
    bfrag<MLP_H>(S.w3t, 0, kt * 16, lane >> 2, t, b0, b1);
    mma_bf16(d, A[kt], b0, b1);
  }
  const int c0 = 2 * t;
  d[0] += S.b3[c0]; d[1] += S.b3[c0 + 1]; d[2] += S.b3[c0]; d[3] += S.b3[c0 + 1];
  if (t == 3) { d[0] = d[1] = d[2] = d[3] = 0.0f; }   // columns 6, 7
  // projection onto sum(c) = 1: the quad of lanes with the same g holds a row
  float sa = d[0] + d[1], sb = d[2] + d[3];
  sa += __shfl_xor_sync(0xffffffffu, sa, 1); sa += __shfl_xor_sync(0xffffffffu, sa, 2);
  sb += __shfl_xor_sync(0xffffffffu, sb, 1); sb += __shfl_xor_sync(0xffffffffu, sb, 2);
  ca = (1.0f - sa) * (1.0f / 6.0f);
  cb = (1.0f - sb) * (1.0f / 6.0f);
}

// One warp, 16 rows starting at r0: x [n][8] -> y [n][8] (pre-projection),
// c [n][6] (projected coefficients); z1, z2 [n][64] pre-activations if given.
__device__ void mlp_rows(const MlpSmem &S, int r0, int n, const float *__restrict__ x, float *y, float *c, float *z1,
                         float *z2, int gelu) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int ra = r0 + g, rb = r0 + g + 8;
  // layer 1: A = x rows (k 0..7, k 8..15 zero)
  uint32_t a[4];
  {
    const float x0 = ra < n ? x[(long)ra * MLP_IN + 2 * t] : 0.0f, x1 = ra < n ? x[(long)ra * MLP_IN + 2 * t + 1] : 0.0f;
    const float x2 = rb < n ? x[(long)rb * MLP_IN + 2 * t] : 0.0f, x3 = rb < n ? x[(long)rb * MLP_IN + 2 * t + 1] : 0.0f;
    a[0] = pack_bf16(x0, x1); a[1] = pack_bf16(x2, x3); a[2] = 0u; a[3] = 0u;
  }
  float d[4], ca, cb;
  mlp_tile(S, a, ra, rb, n, z1, z2, d, ca, cb, gelu);
  const int c0 = 2 * t;
  if (y) {
    if (ra < n) { y[(long)ra * MLP_OUT + c0] = d[0]; y[(long)ra * MLP_OUT + c0 + 1] = d[1]; }
    if (rb < n) { y[(long)rb * MLP_OUT + c0] = d[2]; y[(long)rb * MLP_OUT + c0 + 1] = d[3]; }
  }
  if (c && t < 3) {
    if (ra < n) { c[(long)ra * MLP_NC + c0] = d[0] + ca; c[(long)ra * MLP_NC + c0 + 1] = d[1] + ca; }
    if (rb < n) { c[(long)rb * MLP_NC + c0] = d[2] + cb; c[(long)rb * MLP_NC + c0 + 1] = d[3] + cb; }
  }
}

__global__ void __launch_bounds__(128) k_mlp_forward(const float *__restrict__ params, int n, const float *__restrict__ x,
                                                     float *y, float *c, float *z1, float *z2, int gelu) {
  __shared__ MlpSmem S;
  load_weights(S, params);
  __syncthreads();
  const int warp = (int)(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
  const int nw = (int)(gridDim.x * (blockDim.x >> 5));
  for (int r0 = warp * 16; r0 < n; r0 += nw * 16) mlp_rows(S, r0, n, x, y, c, z1, z2, gelu);
}

// Backward of the forward above for a batch: grad (P_TOTAL floats) +=
// d loss / d params, given dy = d loss / d y (pre-projection outputs).
// A block of 64 threads (one per hidden unit) walks a chunk of rows; each
// thread keeps its row of dW2, its column of dW1 and its row of dW3.
constexpr int BW_NT = 64, BW_ROWS = 256;
__global__ void __launch_bounds__(BW_NT) k_mlp_backward(const float *__restrict__ p, int n, const float *__restrict__ x,
                                                        const float *__restrict__ z1, const float *__restrict__ z2,
                                                        const float *__restrict__ dy, float *grad, int gelu) {
  __shared__ float w2[MLP_H][MLP_H + 1], w3[MLP_H][MLP_OUT];
  __shared__ float h1s[MLP_H], h2s[MLP_H], dz2s[MLP_H], xs[MLP_IN], dys[MLP_OUT];
  const int i = (int)threadIdx.x;
  for (int t = i; t < MLP_H * MLP_H; t += BW_NT) w2[t / MLP_H][t % MLP_H] = bf16r(p[P_W2 + t]);
  for (int t = i; t < MLP_H * MLP_OUT; t += BW_NT) w3[t / MLP_OUT][t % MLP_OUT] = bf16r(p[P_W3 + t]);
  float gw2[MLP_H], gw1[MLP_IN], gw3[MLP_OUT], gb1 = 0.f, gb2 = 0.f, gb3 = 0.f;
#pragma unroll
  for (int j = 0; j < MLP_H; j++) gw2[j] = 0.f;
#pragma unroll
  for (int k = 0; k < MLP_IN; k++) gw1[k] = 0.f;
#pragma unroll
  for (int o = 0; o < MLP_OUT; o++) gw3[o] = 0.f;
  __syncthreads();
  const int r_begin = (int)blockIdx.x * BW_ROWS, r_end = min(n, r_begin + BW_ROWS);
  for (int r = r_begin; r < r_end; r++) {
    const float a1 = z1[(long)r * MLP_H + i], a2 = z2[(long)r * MLP_H + i];
    h1s[i] = bf16r(act(a1, gelu));          // the BF16 operands the forward multiplied
    h2s[i] = bf16r(act(a2, gelu));
    if (i < MLP_IN) xs[i] = bf16r(i < 7 ? x[(long)r * MLP_IN + i] : 0.0f);
    if (i < MLP_OUT) dys[i] = (i < MLP_NC) ? dy[(long)r * MLP_OUT + i] : 0.0f;
    __syncthreads();
    // layer 3: dW3[i][o] += h2[i] dy[o]; dh2[i] = sum_o dy[o] W3[i][o]
    float dh2 = 0.f;
#pragma unroll
    for (int o = 0; o < MLP_OUT; o++) { gw3[o] += h2s[i] * dys[o]; dh2 += dys[o] * w3[i][o]; }
    if (i < MLP_OUT) gb3 += dys[i];
    const float dz2 = dh2 * act_grad(a2, gelu);
    dz2s[i] = dz2;
    gb2 += dz2;
    __syncthreads();
    // layer 2: dW2[i][j] += h1[i] dz2[j]; dh1[i] = sum_j dz2[j] W2[i][j]
    float dh1 = 0.f;
#pragma unroll
    for (int j = 0; j < MLP_H; j++) { gw2[j] += h1s[i] * dz2s[j]; dh1 += dz2s[j] * w2[i][j]; }
    const float dz1 = dh1 * act_grad(a1, gelu);
    gb1 += dz1;
#pragma unroll
    for (int k = 0; k < MLP_IN; k++) gw1[k] += xs[k] * dz1;
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < MLP_H; j++) atomicAdd(&grad[P_W2 + i * MLP_H + j], gw2[j]);
#pragma unroll
  for (int k = 0; k < MLP_IN; k++) atomicAdd(&grad[P_W1 + k * MLP_H + i], gw1[k]);
#pragma unroll
  for (int o = 0; o < MLP_OUT; o++) atomicAdd(&grad[P_W3 + i * MLP_OUT + o], gw3[o]);
  atomicAdd(&grad[P_B1 + i], gb1);
  atomicAdd(&grad[P_B2 + i], gb2);
  if (i < MLP_OUT) atomicAdd(&grad[P_B3 + i], gb3);
}

// Weighted squared error of the face values: phi = m + d * sum_k c_k x_k
// with c = y + (1 - sum y)/6; loss += w (phi - target)^2 and dy = dloss/dy.
__global__ void k_closure_loss(int n, const float *__restrict__ x, const float *__restrict__ y,
                               const float *__restrict__ m, const float *__restrict__ d, const float *__restrict__ target,
                               const float *__restrict__ w, float *dy, double *loss) {
  __shared__ double red[256];
  const int r = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  double l = 0.0;
  if (r < n) {
    float yy[MLP_NC], xx[MLP_NC], s = 0.f;
#pragma unroll
    for (int k = 0; k < MLP_NC; k++) { yy[k] = y[(long)r * MLP_OUT + k]; xx[k] = x[(long)r * MLP_IN + k]; s += yy[k]; }
    const float corr = (1.0f - s) * (1.0f / 6.0f);
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < MLP_NC; k++) acc += (yy[k] + corr) * xx[k];
    const float phi = m[r] + d[r] * acc, e = phi - target[r];
    l = (double)w[r] * (double)e * (double)e;
    float dc[MLP_NC], sdc = 0.f;
#pragma unroll
    for (int k = 0; k < MLP_NC; k++) { dc[k] = 2.0f * w[r] * e * d[r] * xx[k]; sdc += dc[k]; }
#pragma unroll
    for (int k = 0; k < MLP_NC; k++) dy[(long)r * MLP_OUT + k] = dc[k] - sdc * (1.0f / 6.0f);
    dy[(long)r * MLP_OUT + 6] = 0.f; dy[(long)r * MLP_OUT + 7] = 0.f;
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0]);
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
__global__ void k_adam(int np, float *p, const float *__restrict__ g, float *m1, float *m2, int step, float lr,
                       float scale) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (q >= np) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float gq = g[q] * scale;
  const float a = b1 * m1[q] + (1.0f - b1) * gq, b = b2 * m2[q] + (1.0f - b2) * gq * gq;
  m1[q] = a; m2[q] = b;
  const float ah = a / (1.0f - powf(b1, (float)step)), bh = b / (1.0f - powf(b2, (float)step));
  p[q] -= lr * ah / (sqrtf(bh) + eps);
}

// Features of the horizontal faces of a coarse grid (dims of s: NI x NJ x
// (nk+2), Fortran layout with lower bounds 1-ngxy, 0).  dir 0: the x-faces
// i = 1..ni+1 of rows j = 1..nj; dir 1: the y-faces j = 1..nj+1 of columns
// i = 1..ni.  vel is the raw face velocity (u-array for x, v-array for y).
// s is the advected value (with `sadd`, theta0 - 300 + theta' as advs sees it).
// Face order: f = (k-1)*nfx*nfy + (j-1)*nfx + (i-1) with nfx x nfy faces
// per level.  Writes x[f][8], m[f], d[f] and the signed face velocity u[f].
__global__ void k_face_features(int ni, int nj, int nk, int ngxy, int dir, const float *__restrict__ s,
                                const float *__restrict__ th0, int sadd, const float *__restrict__ vel, float dtdx,
                                float *x, float *m, float *dsc, float *uf) {
  const int NI = ni + 2 * ngxy, NJ = nj + 2 * ngxy, ib = 1 - ngxy;
  const int nfx = (dir == 0) ? ni + 1 : ni, nfy = (dir == 0) ? nj : nj + 1;
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x, nf = (long)nfx * nfy * nk;
  if (f >= nf) return;
  const int i = 1 + (int)(f % nfx), j = 1 + (int)((f / nfx) % nfy), k = 1 + (int)(f / ((long)nfx * nfy));
  const long plane = (long)NI * NJ;
  auto S = [&](int ii, int jj) {
    float v = s[(long)(ii - ib) + (long)NI * (jj - ib) + plane * k];
    if (sadd) v = (th0[k] - 300.0f) + v;
    return v;
  };
  const float u = (dir == 0) ? vel[(long)(i - ib) + (long)(NI + 1) * ((j - ib) + (long)NJ * k)]
                             : vel[(long)(i - ib) + (long)NI * ((j - ib) + (long)(NJ + 1) * k)];
  float v[6];
  // upwind-ordered: for u >= 0 the face between cells p-1 and p sees p-3 .. p+2
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const int off = (u >= 0.0f) ? (q - 3) : (2 - q);
    v[q] = (dir == 0) ? S(i + off, j) : S(i, j + off);
  }
  float mn = v[0], mx = v[0], sum = 0.f;
#pragma unroll
  for (int q = 0; q < 6; q++) { mn = fminf(mn, v[q]); mx = fmaxf(mx, v[q]); sum += v[q]; }
  const float mean = sum * (1.0f / 6.0f), sc = (mx - mn) + 1e-6f;
#pragma unroll
  for (int q = 0; q < 6; q++) x[f * MLP_IN + q] = (v[q] - mean) / sc;
  x[f * MLP_IN + 6] = fabsf(u) * dtdx;
  x[f * MLP_IN + 7] = 0.0f;
  m[f] = mean; dsc[f] = sc; uf[f] = u;
}

// p where it lies within the range of the stencil cells 2..5 (the two
// cells on each side of the face), widened on both sides by `widen` times
// the stencil's scale d (plus a tolerance of 1e-6 d), else NaN (the scalar
// kernel then takes the WENO5 value).  widen = 0 is the strict check.
__device__ __forceinline__ float bounded_face(float p, float m, float d, const float *x, float widen) {
  float lo = m + d * x[1], hi = lo;
#pragma unroll
  for (int q = 2; q <= 4; q++) {
    const float v = m + d * x[q];
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
  }
  const float tol = (1e-6f + widen) * d;
  return (p >= lo - tol && p <= hi + tol) ? p : __int_as_float(0x7fc00000);
}

// Face value from the coefficients, bounded as above.
__global__ void k_face_phi(long nf, const float *__restrict__ x, const float *__restrict__ c, const float *__restrict__ m,
                           const float *__restrict__ dsc, float widen, float *phi) {
  const long f = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  float acc = 0.f;
#pragma unroll
  for (int q = 0; q < MLP_NC; q++) acc += c[f * MLP_NC + q] * x[f * MLP_IN + q];
  const float p = m[f] + dsc[f] * acc;
  phi[f] = bounded_face(p, m[f], dsc[f], x + f * MLP_IN, widen);
}

// The closure's face values in one pass: for 32 faces per warp, the
// features (the arithmetic of k_face_features) go to shared memory, the
// MLP runs on the tensor cores (two 16-row tiles), and the bounded face
// value is formed as k_face_phi forms it, with the six coefficients gathered
// to the first lane of each row's quad so that the sum runs in the same
// order.  The result equals features -> forward -> face_phi bit for bit,
// without the 31 floats per face those passes write and read back.
constexpr int CF_WARPS = 4;
struct FaceTile {
  float x[32][MLP_IN + 1];     // pitch 9: the A-fragment reads of a quad fall in different banks
  float m[32], d[32];
};

__global__ void __launch_bounds__(CF_WARPS * 32) k_closure_faces(int ni, int nj, int nk, int ngxy, int dir,
                                                                const float *__restrict__ s,
                                                                const float *__restrict__ th0, int sadd,
                                                                const float *__restrict__ vel, float dtdx,
                                                                const float *__restrict__ params, float widen,
                                                                float *phi, int gelu) {
  __shared__ MlpSmem S;
  __shared__ FaceTile T[CF_WARPS];
  load_weights(S, params);
  __syncthreads();
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
  FaceTile &F = T[wib];
  const int NI = ni + 2 * ngxy, NJ = nj + 2 * ngxy, ib = 1 - ngxy;
  const int nfx = (dir == 0) ? ni + 1 : ni, nfy = (dir == 0) ? nj : nj + 1;
  const long nf = (long)nfx * nfy * nk, plane = (long)NI * NJ;
  const long nw = (long)gridDim.x * CF_WARPS;
  for (long f0 = ((long)blockIdx.x * CF_WARPS + wib) * 32; f0 < nf; f0 += nw * 32) {
    const long f = f0 + lane;
    if (f < nf) {
      const int i = 1 + (int)(f % nfx), j = 1 + (int)((f / nfx) % nfy), k = 1 + (int)(f / ((long)nfx * nfy));
      const float u = (dir == 0) ? vel[(long)(i - ib) + (long)(NI + 1) * ((j - ib) + (long)NJ * k)]
                                 : vel[(long)(i - ib) + (long)NI * ((j - ib) + (long)(NJ + 1) * k)];
      const float add = sadd ? (th0[k] - 300.0f) : 0.0f;
      float v[6];
#pragma unroll
      for (int q = 0; q < 6; q++) {
        const int off = (u >= 0.0f) ? (q - 3) : (2 - q);
        const int ii = (dir == 0) ? i + off : i, jj = (dir == 0) ? j : j + off;
        const float r = s[(long)(ii - ib) + (long)NI * (jj - ib) + plane * k];
        v[q] = sadd ? add + r : r;
      }
      float mn = v[0], mx = v[0], sum = 0.f;
#pragma unroll
      for (int q = 0; q < 6; q++) { mn = fminf(mn, v[q]); mx = fmaxf(mx, v[q]); sum += v[q]; }
      const float mean = sum * (1.0f / 6.0f), sc = (mx - mn) + 1e-6f;
#pragma unroll
      for (int q = 0; q < 6; q++) F.x[lane][q] = (v[q] - mean) / sc;
      F.x[lane][6] = fabsf(u) * dtdx;
      F.x[lane][7] = 0.0f;
      F.m[lane] = mean; F.d[lane] = sc;
    } else {
#pragma unroll
      for (int q = 0; q < MLP_IN; q++) F.x[lane][q] = 0.0f;
      F.m[lane] = 0.0f; F.d[lane] = 1.0f;
    }
    __syncwarp();
#pragma unroll 1
    for (int h = 0; h < 2; h++) {
      const int ra = 16 * h + g, rb = ra + 8;
      uint32_t a[4];
      a[0] = pack_bf16(F.x[ra][2 * t], F.x[ra][2 * t + 1]);
      a[1] = pack_bf16(F.x[rb][2 * t], F.x[rb][2 * t + 1]);
      a[2] = 0u; a[3] = 0u;
      float d[4], ca, cb;
      mlp_tile(S, a, 0, 0, 0, nullptr, nullptr, d, ca, cb, gelu);
      // this lane's coefficients (columns 2t, 2t+1) of rows ra and rb
      const float a0 = d[0] + ca, a1 = d[1] + ca, b0 = d[2] + cb, b1 = d[3] + cb;
      const float a2 = __shfl_down_sync(0xffffffffu, a0, 1), a3 = __shfl_down_sync(0xffffffffu, a1, 1);
      const float a4 = __shfl_down_sync(0xffffffffu, a0, 2), a5 = __shfl_down_sync(0xffffffffu, a1, 2);
      const float b2 = __shfl_down_sync(0xffffffffu, b0, 1), b3 = __shfl_down_sync(0xffffffffu, b1, 1);
      const float b4 = __shfl_down_sync(0xffffffffu, b0, 2), b5 = __shfl_down_sync(0xffffffffu, b1, 2);
      if (t == 0) {
        const float ca6[6] = {a0, a1, a2, a3, a4, a5}, cb6[6] = {b0, b1, b2, b3, b4, b5};
#pragma unroll
        for (int rr = 0; rr < 2; rr++) {
          const int row = rr ? rb : ra;
          const long fr = f0 + row;
          if (fr >= nf) continue;
          const float *cc = rr ? cb6 : ca6;
          float acc = 0.f;
#pragma unroll
          for (int q = 0; q < MLP_NC; q++) acc += cc[q] * F.x[row][q];
          const float mr = F.m[row], dr = F.d[row];
          const float p = mr + dr * acc;
          phi[fr] = bounded_face(p, mr, dr, F.x[row], widen);
        }
      }
    }
    __syncwarp();
  }
}

// ---- launchers ----
static int g_mlp_gelu = 0;   // the hidden activation of every launch below (cm1g_mlp_set_activation)
void mlp_set_gelu(int gelu) { g_mlp_gelu = gelu; }
int mlp_gelu() { return g_mlp_gelu; }
void launch_mlp_forward(const float *params, int n, const float *x, float *y, float *c, float *z1, float *z2,
                        cudaStream_t st) {
  const int warps = (n + 15) / 16, blocks = min(2048, (warps + 3) / 4);
  k_mlp_forward<<<blocks > 0 ? blocks : 1, 128, 0, st>>>(params, n, x, y, c, z1, z2, g_mlp_gelu);
}
void launch_mlp_backward(const float *params, int n, const float *x, const float *z1, const float *z2, const float *dy,
                         float *grad, cudaStream_t st) {
  const int blocks = (n + BW_ROWS - 1) / BW_ROWS;
  if (blocks > 0) k_mlp_backward<<<blocks, BW_NT, 0, st>>>(params, n, x, z1, z2, dy, grad, g_mlp_gelu);
}
void launch_closure_loss(int n, const float *x, const float *y, const float *m, const float *d, const float *target,
                         const float *w, float *dy, double *loss, cudaStream_t st) {
  if (n > 0) k_closure_loss<<<(n + 255) / 256, 256, 0, st>>>(n, x, y, m, d, target, w, dy, loss);
}
void launch_adam(int np, float *p, const float *g, float *m1, float *m2, int step, float lr, float scale,
                 cudaStream_t st) {
  k_adam<<<(np + 255) / 256, 256, 0, st>>>(np, p, g, m1, m2, step, lr, scale);
}
void launch_face_features(int ni, int nj, int nk, int ngxy, int dir, const float *s, const float *th0, int sadd,
                          const float *vel, float dtdx, float *x, float *m, float *d, float *u, cudaStream_t st) {
  const long nf = (long)((dir == 0) ? ni + 1 : ni) * ((dir == 0) ? nj : nj + 1) * nk;
  k_face_features<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(ni, nj, nk, ngxy, dir, s, th0, sadd, vel, dtdx, x, m,
                                                                 d, u);
}
void launch_face_phi(long nf, const float *x, const float *c, const float *m, const float *d, float widen, float *phi,
                     cudaStream_t st) {
  k_face_phi<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(nf, x, c, m, d, widen, phi);
}
void launch_closure_faces(int ni, int nj, int nk, int ngxy, int dir, const float *s, const float *th0, int sadd,
                          const float *vel, float dtdx, const float *params, float widen, float *phi, cudaStream_t st) {
  const long nf = (long)((dir == 0) ? ni + 1 : ni) * ((dir == 0) ? nj : nj + 1) * nk;
  const long tiles = (nf + 31) / 32;
  const long blocks = std::min<long>((tiles + CF_WARPS - 1) / CF_WARPS, 148L * 8);
  if (blocks > 0)
    k_closure_faces<<<(unsigned)blocks, CF_WARPS * 32, 0, st>>>(ni, nj, nk, ngxy, dir, s, th0, sadd, vel, dtdx, params,
                                                                 widen, phi, g_mlp_gelu);
}
int mlp_param_count() { return P_TOTAL; }

}  // namespace cm1g

// ---------------------------------------------------------------------
// C-ABI building blocks of the closure (device pointers, caller's stream).
// They have no counterpart in the reference.
// ---------------------------------------------------------------------
#include "../../include/cm1g.h"

namespace {
int bad(const char *m) { return cm1g::report_error(CM1G_ERR_ARG, m); }
int after_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CM1G_OK : cm1g::report_error(CM1G_ERR_CUDA, cudaGetErrorString(e));
}
}  // namespace

extern "C" int32_t cm1g_mlp_param_count(void) { return cm1g::P_TOTAL; }

extern "C" int cm1g_mlp_set_activation(int32_t act) {
  if (act != 0 && act != 1) return bad("cm1g_mlp_set_activation: act must be 0 (ReLU) or 1 (GELU)");
  cm1g::mlp_set_gelu(act);
  return CM1G_OK;
}
extern "C" int32_t cm1g_mlp_get_activation(void) { return cm1g::mlp_gelu(); }

extern "C" int cm1g_closure_faces(int32_t ni, int32_t nj, int32_t nk, int32_t ngxy, int32_t dir, const float *s,
                                  const float *th0, int32_t sadd, const float *vel, float dtdx, const float *params,
                                  float widen, float *phi, void *stream) {
  if (!s || !vel || !params || !phi || (sadd && !th0) || (dir != 0 && dir != 1) || ni < 1 || nj < 1 || nk < 1 ||
      ngxy < 3 || !(widen >= 0.0f))
    return bad("cm1g_closure_faces: bad argument");
  cm1g::launch_closure_faces(ni, nj, nk, ngxy, dir, s, th0, sadd, vel, dtdx, params, widen, phi, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_mlp_forward(const float *params, int32_t n, const float *x, float *y, float *c, float *z1,
                                float *z2, void *stream) {
  if (!params || !x || n < 0) return bad("cm1g_mlp_forward: null argument");
  cm1g::launch_mlp_forward(params, n, x, y, c, z1, z2, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_mlp_backward(const float *params, int32_t n, const float *x, const float *z1, const float *z2,
                                 const float *dy, float *grad, void *stream) {
  if (!params || !x || !z1 || !z2 || !dy || !grad || n < 0) return bad("cm1g_mlp_backward: null argument");
  cm1g::launch_mlp_backward(params, n, x, z1, z2, dy, grad, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_closure_loss(int32_t n, const float *x, const float *y, const float *m, const float *d,
                                 const float *target, const float *w, float *dy, double *loss, void *stream) {
  if (!x || !y || !m || !d || !target || !w || !dy || !loss || n < 0) return bad("cm1g_closure_loss: null argument");
  cm1g::launch_closure_loss(n, x, y, m, d, target, w, dy, loss, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_adam(int32_t np, float *params, const float *grad, float *m1, float *m2, int32_t step, float lr,
                         float grad_scale, void *stream) {
  if (!params || !grad || !m1 || !m2 || np <= 0 || step < 1) return bad("cm1g_adam: bad argument");
  cm1g::launch_adam(np, params, grad, m1, m2, step, lr, grad_scale, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_face_features(int32_t ni, int32_t nj, int32_t nk, int32_t ngxy, int32_t dir, const float *s,
                                  const float *th0, int32_t sadd, const float *vel, float dtdx, float *x, float *m,
                                  float *d, float *u, void *stream) {
  if (!s || !vel || !x || !m || !d || !u || (sadd && !th0)) return bad("cm1g_face_features: null argument");
  if (ni < 1 || nj < 1 || nk < 1 || ngxy < 3 || (dir != 0 && dir != 1)) return bad("cm1g_face_features: bad size");
  cm1g::launch_face_features(ni, nj, nk, ngxy, dir, s, th0, sadd, vel, dtdx, x, m, d, u, (cudaStream_t)stream);
  return after_launch();
}

extern "C" int cm1g_face_phi(int64_t nf, const float *x, const float *c, const float *m, const float *d, float widen,
                             float *phi, void *stream) {
  if (!x || !c || !m || !d || !phi || nf < 0 || !(widen >= 0.0f)) return bad("cm1g_face_phi: bad argument");
  if (nf) cm1g::launch_face_phi((long)nf, x, c, m, d, widen, phi, (cudaStream_t)stream);
  return after_launch();
}
