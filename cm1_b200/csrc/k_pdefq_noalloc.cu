// k_pdefq_noalloc.cu -- cm1g_pdefq_noalloc: the positive-definite column fix
// of pdefq (src/misclibs.F:1037-1117, pdscheme=1) for callers that cannot
// allocate device memory.
//
// Some host programs must not allocate device memory once they are running:
// a process whose device memory is a pool owned by another component, or an
// embedding that forbids allocation after start-up.  They cannot create a
// context (which allocates its scratch), but they can still clip a moisture
// or tracer field: this entry point takes no context, writes its per-column
// budget into a file-scope device array of fixed size, and calls no
// allocating routine.
//
// The scratch array is held by every GPU that loads the library, for the
// life of the process.  All calls share it, so two calls that overlap on the
// GPU (different streams, or different host threads on one device) race on
// it; serialize them.  Each call overwrites the part it uses before reading
// it, so nothing has to start at zero.
//
// The device address of the array is looked up once per device, on the first
// call made with that device current (cudaGetSymbolAddress).  Every call
// copies asq's increment back and synchronizes the stream, so no call can be
// made while the stream is being captured into a CUDA graph.
//
// The columns are spread over a one-dimensional grid (one thread per column,
// at most CM1G_PDEFQ_NOALLOC_MAX_COLUMNS / 128 = 8192 blocks), so any ni x nj
// within the limit launches, however the columns split between i and j.  The
// budget sum walks each row of columns in order on one thread (the order of
// the context-based entry point): a grid of a few very long rows (ni of
// 10^5-10^6) spends about a millisecond there.
#include <cstdio>
#include <cstring>
#include <mutex>
#include "cm1g_common.cuh"
#include "../../include/cm1g.h"

namespace {

// per-column budgets, then the block partial and the final sum
__device__ __align__(256) double g_pdefq_scratch[CM1G_PDEFQ_NOALLOC_MAX_COLUMNS + 16];

const int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int fail(int code, const char *m) {
  char msg[256];
  snprintf(msg, sizeof msg, "cm1g_pdefq_noalloc: %s", m);
  return cm1g::report_error(code, msg);
}

struct Dims { int ni, nj, nk, NI, NJ, ib, jb; };

__device__ __forceinline__ long sidx(const Dims &d, int i, int j, int k) {
  return (long)(i - d.ib) + (long)d.NI * ((long)(j - d.jb) + (long)d.NJ * (long)k);
}

// one thread per column: pdefq's loops over k (misclibs.F:1063-1081)
__global__ void k_pdefq_na(Dims d, float rmax, const float *__restrict__ ruh, const float *__restrict__ rvh,
                           const float *__restrict__ rmh, const float *__restrict__ rho, float *q, double *bud) {
  const long col = (long)blockIdx.x * blockDim.x + threadIdx.x;   // (j-1)*ni + (i-1)
  if (col >= (long)d.ni * d.nj) return;
  const int j = 1 + (int)(col / d.ni), i = 1 + (int)(col - (long)(j - 1) * d.ni);
  const float ru = ruh[i - d.ib], rv = rvh[j - d.jb];
  double t1 = 0.0, t2 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int k = 1; k <= d.nk; k++) {
    const long o = sidx(d, i, j, k);
    const float r = rho[o], rm = rmh[o];
    float qq = q[o];
    t1 = t1 + (double)(r * qq);
    a1 = a1 + (double)(r * qq * ru * rv * rm);
    if (qq < rmax) { qq = 0.0f; q[o] = qq; }
    t2 = t2 + (double)(r * qq);
  }
  double t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20);
  if (t3 < 0.0) t3 = 1.0;
  for (int k = 1; k <= d.nk; k++) {
    const long o = sidx(d, i, j, k);
    const float r = rho[o], rm = rmh[o];
    const float qq = (float)(t3 * (double)q[o]);
    q[o] = qq;
    a2 = a2 + (double)(r * qq * ru * rv * rm);
  }
  bud[(long)(j - 1) * d.ni + (i - 1)] = a2 - a1;
}

// asq contribution sum_j (sum_i bud) * dx*dy*dz (misclibs.F:1083-1087),
// added in the same order as the context-based entry point; the result
// overwrites out[0].
__global__ void k_pdefq_na_sum(Dims d, double vol, const double *bud, double *out) {
  __shared__ double red[128];
  double s = 0.0;
  for (int j = 1 + (int)threadIdx.x; j <= d.nj; j += blockDim.x) {
    double bj = 0.0;
    for (int i = 0; i < d.ni; i++) bj = bj + bud[(long)(j - 1) * d.ni + i];
    s = s + bj * vol;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 64; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0];
}

bool on_device(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" int cm1g_pdefq_noalloc(const cm1g_config_t *cfg, float rmax, double *asq, const float *ruh,
                                  const float *rvh, const float *rmh, const float *rho, float *q3d, void *stream) {
  if (!cfg || !ruh || !rvh || !rmh || !rho || !q3d) return fail(CM1G_ERR_ARG, "null argument");
  if (cfg->ni < 1 || cfg->nj < 1 || cfg->nk < 1 || cfg->ngxy < 0) return fail(CM1G_ERR_ARG, "bad grid size");
  if ((long)cfg->ni * cfg->nj > (long)CM1G_PDEFQ_NOALLOC_MAX_COLUMNS)
    return fail(CM1G_ERR_ARG, "ni*nj exceeds CM1G_PDEFQ_NOALLOC_MAX_COLUMNS (1048576 columns)");
  const void *dev[] = {ruh, rvh, rmh, rho, q3d};
  for (const void *p : dev)
    if (!on_device(p)) return fail(CM1G_ERR_ARG, "arrays must be device pointers (nothing is staged or allocated)");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return fail(CM1G_ERR_CUDA, "no current CUDA device");
  double *scratch;
  {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[device]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_pdefq_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail(CM1G_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
      }
      g_scratch_addr[device] = (double *)p;
    }
    scratch = g_scratch_addr[device];
  }
  cudaStream_t st = (cudaStream_t)stream;
  Dims d{cfg->ni, cfg->nj, cfg->nk, cfg->ni + 2 * cfg->ngxy, cfg->nj + 2 * cfg->ngxy, 1 - cfg->ngxy, 1 - cfg->ngxy};
  double *bud = scratch, *out = scratch + CM1G_PDEFQ_NOALLOC_MAX_COLUMNS;
  const long ncol = (long)d.ni * d.nj;
  k_pdefq_na<<<(unsigned)((ncol + 127) / 128), 128, 0, st>>>(d, rmax, ruh, rvh, rmh, rho, q3d, bud);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CM1G_ERR_CUDA, cudaGetErrorString(e));
  k_pdefq_na_sum<<<1, 128, 0, st>>>(d, (double)(cfg->dx * cfg->dy * cfg->dz), bud, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CM1G_ERR_CUDA, cudaGetErrorString(e));
  double h = 0.0;
  e = cudaMemcpyAsync(&h, out, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(CM1G_ERR_CUDA, cudaGetErrorString(e));
  if (asq) *asq += h;
  return CM1G_OK;
}
