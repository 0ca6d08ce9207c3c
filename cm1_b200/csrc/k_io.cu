// k_io.cu -- record packing for output and restart files.
//
// The reference writes a field as one record per level of its physical
// points, i fastest then j (writeout.F:8901-8995, writeosp; restart_write.F:
// 2422-2714, writer).  On the device a field's records are one gather: a
// block row of the pack kernel copies one (j, k) row of the physical points
// into the contiguous record buffer, so a whole file's fields leave the GPU in
// one device-to-host copy; unpacking is the same scatter in reverse.
#include "cm1g_common.cuh"

namespace cm1g {

// derived forms of k_pack_records (writeout's output variables)
enum RecMode { REC_PLAIN = 0, REC_ADD_PROFILE, REC_SUB_PROFILE, REC_SUB_FIELD, REC_EXNER, REC_EXNER_PERT };

// extent of the physical points of a field: ie x je, levels k1..k2
__device__ __forceinline__ long rec_src(const DGrid &g, int stag, int i, int j, int k) {
  return stag == 2 ? iU(g, i, j, k) : stag == 3 ? iV(g, i, j, k) : iS(g, i, j, k);
}

// the value written for a point: the field itself or one of writeout's
// derived forms (writeout.F:3205-3480, 6829-6990)
__device__ __forceinline__ float rec_value(const DGrid &g, const float *__restrict__ a, int stag, int i, int j, int k,
                                           int mode, const float *__restrict__ base) {
  const long o = rec_src(g, stag, i, j, k);
  const float v = a[o];
  switch (mode) {
    case REC_ADD_PROFILE: return base[k] + v;            // th = th0 + tha
    case REC_SUB_PROFILE: return v - base[k];            // prspert, rhopert, qvpert
    case REC_SUB_FIELD: return v - base[o];              // upert = ua - u0, vpert = va - v0
    case REC_EXNER:                                      // pi = (prs/p00)**rovcp
    case REC_EXNER_PERT: {                               // pipert = pi - pi0
      // binary64 power rounded once: the correctly rounded binary32 value
      // except in rare double-rounding cases
      const float pi = (float)pow((double)(v * (1.0f / 1.0e5f)), (double)g.c.rovcp);
      return mode == REC_EXNER ? pi : pi - g.pi0[k];
    }
    default: return v;
  }
}

__global__ void k_pack_records(DGrid g, const float *__restrict__ a, int stag, int k1, float *__restrict__ out,
                               int mode, const float *__restrict__ base) {
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3);
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = k1 + (int)blockIdx.z;
  if (i > ie) return;
  out[((long)blockIdx.z * je + (j - 1)) * ie + (i - 1)] = rec_value(g, a, stag, i, j, k, mode, base);
}

__global__ void k_unpack_records(DGrid g, float *__restrict__ a, int stag, int k1, const float *__restrict__ in) {
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3);
  const int i = 1 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int j = 1 + (int)blockIdx.y, k = k1 + (int)blockIdx.z;
  if (i > ie) return;
  a[rec_src(g, stag, i, j, k)] = in[((long)blockIdx.z * je + (j - 1)) * ie + (i - 1)];
}

long record_count(const DGrid &g, int stag, int k1, int k2) {
  const long ie = g.ni + (stag == 2), je = g.nj + (stag == 3);
  return k2 >= k1 ? ie * je * (long)(k2 - k1 + 1) : 0;
}

void launch_pack_records(const DGrid &g, const float *a, int stag, int k1, int k2, float *out, bool unpack,
                         cudaStream_t st, int64_t *nl, int mode, const float *base) {
  if (k2 < k1) return;
  const int ie = g.ni + (stag == 2), je = g.nj + (stag == 3);
  dim3 grid((ie + 127) / 128, je, k2 - k1 + 1);
  if (unpack) {
    ProfScope _ps("k_unpack_records", st);
    k_unpack_records<<<grid, 128, 0, st>>>(g, const_cast<float *>(a), stag, k1, out);
  } else {
    ProfScope _ps("k_pack_records", st);
    k_pack_records<<<grid, 128, 0, st>>>(g, a, stag, k1, out, mode, base);
  }
  if (nl) *nl += 1;
}

}  // namespace cm1g
