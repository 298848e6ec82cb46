// FP64 direct O(N^2) sum on sampled targets (the reference's direct code, DirectCalc3D /
// EvaluateField, bbfmm.c:471-504 and 880-913): out[t] = q_i sum_{x_j != x_i} q_j / |x_j - x_i|
// for i = targets[t]. Used to state the error of every run against an exact sum.
//
// One CTA per 128 targets; source particles are streamed through shared memory in tiles
// of 256 and every thread keeps a Neumaier-compensated FP64 sum.
#include "common.cuh"

namespace bbfmm {

__global__ void __launch_bounds__(128) direct_fp64_kernel(int N, const double *__restrict__ xyz,
                                                          const double *__restrict__ q, int nt,
                                                          const int *__restrict__ targets,
                                                          double *__restrict__ out) {
  __shared__ double sx[256], sy[256], sz[256], sq[256];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t < nt ? targets[t] : 0;
  const double fx = xyz[3 * (int64_t)i], fy = xyz[3 * (int64_t)i + 1], fz = xyz[3 * (int64_t)i + 2];
  double s = 0.0, c = 0.0;
  for (int j0 = 0; j0 < N; j0 += 256) {
    __syncthreads();
    for (int e = threadIdx.x; e < 256; e += blockDim.x) {
      const int j = j0 + e;
      if (j < N) {
        sx[e] = xyz[3 * (int64_t)j]; sy[e] = xyz[3 * (int64_t)j + 1]; sz[e] = xyz[3 * (int64_t)j + 2]; sq[e] = q[j];
      } else {
        sx[e] = fx; sy[e] = fy; sz[e] = fz; sq[e] = 0.0;
      }
    }
    __syncthreads();
#pragma unroll 4
    for (int e = 0; e < 256; ++e) {
      const double dx = sx[e] - fx, dy = sy[e] - fy, dz = sz[e] - fz;
      const double rr = dx * dx + dy * dy + dz * dz;
      if (rr != 0.0) {
        const double v = sq[e] / sqrt(rr);
        const double y = s + v;
        c += (fabs(s) >= fabs(v)) ? ((s - y) + v) : ((v - y) + s);
        s = y;
      }
    }
  }
  if (t < nt) out[t] = q[i] * (s + c);
}

int launch_direct_fp64(int N, const double *xyz, const double *q, int nt, const int *targets, double *out,
                       cudaStream_t s) {
  if (nt <= 0) return BBFMM_OK;
  direct_fp64_kernel<<<(nt + 127) / 128, 128, 0, s>>>(N, xyz, q, nt, targets, out);
  return bbfmm_set_cuda_error(cudaGetLastError(), "direct", __FILE__, __LINE__);
}

}  // namespace bbfmm
