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

__device__ __forceinline__ void neumaier_add(double &s, double &c, double v) {
  const double y = s + v;
  c += (fabs(s) >= fabs(v)) ? ((s - y) + v) : ((v - y) + s);
  s = y;
}

// Potential and its gradient at the targets, without the target-charge factor (the exact
// counterpart of bbfmm_b200_solve_fields): pot[t] = sum_{x_j != x_i} q_j / r_ij and
// field[3t + a] = sum q_j (x_j - x_i)_a / r_ij^3 for i = targets[t]. The reference has no
// gradient code; this is the analytic derivative of its 1/r kernel.
__global__ void __launch_bounds__(128) direct_field_fp64_kernel(int N, const double *__restrict__ xyz,
                                                                const double *__restrict__ q, int nt,
                                                                const int *__restrict__ targets,
                                                                double *__restrict__ pot, double *__restrict__ fld) {
  __shared__ double sx[256], sy[256], sz[256], sq[256];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t < nt ? targets[t] : 0;
  const double fx = xyz[3 * (int64_t)i], fy = xyz[3 * (int64_t)i + 1], fz = xyz[3 * (int64_t)i + 2];
  double s = 0.0, c = 0.0, gx = 0.0, cx = 0.0, gy = 0.0, cy = 0.0, gz = 0.0, cz = 0.0;
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
#pragma unroll 2
    for (int e = 0; e < 256; ++e) {
      const double dx = sx[e] - fx, dy = sy[e] - fy, dz = sz[e] - fz;
      const double rr = dx * dx + dy * dy + dz * dz;
      if (rr != 0.0) {
        const double ir = 1.0 / sqrt(rr);
        const double v = sq[e] * ir, v3 = v * ir * ir;
        neumaier_add(s, c, v);
        neumaier_add(gx, cx, v3 * dx);
        neumaier_add(gy, cy, v3 * dy);
        neumaier_add(gz, cz, v3 * dz);
      }
    }
  }
  if (t < nt) {
    if (pot) pot[t] = s + c;
    if (fld) {
      fld[3 * (int64_t)t] = gx + cx;
      fld[3 * (int64_t)t + 1] = gy + cy;
      fld[3 * (int64_t)t + 2] = gz + cz;
    }
  }
}

int launch_direct_field_fp64(int N, const double *xyz, const double *q, int nt, const int *targets, double *pot,
                             double *fld, cudaStream_t s) {
  if (nt <= 0) return BBFMM_OK;
  direct_field_fp64_kernel<<<(nt + 127) / 128, 128, 0, s>>>(N, xyz, q, nt, targets, pot, fld);
  return bbfmm_set_cuda_error(cudaGetLastError(), "direct_field", __FILE__, __LINE__);
}

}  // namespace bbfmm
