// Near-field P2P: phi_i += q_i * sum_{B in N(A)} sum_{j in B, r_ij != 0} q_j K(x_j - x_i) over
// the <= 27 neighbour leaves of each leaf, K = 1/r (and, in p2p_kernel<T, H>, x/r^3 for H = 2
// and 1/r^4 for H = 4: the reference's LAPLACIANFORCE and ONEOVERR4 builds) (reference:
// anotherNearField.c:141-206 on the CPU, direct.cu:69-209 on the GPU).
//
// One thread per target particle; particles are leaf-sorted, so a warp covers a run of
// neighbouring leaves and the source particles it streams are shared through L1.
//  * p2p_kernel<T>: positions and arithmetic in T (the reference's d and s builds),
//    1/sqrt as in the reference's CPU code.
//  * p2p_mixed_kernel: the pair's separation and its square in FP64 (B200 runs FP64 at half
//    the FP32 rate, and FP32 coordinates would cost up to 2^-24 h / r_ij of relative error on
//    close pairs, h the leaf length), then 1/r in FP32 (rsqrtf with one Newton step) times
//    the FP32 charge; per-target Neumaier-compensated FP32 sums added to an FP64 potential.
#include "common.cuh"

namespace bbfmm {

// H: the kernel's degree of homogeneity, 1 (1/r), 2 (x/r^3 = dx rinv rinv rinv with dx the
// x component of source - target) or 4 (1/r^4 = rinv rinv rinv rinv), each formed as the
// reference's near field forms it (anotherNearField.c:111-124).
template <typename T, int H>
__global__ void __launch_bounds__(256) p2p_kernel(int N, const T *__restrict__ pos4, const int *__restrict__ leaf_start,
                                                  const int *__restrict__ leafm, int maxlev, T *__restrict__ phi) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const T fx = pos4[4 * (int64_t)i], fy = pos4[4 * (int64_t)i + 1], fz = pos4[4 * (int64_t)i + 2];
    const T qi = pos4[4 * (int64_t)i + 3];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    const int64_t sbase = leafm[i] & ~(pow8i(maxlev) - 1);  // first leaf of the particle's set
    T v = 0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int jx = ix + dx;
      if (jx < 0 || jx >= ncpd) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jy = iy + dy;
        if (jy < 0 || jy >= ncpd) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int jz = iz + dz;
          if (jz < 0 || jz >= ncpd) continue;
          const int64_t B = sbase + grid_to_morton(jx, jy, jz, maxlev);
          const int s0 = leaf_start[B], s1 = leaf_start[B + 1];
          for (int s = s0; s < s1; ++s) {
            const T ex = pos4[4 * (int64_t)s] - fx, ey = pos4[4 * (int64_t)s + 1] - fy,
                    ez = pos4[4 * (int64_t)s + 2] - fz;
            const T rr = ex * ex + ey * ey + ez * ez;
            if (rr != (T)0) {
              const T rinv = (T)1 / sqrt(rr);
              const T kern = H == 4 ? rinv * rinv * rinv * rinv : (H == 2 ? ex * rinv * rinv * rinv : rinv);
              v += pos4[4 * (int64_t)s + 3] * kern;
            }
          }
        }
      }
    }
    phi[i] += qi * v;
  }
}

// 1/sqrt(rr) in FP32: the hardware estimate refined by one Newton step.
// The compensated sums below form the term t = q * rsqrt_nr(rr) with __fmul_rn: were the
// product contracted into the addition sum + t, the new sum would not be fl(sum + t) and the
// compensation would no longer be the exact rounding error of that addition.
__device__ __forceinline__ float rsqrt_nr(float rr) {
  const float y = rsqrtf(rr);
  return y * fmaf(-0.5f * rr * y, y, 1.5f);
}

__global__ void __launch_bounds__(256) p2p_mixed_kernel(int N, const double4 *__restrict__ pos4,
                                                        const int *__restrict__ leaf_start,
                                                        const int *__restrict__ leafm, int maxlev,
                                                        double *__restrict__ phi) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double4 f = pos4[i];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    const int64_t sbase = leafm[i] & ~(pow8i(maxlev) - 1);  // first leaf of the particle's set
    float sum = 0.f, comp = 0.f;
    for (int dx = -1; dx <= 1; ++dx) {
      const int jx = ix + dx;
      if (jx < 0 || jx >= ncpd) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jy = iy + dy;
        if (jy < 0 || jy >= ncpd) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int jz = iz + dz;
          if (jz < 0 || jz >= ncpd) continue;
          const int64_t B = sbase + grid_to_morton(jx, jy, jz, maxlev);
          const int s0 = leaf_start[B], s1 = leaf_start[B + 1];
          for (int s = s0; s < s1; ++s) {
            const double4 g = pos4[s];
            const double ex = g.x - f.x, ey = g.y - f.y, ez = g.z - f.z;
            const double rr = fma(ex, ex, fma(ey, ey, ez * ez));
            if (rr != 0.0) {
              const float t = __fmul_rn((float)g.w, rsqrt_nr((float)rr));
              const float y = sum + t;
              comp += (fabsf(sum) >= fabsf(t)) ? ((sum - y) + t) : ((t - y) + sum);
              sum = y;
            }
          }
        }
      }
    }
    phi[i] += f.w * ((double)sum + (double)comp);
  }
}

// Per-particle leaf (Morton) index from the leaf ranges.
__global__ void leaf_of_kernel(int64_t nleaf, const int *__restrict__ leaf_start, int *__restrict__ leafm) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nleaf; m += (int64_t)gridDim.x * blockDim.x)
    for (int p = leaf_start[m]; p < leaf_start[m + 1]; ++p) leafm[p] = (int)m;
}

static int p2p_grid(int64_t n, int threads = 256) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (int)g;
}

template <typename T>
int launch_p2p(int N, const T *pos4, const int *leaf_start, const int *leafm, int maxlev, T *phi, cudaStream_t s,
               int threads, int homogen) {
  if (N <= 0) return BBFMM_OK;
  if (threads < 32 || threads > 256 || threads % 32) return bbfmm_set_error(BBFMM_ERR_ARG, "p2p threads per block");
  if (homogen == 4)
    p2p_kernel<T, 4><<<p2p_grid(N, threads), threads, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, phi);
  else if (homogen == 2)
    p2p_kernel<T, 2><<<p2p_grid(N, threads), threads, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, phi);
  else if (homogen == 1)
    p2p_kernel<T, 1><<<p2p_grid(N, threads), threads, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, phi);
  else
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED,
                           "near field: kernel homogeneity 1 (1/r), 2 (x/r^3) or 4 (1/r^4)");
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p", __FILE__, __LINE__);
}
template int launch_p2p<double>(int, const double *, const int *, const int *, int, double *, cudaStream_t, int, int);
template int launch_p2p<float>(int, const float *, const int *, const int *, int, float *, cudaStream_t, int, int);

int launch_p2p_mixed(int N, const double *pos4, const int *leaf_start, const int *leafm, int maxlev, double *phi,
                     cudaStream_t s, int threads) {
  if (N <= 0) return BBFMM_OK;
  if (threads < 32 || threads > 256 || threads % 32) return bbfmm_set_error(BBFMM_ERR_ARG, "p2p threads per block");
  p2p_mixed_kernel<<<p2p_grid(N, threads), threads, 0, s>>>(N, reinterpret_cast<const double4 *>(pos4), leaf_start,
                                                            leafm, maxlev, phi);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_mixed", __FILE__, __LINE__);
}

int launch_leaf_of(int maxlev, const int *leaf_start, int *leafm, cudaStream_t s, int nsets) {
  const int64_t nleaf = nsets * pow8i(maxlev);
  leaf_of_kernel<<<p2p_grid(nleaf), 256, 0, s>>>(nleaf, leaf_start, leafm);
  return bbfmm_set_cuda_error(cudaGetLastError(), "leaf_of", __FILE__, __LINE__);
}

}  // namespace bbfmm

namespace bbfmm {
// ------------------------------------------------------------- near field with gradient
// pot[i] += sum_j q_j / r_ij and fld[3i + a] += sum_j q_j (x_j - x_i)_a / r_ij^3 (the
// gradient of the potential at x_i), no target factor; sorted order.
template <typename T>
__global__ void __launch_bounds__(256) p2p_field_kernel(int N, const T *__restrict__ pos4,
                                                        const int *__restrict__ leaf_start,
                                                        const int *__restrict__ leafm, int maxlev, T *__restrict__ pot,
                                                        T *__restrict__ fld) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const T fx = pos4[4 * (int64_t)i], fy = pos4[4 * (int64_t)i + 1], fz = pos4[4 * (int64_t)i + 2];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    const int64_t sbase = leafm[i] & ~(pow8i(maxlev) - 1);  // first leaf of the particle's set
    T v = 0, gx = 0, gy = 0, gz = 0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int jx = ix + dx;
      if (jx < 0 || jx >= ncpd) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jy = iy + dy;
        if (jy < 0 || jy >= ncpd) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int jz = iz + dz;
          if (jz < 0 || jz >= ncpd) continue;
          const int64_t B = sbase + grid_to_morton(jx, jy, jz, maxlev);
          for (int s = leaf_start[B]; s < leaf_start[B + 1]; ++s) {
            const T ex = pos4[4 * (int64_t)s] - fx, ey = pos4[4 * (int64_t)s + 1] - fy,
                    ez = pos4[4 * (int64_t)s + 2] - fz;
            const T rr = ex * ex + ey * ey + ez * ez;
            if (rr != (T)0) {
              const T rinv = (T)1 / sqrt(rr), qr = pos4[4 * (int64_t)s + 3] * rinv;
              const T qr3 = qr * rinv * rinv;
              v += qr;
              gx += qr3 * ex;
              gy += qr3 * ey;
              gz += qr3 * ez;
            }
          }
        }
      }
    }
    pot[i] += v;
    fld[3 * (int64_t)i] += gx;
    fld[3 * (int64_t)i + 1] += gy;
    fld[3 * (int64_t)i + 2] += gz;
  }
}

// The same with the arithmetic of p2p_mixed_kernel; FP64 outputs.
__global__ void __launch_bounds__(256) p2p_mixed_field_kernel(int N, const double4 *__restrict__ pos4,
                                                              const int *__restrict__ leaf_start,
                                                              const int *__restrict__ leafm, int maxlev,
                                                              double *__restrict__ pot, double *__restrict__ fld) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const double4 f = pos4[i];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    const int64_t sbase = leafm[i] & ~(pow8i(maxlev) - 1);  // first leaf of the particle's set
    float sum = 0.f, comp = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    for (int dx = -1; dx <= 1; ++dx) {
      const int jx = ix + dx;
      if (jx < 0 || jx >= ncpd) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jy = iy + dy;
        if (jy < 0 || jy >= ncpd) continue;
        for (int dz = -1; dz <= 1; ++dz) {
          const int jz = iz + dz;
          if (jz < 0 || jz >= ncpd) continue;
          const int64_t B = sbase + grid_to_morton(jx, jy, jz, maxlev);
          for (int s = leaf_start[B]; s < leaf_start[B + 1]; ++s) {
            const double4 g = pos4[s];
            const double ex = g.x - f.x, ey = g.y - f.y, ez = g.z - f.z;
            const double rr = fma(ex, ex, fma(ey, ey, ez * ez));
            if (rr != 0.0) {
              const float rinv = rsqrt_nr((float)rr), t = __fmul_rn((float)g.w, rinv), t3 = t * rinv * rinv;
              const float y = sum + t;
              comp += (fabsf(sum) >= fabsf(t)) ? ((sum - y) + t) : ((t - y) + sum);
              sum = y;
              gx += t3 * (float)ex;
              gy += t3 * (float)ey;
              gz += t3 * (float)ez;
            }
          }
        }
      }
    }
    pot[i] += (double)sum + (double)comp;
    fld[3 * (int64_t)i] += gx;
    fld[3 * (int64_t)i + 1] += gy;
    fld[3 * (int64_t)i + 2] += gz;
  }
}

template <typename T>
int launch_p2p_field(int N, const T *pos4, const int *leaf_start, const int *leafm, int maxlev, T *pot, T *fld,
                     cudaStream_t s, int threads) {
  if (N <= 0) return BBFMM_OK;
  if (threads < 32 || threads > 256 || threads % 32) return bbfmm_set_error(BBFMM_ERR_ARG, "p2p threads per block");
  p2p_field_kernel<T><<<p2p_grid(N, threads), threads, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, pot, fld);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_field", __FILE__, __LINE__);
}
template int launch_p2p_field<double>(int, const double *, const int *, const int *, int, double *, double *,
                                      cudaStream_t, int);
template int launch_p2p_field<float>(int, const float *, const int *, const int *, int, float *, float *,
                                     cudaStream_t, int);

int launch_p2p_mixed_field(int N, const double *pos4, const int *leaf_start, const int *leafm, int maxlev,
                           double *pot, double *fld, cudaStream_t s, int threads) {
  if (N <= 0) return BBFMM_OK;
  if (threads < 32 || threads > 256 || threads % 32) return bbfmm_set_error(BBFMM_ERR_ARG, "p2p threads per block");
  p2p_mixed_field_kernel<<<p2p_grid(N, threads), threads, 0, s>>>(N, reinterpret_cast<const double4 *>(pos4),
                                                                  leaf_start, leafm, maxlev, pot, fld);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_mixed_field", __FILE__, __LINE__);
}

}  // namespace bbfmm

// ====================================================== near-field C-ABI entry points
#include <mutex>

#include "../../include/bbfmm_b200.h"

namespace {

// Shared body of the two entry points: given device scratch for the per-particle leaf
// index (N ints), runs the near field on `stream`.
int near_field_run(int N, int maxlev, const double *xyzq, const int *leaf_start, double *phi, int mode,
                   cudaStream_t st, int *leafm) {
  int rc = bbfmm::launch_leaf_of(maxlev, leaf_start, leafm, st, 1);
  if (rc != BBFMM_OK) return rc;
  if (mode == BBFMM_B200_MODE_MIXED) return bbfmm::launch_p2p_mixed(N, xyzq, leaf_start, leafm, maxlev, phi, st, 256);
  return bbfmm::launch_p2p<double>(N, xyzq, leaf_start, leafm, maxlev, phi, st, 256, 1);
}

int near_field_check(int N, int maxlev, double L, const void *xyzq, const void *leaf_start, const void *phi,
                     int mode) {
  if (N < 0 || maxlev < BBFMM_MINLEV || maxlev > 10 || !(L > 0))
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: need N >= 0, 2 <= maxlev <= 10, L > 0");
  if (N > 0 && (!xyzq || !leaf_start || !phi)) return bbfmm_set_error(BBFMM_ERR_ARG, "near field: null pointer");
  if (mode != BBFMM_B200_MODE_D && mode != BBFMM_B200_MODE_MIXED)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: mode must be BBFMM_B200_MODE_D or BBFMM_B200_MODE_MIXED");
  return BBFMM_OK;
}

// Scratch of the allocation-free entry point: room for BBFMM_B200_NOALLOC_MAX_PARTICLES
// particles (one int leaf index each). Every GPU that loads the library holds this array
// until the process exits.
constexpr size_t kNoallocBytes = (size_t)BBFMM_B200_NOALLOC_MAX_PARTICLES * sizeof(int);
static __device__ __align__(256) unsigned char g_near_field_scratch[kNoallocBytes];

// Device addresses of the array, one per device, looked up once with that device current
// (the array's name in host code is only a stand-in and must never reach a kernel).
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_ptr[kMaxDevices] = {};

int noalloc_scratch(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= kMaxDevices) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_near_field_scratch);
    if (e != cudaSuccess || !p)
      return bbfmm_set_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol, "cudaGetSymbolAddress(scratch)",
                                  __FILE__, __LINE__);
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return BBFMM_OK;
}

}  // namespace

extern "C" {

int bbfmm_b200_near_field(int N, int maxlev, double L, const double *xyzq, const int *leaf_start, double *phi,
                          int mode, void *stream) {
  int rc = near_field_check(N, maxlev, L, xyzq, leaf_start, phi, mode);
  if (rc != BBFMM_OK || N == 0) return rc;
  const cudaStream_t st = (cudaStream_t)stream;
  int *leafm = nullptr;
  cudaError_t e = cudaMalloc((void **)&leafm, sizeof(int) * (size_t)N);
  if (e != cudaSuccess) return bbfmm_set_error(BBFMM_ERR_NOMEM, "near field: scratch allocation failed");
  rc = near_field_run(N, maxlev, xyzq, leaf_start, phi, mode, st, leafm);
  e = cudaStreamSynchronize(st);  // the scratch is freed below
  if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(e, "near field", __FILE__, __LINE__);
  cudaFree(leafm);
  return rc;
}

int bbfmm_b200_near_field_noalloc(int N, int maxlev, double L, const double *xyzq, const int *leaf_start,
                                  double *phi, int mode, void *stream) {
  int rc = near_field_check(N, maxlev, L, xyzq, leaf_start, phi, mode);
  if (rc != BBFMM_OK || N == 0) return rc;
  if (N > BBFMM_B200_NOALLOC_MAX_PARTICLES)
    return bbfmm_set_error(BBFMM_ERR_ARG,
                           "near field (no allocation): N exceeds BBFMM_B200_NOALLOC_MAX_PARTICLES = 262144");
  void *base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc != BBFMM_OK) return rc;
  // The scratch is written in full by this call before it is read, so the previous call's
  // contents need no clearing.
  int *leafm = reinterpret_cast<int *>(base);
  return near_field_run(N, maxlev, xyzq, leaf_start, phi, mode, (cudaStream_t)stream, leafm);
}

}  // extern "C"
