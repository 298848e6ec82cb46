// Near-field P2P: phi_i += q_i * sum_{B in N(A)} sum_{j in B, r_ij != 0} q_j / r_ij over
// the <= 27 neighbour leaves of each leaf (reference: anotherNearField.c:141-206 on the
// CPU, direct.cu:69-209 on the GPU).
//
// One thread per target particle; particles are leaf-sorted, so a warp covers a run of
// neighbouring leaves and the source particles it streams are shared through L1.
//  * p2p_kernel<T>: positions and arithmetic in T (the reference's d and s builds),
//    1/sqrt as in the reference's CPU code.
//  * p2p_local_kernel: FP32 arithmetic on leaf-local coordinates. Each particle carries
//    its offset from its own leaf centre in FP32; a pair's separation is
//    (xl_j - xl_i) + (c_B - c_A), where the centre difference is a multiple of the leaf
//    length and exact in FP32, so the separation keeps FP32 relative accuracy instead of
//    losing the bits of the absolute coordinate. Per-target sums are Neumaier-compensated
//    and the result is added to an FP64 potential.
#include "common.cuh"

namespace bbfmm {

template <typename T>
__global__ void __launch_bounds__(256) p2p_kernel(int N, const T *__restrict__ pos4, const int *__restrict__ leaf_start,
                                                  const int *__restrict__ leafm, int maxlev, T *__restrict__ phi) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const T fx = pos4[4 * (int64_t)i], fy = pos4[4 * (int64_t)i + 1], fz = pos4[4 * (int64_t)i + 2];
    const T qi = pos4[4 * (int64_t)i + 3];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
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
          const int64_t B = grid_to_morton(jx, jy, jz, maxlev);
          const int s0 = leaf_start[B], s1 = leaf_start[B + 1];
          for (int s = s0; s < s1; ++s) {
            const T ex = pos4[4 * (int64_t)s] - fx, ey = pos4[4 * (int64_t)s + 1] - fy,
                    ez = pos4[4 * (int64_t)s + 2] - fz;
            const T rr = ex * ex + ey * ey + ez * ez;
            if (rr != (T)0) v += pos4[4 * (int64_t)s + 3] * ((T)1 / sqrt(rr));
          }
        }
      }
    }
    phi[i] += qi * v;
  }
}

// loc4 = (x - c_leaf, y - c_leaf, z - c_leaf, q) in FP32; h = leaf length.
__global__ void __launch_bounds__(256) p2p_local_kernel(int N, const float4 *__restrict__ loc4,
                                                        const int *__restrict__ leaf_start,
                                                        const int *__restrict__ leafm, int maxlev, float h,
                                                        double *__restrict__ phi) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 f = loc4[i];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    float sum = 0.f, comp = 0.f;
    for (int dx = -1; dx <= 1; ++dx) {
      const int jx = ix + dx;
      if (jx < 0 || jx >= ncpd) continue;
      const float ox = (float)dx * h;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jy = iy + dy;
        if (jy < 0 || jy >= ncpd) continue;
        const float oy = (float)dy * h;
        for (int dz = -1; dz <= 1; ++dz) {
          const int jz = iz + dz;
          if (jz < 0 || jz >= ncpd) continue;
          const float oz = (float)dz * h;
          const int64_t B = grid_to_morton(jx, jy, jz, maxlev);
          const int s0 = leaf_start[B], s1 = leaf_start[B + 1];
          for (int s = s0; s < s1; ++s) {
            const float4 g = loc4[s];
            const float ex = (g.x - f.x) + ox, ey = (g.y - f.y) + oy, ez = (g.z - f.z) + oz;
            const float rr = ex * ex + ey * ey + ez * ez;
            if (rr != 0.f) {
              const float t = g.w * rsqrtf(rr);
              const float y = sum + t;
              comp += (fabsf(sum) >= fabsf(t)) ? ((sum - y) + t) : ((t - y) + sum);
              sum = y;
            }
          }
        }
      }
    }
    phi[i] += (double)f.w * ((double)sum + (double)comp);
  }
}

// Leaf-local FP32 coordinates from FP64 sorted positions.
__global__ void make_local_kernel(int N, const double *__restrict__ pos4, const int *__restrict__ leafm, int maxlev,
                                  double L, float4 *__restrict__ loc4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
    loc4[i] = make_float4((float)(pos4[4 * (int64_t)i] - cell_center_1d<double>(ix, maxlev, L)),
                          (float)(pos4[4 * (int64_t)i + 1] - cell_center_1d<double>(iy, maxlev, L)),
                          (float)(pos4[4 * (int64_t)i + 2] - cell_center_1d<double>(iz, maxlev, L)),
                          (float)pos4[4 * (int64_t)i + 3]);
  }
}

// Per-particle leaf (Morton) index from the leaf ranges.
__global__ void leaf_of_kernel(int64_t nleaf, const int *__restrict__ leaf_start, int *__restrict__ leafm) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < nleaf; m += (int64_t)gridDim.x * blockDim.x)
    for (int p = leaf_start[m]; p < leaf_start[m + 1]; ++p) leafm[p] = (int)m;
}

static int p2p_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (int)g;
}

template <typename T>
int launch_p2p(int N, const T *pos4, const int *leaf_start, const int *leafm, int maxlev, T *phi, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  p2p_kernel<T><<<p2p_grid(N), 256, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, phi);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p", __FILE__, __LINE__);
}
template int launch_p2p<double>(int, const double *, const int *, const int *, int, double *, cudaStream_t);
template int launch_p2p<float>(int, const float *, const int *, const int *, int, float *, cudaStream_t);

int launch_p2p_local(int N, const float4 *loc4, const int *leaf_start, const int *leafm, int maxlev, double L,
                     double *phi, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  const float h = (float)cell_length<double>(maxlev, L);
  p2p_local_kernel<<<p2p_grid(N), 256, 0, s>>>(N, loc4, leaf_start, leafm, maxlev, h, phi);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_local", __FILE__, __LINE__);
}

int launch_make_local(int N, const double *pos4, const int *leafm, int maxlev, double L, float4 *loc4,
                      cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  make_local_kernel<<<p2p_grid(N), 256, 0, s>>>(N, pos4, leafm, maxlev, L, loc4);
  return bbfmm_set_cuda_error(cudaGetLastError(), "make_local", __FILE__, __LINE__);
}

int launch_leaf_of(int maxlev, const int *leaf_start, int *leafm, cudaStream_t s) {
  const int64_t nleaf = pow8i(maxlev);
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
          const int64_t B = grid_to_morton(jx, jy, jz, maxlev);
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

// The same on FP32 leaf-local coordinates (see p2p_local_kernel); FP64 outputs.
__global__ void __launch_bounds__(256) p2p_local_field_kernel(int N, const float4 *__restrict__ loc4,
                                                              const int *__restrict__ leaf_start,
                                                              const int *__restrict__ leafm, int maxlev, float h,
                                                              double *__restrict__ pot, double *__restrict__ fld) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float4 f = loc4[i];
    int ix, iy, iz;
    morton_to_grid(leafm[i], maxlev, ix, iy, iz);
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
          const int64_t B = grid_to_morton(jx, jy, jz, maxlev);
          for (int s = leaf_start[B]; s < leaf_start[B + 1]; ++s) {
            const float4 g = loc4[s];
            const float ex = (g.x - f.x) + (float)dx * h, ey = (g.y - f.y) + (float)dy * h,
                        ez = (g.z - f.z) + (float)dz * h;
            const float rr = ex * ex + ey * ey + ez * ez;
            if (rr != 0.f) {
              const float rinv = rsqrtf(rr), t = g.w * rinv, t3 = t * rinv * rinv;
              const float y = sum + t;
              comp += (fabsf(sum) >= fabsf(t)) ? ((sum - y) + t) : ((t - y) + sum);
              sum = y;
              gx += t3 * ex;
              gy += t3 * ey;
              gz += t3 * ez;
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
                     cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  p2p_field_kernel<T><<<p2p_grid(N), 256, 0, s>>>(N, pos4, leaf_start, leafm, maxlev, pot, fld);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_field", __FILE__, __LINE__);
}
template int launch_p2p_field<double>(int, const double *, const int *, const int *, int, double *, double *,
                                      cudaStream_t);
template int launch_p2p_field<float>(int, const float *, const int *, const int *, int, float *, float *,
                                     cudaStream_t);

int launch_p2p_local_field(int N, const float4 *loc4, const int *leaf_start, const int *leafm, int maxlev, double L,
                           double *pot, double *fld, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  const float h = (float)cell_length<double>(maxlev, L);
  p2p_local_field_kernel<<<p2p_grid(N), 256, 0, s>>>(N, loc4, leaf_start, leafm, maxlev, h, pot, fld);
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2p_local_field", __FILE__, __LINE__);
}

}  // namespace bbfmm

// ====================================================== near-field C-ABI entry points
#include <mutex>

#include "../../include/bbfmm_b200.h"

namespace {

// Shared body of the two entry points: given device scratch for the per-particle leaf
// index (N ints) and, in the FP32 mode, the leaf-local coordinates (N float4), runs the
// near field on `stream`.
int near_field_run(int N, int maxlev, double L, const double *xyzq, const int *leaf_start, double *phi, int mode,
                   cudaStream_t st, int *leafm, float4 *loc4) {
  int rc = bbfmm::launch_leaf_of(maxlev, leaf_start, leafm, st);
  if (rc != BBFMM_OK) return rc;
  if (mode == BBFMM_B200_MODE_MIXED) {
    rc = bbfmm::launch_make_local(N, xyzq, leafm, maxlev, L, loc4, st);
    if (rc == BBFMM_OK) rc = bbfmm::launch_p2p_local(N, loc4, leaf_start, leafm, maxlev, L, phi, st);
    return rc;
  }
  return bbfmm::launch_p2p<double>(N, xyzq, leaf_start, leafm, maxlev, phi, st);
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
// particles (one float4 of leaf-local coordinates and one int leaf index each). Every GPU
// that loads the library holds this array until the process exits.
constexpr size_t kNoallocLoc4Bytes = (size_t)BBFMM_B200_NOALLOC_MAX_PARTICLES * sizeof(float4);
constexpr size_t kNoallocBytes = kNoallocLoc4Bytes + (size_t)BBFMM_B200_NOALLOC_MAX_PARTICLES * sizeof(int);
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
  float4 *loc4 = nullptr;
  cudaError_t e = cudaMalloc((void **)&leafm, sizeof(int) * (size_t)N);
  if (e == cudaSuccess && mode == BBFMM_B200_MODE_MIXED) e = cudaMalloc((void **)&loc4, sizeof(float4) * (size_t)N);
  if (e != cudaSuccess) {
    if (leafm) cudaFree(leafm);
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "near field: scratch allocation failed");
  }
  rc = near_field_run(N, maxlev, L, xyzq, leaf_start, phi, mode, st, leafm, loc4);
  e = cudaStreamSynchronize(st);  // the scratch is freed below
  if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(e, "near field", __FILE__, __LINE__);
  cudaFree(leafm);
  if (loc4) cudaFree(loc4);
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
  // Both scratch arrays are written in full by this call before they are read, so the
  // previous call's contents need no clearing.
  float4 *loc4 = reinterpret_cast<float4 *>(base);
  int *leafm = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(base) + kNoallocLoc4Bytes);
  return near_field_run(N, maxlev, L, xyzq, leaf_start, phi, mode, (cudaStream_t)stream, leafm, loc4);
}

}  // extern "C"
