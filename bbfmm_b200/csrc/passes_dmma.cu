// M2M and L2L for n = 8 in FP64 on the FP64 tensor path (mma.sync m8n8k4 f64).
//
// Each of the three one-axis contractions of M2M (anotherUpwardPass.c:345-539: z, then y,
// then x with Cweights) and of L2L (anotherDownwardPassX.c:40-211: x, then y, then z) is a
// product (rows x 16) x (16 x 8) or (rows x 8) x (8 x 8) with a fixed 8 x 8 Cweights block
// as B, i.e. whole m8n8k4 fragments: the B fragments live in registers and each A fragment
// is one shared-memory load per lane, where the CUDA-core kernels (passes.cu) load every
// operand for every multiply-add and are bound by shared-memory bandwidth. Shared arrays
// whose fragment rows would fall on the same banks are padded (row pitch 12 or 72 doubles).
// One CTA of 256 threads per parent (grid-stride); the next parent's values are prefetched
// into registers while the current one is contracted.
#include "common.cuh"

namespace bbfmm {
namespace pd {

constexpr int N3 = 512, PC = 12, SYM = 72, SYX = 8 * SYM, FPM = 72;

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Shared layout of M2M (doubles): children [512 rows (child, l12)][PC] | sz [4][512] | sy [2][SYX]
constexpr int M2M_SMEM = (8 * 64 * PC + 4 * N3 + 2 * SYX) * 8;

// Children S (level l+1, 8 n^3 contiguous per parent) -> parent S (level l), parents A0 + a.
__global__ void __launch_bounds__(256) m2m_dmma_kernel(const double *__restrict__ Sc, double *__restrict__ Sp,
                                                       const double *__restrict__ cwg, int64_t A0, int64_t count) {
  extern __shared__ __align__(16) double sm[];
  double *sc = sm, *sz = sc + 8 * 64 * PC, *sy = sz + 4 * N3;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r8 = lane >> 2, c4 = lane & 3;
  // B fragments of C[bit][n][m] (n = lane / 4), identical for the three phases
  double bfr[4];
#pragma unroll
  for (int ks = 0; ks < 4; ++ks) bfr[ks] = cwg[(ks >> 1) * 64 + r8 * 8 + (ks & 1) * 4 + c4];
  const double pre3 = 1.0 / 64.0;  // (2/n)^3
  double nxt[16];
  auto fetch = [&](int64_t a) {
    const double *src = Sc + a * 8 * N3 + tid;
#pragma unroll
    for (int k = 0; k < 16; ++k) nxt[k] = src[256 * k];
  };
  if ((int64_t)blockIdx.x < count) fetch(blockIdx.x);
  for (int64_t a = blockIdx.x; a < count; a += gridDim.x) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int e = tid + 256 * k;
      sc[(e >> 3) * PC + (e & 7)] = nxt[k];
    }
    if (a + gridDim.x < count) fetch(a + gridDim.x);
    __syncthreads();
    // z: sz[jj][l12][l3] = sum_{zb, m} child[2 jj + zb][l12][m] C[zb][l3][m]
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int mt = warp + 8 * i, R = 8 * mt + r8, jj = R >> 6, l12 = R & 63;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        dmma(d0, d1, sc[((2 * jj + (ks >> 1)) * 64 + l12) * PC + (ks & 1) * 4 + c4], bfr[ks]);
      *reinterpret_cast<double2 *>(sz + jj * N3 + l12 * 8 + 2 * c4) = make_double2(d0, d1);
    }
    __syncthreads();
    // y: sy[xb][l1][l2][l3] = sum_{yb, m} sz[2 xb + yb][l1][m][l3] C[yb][l2][m]
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int mt = warp + 8 * i, xb = mt >> 3, l1 = mt & 7, l3 = r8;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
        dmma(d0, d1, sz[(2 * xb + (ks >> 1)) * N3 + l1 * 64 + ((ks & 1) * 4 + c4) * 8 + l3], bfr[ks]);
      sy[xb * SYX + l1 * SYM + (2 * c4) * 8 + l3] = d0;
      sy[xb * SYX + l1 * SYM + (2 * c4 + 1) * 8 + l3] = d1;
    }
    __syncthreads();
    // x: S[l1][l2][l3] = pre3 sum_{xb, m} sy[xb][m][l2][l3] C[xb][l1][m]
    {
      const int l2 = warp, l3 = r8;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) dmma(d0, d1, sy[(ks >> 1) * SYX + ((ks & 1) * 4 + c4) * SYM + l2 * 8 + l3], bfr[ks]);
      double *dst = Sp + (A0 + a) * N3;
      dst[(2 * c4) * 64 + l2 * 8 + l3] = d0 * pre3;
      dst[(2 * c4 + 1) * 64 + l2 * 8 + l3] = d1 * pre3;
    }
  }
}

// Shared layout of L2L (doubles): fp [8 (m)][FPM] | fx [2][512] | fy [4 * 64 rows (j, l12)][PC]
constexpr int L2L_SMEM = (8 * FPM + 2 * N3 + 4 * 64 * PC) * 8;

// Parent F (level l) -> children F (level l+1, added), parents A0 + a.
__global__ void __launch_bounds__(256) l2l_dmma_kernel(const double *__restrict__ Fp, double *__restrict__ Fc,
                                                       const double *__restrict__ cwg, int64_t A0, int64_t count) {
  extern __shared__ __align__(16) double sm[];
  double *fp = sm, *fx = fp + 8 * FPM, *fy = fx + 2 * N3;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r8 = lane >> 2, c4 = lane & 3;
  // B fragments of C[bit][m][n] (n = lane / 4), m = 4 ks + lane % 4
  double bfr[2][2];
#pragma unroll
  for (int bit = 0; bit < 2; ++bit)
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) bfr[bit][ks] = cwg[bit * 64 + (ks * 4 + c4) * 8 + r8];
  const double pre3 = 1.0 / 64.0;
  // this lane's 16 child outputs: task i -> (j, mt) = ((warp + 8 i) / 8, (warp + 8 i) % 8),
  // entries l12 = 8 mt + lane / 4, l3 = 2 (lane % 4) + {0, 1}
  double np[2];
  double2 nc[8], old[8];
  auto child_off = [&](int i) {
    const int tk = warp + 8 * i, j = tk >> 3, mt = tk & 7;
    return j * N3 + (8 * mt + r8) * 8 + 2 * c4;
  };
  auto fetch = [&](int64_t a) {
    const double *pp = Fp + (A0 + a) * N3;
    np[0] = pp[tid];
    np[1] = pp[tid + 256];
    const double *cc = Fc + a * 8 * N3;
#pragma unroll
    for (int i = 0; i < 8; ++i) nc[i] = *reinterpret_cast<const double2 *>(cc + child_off(i));
  };
  if ((int64_t)blockIdx.x < count) fetch(blockIdx.x);
  for (int64_t a = blockIdx.x; a < count; a += gridDim.x) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int e = tid + 256 * k;  // e = m 64 + l23
      fp[(e >> 6) * FPM + (e & 63)] = np[k];
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) old[i] = nc[i];
    if (a + gridDim.x < count) fetch(a + gridDim.x);
    __syncthreads();
    // x: fx[j][l1][l2][l3] = sum_m F[m][l2][l3] C[j][m][l1]; task (j, l2) per warp pair
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int tk = warp + 8 * i, j = tk >> 3, l2 = tk & 7, l3 = r8;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) dmma(d0, d1, fp[(ks * 4 + c4) * FPM + l2 * 8 + l3], bfr[j][ks]);
      fx[j * N3 + (2 * c4) * 64 + l2 * 8 + l3] = d0;
      fx[j * N3 + (2 * c4 + 1) * 64 + l2 * 8 + l3] = d1;
    }
    __syncthreads();
    // y: fy[j][l1][l2][l3] = sum_m fx[j/2][l1][m][l3] C[j%2][m][l2]; task (j, l1)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int tk = warp + 8 * i, j = tk >> 3, l1 = tk & 7, l3 = r8;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) dmma(d0, d1, fx[(j >> 1) * N3 + l1 * 64 + (ks * 4 + c4) * 8 + l3], bfr[j & 1][ks]);
      fy[(j * 64 + l1 * 8 + 2 * c4) * PC + l3] = d0;
      fy[(j * 64 + l1 * 8 + 2 * c4 + 1) * PC + l3] = d1;
    }
    __syncthreads();
    // z: child_j[l12][l3] += pre3 sum_m fy[j/2][l12][m] C[j%2][m][l3]; task (j, mt)
    double *cc = Fc + a * 8 * N3;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int tk = warp + 8 * i, j = tk >> 3, mt = tk & 7, l12 = 8 * mt + r8;
      double d0 = 0.0, d1 = 0.0;
#pragma unroll
      for (int ks = 0; ks < 2; ++ks) dmma(d0, d1, fy[((j >> 1) * 64 + l12) * PC + ks * 4 + c4], bfr[j & 1][ks]);
      *reinterpret_cast<double2 *>(cc + child_off(i)) = make_double2(old[i].x + pre3 * d0, old[i].y + pre3 * d1);
    }
  }
}

}  // namespace pd

int launch_m2m_dmma(const double *Sc, double *Sp, const double *cw, int64_t first, int64_t count, cudaStream_t s) {
  if (count <= 0) return BBFMM_OK;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(pd::m2m_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, pd::M2M_SMEM);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "m2m_dmma smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  int64_t g = count < 148 * 3 * 4 ? count : 148 * 3 * 4;
  pd::m2m_dmma_kernel<<<(int)g, 256, pd::M2M_SMEM, s>>>(Sc, Sp, cw, first, count);
  return bbfmm_set_cuda_error(cudaGetLastError(), "m2m_dmma", __FILE__, __LINE__);
}

int launch_l2l_dmma(const double *Fp, double *Fc, const double *cw, int64_t first, int64_t count, cudaStream_t s) {
  if (count <= 0) return BBFMM_OK;
  int64_t g = count < 148 * 3 * 4 ? count : 148 * 3 * 4;
  pd::l2l_dmma_kernel<<<(int)g, 256, pd::L2L_SMEM, s>>>(Fp, Fc, cw, first, count);
  return bbfmm_set_cuda_error(cudaGetLastError(), "l2l_dmma", __FILE__, __LINE__);
}

}  // namespace bbfmm
