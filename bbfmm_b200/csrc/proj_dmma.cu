// FP64 U-projections around M2L on the FP64 tensor path (mma.sync m8n8k4 f64):
//   up   : M[cpg(m)][i] = sum_l S[m][l] (Kweights[l] U(l, i))           (P2M/M2M -> M2L)
//   down : F[m][l] = (1/L_l) Kweights[l] sum_j U(l, j) L[cpg(m)][j]      (M2L -> L2L/L2P)
// (anotherUpwardPass.c:311-324 with atransx.c:48-86; auxAnotherFMMInteraction.c:398-416).
// C[out(m)][n] = scale * cs[n] * sum_k A[in(m)][k] B[k][n] with rows remapped between
// Morton and cpg order. CTA tile 64 rows x 256 columns, K-chunks of 16 double-buffered
// with cp.async, 8 warps in a 2 x 4 grid of 32 x 64 warp tiles.
#include "common.cuh"

namespace bbfmm {

namespace pj {

constexpr int BM = 64, BN = 256, BK = 16;
constexpr int AST = BK + 4;   // A stored [row][k]: fragment reads hit distinct banks
constexpr int BST = BN + 4;   // B stored [k][n]
constexpr int STAGE_DOUBLES = BM * AST + BK * BST;
constexpr int SMEM_BYTES = 2 * STAGE_DOUBLES * 8;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Local row m of a pass (the slab from cell row0, or the row list `rows`): the cpg row of its
// cell (to_cpg) or m itself.
__device__ __forceinline__ int64_t remap(int64_t m, int64_t row0, const int64_t *rows, int level, bool to_cpg) {
  return to_cpg ? morton_to_cpg_row(pass_cell(rows, row0, m), level) : m;
}

__global__ void __launch_bounds__(256, 1) proj_dmma_kernel(int64_t M, int K, int N, const double *__restrict__ A,
                                                           const double *__restrict__ B,
                                                           const double *__restrict__ cs, double scale,
                                                           double *__restrict__ C, int level, int mapmode,
                                                           int64_t row0, int lda, const int64_t *__restrict__ rows) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int64_t arow[BM];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp & 1, wn = warp >> 1;
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const int nk = K / BK;
  if (tid < BM) {
    const int64_t m = m0 + tid;
    arow[tid] = m < M ? remap(m, row0, rows, level, mapmode == MAP_IN_CPG) : -1;
  }
  __syncthreads();

  auto issue = [&](int kc, int buf) {
    const uint32_t sa = sbase + (uint32_t)(buf * STAGE_DOUBLES) * 8u;
    const uint32_t sb = sa + (uint32_t)(BM * AST) * 8u;
    const int k0 = kc * BK;
    for (int e = tid; e < BM * (BK / 2); e += 256) {  // 64 rows x 8 pairs
      const int row = e / (BK / 2), k2 = (e % (BK / 2)) * 2;
      const int64_t ar = arow[row];
      const double *src = ar >= 0 ? A + ar * lda + k0 + k2 : A;
      cp_async16(sa + (uint32_t)(row * AST + k2) * 8u, src, ar >= 0);
    }
    for (int e = tid; e < BK * (BN / 2); e += 256) {  // 16 rows x 128 pairs
      const int k = e / (BN / 2), n2 = (e % (BN / 2)) * 2;
      cp_async16(sb + (uint32_t)(k * BST + n2) * 8u, B + (int64_t)(k0 + k) * N + n0 + n2, true);
    }
    cp_commit();
  };

  double acc[4][8][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  issue(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) {
      issue(kc + 1, buf ^ 1);
      cp_wait_one();
    } else {
      cp_wait_all();
    }
    __syncthreads();
    const double *As = smem + buf * STAGE_DOUBLES;
    const double *Bs = As + BM * AST;
#pragma unroll
    for (int ks = 0; ks < BK / 4; ++ks) {
      const int k = ks * 4 + (lane & 3);
      double af[4], bf[8];
#pragma unroll
      for (int mf = 0; mf < 4; ++mf) af[mf] = As[(wm * 32 + mf * 8 + (lane >> 2)) * AST + k];
#pragma unroll
      for (int nf = 0; nf < 8; ++nf) bf[nf] = Bs[k * BST + wn * 64 + nf * 8 + (lane >> 2)];
#pragma unroll
      for (int mf = 0; mf < 4; ++mf)
#pragma unroll
        for (int nf = 0; nf < 8; ++nf) dmma(acc[mf][nf][0], acc[mf][nf][1], af[mf], bf[nf]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mf = 0; mf < 4; ++mf) {
    const int64_t m = m0 + wm * 32 + mf * 8 + (lane >> 2);
    if (m >= M) continue;
    double *dst = C + remap(m, row0, rows, level, mapmode == MAP_OUT_CPG) * N;
#pragma unroll
    for (int nf = 0; nf < 8; ++nf) {
      const int n = n0 + wn * 64 + nf * 8 + 2 * (lane & 3);
      const double c0 = cs ? scale * cs[n] : scale, c1 = cs ? scale * cs[n + 1] : scale;
      *reinterpret_cast<double2 *>(dst + n) = make_double2(c0 * acc[mf][nf][0], c1 * acc[mf][nf][1]);
    }
  }
}

// Narrow form for the FP64 leading columns of the mixed-mode up projection:
// C[out(m)][0:16] = sum_k A[m][k] B[k][0:16], CTA tile 128 rows x 16 columns, 8 warps of
// 16 rows, K-chunks of 16 double-buffered with cp.async; rows of C ldc apart.
namespace nw {
constexpr int BM = 128, BN = 16, BK = 16, AST = BK + 4, BST = BN + 8;
constexpr int STAGE = BM * AST + BK * BST;
constexpr int SMEM_BYTES = 2 * STAGE * 8;
}  // namespace nw

__global__ void __launch_bounds__(256) proj_narrow_kernel(int64_t M, int K, const double *__restrict__ A,
                                                          const double *__restrict__ B, double *__restrict__ C,
                                                          int ldc, int level, int mapmode, int64_t row0,
                                                          const int64_t *__restrict__ rows) {
  extern __shared__ __align__(16) double smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, r8 = lane >> 2, c4 = lane & 3;
  const int64_t m0 = (int64_t)blockIdx.x * nw::BM;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  const int nk = K / nw::BK;
  auto issue = [&](int kc, int buf) {
    const uint32_t sa = sbase + (uint32_t)(buf * nw::STAGE) * 8u;
    const uint32_t sb = sa + (uint32_t)(nw::BM * nw::AST) * 8u;
    const int k0 = kc * nw::BK;
    for (int e = tid; e < nw::BM * (nw::BK / 2); e += 256) {  // 128 rows x 8 pairs
      const int row = e / (nw::BK / 2), k2 = (e % (nw::BK / 2)) * 2;
      const int64_t m = m0 + row;
      const int64_t ar = m < M ? remap(m, row0, rows, level, mapmode == MAP_IN_CPG) : -1;
      cp_async16(sa + (uint32_t)(row * nw::AST + k2) * 8u, ar >= 0 ? A + ar * K + k0 + k2 : A, ar >= 0);
    }
    for (int e = tid; e < nw::BK * (nw::BN / 2); e += 256) {  // 16 rows x 8 pairs
      const int k = e / (nw::BN / 2), n2 = (e % (nw::BN / 2)) * 2;
      cp_async16(sb + (uint32_t)(k * nw::BST + n2) * 8u, B + (int64_t)(k0 + k) * nw::BN + n2, true);
    }
    cp_commit();
  };
  constexpr int NF = nw::BN / 8;
  double acc[2][NF][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < NF; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
  issue(0, 0);
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) {
      issue(kc + 1, buf ^ 1);
      cp_wait_one();
    } else {
      cp_wait_all();
    }
    __syncthreads();
    const double *As = smem + buf * nw::STAGE;
    const double *Bs = As + nw::BM * nw::AST;
#pragma unroll
    for (int ks = 0; ks < nw::BK / 4; ++ks) {
      const int k = ks * 4 + c4;
      double af[2], bf[NF];
#pragma unroll
      for (int mf = 0; mf < 2; ++mf) af[mf] = As[(warp * 16 + mf * 8 + r8) * nw::AST + k];
#pragma unroll
      for (int nf = 0; nf < NF; ++nf) bf[nf] = Bs[k * nw::BST + nf * 8 + r8];
#pragma unroll
      for (int mf = 0; mf < 2; ++mf)
#pragma unroll
        for (int nf = 0; nf < NF; ++nf) dmma(acc[mf][nf][0], acc[mf][nf][1], af[mf], bf[nf]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mf = 0; mf < 2; ++mf) {
    const int64_t m = m0 + warp * 16 + mf * 8 + r8;
    if (m >= M) continue;
    double *dst = C + remap(m, row0, rows, level, mapmode == MAP_OUT_CPG) * ldc;
#pragma unroll
    for (int nf = 0; nf < NF; ++nf)
      *reinterpret_cast<double2 *>(dst + nf * 8 + 2 * c4) = make_double2(acc[mf][nf][0], acc[mf][nf][1]);
  }
}

}  // namespace pj

int launch_proj_narrow(int64_t M, int K, const double *A, const double *B, double *C, int ldc, int level,
                       int mapmode, cudaStream_t s, int64_t row0, const int64_t *rows) {
  if (K % pj::nw::BK) return bbfmm_set_error(BBFMM_ERR_ARG, "narrow projection: K must be a multiple of 16");
  if (M <= 0) return BBFMM_OK;
  static bool attr = false;  // 47 KB of dynamic shared memory
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(pj::proj_narrow_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         pj::nw::SMEM_BYTES);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "proj_narrow smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  pj::proj_narrow_kernel<<<(unsigned)((M + pj::nw::BM - 1) / pj::nw::BM), 256, pj::nw::SMEM_BYTES, s>>>(
      M, K, A, B, C, ldc, level, mapmode, row0, rows);
  return bbfmm_set_cuda_error(cudaGetLastError(), "proj_narrow", __FILE__, __LINE__);
}

// Returns BBFMM_ERR_UNSUPPORTED (without recording an error) when the shape does not fit
// the tile (K % 16, N % 256); the caller then uses the CUDA-core GEMM.
int launch_proj_dmma(int64_t M, int K, int N, const double *A, const double *B, const double *cs, double scale,
                     double *C, int level, int mapmode, cudaStream_t s, int64_t row0, int lda,
                     const int64_t *rows) {
  if (K % pj::BK || N % pj::BN) return BBFMM_ERR_UNSUPPORTED;
  if (M <= 0) return BBFMM_OK;
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(pj::proj_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, pj::SMEM_BYTES);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "proj_dmma smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  dim3 grid((unsigned)((M + pj::BM - 1) / pj::BM), (unsigned)(N / pj::BN));
  pj::proj_dmma_kernel<<<grid, 256, pj::SMEM_BYTES, s>>>(M, K, N, A, B, cs, scale, C, level, mapmode, row0,
                                                          lda > 0 ? lda : K, rows);
  return bbfmm_set_cuda_error(cudaGetLastError(), "proj_dmma", __FILE__, __LINE__);
}

}  // namespace bbfmm
