// Upward and downward passes on the device (P2M, M2M, L2L, L2P), the U-projections
// around M2L, and the particle permutations. Expansions stay resident in HBM.
//
// Reference semantics (all CPU in the reference):
//   P2M  anotherUpwardPass.c:61-330   S = (2/n)^3 sum_p q_p Sx(x_p) Sy(y_p) Sz(z_p)
//   M2M  anotherUpwardPass.c:345-539  z, then y, then x contraction with Cweights
//   proj anotherUpwardPass.c:311-324  P = U^T (S o Kweights)       (atransx.c:48-86)
//   post auxAnotherFMMInteraction.c:398-416  F = (1/L_l) Kweights o (U PF)
//   L2L  anotherDownwardPassX.c:40-211  x, then y, then z interpolation, accumulated
//   L2P  anotherDownwardPassX.c:226-331  phi_p = q_p (2/n)^3 sum F Sx Sy Sz
// The summation order of each output follows the reference loops.
#include <cuda_bf16.h>

#include "common.cuh"

namespace bbfmm {

// FP64 tensor-path M2M / L2L for n = 8 (passes_dmma.cu).
int launch_m2m_dmma(const double *Sc, double *Sp, const double *cw, int64_t first, int64_t count, cudaStream_t s);
int launch_l2l_dmma(const double *Fp, double *Fc, const double *cw, int64_t first, int64_t count, cudaStream_t s);

// Lane t < 3 NN of a warp: S(x_m, c) for axis t / NN (c = x, y, z) and node m = t % NN by
// the Clenshaw recurrence of ComputeSn2 (bbfmm.c:1682-1690), S = 1/2 T_0(x_m) + sum_k
// T_k(x_m) T_k(c) with Tkz[m n + k] = T_k(x_m); other lanes return 0. The warp shares the
// 3 NN values by shuffles instead of every lane evaluating all of them.
template <typename T, int NN>
__device__ __forceinline__ T sn_lane(const T *__restrict__ tkz, int lane, T x, T y, T z) {
  if (lane >= 3 * NN) return (T)0;
  const int a = lane / NN, m = lane % NN;
  const T c = a == 0 ? x : (a == 1 ? y : z);
  T d1 = 0, d2 = 0;
#pragma unroll
  for (int j = NN - 1; j > 0; --j) {
    const T d0 = 2 * c * d1 - d2 + tkz[m * NN + j];
    d2 = d1;
    d1 = d0;
  }
  return c * d1 - d2 + (T)0.5 * tkz[m * NN];
}

// S(x_m, c) for axis idx / NN (c = x, y, z) and node m = idx % NN, idx < 3 NN: the value
// lane idx of sn_lane returns, from the transposed table tkzT[j n + m] = T_j(x_m) (lanes of
// consecutive nodes read consecutive words).
template <typename T, int NN>
__device__ __forceinline__ T sn_value(const T *__restrict__ tkzT, int idx, T x, T y, T z) {
  const int a = idx / NN, m = idx % NN;
  const T c = a == 0 ? x : (a == 1 ? y : z);
  T d1 = 0, d2 = 0;
#pragma unroll
  for (int j = NN - 1; j > 0; --j) {
    const T d0 = 2 * c * d1 - d2 + tkzT[j * NN + m];
    d2 = d1;
    d1 = d0;
  }
  return c * d1 - d2 + (T)0.5 * tkzT[m];
}

template <typename T>
__device__ __forceinline__ T wshfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }

template <typename T> __device__ __forceinline__ const T *tab_tkz(const Tables &t);
template <> __device__ __forceinline__ const double *tab_tkz<double>(const Tables &t) { return t.tkz_d; }
template <> __device__ __forceinline__ const float *tab_tkz<float>(const Tables &t) { return t.tkz_f; }
template <typename T> __device__ __forceinline__ const T *tab_cw(const Tables &t);
template <> __device__ __forceinline__ const double *tab_cw<double>(const Tables &t) { return t.cw_d; }
template <> __device__ __forceinline__ const float *tab_cw<float>(const Tables &t) { return t.cw_f; }

// ----------------------------------------------------------------------------- P2M
// One warp per leaf (grid-stride). pos4 = (x, y, z, q) in leaf-sorted order.
// S_leaf[m * n3 + l], Morton order at maxlev. With Ssplit (mixed mode) the kernel also writes
// the [hi | lo] BF16 split of the same rows (hi plane count x n3, then the lo plane), as
// split_rows_kernel would from S, for the tensor-core up projection.
template <typename T, int NN>
__global__ void __launch_bounds__(128) p2m_kernel(const T *__restrict__ pos4, const int *__restrict__ leaf_start,
                                                  int maxlev, T L, Tables tabs, T *__restrict__ S, int64_t m0,
                                                  int64_t count, __nv_bfloat16 *__restrict__ Ssplit,
                                                  const int64_t *__restrict__ rows) {
  constexpr int N3 = NN * NN * NN;
  constexpr int PER = (N3 + 31) / 32;
  __shared__ T s_tkz[NN * NN];
  const T *tkz = tab_tkz<T>(tabs);
  for (int i = threadIdx.x; i < NN * NN; i += blockDim.x) s_tkz[i] = tkz[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const T len = cell_length<T>(maxlev, L);
  const T ihalf = (T)1 / (len / (T)2);
  const T prefac = (T)2 / (T)NN;
  const T pre3 = prefac * prefac * prefac;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t mm = warp; mm < count; mm += nwarps) {
    const int64_t m = pass_cell(rows, m0, mm);  // leaf; S holds the pass's leaves in order
    int ix, iy, iz;
    morton_to_grid(m, maxlev, ix, iy, iz);  // the set index above bit 3 maxlev is ignored
    const T cx = cell_center_1d<T>(ix, maxlev, L), cy = cell_center_1d<T>(iy, maxlev, L),
            cz = cell_center_1d<T>(iz, maxlev, L);
    T acc[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) acc[k] = 0;
    const int p0 = leaf_start[m], p1 = leaf_start[m + 1];
    for (int p = p0; p < p1; ++p) {
      const T x = ihalf * (pos4[4 * (int64_t)p] - cx);
      const T y = ihalf * (pos4[4 * (int64_t)p + 1] - cy);
      const T z = ihalf * (pos4[4 * (int64_t)p + 2] - cz);
      const T q = pos4[4 * (int64_t)p + 3];
      const T val = sn_lane<T, NN>(s_tkz, lane, x, y, z);
      const T szl = wshfl(val, 2 * NN + lane % NN);  // l3 = lane % NN for every k (32 % NN == 0)
#pragma unroll
      for (int k = 0; k < PER; ++k) {  // N3 is a multiple of 32: every lane has PER outputs
        const int l = lane + 32 * k;
        const int l1 = l / (NN * NN), l2 = (l / NN) % NN;
        const T w = q * wshfl(val, l1) * wshfl(val, NN + l2);
        acc[k] += w * szl;
      }
    }
    T *out = S + mm * N3;
#pragma unroll
    for (int k = 0; k < PER; ++k) out[lane + 32 * k] = pre3 * acc[k];
    if (Ssplit) {
      __nv_bfloat16 *hi = Ssplit + mm * N3, *lo = Ssplit + (count + mm) * N3;
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const double x = (double)(pre3 * acc[k]);
        const __nv_bfloat16 h = __double2bfloat16(x);
        hi[lane + 32 * k] = h;
        lo[lane + 32 * k] = __double2bfloat16(x - (double)__bfloat162float(h));
      }
    }
  }
}

// ----------------------------------------------------------------------------- M2M
// One CTA of 256 threads per parent (grid-stride): children S (level l+1, Morton,
// contiguous block of 8 n^3) -> parent S (level l). All eight children are visited. Each
// thread holds its share of the NEXT parent's children in registers, loaded while the
// current parent is contracted, so the loads of a parent are all in flight at once and
// overlap the arithmetic instead of following it.
template <typename T, int NN>
__global__ void __launch_bounds__(256) m2m_kernel(const T *__restrict__ Sc, T *__restrict__ Sp, int level,
                                                  Tables tabs, int64_t A0, int64_t count) {
  constexpr int N2 = NN * NN, N3 = N2 * NN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sc = reinterpret_cast<T *>(smem_raw);  // 8 * N3
  T *sz = sc + 8 * N3;                       // 4 * N3
  T *sy = sz + 4 * N3;                       // 2 * N3
  __shared__ T cw[2 * N2];
  const T *cwg = tab_cw<T>(tabs);
  for (int i = threadIdx.x; i < 2 * N2; i += blockDim.x) cw[i] = cwg[i];
  const T prefac = (T)2 / (T)NN;
  const T pre3 = prefac * prefac * prefac;
  constexpr int PER = 8 * N3 / 256;  // children values per thread (blockDim = 256)
  T nxt[PER];
  auto fetch = [&](int64_t a) {
    const T *src = Sc + a * 8 * N3 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < PER; ++k) nxt[k] = src[256 * k];
  };
  if ((int64_t)blockIdx.x < count) fetch(blockIdx.x);
  for (int64_t a = blockIdx.x; a < count; a += gridDim.x) {
    const int64_t A = A0 + a;  // parent; Sc holds the children of parents A0 .. A0 + count - 1
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PER; ++k) sc[threadIdx.x + 256 * k] = nxt[k];
    if (a + gridDim.x < count) fetch(a + gridDim.x);
    __syncthreads();
    // z: sz[(j/2) n3 + l1 n + l3] = sum over zbit of sum_m child_j[l1 n + m] C[zbit][l3][m]
    for (int o = threadIdx.x; o < 4 * N3; o += blockDim.x) {
      const int jj = o / N3, rem = o % N3, l1 = rem / NN, l3 = rem % NN;
      T v = 0;
#pragma unroll
      for (int zb = 0; zb < 2; ++zb) {
        const T *ch = sc + (2 * jj + zb) * N3 + l1 * NN;
        const T *c = cw + zb * N2 + l3 * NN;
        T s = 0;
#pragma unroll
        for (int m = 0; m < NN; ++m) s += ch[m] * c[m];
        v += s;
      }
      sz[o] = v;
    }
    __syncthreads();
    // y: sy[(j/2) n3 + l1 n2 + l2 n + l3] = sum over ybit of sum_m sz[j n3 + l1 n2 + m n + l3] C[ybit][l2][m]
    for (int o = threadIdx.x; o < 2 * N3; o += blockDim.x) {
      const int xb = o / N3, rem = o % N3, l1 = rem / N2, l2 = (rem / NN) % NN, l3 = rem % NN;
      T v = 0;
#pragma unroll
      for (int yb = 0; yb < 2; ++yb) {
        const int j = 2 * xb + yb;
        const T *c = cw + yb * N2 + l2 * NN;
        T s = 0;
#pragma unroll
        for (int m = 0; m < NN; ++m) s += sz[j * N3 + l1 * N2 + m * NN + l3] * c[m];
        v += s;
      }
      sy[o] = v;
    }
    __syncthreads();
    // x: S[l1 n2 + l2 n + l3] = sum over xbit of sum_m sy[j n3 + m n2 + l2 n + l3] C[xbit][l1][m]
    T *dst = Sp + A * N3;
    for (int o = threadIdx.x; o < N3; o += blockDim.x) {
      const int l1 = o / N2, l2 = (o / NN) % NN, l3 = o % NN;
      T v = 0;
#pragma unroll
      for (int xb = 0; xb < 2; ++xb) {
        const T *c = cw + xb * N2 + l1 * NN;
        T s = 0;
#pragma unroll
        for (int m = 0; m < NN; ++m) s += sy[xb * N3 + m * N2 + l2 * NN + l3] * c[m];
        v += s;
      }
      dst[o] = v * pre3;
    }
  }
}

// ----------------------------------------------------------------------------- L2L
// One CTA of 256 threads per parent: F_child[j] += (2/n)^3 * interp_j(F_parent), children
// contiguous. The next parent's F and its children's current values are loaded into
// registers while the current parent is interpolated (as in M2M).
template <typename T, int NN>
__global__ void __launch_bounds__(256) l2l_kernel(const T *__restrict__ Fp, T *__restrict__ Fc, int level,
                                                  Tables tabs, int64_t A0, int64_t count) {
  constexpr int N2 = NN * NN, N3 = N2 * NN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *fp = reinterpret_cast<T *>(smem_raw);  // N3
  T *fx = fp + N3;                           // 2 * N3
  T *fy = fx + 2 * N3;                       // 4 * N3
  __shared__ T cw[2 * N2];
  const T *cwg = tab_cw<T>(tabs);
  for (int i = threadIdx.x; i < 2 * N2; i += blockDim.x) cw[i] = cwg[i];
  const T prefac = (T)2 / (T)NN;
  const T pre3 = prefac * prefac * prefac;
  constexpr int PERC = 8 * N3 / 256;         // children values per thread (blockDim = 256)
  constexpr int PERP = (N3 + 255) / 256;     // parent values per thread
  T nc[PERC], np[PERP], old[PERC];
  auto fetch = [&](int64_t a) {
    const T *pp = Fp + (A0 + a) * N3;
#pragma unroll
    for (int k = 0; k < PERP; ++k)
      if (threadIdx.x + 256 * k < N3) np[k] = pp[threadIdx.x + 256 * k];
    const T *cc = Fc + a * 8 * N3 + threadIdx.x;
#pragma unroll
    for (int k = 0; k < PERC; ++k) nc[k] = cc[256 * k];
  };
  if ((int64_t)blockIdx.x < count) fetch(blockIdx.x);
  for (int64_t a = blockIdx.x; a < count; a += gridDim.x) {
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PERP; ++k)
      if (threadIdx.x + 256 * k < N3) fp[threadIdx.x + 256 * k] = np[k];
#pragma unroll
    for (int k = 0; k < PERC; ++k) old[k] = nc[k];
    if (a + gridDim.x < count) fetch(a + gridDim.x);
    __syncthreads();
    // Fx[j n3 + l1 n2 + l2 n + l3] = sum_m F[m n2 + l2 n + l3] C[j][m][l1]
    for (int o = threadIdx.x; o < 2 * N3; o += blockDim.x) {
      const int j = o / N3, rem = o % N3, l1 = rem / N2, l2 = (rem / NN) % NN, l3 = rem % NN;
      T s = 0;
#pragma unroll
      for (int m = 0; m < NN; ++m) s += fp[m * N2 + l2 * NN + l3] * cw[j * N2 + m * NN + l1];
      fx[o] = s;
    }
    __syncthreads();
    // Fy[j n3 + l1 n2 + l2 n + l3] = sum_m Fx[(j/2) n3 + l1 n2 + m n + l3] C[j%2][m][l2]
    for (int o = threadIdx.x; o < 4 * N3; o += blockDim.x) {
      const int j = o / N3, rem = o % N3, l1 = rem / N2, l2 = (rem / NN) % NN, l3 = rem % NN;
      T s = 0;
#pragma unroll
      for (int m = 0; m < NN; ++m) s += fx[(j / 2) * N3 + l1 * N2 + m * NN + l3] * cw[(j % 2) * N2 + m * NN + l2];
      fy[o] = s;
    }
    __syncthreads();
    // Fchild_j[l1l2 n + l3] += pre3 * sum_m Fy[(j/2) n3 + l1l2 n + m] C[j%2][m][l3]
#pragma unroll
    for (int k = 0; k < PERC; ++k) {
      const int o = threadIdx.x + 256 * k;
      const int j = o / N3, rem = o % N3, l12 = rem / NN, l3 = rem % NN;
      T s = 0;
#pragma unroll
      for (int m = 0; m < NN; ++m) s += fy[(j / 2) * N3 + l12 * NN + m] * cw[(j % 2) * N2 + m * NN + l3];
      Fc[a * 8 * N3 + o] = old[k] + pre3 * s;
    }
  }
}

// ----------------------------------------------------------------------------- L2P
// Status word of the passes' bounded waits (0 = every wait completed).
__device__ int g_pass_status = 0;
constexpr uint32_t PASS_WAIT_LIMIT = 1u << 26;
constexpr int PASS_WAIT_CODE = 31;  // an L2P leaf copy did not arrive

constexpr int L2P_DEPTH = 3;   // leaf slots per warp (51 KB per CTA at n = 8 in FP64: 4 CTAs per SM)
constexpr int L2P_WARPS = 4;   // warps per CTA (128 threads)
constexpr int L2P_PCAP = 8;    // particle positions a slot carries (the leaf's first ones)
// one slot: the leaf's n^3 values, then up to L2P_PCAP positions (x, y, z, q)
template <typename T, int NN>
constexpr int l2p_slot_elems() { return NN * NN * NN + 4 * L2P_PCAP; }
template <typename T, int NN>
constexpr int l2p_smem_bytes() { return L2P_WARPS * L2P_DEPTH * l2p_slot_elems<T, NN>() * (int)sizeof(T); }

__device__ __forceinline__ uint32_t pass_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Warp-per-leaf pipeline shared by the L2P kernels: each warp keeps a ring of L2P_DEPTH leaf
// slots in shared memory, filled by bulk copies that complete on the slot's mbarrier -- the
// leaf's n^3 values (one contiguous row of F) and the positions of its first L2P_PCAP
// particles (contiguous in the sorted order) -- so L2P_DEPTH - 1 leaves, positions included,
// are on their way from HBM while one is evaluated, without holding them in registers. The
// warp's leaves are taken in chunks of 32 whose cells and offsets its lanes load together one
// chunk ahead (and whose centres they compute, one leaf per lane), so no leaf waits for its own
// offset loads. Empty leaves take no copy (the slot's barrier is arrived at without bytes).
// body(p0, p1, the slot -- the leaf's n^3 values, then the positions of particles
// p0 .. p0 + L2P_PCAP - 1 --, leaf centre) does the arithmetic. A wait that gives up records
// PASS_WAIT_CODE in g_pass_status and ends the warp's work.
template <typename T, int NN, typename Body>
__device__ __forceinline__ void l2p_pipeline(const int *__restrict__ leaf_start, const T *__restrict__ F,
                                             const T *__restrict__ pos4, int maxlev, T L, int64_t m0, int64_t count,
                                             const int64_t *__restrict__ rows, T *ring_all, uint64_t *bars_all,
                                             int2 *offs_all, Body body) {
  constexpr int N3 = NN * NN * NN, D = L2P_DEPTH, SLOT = l2p_slot_elems<T, NN>();
  static_assert(D < 32, "the slots run at most one offset chunk ahead");
  constexpr uint32_t BYTES = N3 * sizeof(T);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  // leaves of this warp: index i is local row warp + i nwarps
  const int64_t nmine = warp < count ? (count - warp + nwarps - 1) / nwarps : 0;
  T *ring = ring_all + (size_t)wib * D * SLOT;
  uint64_t *bars = bars_all + wib * D;
  int2 *offs = offs_all + wib * D;
  if (lane == 0) {
    for (int d = 0; d < D; ++d)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(pass_smem_u32(bars + d)), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  // chunk c of 32 leaves: lane j holds leaf 32 c + j's cell and offsets (loaded one chunk
  // ahead) and, for the current chunk, its centre
  auto load_chunk = [&](int64_t c, int64_t &m, int &p0, int &p1) {
    const int64_t i = 32 * c + lane;
    m = 0;
    p0 = p1 = 0;
    if (i < nmine) {
      m = pass_cell(rows, m0, warp + i * nwarps);
      p0 = leaf_start[m];
      p1 = leaf_start[m + 1];
    }
  };
  T ccx, ccy, ccz;  // centre of this lane's leaf of the current chunk
  auto centre = [&](int64_t m) {
    int ix, iy, iz;
    morton_to_grid(m, maxlev, ix, iy, iz);
    ccx = cell_center_1d<T>(ix, maxlev, L);
    ccy = cell_center_1d<T>(iy, maxlev, L);
    ccz = cell_center_1d<T>(iz, maxlev, L);
  };
  int64_t cm, nm;  // cells of the current chunk and the next one
  int c0, c1, n0, n1;
  load_chunk(0, cm, c0, c1);
  load_chunk(1, nm, n0, n1);
  centre(cm);
  // lane 0: slot (i % D) <- leaf i, whose offsets are (p0, p1)
  auto issue = [&](int64_t i, int p0, int p1) {
    const int d = (int)(i % D);
    offs[d] = make_int2(p0, p1);
    const uint32_t bar = pass_smem_u32(bars + d);
    const int np = p1 - p0 < L2P_PCAP ? p1 - p0 : L2P_PCAP;
    const uint32_t pbytes = np > 0 ? (uint32_t)np * 4u * (uint32_t)sizeof(T) : 0u;
    const uint32_t tx = p1 > p0 ? BYTES + pbytes : 0u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx) : "memory");
    if (tx) {
      T *slot = ring + (size_t)d * SLOT;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the slot's earlier lane reads
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              pass_smem_u32(slot)),
          "l"(F + (warp + i * nwarps) * N3), "r"(BYTES), "r"(bar)
          : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              pass_smem_u32(slot + N3)),
          "l"(pos4 + 4 * (int64_t)p0), "r"(pbytes), "r"(bar)
          : "memory");
    }
  };
  // offsets of leaf j (in the current chunk of leaf i or the next one), from its lane
  auto offsets_of = [&](int64_t j, int64_t i, int &p0, int &p1) {
    const bool here = (j >> 5) == (i >> 5);
    const int a0 = __shfl_sync(0xffffffffu, c0, (int)(j & 31)), a1 = __shfl_sync(0xffffffffu, c1, (int)(j & 31));
    const int b0 = __shfl_sync(0xffffffffu, n0, (int)(j & 31)), b1 = __shfl_sync(0xffffffffu, n1, (int)(j & 31));
    p0 = here ? a0 : b0;
    p1 = here ? a1 : b1;
  };
  int64_t nxt = 0;  // next leaf to issue
  for (; nxt < D && nxt < nmine; ++nxt) {
    int p0, p1;
    offsets_of(nxt, 0, p0, p1);
    if (lane == 0) issue(nxt, p0, p1);
  }
  auto wait_slot = [&](int64_t i) -> bool {  // bounded wait for leaf i's slot
    const uint32_t bar = pass_smem_u32(bars + (int)(i % D));
    const uint32_t par = (uint32_t)(i / D) & 1u;
    uint32_t done = 0;
    for (uint32_t it = 0; it < PASS_WAIT_LIMIT && !done; ++it)
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(bar), "r"(par)
          : "memory");
    return done != 0;
  };
  int64_t i = 0;
  for (; i < nmine; ++i) {
    if (i > 0 && (i & 31) == 0) {  // next chunk: shift, and fetch the one after it
      cm = nm;
      c0 = n0;
      c1 = n1;
      load_chunk((i >> 5) + 1, nm, n0, n1);
      centre(cm);
    }
    if (!wait_slot(i)) {
      if (lane == 0) atomicCAS(&g_pass_status, 0, PASS_WAIT_CODE);
      break;
    }
    const int d = (int)(i % D);
    const int2 po = offs[d];
    if (po.y > po.x) {
      const int src = (int)(i & 31);
      const T cx = wshfl(ccx, src), cy = wshfl(ccy, src), cz = wshfl(ccz, src);
      body(po.x, po.y, ring + (size_t)d * SLOT, cx, cy, cz);
    }
    __syncwarp();  // every lane has used the slot's values
    if (nxt < nmine) {
      int p0, p1;
      offsets_of(nxt, i, p0, p1);
      if (lane == 0) issue(nxt, p0, p1);
      ++nxt;
    }
  }
  // a warp that gave up still lets the copies it issued land (each wait bounded) before its
  // shared memory can be reused
  for (int64_t j = i + 1; j < nxt; ++j) wait_slot(j);
}

template <typename T> struct Vec4;
template <> struct Vec4<double> { using type = double4; };
template <> struct Vec4<float> { using type = float4; };

// One warp per leaf; phi_sorted[p] = q_p (2/n)^3 sum_l F[l] Sx Sy Sz (assign), the leaf's
// values and first positions taken from its ring slot (l2p_pipeline), two particles per pass.
template <typename T, int NN>
__global__ void __launch_bounds__(128, 4) l2p_kernel(const T *__restrict__ pos4, const int *__restrict__ leaf_start,
                                                  int maxlev, T L, Tables tabs, const T *__restrict__ F,
                                                  T *__restrict__ phi, int64_t m0, int64_t count,
                                                  const int64_t *__restrict__ rows) {
  __shared__ T s_tkzT[NN * NN];  // transposed: s_tkzT[j n + m] = T_j(x_m)
  const T *tkz = tab_tkz<T>(tabs);
  for (int i = threadIdx.x; i < NN * NN; i += blockDim.x) s_tkzT[(i % NN) * NN + i / NN] = tkz[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const T len = cell_length<T>(maxlev, L);
  const T ihalf = (T)1 / (len / (T)2);
  const T prefac = (T)2 / (T)NN;
  const T pre3 = prefac * prefac * prefac;
  using V4 = typename Vec4<T>::type;
  const V4 *p4 = reinterpret_cast<const V4 *>(pos4);
  extern __shared__ __align__(128) unsigned char l2p_ring[];  // l2p_smem_bytes<T, NN>()
  __shared__ __align__(8) uint64_t l2p_bars[L2P_WARPS * L2P_DEPTH];
  __shared__ int2 l2p_offs[L2P_WARPS * L2P_DEPTH];
  // two particles at a time, one per half-warp: lanes s = lane mod 16 of half h hold the
  // leaf's values s + 16 k, evaluate the half's particle's 3 n S values (two per lane at
  // most) into shared memory, read the ones their values need, and reduce over the half
  __shared__ T s_S[L2P_WARPS][2][3 * NN];
  const int h = lane >> 4, s = lane & 15;
  T *sS = s_S[threadIdx.x >> 5][h];
  l2p_pipeline<T, NN>(leaf_start, F, pos4, maxlev, L, m0, count, rows, reinterpret_cast<T *>(l2p_ring), l2p_bars,
                      l2p_offs, [&](int p0, int p1, const T *slot, T cx, T cy, T cz) {
    const T *spos = slot + NN * NN * NN;
    const T *sF = slot + s;  // this lane's values s + 16 k are sF[16 k]
    for (int pb = p0; pb < p1; pb += 2) {
      const int p = pb + h;
      const bool has = p < p1;
      // the slot holds the first L2P_PCAP positions; later ones come from global memory
      const V4 me = !has ? V4{} : (p - p0 < L2P_PCAP ? reinterpret_cast<const V4 *>(spos)[p - p0] : p4[p]);
      const T x = ihalf * (me.x - cx), y = ihalf * (me.y - cy), z = ihalf * (me.z - cz);
      for (int idx = s; idx < 3 * NN; idx += 16) sS[idx] = sn_value<T, NN>(s_tkzT, idx, x, y, z);
      __syncwarp();
      T part = 0;
      if constexpr (NN == 8) {  // value s + 16 k: l1 = k / 4, l2 = s / 8 + 2 (k mod 4), l3 = s mod 8
        T sy[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) sy[b] = sS[NN + (s >> 3) + 2 * b];
#pragma unroll
        for (int a = 0; a < NN; ++a)
          part += sS[a] * (sF[64 * a] * sy[0] + sF[64 * a + 16] * sy[1] + sF[64 * a + 32] * sy[2] +
                           sF[64 * a + 48] * sy[3]);
      } else {  // n = 4, value s + 16 k: l1 = k, l2 = s / 4, l3 = s mod 4
#pragma unroll
        for (int k = 0; k < NN; ++k) part += sF[16 * k] * sS[k];
        part *= sS[NN + (s >> 2)];
      }
      part *= sS[2 * NN + (s & (NN - 1))];
#pragma unroll
      for (int off = 8; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
      if (s == 0 && has) phi[p] = me.w * pre3 * part;
      __syncwarp();  // sS is rewritten for the next pair
    }
  });
}

// --------------------------------------------------------------- projections (GEMM)
// C[out_row(m)][0:N] = scale * cs[0:N] o sum_k A[in_row(m)][k] B[k][0:N] for m < M,
// where rows are mapped between Morton and cpg order at the given level.
// A may be the sum of two sources (T and float) for the split M2L output.
// Register-blocked SIMT GEMM: CTA tile 128 x BN, K-chunks of 16, 256 threads.
// Local row m of a slab starting at cell row0: its cpg index when `which` is the mapped
// side, else m itself.
__device__ __forceinline__ int64_t map_row(int64_t m, int64_t row0, const int64_t *rows, int level, int which,
                                           int mode) {
  return mode == which ? morton_to_cpg_row(pass_cell(rows, row0, m), level) : m;
}

template <typename T, int BN>
__global__ void __launch_bounds__(256) proj_gemm_kernel(int64_t M, int K, int N, const T *__restrict__ A,
                                                        const float *__restrict__ A2, const T *__restrict__ B,
                                                        const T *__restrict__ cs, T scale, T *__restrict__ C,
                                                        int level, int mapmode, int64_t row0, int ldc, int lda,
                                                        const int64_t *__restrict__ rows) {
  constexpr int BM = 128, BK = 16, TN = BN / 16;
  __shared__ T sa[BK][BM + 1];
  __shared__ T sb[BK][BN];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const int64_t m0 = (int64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  T acc[8][TN];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0;
  // each thread loads 8 A elements (rows) per chunk
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = threadIdx.x; e < BM * BK; e += 256) {
      const int r = e / BK, c = e % BK;
      const int64_t m = m0 + r;
      T v = 0;
      if (m < M && k0 + c < K) {
        const int64_t ar = map_row(m, row0, rows, level, MAP_IN_CPG, mapmode);
        v = A[ar * lda + k0 + c];
        if (A2) v += (T)A2[ar * lda + k0 + c];
      }
      sa[c][r] = v;
    }
    for (int e = threadIdx.x; e < BK * BN; e += 256) {
      const int r = e / BN, c = e % BN;
      sb[r][c] = (k0 + r < K && n0 + c < N) ? B[(int64_t)(k0 + r) * N + n0 + c] : (T)0;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      T a[8], b[TN];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = sa[k][ty * 8 + i];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = sb[k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t m = m0 + ty * 8 + i;
    if (m >= M) continue;
    const int64_t cr = map_row(m, row0, rows, level, MAP_OUT_CPG, mapmode);
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const int n = n0 + tx + 16 * j;
      if (n < N) C[cr * ldc + n] = scale * (cs ? cs[n] : (T)1) * acc[i][j];
    }
  }
}

// ----------------------------------------------------------------- permutations
template <typename T, typename TI>
__global__ void gather_pos4_kernel(int N, const int *__restrict__ perm, const TI *__restrict__ xyz,
                                   const TI *__restrict__ q, T *__restrict__ pos4) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int k = perm[i];
    if (xyz) {
      pos4[4 * (int64_t)i] = (T)xyz[3 * (int64_t)k];
      pos4[4 * (int64_t)i + 1] = (T)xyz[3 * (int64_t)k + 1];
      pos4[4 * (int64_t)i + 2] = (T)xyz[3 * (int64_t)k + 2];
    }
    if (q) pos4[4 * (int64_t)i + 3] = (T)q[k];
  }
}

template <typename T, typename TO>
__global__ void scatter_phi_kernel(int N, const int *__restrict__ perm, const T *__restrict__ phis,
                                   TO *__restrict__ phi) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
    phi[perm[i]] = (TO)phis[i];
}

// Morton-ordered r-vectors (reference layout, one level) <-> cpg layout.
template <typename T>
__global__ void morton_to_cpg_kernel(int level, int r, const T *__restrict__ src, T *__restrict__ dst, int inverse) {
  const int64_t total = pow8i(level) * r;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = e / r;
    const int j = (int)(e % r);
    int ix, iy, iz;
    morton_to_grid(m, level, ix, iy, iz);
    const int64_t c = grid_to_cpg(ix, iy, iz, level);
    if (inverse) dst[m * r + j] = src[c * r + j];
    else dst[c * r + j] = src[m * r + j];
  }
}

// ------------------------------------------------------------------ launchers
static int grid_for(int64_t work, int per_block, int cap) {
  int64_t g = (work + per_block - 1) / per_block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

// One wave of `kernel` at `threads` per CTA: SMs x resident CTAs per SM (looked up once per
// kernel), so that grid-stride pipelines run for the whole launch.
template <auto Kernel>
static int resident_grid(int threads, int smem = 0) {
  static int blocks = 0;  // one cache per kernel
  if (!blocks) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // dynamic plus static shared memory above 48 KB needs the opt-in
    if (smem > 0) cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, Kernel, threads, smem);
    blocks = sms * (per > 0 ? per : 1);
  }
  return blocks;
}

// Reads (and with clear, resets) the passes' status word: PASS_WAIT_CODE when an L2P wait gave up.
int pass_status(int clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_pass_status, sizeof(int)) != cudaSuccess) return -1;
  if (clear && v) {
    int z = 0;
    cudaMemcpyToSymbol(g_pass_status, &z, sizeof(int));
  }
  return v;
}

template <typename T>
int launch_p2m(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, T *S, cudaStream_t s,
               int nsets, int64_t first, int64_t count, void *Ssplit, const int64_t *rows) {
  if (count < 0) count = nsets * pow8i(maxlev) - first;
  if (count <= 0) return BBFMM_OK;
  const int grid = grid_for(count, 4, 148 * 64);
  __nv_bfloat16 *sp = (__nv_bfloat16 *)Ssplit;
  if (n == 4) p2m_kernel<T, 4><<<grid, 128, 0, s>>>(pos4, leaf_start, maxlev, L, t, S, first, count, sp, rows);
  else if (n == 8) p2m_kernel<T, 8><<<grid, 128, 0, s>>>(pos4, leaf_start, maxlev, L, t, S, first, count, sp, rows);
  else return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  return bbfmm_set_cuda_error(cudaGetLastError(), "p2m", __FILE__, __LINE__);
}

template <typename T>
int launch_m2m(int n, const T *Sc, T *Sp, int level, const Tables &t, cudaStream_t s, int nsets, int64_t first,
               int64_t count) {
  const int n3 = n * n * n;
  const size_t smem = sizeof(T) * 14 * n3;
  if (count < 0) count = nsets * pow8i(level) - first;
  if (count <= 0) return BBFMM_OK;
  if (sizeof(T) == 8 && n == 8)
    return launch_m2m_dmma((const double *)Sc, (double *)Sp, t.cw_d, first, count, s);
  const int grid = grid_for(count, 1, 148 * 8);
  if (n == 4) {
    m2m_kernel<T, 4><<<grid, 256, smem, s>>>(Sc, Sp, level, t, first, count);
  } else if (n == 8) {
    cudaFuncSetAttribute(m2m_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    m2m_kernel<T, 8><<<grid, 256, smem, s>>>(Sc, Sp, level, t, first, count);
  } else return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  return bbfmm_set_cuda_error(cudaGetLastError(), "m2m", __FILE__, __LINE__);
}

template <typename T>
int launch_l2l(int n, const T *Fp, T *Fc, int level, const Tables &t, cudaStream_t s, int nsets, int64_t first,
               int64_t count) {
  const int n3 = n * n * n;
  const size_t smem = sizeof(T) * 7 * n3;
  if (count < 0) count = nsets * pow8i(level) - first;
  if (count <= 0) return BBFMM_OK;
  if (sizeof(T) == 8 && n == 8)
    return launch_l2l_dmma((const double *)Fp, (double *)Fc, t.cw_d, first, count, s);
  const int grid = grid_for(count, 1, 148 * 8);
  if (n == 4) {
    l2l_kernel<T, 4><<<grid, 256, smem, s>>>(Fp, Fc, level, t, first, count);
  } else if (n == 8) {
    cudaFuncSetAttribute(l2l_kernel<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    l2l_kernel<T, 8><<<grid, 256, smem, s>>>(Fp, Fc, level, t, first, count);
  } else return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  return bbfmm_set_cuda_error(cudaGetLastError(), "l2l", __FILE__, __LINE__);
}

template <typename T>
int launch_l2p(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, const T *F, T *phi,
               cudaStream_t s, int nsets, int64_t first, int64_t count, const int64_t *rows) {
  if (count < 0) count = nsets * pow8i(maxlev) - first;
  if (count <= 0) return BBFMM_OK;
  constexpr int sm4 = l2p_smem_bytes<T, 4>(), sm8 = l2p_smem_bytes<T, 8>();
  if (n == 4)
    l2p_kernel<T, 4><<<grid_for(count, 4, resident_grid<l2p_kernel<T, 4>>(128, sm4)), 128, sm4, s>>>(
        pos4, leaf_start, maxlev, L, t, F, phi, first, count, rows);
  else if (n == 8)
    l2p_kernel<T, 8><<<grid_for(count, 4, resident_grid<l2p_kernel<T, 8>>(128, sm8)), 128, sm8, s>>>(
        pos4, leaf_start, maxlev, L, t, F, phi, first, count, rows);
  else return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  return bbfmm_set_cuda_error(cudaGetLastError(), "l2p", __FILE__, __LINE__);
}

template <typename T>
int launch_proj(int64_t M, int K, int N, const T *A, const float *A2, const T *B, const T *cs, T scale, T *C,
                int level, int mapmode, cudaStream_t s, int64_t row0, int ldc, int lda, const int64_t *rows) {
  if (M <= 0) return BBFMM_OK;
  if (ldc <= 0) ldc = N;
  if (lda <= 0) lda = K;
  if (N >= 64) {
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)((N + 63) / 64));
    proj_gemm_kernel<T, 64><<<grid, 256, 0, s>>>(M, K, N, A, A2, B, cs, scale, C, level, mapmode, row0, ldc, lda,
                                                 rows);
  } else {
    dim3 grid((unsigned)((M + 127) / 128), (unsigned)((N + 31) / 32));
    proj_gemm_kernel<T, 32><<<grid, 256, 0, s>>>(M, K, N, A, A2, B, cs, scale, C, level, mapmode, row0, ldc, lda,
                                                 rows);
  }
  return bbfmm_set_cuda_error(cudaGetLastError(), "proj", __FILE__, __LINE__);
}

template <typename T, typename TI>
int launch_gather(int N, const int *perm, const TI *xyz, const TI *q, T *pos4, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  gather_pos4_kernel<T, TI><<<grid_for(N, 256, 148 * 32), 256, 0, s>>>(N, perm, xyz, q, pos4);
  return bbfmm_set_cuda_error(cudaGetLastError(), "gather", __FILE__, __LINE__);
}

template <typename T, typename TO>
int launch_scatter(int N, const int *perm, const T *phis, TO *phi, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  scatter_phi_kernel<T, TO><<<grid_for(N, 256, 148 * 32), 256, 0, s>>>(N, perm, phis, phi);
  return bbfmm_set_cuda_error(cudaGetLastError(), "scatter", __FILE__, __LINE__);
}

template <typename T>
int launch_morton_cpg(int level, int r, const T *src, T *dst, int inverse, cudaStream_t s) {
  morton_to_cpg_kernel<T><<<grid_for(pow8i(level) * r, 256, 148 * 32), 256, 0, s>>>(level, r, src, dst, inverse);
  return bbfmm_set_cuda_error(cudaGetLastError(), "morton_cpg", __FILE__, __LINE__);
}

#define INST(T)                                                                                           \
  template int launch_p2m<T>(int, const T *, const int *, int, T, const Tables &, T *, cudaStream_t, int,   \
                             int64_t, int64_t, void *, const int64_t *);                                   \
  template int launch_m2m<T>(int, const T *, T *, int, const Tables &, cudaStream_t, int, int64_t, int64_t); \
  template int launch_l2l<T>(int, const T *, T *, int, const Tables &, cudaStream_t, int, int64_t, int64_t); \
  template int launch_l2p<T>(int, const T *, const int *, int, T, const Tables &, const T *, T *,          \
                             cudaStream_t, int, int64_t, int64_t, const int64_t *);                        \
  template int launch_proj<T>(int64_t, int, int, const T *, const float *, const T *, const T *, T, T *,   \
                              int, int, cudaStream_t, int64_t, int, int, const int64_t *);                 \
  template int launch_morton_cpg<T>(int, int, const T *, T *, int, cudaStream_t);
INST(float)
INST(double)
// y[i] += x[i].
template <typename T>
__global__ void add_kernel(int64_t n, const T *__restrict__ x, T *__restrict__ y) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += x[i];
}

template <typename T>
int launch_add(int64_t n, const T *x, T *y, cudaStream_t s) {
  if (n <= 0) return BBFMM_OK;
  add_kernel<T><<<grid_for(n, 256, 148 * 32), 256, 0, s>>>(n, x, y);
  return bbfmm_set_cuda_error(cudaGetLastError(), "add", __FILE__, __LINE__);
}
template int launch_add<double>(int64_t, const double *, double *, cudaStream_t);
template int launch_add<float>(int64_t, const float *, float *, cudaStream_t);

// q[i] = the charge of sorted particle i (pos4's fourth component).
template <typename T>
__global__ void charges_of_kernel(int N, const T *__restrict__ pos4, T *__restrict__ q) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) q[i] = pos4[4 * (int64_t)i + 3];
}

template <typename T>
int launch_charges_of(int N, const T *pos4, T *q, cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  charges_of_kernel<T><<<grid_for(N, 256, 148 * 32), 256, 0, s>>>(N, pos4, q);
  return bbfmm_set_cuda_error(cudaGetLastError(), "charges", __FILE__, __LINE__);
}
template int launch_charges_of<double>(int, const double *, double *, cudaStream_t);
template int launch_charges_of<float>(int, const float *, float *, cudaStream_t);

template int launch_gather<double, double>(int, const int *, const double *, const double *, double *, cudaStream_t);
template int launch_gather<float, double>(int, const int *, const double *, const double *, float *, cudaStream_t);
template int launch_gather<float, float>(int, const int *, const float *, const float *, float *, cudaStream_t);
template int launch_gather<double, float>(int, const int *, const float *, const float *, double *, cudaStream_t);
template int launch_scatter<double, double>(int, const int *, const double *, double *, cudaStream_t);
template int launch_scatter<float, float>(int, const int *, const float *, float *, cudaStream_t);
template int launch_scatter<float, double>(int, const int *, const float *, double *, cudaStream_t);
template int launch_scatter<double, float>(int, const int *, const double *, float *, cudaStream_t);

}  // namespace bbfmm

// ------------------------------------------------------------ L2P with gradient
namespace bbfmm {

// S and dS/dc of sn_value for idx < 3 NN, from the transposed table tkzT[j n + m] = T_j(x_m):
// the Clenshaw recurrence differentiated term by term (e_j = d'_j).
template <typename T, int NN>
__device__ __forceinline__ void sn_value_d(const T *__restrict__ tkzT, int idx, T x, T y, T z, T &sv, T &dv) {
  const int a = idx / NN, m = idx % NN;
  const T c = a == 0 ? x : (a == 1 ? y : z);
  T d1 = 0, d2 = 0, e1 = 0, e2 = 0;
#pragma unroll
  for (int j = NN - 1; j > 0; --j) {
    const T d0 = 2 * c * d1 - d2 + tkzT[j * NN + m];
    const T e0 = 2 * d1 + 2 * c * e1 - e2;
    d2 = d1; d1 = d0;
    e2 = e1; e1 = e0;
  }
  sv = c * d1 - d2 + (T)0.5 * tkzT[m];
  dv = d1 + c * e1 - e2;
}

// One warp per leaf: pot[p] = (2/n)^3 sum_l F[l] Sx Sy Sz (no target factor) and
// fld[3p + a] = d pot / d x_a, with the chain factor 2 / leaf length of the leaf map; the
// same pipeline and particle pairs as l2p_kernel, each half-warp also evaluating dS.
template <typename T, int NN>
__global__ void __launch_bounds__(128, 4) l2p_field_kernel(const T *__restrict__ pos4, const int *__restrict__ leaf_start,
                                                        int maxlev, T L, Tables tabs, const T *__restrict__ F,
                                                        T *__restrict__ pot, T *__restrict__ fld, int64_t m0,
                                                        int64_t count, const int64_t *__restrict__ rows) {
  __shared__ T s_tkzT[NN * NN];  // transposed: s_tkzT[j n + m] = T_j(x_m)
  const T *tkz = tab_tkz<T>(tabs);
  for (int i = threadIdx.x; i < NN * NN; i += blockDim.x) s_tkzT[(i % NN) * NN + i / NN] = tkz[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const T len = cell_length<T>(maxlev, L);
  const T ihalf = (T)1 / (len / (T)2);
  const T prefac = (T)2 / (T)NN;
  const T pre3 = prefac * prefac * prefac;
  using V4 = typename Vec4<T>::type;
  const V4 *p4 = reinterpret_cast<const V4 *>(pos4);
  extern __shared__ __align__(128) unsigned char l2p_ring[];  // l2p_smem_bytes<T, NN>()
  __shared__ __align__(8) uint64_t l2p_bars[L2P_WARPS * L2P_DEPTH];
  __shared__ int2 l2p_offs[L2P_WARPS * L2P_DEPTH];
  // S and dS of the half-warp's particle (3 n each)
  __shared__ T s_S[L2P_WARPS][2][3 * NN], s_D[L2P_WARPS][2][3 * NN];
  const int h = lane >> 4, s = lane & 15;
  T *sS = s_S[threadIdx.x >> 5][h], *sD = s_D[threadIdx.x >> 5][h];
  l2p_pipeline<T, NN>(leaf_start, F, pos4, maxlev, L, m0, count, rows, reinterpret_cast<T *>(l2p_ring), l2p_bars,
                      l2p_offs, [&](int p0, int p1, const T *slot, T cx, T cy, T cz) {
    const T *spos = slot + NN * NN * NN;
    const T *sF = slot + s;  // this lane's values s + 16 k are sF[16 k]
    for (int pb = p0; pb < p1; pb += 2) {
      const int p = pb + h;
      const bool has = p < p1;
      const V4 me = !has ? V4{} : (p - p0 < L2P_PCAP ? reinterpret_cast<const V4 *>(spos)[p - p0] : p4[p]);
      const T x = ihalf * (me.x - cx), y = ihalf * (me.y - cy), z = ihalf * (me.z - cz);
      for (int idx = s; idx < 3 * NN; idx += 16) sn_value_d<T, NN>(s_tkzT, idx, x, y, z, sS[idx], sD[idx]);
      __syncwarp();
      // per l1 row a: A = sum F Sy[l2], B = sum F dSy[l2]; then v = sum Sx A, gx = sum dSx A,
      // gy = sum Sx B (times Sz, or dSz for gz, below)
      T v = 0, gx = 0, gy = 0;
      if constexpr (NN == 8) {  // value s + 16 k: l1 = k / 4, l2 = s / 8 + 2 (k mod 4), l3 = s mod 8
        T sy[4], dy[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          sy[b] = sS[NN + (s >> 3) + 2 * b];
          dy[b] = sD[NN + (s >> 3) + 2 * b];
        }
#pragma unroll
        for (int a = 0; a < NN; ++a) {
          const T f0 = sF[64 * a], f1 = sF[64 * a + 16], f2 = sF[64 * a + 32], f3 = sF[64 * a + 48];
          const T A = f0 * sy[0] + f1 * sy[1] + f2 * sy[2] + f3 * sy[3];
          const T B = f0 * dy[0] + f1 * dy[1] + f2 * dy[2] + f3 * dy[3];
          v += sS[a] * A;
          gx += sD[a] * A;
          gy += sS[a] * B;
        }
      } else {  // n = 4, value s + 16 k: l1 = k, l2 = s / 4, l3 = s mod 4
        T A = 0, Bx = 0;
#pragma unroll
        for (int k = 0; k < NN; ++k) {
          A += sF[16 * k] * sS[k];
          Bx += sF[16 * k] * sD[k];
        }
        const T sy = sS[NN + (s >> 2)], dy = sD[NN + (s >> 2)];
        v = A * sy;
        gx = Bx * sy;
        gy = A * dy;
      }
      const int c = 2 * NN + (s & (NN - 1));
      const T sz = sS[c], dz = sD[c];
      T gz = v * dz;
      v *= sz;
      gx *= sz;
      gy *= sz;
#pragma unroll
      for (int off = 8; off > 0; off >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, off);
        gx += __shfl_xor_sync(0xffffffffu, gx, off);
        gy += __shfl_xor_sync(0xffffffffu, gy, off);
        gz += __shfl_xor_sync(0xffffffffu, gz, off);
      }
      if (s == 0 && has) {
        pot[p] = pre3 * v;
        fld[3 * (int64_t)p] = pre3 * ihalf * gx;
        fld[3 * (int64_t)p + 1] = pre3 * ihalf * gy;
        fld[3 * (int64_t)p + 2] = pre3 * ihalf * gz;
      }
      __syncwarp();  // sS, sD are rewritten for the next pair
    }
  });
}

// Sorted (potential, field) -> caller's order.
template <typename T, typename TO>
__global__ void scatter_field_kernel(int N, const int *__restrict__ perm, const T *__restrict__ pot,
                                     const T *__restrict__ fld, TO *__restrict__ pot_out, TO *__restrict__ fld_out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int k = perm[i];
    if (pot_out) pot_out[k] = (TO)pot[i];
    if (fld_out) {
      fld_out[3 * (int64_t)k] = (TO)fld[3 * (int64_t)i];
      fld_out[3 * (int64_t)k + 1] = (TO)fld[3 * (int64_t)i + 1];
      fld_out[3 * (int64_t)k + 2] = (TO)fld[3 * (int64_t)i + 2];
    }
  }
}

template <typename T>
int launch_l2p_field(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, const T *F,
                     T *pot, T *fld, cudaStream_t s, int nsets, int64_t first, int64_t count, const int64_t *rows) {
  if (count < 0) count = nsets * pow8i(maxlev) - first;
  if (count <= 0) return BBFMM_OK;
  constexpr int sm4 = l2p_smem_bytes<T, 4>(), sm8 = l2p_smem_bytes<T, 8>();
  if (n == 4)
    l2p_field_kernel<T, 4><<<grid_for(count, 4, resident_grid<l2p_field_kernel<T, 4>>(128, sm4)), 128, sm4, s>>>(
        pos4, leaf_start, maxlev, L, t, F, pot, fld, first, count, rows);
  else if (n == 8)
    l2p_field_kernel<T, 8><<<grid_for(count, 4, resident_grid<l2p_field_kernel<T, 8>>(128, sm8)), 128, sm8, s>>>(
        pos4, leaf_start, maxlev, L, t, F, pot, fld, first, count, rows);
  else return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "order n must be 4 or 8");
  return bbfmm_set_cuda_error(cudaGetLastError(), "l2p_field", __FILE__, __LINE__);
}

template <typename T, typename TO>
int launch_scatter_field(int N, const int *perm, const T *pot, const T *fld, TO *pot_out, TO *fld_out,
                         cudaStream_t s) {
  if (N <= 0) return BBFMM_OK;
  scatter_field_kernel<T, TO><<<grid_for(N, 256, 148 * 32), 256, 0, s>>>(N, perm, pot, fld, pot_out, fld_out);
  return bbfmm_set_cuda_error(cudaGetLastError(), "scatter_field", __FILE__, __LINE__);
}

template int launch_l2p_field<double>(int, const double *, const int *, int, double, const Tables &, const double *,
                                      double *, double *, cudaStream_t, int, int64_t, int64_t, const int64_t *);
template int launch_l2p_field<float>(int, const float *, const int *, int, float, const Tables &, const float *,
                                     float *, float *, cudaStream_t, int, int64_t, int64_t, const int64_t *);
template int launch_scatter_field<double, double>(int, const int *, const double *, const double *, double *,
                                                  double *, cudaStream_t);
template int launch_scatter_field<float, float>(int, const int *, const float *, const float *, float *, float *,
                                                cudaStream_t);

}  // namespace bbfmm
