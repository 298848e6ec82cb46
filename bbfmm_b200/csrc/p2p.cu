// Near-field P2P: phi_i += q_i * sum_{B in N(A)} sum_{j in B, r_ij != 0} q_j K(x_j - x_i) over
// the <= 27 neighbour leaves of each leaf, K = 1/r, x/r^3 (homogeneity 2, the reference's
// LAPLACIANFORCE build) or 1/r^4 (homogeneity 4, ONEOVERR4) (reference: anotherNearField.c:
// 141-206 on the CPU, direct.cu:69-209 on the GPU, pair values anotherNearField.c:111-124).
//
// Leaf-tiled design. Source particles are staged in shared memory once per CTA and reused by
// every target of the CTA; the CTA's work is one item of a work list built on the device from
// the leaf offsets (near_work_build):
//  * sparse item: a block of 4 x 4 x 4 leaves (a cell of level maxlev - 2) holding at most
//    2 x (threads per CTA) particles. The 6 x 6 x 6 leaves around it are staged (their
//    particles in x-major, z-fastest leaf order, so the three leaves of each z-row of a
//    target's 3 x 3 x 3 neighbourhood are one contiguous run); each thread takes one or two
//    targets and walks its nine runs in shared memory.
//  * dense item: up to (threads per CTA) targets of one leaf of a block that holds more. Every
//    source of the 27 neighbour leaves interacts with every target, so the CTA streams them
//    through shared memory in tiles and all threads work on every tile; when the chunk has
//    fewer targets than threads, g = threads / targets groups of threads split each tile's
//    sources and their partial sums are added in a fixed order at the end.
// Regions larger than one tile (dense neighbours) stream in tiles in both kinds.
//
// Arithmetic (MODE):
//  * FP64 / FP32: positions and arithmetic in the working precision, 1/sqrt as the reference
//    (the d and s builds).
//  * mixed: the pair's separation and its square in FP64 (FP32 coordinates would cost up to
//    2^-24 h / r_ij of relative error on close pairs, h the leaf length), then 1/r in FP32
//    (rsqrtf and one Newton step) and the pair value times the FP32 charge; per-target
//    Neumaier-compensated FP32 sums added to an FP64 potential.
//
// Robustness: every leaf offset read is clamped to [0, N] and a decreasing or out-of-range
// offset is recorded (the work list's flag and this file's status word), so a malformed
// leaf_start never makes a kernel read or write outside the caller's arrays.
#include <type_traits>

#include "common.cuh"
#include "solver.cuh"

namespace bbfmm {

__device__ int g_p2p_status = 0;  // 0 = ok; else BBFMM_B200_LEAF_RANGE_CODE (leaf offsets out of order)

constexpr int P2P_TILE = 512;        // staged source particles per tile
constexpr int P2P_REGION = 216;      // leaves around a sparse block (6 x 6 x 6)
constexpr int P2P_SCAN_THREADS = 256;  // builder CTA: one block of leaves per thread
constexpr int LEAF_RANGE_CODE = 98;  // = BBFMM_B200_LEAF_RANGE_CODE

__device__ __forceinline__ int clamp_n(int v, int N) { return v < 0 ? 0 : (v > N ? N : v); }

__device__ __forceinline__ void flag_leaf_range(int *flag) {
  atomicExch(flag, 1);
  atomicCAS(&g_p2p_status, 0, LEAF_RANGE_CODE);
}

// ------------------------------------------------------------------ pair arithmetic
// 1/sqrt(rr) in FP32: the hardware estimate refined by one Newton step.
__device__ __forceinline__ float rsqrt_nr(float rr) {
  const float y = rsqrtf(rr);
  return y * fmaf(-0.5f * rr * y, y, 1.5f);
}

// Source particles as staged in shared memory: FP64 / FP32 (x, y, z, q); mixed: FP64
// position and the FP32 charge (converted once per staged source, not once per pair).
struct MixedSrc {
  double x, y, z;
  float q, pad;
};

template <int MODE> struct NearTypes;
template <> struct NearTypes<MODE_D> {
  using P4 = double4; using S = double4; using C = double; using A = double; using R = double;
};
template <> struct NearTypes<MODE_S> {
  using P4 = float4; using S = float4; using C = float; using A = float; using R = float;
};
template <> struct NearTypes<MODE_MIXED> {
  using P4 = double4; using S = MixedSrc; using C = double; using A = float; using R = double;
};

template <int MODE>
__device__ __forceinline__ typename NearTypes<MODE>::S stage_src(const typename NearTypes<MODE>::P4 &p) {
  if constexpr (MODE == MODE_MIXED) return MixedSrc{p.x, p.y, p.z, (float)p.w, 0.f};
  else return p;
}

// Per-target accumulator. v: sum of q_j K (FIELD: q_j / r), c: Neumaier compensation of v
// (mixed), g*: sum of q_j (x_j - x_i) / r^3 (FIELD). H: homogeneity of the kernel.
template <int MODE, int H, bool FIELD>
struct NearAcc {
  using T = NearTypes<MODE>;
  using C = typename T::C;
  using A = typename T::A;
  using Src = typename T::S;
  A v, c, gx, gy, gz;
  __device__ __forceinline__ void zero() { v = c = gx = gy = gz = (A)0; }
  // The pair's contribution to v (0 for coincident points); FIELD: the gradient terms are
  // added here.
  __device__ __forceinline__ A term(C fx, C fy, C fz, const Src &g) {
    const C ex = g.x - fx, ey = g.y - fy, ez = g.z - fz;
    if constexpr (MODE == MODE_MIXED) {
      const double rr = fma(ex, ex, fma(ey, ey, ez * ez));
      const float rrf = (float)rr;
      // rrf = 0 only for coincident points (positions in the unit-scale root cell)
      const float rinv = rrf > 0.f ? rsqrt_nr(rrf) : 0.f;
      // the term enters the sum rounded (an explicit __fmul_rn is never contracted into an
      // addition), so the compensation below sees the exact rounding error of each addition
      float t;
      if constexpr (H == 4) t = __fmul_rn(g.q, (rinv * rinv) * (rinv * rinv));
      else if constexpr (H == 2) t = __fmul_rn(g.q, (float)ex * (rinv * rinv * rinv));
      else t = __fmul_rn(g.q, rinv);
      if constexpr (FIELD) {
        const float t3 = t * rinv * rinv;
        gx += t3 * (float)ex;
        gy += t3 * (float)ey;
        gz += t3 * (float)ez;
      }
      return t;
    } else {
      const C rr = ex * ex + ey * ey + ez * ez;
      if (rr == (C)0) return (C)0;
      const C rinv = (C)1 / sqrt(rr);
      if constexpr (FIELD) {
        const C qr = g.w * rinv, qr3 = qr * rinv * rinv;
        gx += qr3 * ex;
        gy += qr3 * ey;
        gz += qr3 * ez;
        return qr;
      } else {
        const C kern = H == 4 ? rinv * rinv * rinv * rinv : (H == 2 ? ex * rinv * rinv * rinv : rinv);
        return g.w * kern;
      }
    }
  }
  // v += t: plain in FP64 / FP32; mixed: Neumaier-compensated.
  __device__ __forceinline__ void accum(A t) {
    if constexpr (MODE == MODE_MIXED) {
      const float y = v + t;
      c += (fabsf(v) >= fabsf(t)) ? ((v - y) + t) : ((t - y) + v);
      v = y;
    } else {
      v += t;
    }
  }
  __device__ __forceinline__ void add(C fx, C fy, C fz, const Src &g) { accum(term(fx, fy, fz, g)); }
  // Four consecutive sources: mixed mode adds their FP32 sum (t1 + t2) + (t3 + t4) to the
  // compensated sum, a quarter of the compensation work per pair; each partial sum is
  // rounded once, so the error stays of the order of the terms' own FP32 rounding. The other
  // modes add the terms one after the other.
  __device__ __forceinline__ void add4(C fx, C fy, C fz, const Src *g) {
    if constexpr (MODE == MODE_MIXED) {
      const A t1 = term(fx, fy, fz, g[0]), t2 = term(fx, fy, fz, g[1]);
      const A t3 = term(fx, fy, fz, g[2]), t4 = term(fx, fy, fz, g[3]);
      accum((t1 + t2) + (t3 + t4));
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) accum(term(fx, fy, fz, g[k]));
    }
  }
  // Two charge vectors (FIELD, 1/r): the pair's geometry once; this accumulator takes the
  // staged charge and o the source's second charge q2, each with the arithmetic of term/add.
  __device__ __forceinline__ void add2(NearAcc &o, C fx, C fy, C fz, const Src &g, A q2) {
    static_assert(FIELD && H == 1, "two charge vectors: potentials and fields of 1/r");
    const C ex = g.x - fx, ey = g.y - fy, ez = g.z - fz;
    if constexpr (MODE == MODE_MIXED) {
      const double rr = fma(ex, ex, fma(ey, ey, ez * ez));
      const float rrf = (float)rr;
      const float rinv = rrf > 0.f ? rsqrt_nr(rrf) : 0.f;
      const float t = __fmul_rn(g.q, rinv), u = __fmul_rn(q2, rinv);
      const float t3 = t * rinv * rinv, u3 = u * rinv * rinv;
      gx += t3 * (float)ex;
      gy += t3 * (float)ey;
      gz += t3 * (float)ez;
      o.gx += u3 * (float)ex;
      o.gy += u3 * (float)ey;
      o.gz += u3 * (float)ez;
      accum(t);
      o.accum(u);
    } else {
      const C rr = ex * ex + ey * ey + ez * ez;
      if (rr == (C)0) return;  // both terms 0, as add adds
      const C rinv = (C)1 / sqrt(rr);
      const C qr = g.w * rinv, qr3 = qr * rinv * rinv;
      const C ur = q2 * rinv, ur3 = ur * rinv * rinv;
      gx += qr3 * ex;
      gy += qr3 * ey;
      gz += qr3 * ez;
      o.gx += ur3 * ex;
      o.gy += ur3 * ey;
      o.gz += ur3 * ez;
      accum(qr);
      o.accum(ur);
    }
  }
  // add4 for two charge vectors: the same grouping of the four terms in each sum.
  __device__ __forceinline__ void add2x4(NearAcc &o, C fx, C fy, C fz, const Src *g, const A *q2) {
    if constexpr (MODE == MODE_MIXED) {
      NearAcc a = *this, b = o;  // the gradients accumulate term by term; the potentials in fours
      float t[4], u[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const C ex = g[k].x - fx, ey = g[k].y - fy, ez = g[k].z - fz;
        const double rr = fma(ex, ex, fma(ey, ey, ez * ez));
        const float rrf = (float)rr;
        const float rinv = rrf > 0.f ? rsqrt_nr(rrf) : 0.f;
        t[k] = __fmul_rn(g[k].q, rinv);
        u[k] = __fmul_rn(q2[k], rinv);
        const float t3 = t[k] * rinv * rinv, u3 = u[k] * rinv * rinv;
        a.gx += t3 * (float)ex;
        a.gy += t3 * (float)ey;
        a.gz += t3 * (float)ez;
        b.gx += u3 * (float)ex;
        b.gy += u3 * (float)ey;
        b.gz += u3 * (float)ez;
      }
      a.accum((t[0] + t[1]) + (t[2] + t[3]));
      b.accum((u[0] + u[1]) + (u[2] + u[3]));
      *this = a;
      o = b;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) add2(o, fx, fy, fz, g[k], q2[k]);
    }
  }
  // potential part in the output precision
  __device__ __forceinline__ typename T::R pot() const {
    if constexpr (MODE == MODE_MIXED) return (double)v + (double)c;
    else return v;
  }
};

// ------------------------------------------------------------------ work list
// Scratch layout: [int64 item count, int flag, int spare][int64 per tile][items: int2].
// item.x >= 0: sparse block (cell item.x of level maxlev - 2 over the stacked sets; its
// leaves are [64 item.x, 64 item.x + 64)); item.x < 0: leaf m = -item.x - 1, chunk item.y
// (targets leaf_start[m] + item.y * threads ...). With consistent offsets the list never has
// more items than particles: a sparse block holds at least one particle, and a dense block
// (more than 2 x threads >= 128 particles) gives at most particles / threads + 64 items.
// Malformed offsets can ask for more; the list then keeps its first N items and the flag is
// set.
static int64_t near_blocks(int maxlev, int nsets) { return (int64_t)nsets * pow8i(maxlev - 2); }
static int64_t near_tiles(int maxlev, int nsets) {
  return (near_blocks(maxlev, nsets) + P2P_SCAN_THREADS - 1) / P2P_SCAN_THREADS;
}
static size_t near_items_offset(int maxlev, int nsets) { return 16 + 8 * (size_t)near_tiles(maxlev, nsets); }

size_t near_work_bytes(int N, int maxlev, int nsets) {
  return near_items_offset(maxlev, nsets) + sizeof(int2) * (size_t)(N > 0 ? N : 1);
}
const int2 *near_work_items(const void *scratch, int maxlev, int nsets) {
  return (const int2 *)((const char *)scratch + near_items_offset(maxlev, nsets));
}
static int *near_work_flag(void *scratch) { return (int *)((char *)scratch + 8); }

// Items of block b (leaves [64 b, 64 b + 64)): 0 when empty, 1 (sparse) when it holds at
// most 2 x threads particles, else one per `threads` particles of each of its leaves. With
// `items`, writes them at items[base ...], skipping indices >= cap.
// mask (optional): target mask over the cells of a level R <= maxlev (stacked numbering); a
// leaf m is active when mask[m >> mask_shift] is set, mask_shift = 3 (maxlev - R). Only active
// leaves' targets are computed: dense chunks of inactive leaves are not emitted, sparse blocks
// only when one of their leaves is active (the kernel skips the inactive ones' targets).
__device__ __forceinline__ bool leaf_active(const unsigned char *mask, int shift, int64_t m) {
  return !mask || mask[m >> shift];
}

__device__ int64_t block_items(const int *__restrict__ ls, int64_t b, int N, int threads,
                               const unsigned char *__restrict__ mask, int mask_shift, int2 *items = nullptr,
                               int64_t base = 0, int64_t cap = 0) {
  const int64_t m0 = b * 64;
  const int first = clamp_n(ls[m0], N), last = max(first, clamp_n(ls[m0 + 64], N));
  if (last == first) return 0;
  if (last - first <= 2 * threads) {
    bool any = !mask;
    for (int k = 0; k < 64 && !any; ++k) any = leaf_active(mask, mask_shift, m0 + k);
    if (!any) return 0;
    if (items && base < cap) items[base] = make_int2((int)b, 0);
    return 1;
  }
  int64_t n = 0;
  int prev = first;
  for (int k = 1; k <= 64; ++k) {
    const int v = max(prev, min(clamp_n(ls[m0 + k], N), last));
    const int ch = leaf_active(mask, mask_shift, m0 + k - 1) ? (v - prev + threads - 1) / threads : 0;
    if (items)
      for (int j = 0; j < ch && base + n + j < cap; ++j) items[base + n + j] = make_int2(-(int)(m0 + k - 1) - 1, j);
    n += ch;
    prev = v;
  }
  return n;
}

// Exclusive scan of one value per thread over the CTA (blockDim a multiple of 32, <= 1024);
// returns the thread's prefix, *total the CTA's sum.
__device__ int64_t cta_exclusive_scan(int64_t x, int64_t *s_warp, int64_t *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int64_t incl = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    const int64_t v = lane < nw ? s_warp[lane] : 0;
    int64_t wi = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) s_warp[lane] = wi - v;
    if (lane == 31) s_warp[32] = wi;
  }
  __syncthreads();
  const int64_t r = s_warp[w] + incl - x;
  *total = s_warp[32];
  __syncthreads();
  return r;
}

// Pass 1: items per tile of P2P_SCAN_THREADS blocks, and the leaf-range checks (offsets in
// [0, N], non-decreasing, leaf_start[0] = 0, leaf_start[nleaf] = N), swept coalesced.
__global__ void __launch_bounds__(P2P_SCAN_THREADS) near_count_kernel(int64_t nblocks, const int *__restrict__ ls,
                                                                      int N, int threads, int64_t *tiles, int *flag,
                                                                      const unsigned char *mask, int mask_shift) {
  __shared__ int64_t s_warp[33];
  const int64_t b = (int64_t)blockIdx.x * P2P_SCAN_THREADS + threadIdx.x;
  const int64_t x = b < nblocks ? block_items(ls, b, N, threads, mask, mask_shift) : 0;
  int64_t total = 0;
  cta_exclusive_scan(x, s_warp, &total);
  if (threadIdx.x == 0) tiles[blockIdx.x] = total;
  const int64_t nleaf = nblocks * 64;
  const int64_t m0 = (int64_t)blockIdx.x * P2P_SCAN_THREADS * 64;
  const int64_t m1 = min(nleaf, m0 + (int64_t)P2P_SCAN_THREADS * 64);
  bool bad = false;
  for (int64_t m = m0 + threadIdx.x; m < m1; m += P2P_SCAN_THREADS) {
    const int a = ls[m], e = ls[m + 1];
    bad |= a < 0 || e < a || e > N;
    if (m == 0) bad |= a != 0;
    if (m + 1 == nleaf) bad |= e != N;
  }
  if (bad) flag_leaf_range(flag);
}

// Pass 2 (one CTA): exclusive scan of the tile counts in place; *count = items.
__global__ void __launch_bounds__(1024) near_scan_tiles_kernel(int64_t ntiles, int64_t *tiles, int64_t *count) {
  __shared__ int64_t s_warp[33];
  int64_t carry = 0;
  for (int64_t t0 = 0; t0 < ntiles; t0 += blockDim.x) {
    const int64_t t = t0 + threadIdx.x;
    const int64_t x = t < ntiles ? tiles[t] : 0;
    int64_t total = 0;
    const int64_t ex = cta_exclusive_scan(x, s_warp, &total);
    if (t < ntiles) tiles[t] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *count = carry;
}

// Pass 3: every block writes its items at its offset (indices below cap only).
__global__ void __launch_bounds__(P2P_SCAN_THREADS) near_emit_kernel(int64_t nblocks, const int *__restrict__ ls,
                                                                     int N, int threads, const int64_t *tiles,
                                                                     int2 *items, int64_t cap,
                                                                     const unsigned char *mask, int mask_shift) {
  __shared__ int64_t s_warp[33];
  const int64_t b = (int64_t)blockIdx.x * P2P_SCAN_THREADS + threadIdx.x;
  const int64_t x = b < nblocks ? block_items(ls, b, N, threads, mask, mask_shift) : 0;
  int64_t total = 0;
  const int64_t ex = cta_exclusive_scan(x, s_warp, &total);
  if (x > 0) block_items(ls, b, N, threads, mask, mask_shift, items, tiles[blockIdx.x] + ex, cap);
}

// Builds the work list for `threads` threads per CTA into `scratch` (near_work_bytes). With
// nitems_host, synchronises `s` and returns the item count (at most N; a larger count sets
// *flag_host) and the leaf-range flag.
int near_work_build(int N, const int *leaf_start, int maxlev, int nsets, int threads, void *scratch, cudaStream_t s,
                    int *nitems_host, int *flag_host, const unsigned char *mask, int mask_level) {
  const int mask_shift = mask ? 3 * (maxlev - mask_level) : 0;
  if (mask && (mask_level < 0 || mask_level > maxlev)) return bbfmm_set_error(BBFMM_ERR_ARG, "mask level out of range");
  if (maxlev < BBFMM_MINLEV) return bbfmm_set_error(BBFMM_ERR_ARG, "near field: maxlev >= 2");
  if (threads != 64 && threads != 128 && threads != 256)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: 64, 128 or 256 threads per block");
  int64_t *count = (int64_t *)scratch;
  int64_t *tiles = count + 2;
  int2 *items = (int2 *)((char *)scratch + near_items_offset(maxlev, nsets));
  const int64_t nblocks = near_blocks(maxlev, nsets), ntiles = near_tiles(maxlev, nsets);
  BBFMM_CUDA_OK(cudaMemsetAsync(scratch, 0, 16, s));
  near_count_kernel<<<(unsigned)ntiles, P2P_SCAN_THREADS, 0, s>>>(nblocks, leaf_start, N, threads, tiles,
                                                                  near_work_flag(scratch), mask, mask_shift);
  near_scan_tiles_kernel<<<1, 1024, 0, s>>>(ntiles, tiles, count);
  near_emit_kernel<<<(unsigned)ntiles, P2P_SCAN_THREADS, 0, s>>>(nblocks, leaf_start, N, threads, tiles, items,
                                                                 (int64_t)N, mask, mask_shift);
  BBFMM_CUDA_OK(cudaGetLastError());
  if (nitems_host || flag_host) {
    int64_t h[2] = {0, 0};
    BBFMM_CUDA_OK(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
    BBFMM_CUDA_OK(cudaStreamSynchronize(s));
    const int64_t n = h[0];
    const int flag = (int)(h[1] & 0xffffffff) != 0 || n > N;
    if (nitems_host) *nitems_host = (int)(n > N ? N : n);
    if (flag_host) *flag_host = flag;
  }
  return BBFMM_OK;
}

// ------------------------------------------------------------------ the near-field kernel
// RHS2: a second charge vector q2 (sorted order) whose potentials and fields go to pot2 and
// fld2, from the same pair evaluations.
template <int MODE, int H, bool FIELD, bool RHS2 = false>
__global__ void __launch_bounds__(256) near_kernel(int N, const typename NearTypes<MODE>::P4 *__restrict__ pos4,
                                                   const int *__restrict__ leaf_start, int maxlev,
                                                   const int2 *__restrict__ items, int nitems,
                                                   typename NearTypes<MODE>::R *__restrict__ pot,
                                                   typename NearTypes<MODE>::R *__restrict__ fld, int *flag,
                                                   const unsigned char *__restrict__ mask, int mask_shift,
                                                   const typename NearTypes<MODE>::R *__restrict__ q2 = nullptr,
                                                   typename NearTypes<MODE>::R *__restrict__ pot2 = nullptr,
                                                   typename NearTypes<MODE>::R *__restrict__ fld2 = nullptr) {
  using NT = NearTypes<MODE>;
  using P4 = typename NT::P4;
  using C = typename NT::C;
  using R = typename NT::R;
  using Src = typename NT::S;
  using Acc = NearAcc<MODE, H, FIELD>;
  using A = typename NT::A;
  static_assert(sizeof(Acc) * 256 <= sizeof(Src) * P2P_TILE, "group partials fit the tile buffer");
  __shared__ __align__(16) unsigned char s_buf[sizeof(Src) * P2P_TILE];
  __shared__ A s_q2[RHS2 ? P2P_TILE : 1];  // the staged sources' second charges
  __shared__ int s_start[P2P_REGION], s_off[P2P_REGION + 1];
  __shared__ unsigned char s_tleaf[512], s_act[P2P_REGION];
  Src *s_src = reinterpret_cast<Src *>(s_buf);
  const int nt = blockDim.x, tid = threadIdx.x;
  const int ncpd = 1 << maxlev;
  const int64_t per_set = pow8i(maxlev), per_set_b = pow8i(maxlev - 2);
  for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
    const int2 item = items[it];
    const bool dense = item.x < 0;
    int64_t setbase;
    int ox, oy, oz, RR, t0, t1;
    if (dense) {
      const int64_t m = -(int64_t)item.x - 1;
      setbase = m - (m & (per_set - 1));
      int ix, iy, iz;
      morton_to_grid(m & (per_set - 1), maxlev, ix, iy, iz);
      ox = ix - 1; oy = iy - 1; oz = iz - 1;
      RR = 3;
      const int a = clamp_n(leaf_start[m], N), e = max(a, clamp_n(leaf_start[m + 1], N));
      t0 = min(e, a + item.y * nt);
      t1 = min(e, t0 + nt);
    } else {
      const int64_t b = item.x;
      setbase = (b - (b & (per_set_b - 1))) * 64;
      int bx, by, bz;
      morton_to_grid(b & (per_set_b - 1), maxlev - 2, bx, by, bz);
      ox = 4 * bx - 1; oy = 4 * by - 1; oz = 4 * bz - 1;
      RR = 6;
      t0 = clamp_n(leaf_start[b * 64], N);
      t1 = max(t0, clamp_n(leaf_start[b * 64 + 64], N));
      if (t1 - t0 > 2 * nt) {  // only a leaf_start changed since the list was built gets here
        if (tid == 0) flag_leaf_range(flag);
        t1 = t0 + 2 * nt;
      }
    }
    const int nreg = RR * RR * RR;
    __syncthreads();  // the previous item is done with shared memory
    // region leaves (x-major, z fastest): first particle and count
    for (int rho = tid; rho < nreg; rho += nt) {
      const int rx = rho / (RR * RR), ry = (rho / RR) % RR, rz = rho % RR;
      const int gx = ox + rx, gy = oy + ry, gz = oz + rz;
      int s0 = 0, cnt = 0;
      bool act = false;
      if (gx >= 0 && gx < ncpd && gy >= 0 && gy < ncpd && gz >= 0 && gz < ncpd) {
        const int64_t B = setbase + grid_to_morton(gx, gy, gz, maxlev);
        s0 = clamp_n(leaf_start[B], N);
        cnt = max(0, clamp_n(leaf_start[B + 1], N) - s0);
        act = leaf_active(mask, mask_shift, B);
      }
      s_start[rho] = s0;
      s_off[rho] = cnt;
      s_act[rho] = act;
    }
    __syncthreads();
    // exclusive scan of the counts (one warp; <= 7 entries per lane)
    if (tid < 32) {
      const int per = (nreg + 31) / 32, b0 = tid * per;
      int loc = 0;
      for (int k = 0; k < per; ++k)
        if (b0 + k < nreg) loc += s_off[b0 + k];
      int incl = loc;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (tid >= o) incl += y;
      }
      int run = incl - loc;
      for (int k = 0; k < per; ++k)
        if (b0 + k < nreg) {
          const int cnt = s_off[b0 + k];
          s_off[b0 + k] = run;
          run += cnt;
        }
      if (tid == 31) s_off[nreg] = incl;
    }
    // sparse: the region leaf of every target (the 4 x 4 x 4 central leaves hold them)
    const int ntg = t1 - t0;
    if (!dense)
      for (int k = tid; k < ntg; k += nt) s_tleaf[k] = 255;
    __syncthreads();
    if (!dense) {
      for (int rho = tid; rho < nreg; rho += nt) {
        const int rx = rho / 36, ry = (rho / 6) % 6, rz = rho % 6;
        if (rx < 1 || rx > 4 || ry < 1 || ry > 4 || rz < 1 || rz > 4 || !s_act[rho]) continue;
        const int a = max(s_start[rho], t0), e = min(s_start[rho] + s_off[rho + 1] - s_off[rho], t1);
        for (int p = a; p < e; ++p) s_tleaf[p - t0] = (unsigned char)rho;
      }
    }
    __syncthreads();
    const int total = s_off[nreg];
    // targets: dense -> one per thread of group 0 .. g-1 (slot = tid % ntg); sparse -> tid, tid + nt
    const int g = dense && ntg > 0 ? nt / ntg : 1;
    const int slot = dense && ntg > 0 ? tid % ntg : tid, grp = dense && ntg > 0 ? tid / ntg : 0;
    const bool active = dense ? (ntg > 0 && grp < g) : true;
    Acc acc[2], acc2[2];
    C fx[2], fy[2], fz[2];
    int trho[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      acc[k].zero();
      acc2[k].zero();
      fx[k] = fy[k] = fz[k] = (C)0;
      trho[k] = 255;
      const int i = t0 + slot + k * nt;
      if (active && (dense ? k == 0 : slot + k * nt < ntg)) {
        const P4 f = pos4[i];
        fx[k] = f.x; fy[k] = f.y; fz[k] = f.z;
        trho[k] = dense ? 13 : s_tleaf[i - t0];
      }
    }
    for (int tile0 = 0; tile0 < total; tile0 += P2P_TILE) {
      const int tn = min(P2P_TILE, total - tile0);
      __syncthreads();  // the previous tile is consumed
      for (int k = tid; k < tn; k += nt) {
        const int v = tile0 + k;
        int lo = 0, hi = nreg;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= v) lo = mid;
          else hi = mid;
        }
        const int src = s_start[lo] + (v - s_off[lo]);
        s_src[k] = stage_src<MODE>(pos4[src]);
        if constexpr (RHS2) s_q2[k] = (A)q2[src];
      }
      __syncthreads();
      if (dense) {
        if (trho[0] != 255) {
          // group grp takes the contiguous slice [j0, j1) of the tile
          const int j0 = (int)((int64_t)tn * grp / g), j1 = (int)((int64_t)tn * (grp + 1) / g);
          int j = j0;
          if constexpr (RHS2) {
            for (; j + 4 <= j1; j += 4) acc[0].add2x4(acc2[0], fx[0], fy[0], fz[0], s_src + j, s_q2 + j);
            for (; j < j1; ++j) acc[0].add2(acc2[0], fx[0], fy[0], fz[0], s_src[j], s_q2[j]);
          } else {
            for (; j + 4 <= j1; j += 4) acc[0].add4(fx[0], fy[0], fz[0], s_src + j);
            for (; j < j1; ++j) acc[0].add(fx[0], fy[0], fz[0], s_src[j]);
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          if (trho[k] == 255) continue;
          const int rx = trho[k] / 36, ry = (trho[k] / 6) % 6, rz = trho[k] % 6;
          // the nine z-runs rz-1 .. rz+1 of rows (rx + dx, ry + dy), walked as one sequence so
          // that lanes with short runs do not wait at every run's end
          auto run = [&](int u, int &a, int &e) {
            const int r0 = ((rx + u / 3 - 1) * 6 + ry + u % 3 - 1) * 6 + rz - 1;
            a = max(s_off[r0], tile0) - tile0;
            e = min(s_off[r0 + 3], tile0 + tn) - tile0;
          };
          int u = 0, j, e;
          run(0, j, e);
          for (;;) {
            if (j >= e) {
              if (++u == 9) break;
              run(u, j, e);
              continue;
            }
            if constexpr (RHS2) acc[k].add2(acc2[k], fx[k], fy[k], fz[k], s_src[j], s_q2[j]);
            else acc[k].add(fx[k], fy[k], fz[k], s_src[j]);
            ++j;
          }
        }
      }
    }
    // outputs
    if (dense) {
      if (ntg <= 0) continue;
      Acc *red = reinterpret_cast<Acc *>(s_buf);
      // the groups' partial sums of one charge vector, added in a fixed order
      auto flush = [&](const Acc &mine, R *po, R *fl) {
        __syncthreads();  // the last tile (or the previous flush) is consumed
        if (active) red[tid] = mine;
        __syncthreads();
        if (tid < ntg) {
          R p = (R)0, qx = (R)0, qy = (R)0, qz = (R)0;
          for (int k = 0; k < g; ++k) {
            const Acc &a = red[tid + k * ntg];
            p += a.pot();
            if constexpr (FIELD) {
              qx += (R)a.gx;
              qy += (R)a.gy;
              qz += (R)a.gz;
            }
          }
          const int i = t0 + tid;
          if constexpr (FIELD) {
            po[i] += p;
            fl[3 * (int64_t)i] += qx;
            fl[3 * (int64_t)i + 1] += qy;
            fl[3 * (int64_t)i + 2] += qz;
          } else {
            po[i] += (R)pos4[i].w * p;
          }
        }
      };
      flush(acc[0], pot, fld);
      if constexpr (RHS2) flush(acc2[0], pot2, fld2);
    } else {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (trho[k] == 255) continue;
        const int i = t0 + slot + k * nt;
        if constexpr (FIELD) {
          pot[i] += acc[k].pot();
          fld[3 * (int64_t)i] += (R)acc[k].gx;
          fld[3 * (int64_t)i + 1] += (R)acc[k].gy;
          fld[3 * (int64_t)i + 2] += (R)acc[k].gz;
          if constexpr (RHS2) {
            pot2[i] += acc2[k].pot();
            fld2[3 * (int64_t)i] += (R)acc2[k].gx;
            fld2[3 * (int64_t)i + 1] += (R)acc2[k].gy;
            fld2[3 * (int64_t)i + 2] += (R)acc2[k].gz;
          }
        } else {
          pot[i] += (R)pos4[i].w * acc[k].pot();
        }
      }
    }
  }
}

template <int MODE, int H, bool FIELD>
static void near_launch(int N, const void *pos4, const int *leaf_start, int maxlev, const int2 *items, int nitems,
                        int threads, void *pot, void *fld, int *flag, const unsigned char *mask, int mask_shift,
                        cudaStream_t s) {
  using NT = NearTypes<MODE>;
  near_kernel<MODE, H, FIELD><<<nitems, threads, 0, s>>>(N, (const typename NT::P4 *)pos4, leaf_start, maxlev, items,
                                                         nitems, (typename NT::R *)pot, (typename NT::R *)fld, flag,
                                                         mask, mask_shift);
}

int launch_near(int mode, int homogen, int N, const void *pos4, const int *leaf_start, int maxlev,
                const void *work, int nsets, int nitems, int threads, void *pot, void *fld, cudaStream_t s,
                const unsigned char *mask, int mask_level) {
  const int mask_shift = mask ? 3 * (maxlev - mask_level) : 0;
  if (N <= 0 || nitems <= 0) return BBFMM_OK;
  if (threads != 64 && threads != 128 && threads != 256)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: 64, 128 or 256 threads per block");
  if (homogen != 1 && homogen != 2 && homogen != 4)
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "near field: kernel homogeneity 1 (1/r), 2 (x/r^3) or 4 (1/r^4)");
  if (fld && homogen != 1) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "near-field gradients are for 1/r");
  const int2 *items = near_work_items(work, maxlev, nsets);
  int *flag = near_work_flag(const_cast<void *>(work));
#define NEAR_CASE(M)                                                                                     \
  if (fld) near_launch<M, 1, true>(N, pos4, leaf_start, maxlev, items, nitems, threads, pot, fld, flag, mask, mask_shift, s); \
  else if (homogen == 1) near_launch<M, 1, false>(N, pos4, leaf_start, maxlev, items, nitems, threads, pot, nullptr, flag, mask, mask_shift, s); \
  else if (homogen == 2) near_launch<M, 2, false>(N, pos4, leaf_start, maxlev, items, nitems, threads, pot, nullptr, flag, mask, mask_shift, s); \
  else near_launch<M, 4, false>(N, pos4, leaf_start, maxlev, items, nitems, threads, pot, nullptr, flag, mask, mask_shift, s);
  if (mode == MODE_D) { NEAR_CASE(MODE_D) }
  else if (mode == MODE_S) { NEAR_CASE(MODE_S) }
  else if (mode == MODE_MIXED) { NEAR_CASE(MODE_MIXED) }
  else return bbfmm_set_error(BBFMM_ERR_ARG, "near field: unknown precision mode");
#undef NEAR_CASE
  return bbfmm_set_cuda_error(cudaGetLastError(), "near field", __FILE__, __LINE__);
}

// Potentials and fields of 1/r for two charge vectors in one pass over the pairs: the charges
// in pos4's fourth component into (pot, fld), the sorted charges q2 into (pot2, fld2), each
// added and each with the arithmetic of a launch_near call of its own.
int launch_near2(int mode, int N, const void *pos4, const int *leaf_start, int maxlev, const void *work, int nsets,
                 int nitems, int threads, const void *q2, void *pot, void *fld, void *pot2, void *fld2, cudaStream_t s,
                 const unsigned char *mask, int mask_level) {
  const int mask_shift = mask ? 3 * (maxlev - mask_level) : 0;
  if (N <= 0 || nitems <= 0) return BBFMM_OK;
  if (threads != 64 && threads != 128 && threads != 256)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: 64, 128 or 256 threads per block");
  if (!q2 || !pot || !fld || !pot2 || !fld2) return bbfmm_set_error(BBFMM_ERR_ARG, "near field: null pointer");
  const int2 *items = near_work_items(work, maxlev, nsets);
  int *flag = near_work_flag(const_cast<void *>(work));
#define NEAR2_CASE(M)                                                                                       \
  {                                                                                                          \
    using NT = NearTypes<M>;                                                                                 \
    using R = typename NT::R;                                                                                \
    near_kernel<M, 1, true, true><<<nitems, threads, 0, s>>>(                                                \
        N, (const typename NT::P4 *)pos4, leaf_start, maxlev, items, nitems, (R *)pot, (R *)fld, flag, mask, \
        mask_shift, (const R *)q2, (R *)pot2, (R *)fld2);                                                    \
  }
  if (mode == MODE_D) NEAR2_CASE(MODE_D)
  else if (mode == MODE_S) NEAR2_CASE(MODE_S)
  else if (mode == MODE_MIXED) NEAR2_CASE(MODE_MIXED)
  else return bbfmm_set_error(BBFMM_ERR_ARG, "near field: unknown precision mode");
#undef NEAR2_CASE
  return bbfmm_set_cuda_error(cudaGetLastError(), "near field (two charge vectors)", __FILE__, __LINE__);
}

// Reads and clears this file's status word (0, or LEAF_RANGE_CODE after malformed offsets).
int near_status(int clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_p2p_status, sizeof(int)) != cudaSuccess) return -1;
  if (clear && v) {
    const int z = 0;
    cudaMemcpyToSymbol(g_p2p_status, &z, sizeof(int));
  }
  return v;
}

}  // namespace bbfmm

// ====================================================== near-field C-ABI entry points
#include <mutex>

#include "../../include/bbfmm_b200.h"

static_assert(bbfmm::LEAF_RANGE_CODE == BBFMM_B200_LEAF_RANGE_CODE, "status code");

namespace {

// Shared body of the two entry points: builds the work list in `scratch` (sized by
// near_work_bytes), runs the near field and synchronises `st` to check the leaf offsets.
int near_field_run(int N, int maxlev, const double *xyzq, const int *leaf_start, double *phi, int mode,
                   cudaStream_t st, void *scratch) {
  int nitems = 0, flag = 0;
  int rc = bbfmm::near_work_build(N, leaf_start, maxlev, 1, 128, scratch, st, &nitems, &flag);
  if (rc != BBFMM_OK) return rc;
  if (!flag) {
    const int m = mode == BBFMM_B200_MODE_MIXED ? bbfmm::MODE_MIXED : bbfmm::MODE_D;
    rc = bbfmm::launch_near(m, 1, N, xyzq, leaf_start, maxlev, scratch, 1, nitems, 128, phi, nullptr, st);
    if (rc != BBFMM_OK) return rc;
    cudaError_t e = cudaMemcpyAsync(&flag, (char *)scratch + 8, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    rc = bbfmm_set_cuda_error(e, "near field", __FILE__, __LINE__);
    if (rc != BBFMM_OK) return rc;
  }
  if (flag)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field: leaf_start must rise from 0 to N without decreasing");
  return BBFMM_OK;
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

// Scratch of the allocation-free entry point: the work list of up to
// BBFMM_B200_NOALLOC_MAX_PARTICLES particles at any depth up to 10 (near_work_bytes). Every
// GPU that loads the library holds this array until the process exits.
constexpr size_t kNoallocBytes = (size_t)BBFMM_B200_NOALLOC_SCRATCH_BYTES;
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
  void *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, bbfmm::near_work_bytes(N, maxlev, 1));
  if (e != cudaSuccess) return bbfmm_set_error(BBFMM_ERR_NOMEM, "near field: scratch allocation failed");
  rc = near_field_run(N, maxlev, xyzq, leaf_start, phi, mode, st, scratch);
  e = cudaStreamSynchronize(st);  // the scratch is freed below
  if (rc == BBFMM_OK) rc = bbfmm_set_cuda_error(e, "near field", __FILE__, __LINE__);
  cudaFree(scratch);
  return rc;
}

int bbfmm_b200_near_field_noalloc(int N, int maxlev, double L, const double *xyzq, const int *leaf_start,
                                  double *phi, int mode, void *stream) {
  int rc = near_field_check(N, maxlev, L, xyzq, leaf_start, phi, mode);
  if (rc != BBFMM_OK || N == 0) return rc;
  if (N > BBFMM_B200_NOALLOC_MAX_PARTICLES)
    return bbfmm_set_error(BBFMM_ERR_ARG,
                           "near field (no allocation): N exceeds BBFMM_B200_NOALLOC_MAX_PARTICLES = 262144");
  if (bbfmm::near_work_bytes(N, maxlev, 1) > kNoallocBytes)
    return bbfmm_set_error(BBFMM_ERR_ARG, "near field (no allocation): work list exceeds the static scratch");
  void *base = nullptr;
  rc = noalloc_scratch(&base);
  if (rc != BBFMM_OK) return rc;
  // The call clears the list's counters and then writes every entry it reads, so the
  // previous call's contents need no clearing.
  return near_field_run(N, maxlev, xyzq, leaf_start, phi, mode, (cudaStream_t)stream, base);
}

}  // extern "C"
