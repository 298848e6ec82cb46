// Octree build on the device: the leaf assignment of anotherFMMDistribute.c:258-298
// (truncating (x + L/2) / leaf_length, clamped to the last leaf) and the stable sort of the
// particles into leaves in Morton (reference) order, i.e. the particle order of the
// reference's fieldlist (anotherFMMDistribute.c:431-473) -- the same perm and leaf_start as
// the host routine bbfmm_sort_particles, for positions that are already on the GPU.
//
//  * tree_keys_kernel: Morton leaf index of every particle (additions and products with
//    explicit rounding, so no contraction can move a particle across a leaf boundary that
//    the host arithmetic puts it on one side of).
//  * an LSD radix sort of (key, index) with 4-bit digits, 3 maxlev bits in all: per pass,
//    per-block digit counts (blocks of 4,096 particles), one exclusive scan over (digit,
//    block), and a stable scatter in which every thread's 16 consecutive items get their
//    ranks from a block-wide scan of the per-thread digit counts. Each pass keeps the
//    relative order of equal digits, so the result is the stable order by key.
//  * leaf_start[m] = the first sorted position whose key is >= m (a binary search per leaf).
//
// Several particle sets stacked for one solver (a batch group: set slot j owns the leaves
// [j 8^maxlev, (j+1) 8^maxlev)) are one sort: slot j's particles are the range [off_j, off_j +
// count_j) of the positions array, their keys j 8^maxlev + leaf and their indices global, so
// the stable order is each set's own stable leaf order, set after set -- what per-set host
// sorts concatenated give.
#include <utility>
#include <vector>

#include "common.cuh"

namespace bbfmm {
namespace tr {

constexpr int THREADS = 256, ITEMS = 16, TILE = THREADS * ITEMS, DIGITS = 16;

__device__ int g_tree_status;  // 1: a particle outside the root cell

template <typename T> __device__ __forceinline__ T add_rn(T a, T b);
template <> __device__ __forceinline__ double add_rn<double>(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float add_rn<float>(float a, float b) { return __fadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T mul_rn(T a, T b);
template <> __device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }

// Sort item i belongs to slot j with base[j] <= i < base[j + 1] (base[0] = 0, base[nseg] = N;
// empty slots repeat a base) and is particle g = off[j] + i - base[j] of xyz.
template <typename T>
__global__ void tree_keys_kernel(int N, int nseg, const int *__restrict__ base, const int *__restrict__ off,
                                 const T *__restrict__ xyz, T L0half, T iLm, int maxlev, int *__restrict__ key,
                                 int *__restrict__ idx) {
  const int ncpd = 1 << maxlev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    int lo = 0, hi = nseg;  // base[lo] <= i < base[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (base[mid] <= i) lo = mid;
      else hi = mid;
    }
    const int g = off[lo] + (i - base[lo]);
    const T x = xyz[3 * (int64_t)g], y = xyz[3 * (int64_t)g + 1], z = xyz[3 * (int64_t)g + 2];
    if (!(x >= -L0half && x <= L0half && y >= -L0half && y <= L0half && z >= -L0half && z <= L0half)) {
      g_tree_status = 1;
      key[i] = 0;
      idx[i] = g;
      continue;
    }
    int ix = (int)mul_rn<T>(add_rn<T>(x, L0half), iLm);
    int iy = (int)mul_rn<T>(add_rn<T>(y, L0half), iLm);
    int iz = (int)mul_rn<T>(add_rn<T>(z, L0half), iLm);
    if (ix > ncpd - 1) ix = ncpd - 1;
    if (iy > ncpd - 1) iy = ncpd - 1;
    if (iz > ncpd - 1) iz = ncpd - 1;
    key[i] = (int)(((int64_t)lo << (3 * maxlev)) + grid_to_morton(ix, iy, iz, maxlev));
    idx[i] = g;
  }
}

// hist[d * nb + b] = number of items of block b whose digit (key >> shift) & 15 is d.
__global__ void __launch_bounds__(THREADS) radix_hist_kernel(int N, const int *__restrict__ key, int shift,
                                                              int *__restrict__ hist) {
  __shared__ int cnt[DIGITS];
  if (threadIdx.x < DIGITS) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t b0 = (int64_t)blockIdx.x * TILE;
  for (int u = 0; u < ITEMS; ++u) {
    const int64_t i = b0 + u * THREADS + threadIdx.x;
    if (i < N) atomicAdd(&cnt[(key[i] >> shift) & (DIGITS - 1)], 1);
  }
  __syncthreads();
  if (threadIdx.x < DIGITS) hist[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Exclusive scan of one chunk of CHUNK = THREADS * ITEMS ints in place (block-wide), the chunk
// total to sums[blockIdx.x].
__global__ void __launch_bounds__(THREADS) scan_chunk_kernel(int64_t n, int *__restrict__ data, int *__restrict__ sums) {
  __shared__ int wsum[THREADS / 32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t base = (int64_t)blockIdx.x * TILE + (int64_t)t * ITEMS;
  int v[ITEMS], run = 0;
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    v[u] = base + u < n ? data[base + u] : 0;
    const int x = v[u];
    v[u] = run;
    run += x;
  }
  // exclusive scan of the per-thread totals across the block
  int incl = run;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int s = lane < THREADS / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, off);
      if (lane >= off) s += y;
    }
    if (lane < THREADS / 32) wsum[lane] = s;  // inclusive over warps
  }
  __syncthreads();
  const int excl = incl - run + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll
  for (int u = 0; u < ITEMS; ++u)
    if (base + u < n) data[base + u] = v[u] + excl;
  if (t == THREADS - 1) sums[blockIdx.x] = excl + run;
}

__global__ void scan_add_kernel(int64_t n, int *__restrict__ data, const int *__restrict__ sums) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    data[i] += sums[i / TILE];
}

// Stable scatter of one pass: block b's items go to off[d * nb + b] + their rank among the
// block's items of digit d (in item order).
__global__ void __launch_bounds__(THREADS) radix_scatter_kernel(int N, const int *__restrict__ kin,
                                                                 const int *__restrict__ iin, int shift,
                                                                 const int *__restrict__ off, int *__restrict__ kout,
                                                                 int *__restrict__ iout) {
  __shared__ int s[DIGITS * THREADS];  // per (digit, thread) counts, then their exclusive scan
  __shared__ int wsum[THREADS / 32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int64_t b0 = (int64_t)blockIdx.x * TILE + (int64_t)t * ITEMS;  // this thread's 16 consecutive items
  int k[ITEMS], v[ITEMS], c[DIGITS];
#pragma unroll
  for (int d = 0; d < DIGITS; ++d) c[d] = 0;
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    const int64_t i = b0 + u;
    k[u] = i < N ? kin[i] : -1;
    v[u] = i < N ? iin[i] : 0;
    if (i < N) ++c[(k[u] >> shift) & (DIGITS - 1)];
  }
#pragma unroll
  for (int d = 0; d < DIGITS; ++d) s[d * THREADS + t] = c[d];
  __syncthreads();
  // exclusive scan of s in (digit, thread) order: thread t owns entries [16 t, 16 t + 16)
  int e[ITEMS], run = 0;
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    e[u] = run;
    run += s[t * ITEMS + u];
  }
  int incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int x = lane < THREADS / 32 ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane < THREADS / 32) wsum[lane] = x;
  }
  __syncthreads();
  const int excl = incl - run + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) s[t * ITEMS + u] = e[u] + excl;
  __syncthreads();
  // s[d * THREADS + t] = items of digit < d in the block + items of digit d in threads < t
  int pos[DIGITS];
#pragma unroll
  for (int d = 0; d < DIGITS; ++d) pos[d] = off[(int64_t)d * gridDim.x + blockIdx.x] + s[d * THREADS + t] - s[d * THREADS];
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    if (b0 + u >= N) break;
    const int d = (k[u] >> shift) & (DIGITS - 1);
    int p = 0;
#pragma unroll
    for (int dd = 0; dd < DIGITS; ++dd)
      if (dd == d) p = pos[dd]++;
    kout[p] = k[u];
    iout[p] = v[u];
  }
}

// leaf_start[m] = first position p with key[p] >= m, for m in [0, nleaf] (N for m = nleaf).
__global__ void leaf_bounds_kernel(int N, const int *__restrict__ key, int64_t nleaf, int *__restrict__ leaf_start) {
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m <= nleaf; m += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = N;
    while (lo < hi) {
      const int mid = lo + ((hi - lo) >> 1);
      if ((int64_t)key[mid] < m) lo = mid + 1;
      else hi = mid;
    }
    leaf_start[m] = lo;
  }
}

}  // namespace tr

// Exclusive scan of n ints in place (n <= TILE * TILE): chunks of TILE, then their totals.
static int scan_exclusive(int64_t n, int *data, int *sums, cudaStream_t s) {
  const int64_t nch = (n + tr::TILE - 1) / tr::TILE;
  if (nch > tr::TILE) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "device tree build: too many particles");
  tr::scan_chunk_kernel<<<(int)nch, tr::THREADS, 0, s>>>(n, data, sums);
  if (nch > 1) {
    tr::scan_chunk_kernel<<<1, tr::THREADS, 0, s>>>(nch, sums, sums + nch);
    tr::scan_add_kernel<<<148 * 8, 256, 0, s>>>(n, data, sums);
  }
  return bbfmm_set_cuda_error(cudaGetLastError(), "tree scan", __FILE__, __LINE__);
}

// perm (N = sum of counts) and leaf_start (nseg 8^maxlev + 1) on the device for the stacked
// sets whose particles are xyz[off[j] .. off[j] + count[j]) (device, [..][3]; off and count on
// the host). Scratch: 4 N + 16 ceil(N / 4096) + ceil(that / 4096) + 1 + 2 nseg + 1 ints,
// allocated here.
template <typename T>
int build_tree_device_sets(int nseg, const int *off_h, const int *count_h, const T *xyz, T L, int maxlev, int *perm,
                           int *leaf_start, cudaStream_t s) {
  if (nseg < 1 || maxlev < BBFMM_MINLEV || maxlev > 10 || nseg * pow8i(maxlev) > ((int64_t)1 << 30))
    return bbfmm_set_error(BBFMM_ERR_ARG, "need 1 <= sets, 2 <= maxlev <= 10 and sets x 8^maxlev <= 2^30");
  std::vector<int> seg(2 * (size_t)nseg + 1);  // base[0..nseg], then off[0..nseg)
  int64_t total = 0;
  for (int j = 0; j < nseg; ++j) {
    if (count_h[j] < 0 || off_h[j] < 0) return bbfmm_set_error(BBFMM_ERR_ARG, "negative set offset or size");
    seg[j] = (int)total;
    seg[nseg + 1 + j] = off_h[j];
    total += count_h[j];
    if (total > 0x7fffffff) return bbfmm_set_error(BBFMM_ERR_ARG, "more than 2^31 - 1 particles");
  }
  seg[nseg] = (int)total;
  const int N = (int)total;
  const int64_t nleaf = nseg * pow8i(maxlev);
  if (N == 0) {
    BBFMM_CUDA_OK(cudaMemsetAsync(leaf_start, 0, sizeof(int) * (nleaf + 1), s));
    return bbfmm_set_cuda_error(cudaStreamSynchronize(s), "tree build", __FILE__, __LINE__);
  }
  T celeng = L;
  for (int l = 1; l <= maxlev; ++l) celeng *= (T)0.5;
  const T L0half = L / 2, iLm = 1 / celeng;  // the host routine's values, bit for bit
  const int nb = (int)((N + tr::TILE - 1) / tr::TILE);
  const int64_t nh = (int64_t)tr::DIGITS * nb;
  const int64_t nsum = (nh + tr::TILE - 1) / tr::TILE + 1;
  int *buf = nullptr;
  const size_t words = 4 * (size_t)N + nh + nsum + 1 + seg.size();
  cudaError_t e = cudaMalloc(&buf, words * sizeof(int));
  if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "tree build scratch", __FILE__, __LINE__);
  int *k0 = buf, *i0 = buf + N, *k1 = buf + 2 * (size_t)N, *i1 = buf + 3 * (size_t)N;
  int *hist = buf + 4 * (size_t)N, *sums = hist + nh, *seg_d = sums + nsum + 1;
  int rc = BBFMM_OK;
  const int zero = 0;
  e = cudaMemcpyAsync(seg_d, seg.data(), sizeof(int) * seg.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(tr::g_tree_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    const int g = (int)((N + 255) / 256 < 148 * 32 ? (N + 255) / 256 : 148 * 32);
    tr::tree_keys_kernel<T><<<g, 256, 0, s>>>(N, nseg, seg_d, seg_d + nseg + 1, xyz, L0half, iLm, maxlev, k0, i0);
    e = cudaGetLastError();
  }
  int bits = 3 * maxlev;  // keys < nseg 8^maxlev
  while (((int64_t)1 << bits) < nleaf) ++bits;
  for (int shift = 0; e == cudaSuccess && rc == BBFMM_OK && shift < bits; shift += 4) {
    tr::radix_hist_kernel<<<nb, tr::THREADS, 0, s>>>(N, k0, shift, hist);
    rc = scan_exclusive(nh, hist, sums, s);
    if (rc != BBFMM_OK) break;
    tr::radix_scatter_kernel<<<nb, tr::THREADS, 0, s>>>(N, k0, i0, shift, hist, k1, i1);
    e = cudaGetLastError();
    std::swap(k0, k1);
    std::swap(i0, i1);
  }
  if (e == cudaSuccess && rc == BBFMM_OK) {
    e = cudaMemcpyAsync(perm, i0, sizeof(int) * N, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) {
      tr::leaf_bounds_kernel<<<148 * 16, 256, 0, s>>>(N, k0, nleaf, leaf_start);
      e = cudaGetLastError();
    }
  }
  int status = 0;
  if (e == cudaSuccess) e = cudaMemcpyFromSymbolAsync(&status, tr::g_tree_status, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(buf);
  if (rc != BBFMM_OK) return rc;
  if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "tree build", __FILE__, __LINE__);
  if (status) return bbfmm_set_error(BBFMM_ERR_ARG, "particle outside the root cell [-L/2, L/2]^3");
  return BBFMM_OK;
}

// One set: perm (N) and leaf_start (8^maxlev + 1) for the N particles at xyz.
template <typename T>
int build_tree_device(int N, const T *xyz, T L, int maxlev, int *perm, int *leaf_start, cudaStream_t s) {
  if (N < 0) return bbfmm_set_error(BBFMM_ERR_ARG, "need N >= 0");
  const int off = 0;
  return build_tree_device_sets<T>(1, &off, &N, xyz, L, maxlev, perm, leaf_start, s);
}

template int build_tree_device<double>(int, const double *, double, int, int *, int *, cudaStream_t);
template int build_tree_device<float>(int, const float *, float, int, int *, int *, cudaStream_t);
template int build_tree_device_sets<double>(int, const int *, const int *, const double *, double, int, int *, int *,
                                            cudaStream_t);
template int build_tree_device_sets<float>(int, const int *, const int *, const float *, float, int, int *, int *,
                                           cudaStream_t);

}  // namespace bbfmm
