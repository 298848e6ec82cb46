// M2L on CUDA cores over the dense class-major grid of one level.
//
//   L(F) = sum_{S in IL(F)} E_{k(F,S)} M(S)     (m2l_kern_basic.cu:82-130 semantics,
//                                                k from m2l_aux.c:1135-1191)
//
// For a target of sibling class b = (bx,by,bz) the interaction list is the set of
// offsets v with v_a in [-2-b_a, 3-b_a] and max|v_a| > 1: 189 offsets per class
// (anotherInteractionList.c:46-110 on a full tree). Out-of-grid sources contribute
// zero, which reproduces the shorter lists of boundary cells.
//
// CTA tile: a box of up to 4x4x4 targets of one class x all r outputs. The kernel loops
// over the class's offsets and over chunks of 16 contraction indices j in [j0, j1),
// staging the shifted source box and the operator chunk in shared memory, and keeps a
// register-blocked accumulator. With [j0, j1) = [0, r) this is the plain FP64 (or FP32)
// M2L; with [0, 16) it is the FP64 leading-component part of the mixed-precision M2L.
// With a box list (a target region) a tile is instead 8 listed 2 x 2 x 2 blocks of parent
// cells of one class, each of its own set and origin (slots past the list's end are not
// written).
//
// Operators: Ert[k][i][j] = E_k(i, j) (row-major), i.e. the transpose of the
// reference's column-major K file blocks.
#include "common.cuh"

namespace bbfmm {

struct OffsetTable {
  // per class c: 189 entries (k, vx, vy, vz) packed as int4
  const int4 *offs;
};

// TM x TN outputs per thread; the CTA has (64 / TM) (R / TN) threads (256 at r = 256 with an
// 8 x 8 tile, 128 at r = 32 with a 4 x 4 tile: 8 shared-memory loads per 16 FMAs).
template <typename T, int R, int TM, int TN>
__global__ void __launch_bounds__((64 / TM) * (R / TN)) m2l_simt_kernel(const T *__restrict__ M, const T *__restrict__ Ert,
                                                       T *__restrict__ Lout, int level, int j0, int j1,
                                                       const int4 *__restrict__ offs, int accumulate,
                                                       const int4 *__restrict__ boxes, int nboxes, int nsets) {
  constexpr int BK = 16;
  constexpr int NT = 64;  // targets per tile (4x4x4 box)
  constexpr int THREADS = (NT / TM) * (R / TN);
  constexpr int TGX = NT / TM;  // thread groups along targets
  __shared__ T sa[BK][NT];
  __shared__ T sb[BK][R + (sizeof(T) == 8 ? 1 : 0)];
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;  // box width per dimension
  const int nbox = P / bw;
  const int tiles_per_class = nbox * nbox * nbox;
  // sibling class fastest (the set above it): the CTAs resident at one time are the 8 classes
  // of neighbouring boxes, which read one source region that stays in L2
  const bool listed = boxes != nullptr;
  const int tpc = listed ? 1 : tiles_per_class;
  const int set_ = (int)(blockIdx.x / (8 * tpc)), loc_ = (int)(blockIdx.x % (8 * tpc));
  const int c = (listed ? 0 : set_ * 8) + loc_ % 8;  // class (and set base when not listed)
  const int tb = loc_ / 8;
  const int bxo = (tb % nbox) * bw, byo = ((tb / nbox) % nbox) * bw, bzo = (tb / (nbox * nbox)) * bw;
  const int cbx = (c >> 2) & 1, cby = (c >> 1) & 1, cbz = c & 1;
  const int nt = listed ? NT : bw * bw * bw;
  const int tid = threadIdx.x;
  __shared__ int4 s_box[8];  // listed: (set, or -1 - set past the list; x0, y0, z0) of the 8 slots
  if (listed && tid < 8) {
    const int bi = set_ * 8 + tid;
    int4 b = boxes[bi < nboxes ? bi : nboxes - 1];
    if (bi >= nboxes) b.x = -1 - b.x;
    s_box[tid] = b;
  }
  __syncthreads();
  // target t of the tile: set base (8 set), class-grid position, whether it is written
  auto cell = [&](int t, int &sb, int &px, int &py, int &pz, bool &ok) {
    if (listed) {
      const int4 b = s_box[t >> 3];
      ok = b.x >= 0;
      sb = 8 * (ok ? b.x : -1 - b.x);
      px = b.y + (t & 1);
      py = b.z + ((t >> 1) & 1);
      pz = b.w + ((t >> 2) & 1);
    } else {
      ok = t < nt;
      sb = c & ~7;
      px = bxo + (t % bw);
      py = byo + ((t / bw) % bw);
      pz = bzo + (t / (bw * bw));
    }
  };
  const int tg = tid % TGX, og = tid / TGX;
  T acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = 0;
  const int64_t P3 = (int64_t)P * P * P;
  // blockIdx.y selects one of gridDim.y groups of the 189 offsets; with several groups each
  // writes its partial sums to its own slice of Lout (all classes of all sets apart)
  const int grp = blockIdx.y, ngrp = gridDim.y;
  const int o0 = (189 * grp) / ngrp, o1 = (189 * (grp + 1)) / ngrp;
  Lout += (int64_t)grp * 8 * nsets * P3 * R;  // all classes of all sets
  for (int o = o0; o < o1; ++o) {
    const int4 ov = offs[(c & 7) * 189 + o];
    const int k = ov.x;
    // source class and parent-grid shift for this class/offset
    const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
    const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
    const int shx = (gx - scx) / 2, shy = (gy - scy) / 2, shz = (gz - scz) / 2;
    const int sc = (scx << 2) | (scy << 1) | scz;
    for (int jc = j0; jc < j1; jc += BK) {
      __syncthreads();
      for (int e = tid; e < NT * BK; e += THREADS) {
        const int t = e / BK, jj = e % BK;
        T v = 0;
        int sb, px, py, pz;
        bool ok;
        cell(t, sb, px, py, pz, ok);
        if (t < nt && jc + jj < j1) {
          px += shx;
          py += shy;
          pz += shz;
          if (px >= 0 && px < P && py >= 0 && py < P && pz >= 0 && pz < P)
            v = M[(((int64_t)(sb + sc) * P3 + ((int64_t)pz * P + py) * P + px)) * R + jc + jj];
        }
        sa[jj][t] = v;
      }
      const T *Ek = Ert + (int64_t)k * R * R;
      for (int e = tid; e < R * BK; e += THREADS) {
        const int i = e / BK, jj = e % BK;
        sb[jj][i] = (jc + jj < j1) ? Ek[(int64_t)i * R + jc + jj] : (T)0;
      }
      __syncthreads();
#pragma unroll
      for (int jj = 0; jj < BK; ++jj) {
        T a[TM], b[TN];
#pragma unroll
        for (int x = 0; x < TM; ++x) a[x] = sa[jj][tg + TGX * x];
#pragma unroll
        for (int y = 0; y < TN; ++y) b[y] = sb[jj][og + (R / TN) * y];
#pragma unroll
        for (int x = 0; x < TM; ++x)
#pragma unroll
          for (int y = 0; y < TN; ++y) acc[x][y] += a[x] * b[y];
      }
    }
  }
#pragma unroll
  for (int x = 0; x < TM; ++x) {
    const int t = tg + TGX * x;
    int sb, px, py, pz;
    bool ok;
    cell(t, sb, px, py, pz, ok);
    if (!ok) continue;
    T *dst = Lout + (((int64_t)(sb + (c & 7)) * P3 + ((int64_t)pz * P + py) * P + px)) * R;
#pragma unroll
    for (int y = 0; y < TN; ++y) {
      const int i = og + (R / TN) * y;
      if (accumulate) dst[i] += acc[x][y];
      else dst[i] = acc[x][y];
    }
  }
}

int m2l_simt_tiles(int level) {
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;
  const int nbox = P / bw;
  return 8 * nbox * nbox * nbox;
}

// Lout[e] = sum_g part[g][e], in a fixed order.
template <typename T>
__global__ void simt_sum_parts_kernel(int64_t count, int ng, const T *__restrict__ part, T *__restrict__ Lout) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x) {
    T v = 0;
    for (int g = 0; g < ng; ++g) v += part[(int64_t)g * count + e];
    Lout[e] = v;
  }
}

// ngroups > 1 splits the 189 offsets over that many CTAs per target tile; their partials go
// to `part` (part_elems elements) and are summed in a fixed order (groups are reduced to
// fit the scratch; accumulate then does not apply). With a list of nboxes 2 x 2 x 2 blocks of
// parent cells (set, x0, y0, z0) only their targets are computed, in one group, and the rest
// of Lout is left as it is.
template <typename T>
int launch_m2l_simt(int r, const T *M, const T *Ert, T *Lout, int level, int j0, int j1, const int4 *offs,
                    int accumulate, cudaStream_t s, int nsets, int ngroups, T *part, int64_t part_elems,
                    const int4 *boxes, int nboxes) {
  const int64_t P = (int64_t)1 << (level - 1);
  if (boxes && (nboxes < 0 || nboxes > nsets * P * P * P / 8 || P < 2))
    return bbfmm_set_error(BBFMM_ERR_ARG, "box list longer than the level");
  if (boxes && nboxes == 0) return BBFMM_OK;
  // the class index runs over all sets' 8 classes; a box list: 8 classes x groups of 8 blocks
  const int tiles = boxes ? 8 * ((nboxes + 7) / 8) : nsets * m2l_simt_tiles(level);
  const int64_t count = 8 * nsets * P * P * P * r;
  int ng = ngroups > 0 ? ngroups : 1;
  if (ng > 21) ng = 21;
  if (!part || boxes) ng = 1;
  else if ((int64_t)ng * count > part_elems) ng = (int)(part_elems / count);
  if (ng < 1) ng = 1;
  T *dst = ng > 1 ? part : Lout;
  const dim3 grid(tiles, ng);
  if (r == 256) {
    m2l_simt_kernel<T, 256, 8, 8><<<grid, 256, 0, s>>>(M, Ert, dst, level, j0, j1, offs, ng > 1 ? 0 : accumulate,
                                                       boxes, nboxes, nsets);
  } else if (r == 32) {
    m2l_simt_kernel<T, 32, 4, 4><<<grid, 128, 0, s>>>(M, Ert, dst, level, j0, j1, offs, ng > 1 ? 0 : accumulate,
                                                     boxes, nboxes, nsets);
  } else {
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "M2L rank must be 32 or 256 (n = 4 or 8)");
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || ng == 1) return bbfmm_set_cuda_error(e, "m2l_simt", __FILE__, __LINE__);
  int sg = (int)((count + 255) / 256);
  if (sg > 148 * 32) sg = 148 * 32;
  simt_sum_parts_kernel<T><<<sg, 256, 0, s>>>(count, ng, part, Lout);
  return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_simt parts", __FILE__, __LINE__);
}

template int launch_m2l_simt<double>(int, const double *, const double *, double *, int, int, int, const int4 *, int,
                                     cudaStream_t, int, int, double *, int64_t, const int4 *, int);
template int launch_m2l_simt<float>(int, const float *, const float *, float *, int, int, int, const int4 *, int,
                                    cudaStream_t, int, int, float *, int64_t, const int4 *, int);

// Host table of the 189 offsets of each sibling class, as (k, vx, vy, vz).
void build_offset_table(int *out /* 8*189*4 */) {
  for (int c = 0; c < 8; ++c) {
    const int b[3] = {(c >> 2) & 1, (c >> 1) & 1, c & 1};
    int cnt = 0;
    int k = 0;
    for (int vx = -3; vx <= 3; ++vx)
      for (int vy = -3; vy <= 3; ++vy)
        for (int vz = -3; vz <= 3; ++vz) {
          const bool far = vx < -1 || vx > 1 || vy < -1 || vy > 1 || vz < -1 || vz > 1;
          if (!far) continue;
          const int v[3] = {vx, vy, vz};
          bool ok = true;
          for (int a = 0; a < 3; ++a) ok = ok && v[a] >= -2 - b[a] && v[a] <= 3 - b[a];
          if (ok) {
            int *e = out + 4 * (c * 189 + cnt);
            e[0] = k; e[1] = vx; e[2] = vy; e[3] = vz;
            ++cnt;
          }
          ++k;
        }
  }
}

}  // namespace bbfmm
