// FP64 M2L on the FP64 tensor path (mma.sync m8n8k4 f64) over the dense class-major grid.
//
// Same contraction and tiling as m2l_simt.cu (one CTA per 4x4x4 box of targets of one
// sibling class), restricted to contraction components j in [j0, j1) and outputs
// i in [0, ni):
//   j in [0, 256), i in [0, 256)   the plain FP64 M2L,
//   j in [0, lead), i in [0, ilead) the FP64 leading block of the mixed-precision M2L.
// The A tile (sources x 16 j) is gathered from the cpg multipole grid and the B tile
// (16 j x 256 i) is read from the operators in the reference's own column-major layout
// E[k][j][i] (K file, bbfmm.c:1384-1405), so both global reads are contiguous. Tiles are
// double-buffered with cp.async; 8 warps in a 2 x 4 grid each own a 32-target x 64-output
// accumulator (4 x 8 fragments of 8x8); warps whose outputs lie beyond ni skip the math.
#include "solver.cuh"

namespace bbfmm {

namespace dm {

constexpr int NT = 64, R = 256, BK = 16;
constexpr int AST = NT + 4;   // padded row strides (doubles): conflict-free fragment reads
constexpr int BST = R + 4;
constexpr int STAGE_DOUBLES = BK * AST + BK * BST;
constexpr int SMEM_BYTES = 2 * STAGE_DOUBLES * 8;

__device__ __forceinline__ void cp_async8(uint32_t dst, const void *src, bool valid) {
  const int n = valid ? 8 : 0;  // zero-fill when the source lies outside the grid
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256, 1) m2l_dmma_kernel(const double *__restrict__ M,
                                                          const double *__restrict__ Ecol,
                                                          double *__restrict__ Lout, int level, int j0, int j1,
                                                          int ni, const int4 *__restrict__ offs,
                                                          const int4 *__restrict__ boxes, int nboxes, int nsets) {
  // blockIdx.y selects one of gridDim.y groups of the 189 offsets; with several groups each
  // writes its partial sums to its own slice of Lout (level cells x R apart)
  extern __shared__ __align__(16) double smem[];
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;
  const int nbox = P / bw;
  const int tiles_per_class = nbox * nbox * nbox;
  // sibling class fastest (the set above it): the CTAs resident at one time are the 8 classes
  // of neighbouring boxes, which read one source region that stays in L2
  // a box list (a target region): 8 listed 2 x 2 x 2 blocks of parent cells of one class per tile
  const bool listed = boxes != nullptr;
  const int tpc = listed ? 1 : tiles_per_class;
  const int set_ = (int)(blockIdx.x / (8 * tpc)), loc_ = (int)(blockIdx.x % (8 * tpc));
  const int c = (listed ? 0 : set_ * 8) + loc_ % 8;  // class (and set base when not listed)
  const int tb = loc_ / 8;
  const int bxo = (tb % nbox) * bw, byo = ((tb / nbox) % nbox) * bw, bzo = (tb / (nbox * nbox)) * bw;
  const int cbx = (c >> 2) & 1, cby = (c >> 1) & 1, cbz = c & 1;
  const int nt = listed ? NT : bw * bw * bw;
  const int64_t P3 = (int64_t)P * P * P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
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
  const int wm = warp & 1, wn = warp >> 1;  // 2 x 4 warp grid
  const bool active = wn * 64 < ni;         // this warp has outputs to compute
  const int nb = ni < R ? ((ni + 63) / 64) * 64 : R;  // B columns staged
  const int nchunk = (j1 - j0 + BK - 1) / BK;
  const int og = blockIdx.y, ng = gridDim.y;
  const int o0 = (189 * og) / ng, o1 = (189 * (og + 1)) / ng;
  const int niter = (o1 - o0) * nchunk;
  Lout += (int64_t)og * 8 * nsets * P3 * R;  // all classes of all sets
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);

  auto issue = [&](int it, int buf) {
    const int o = o0 + it / nchunk, jc = j0 + (it % nchunk) * BK;
    const int4 ov = offs[(c & 7) * 189 + o];
    const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
    const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
    const int shx = (gx - scx) / 2, shy = (gy - scy) / 2, shz = (gz - scz) / 2;
    const int sc = (scx << 2) | (scy << 1) | scz;
    const uint32_t sa = sbase + (uint32_t)(buf * STAGE_DOUBLES) * 8u;
    const uint32_t sb = sa + (uint32_t)(BK * AST) * 8u;
    // A: 64 targets x 16 j, 8-byte copies, zero outside the grid / j range
    for (int e = tid; e < NT * BK; e += 256) {
      const int t = e / BK, jj = e % BK;
      int sb, px, py, pz;
      bool wr;
      cell(t, sb, px, py, pz, wr);
      px += shx;
      py += shy;
      pz += shz;
      const bool ok = t < nt && jc + jj < j1 && px >= 0 && px < P && py >= 0 && py < P && pz >= 0 && pz < P;
      const double *src = ok ? M + ((int64_t)(sb + sc) * P3 + ((int64_t)pz * P + py) * P + px) * R + jc + jj : M;
      cp_async8(sa + (uint32_t)(jj * AST + t) * 8u, src, ok);
    }
    // B: 16 rows j of E_k (the first nb outputs i), 16-byte copies
    const double *Ek = Ecol + (int64_t)ov.x * R * R;
    for (int e = tid; e < BK * (nb / 2); e += 256) {
      const int jj = e / (nb / 2), i2 = (e % (nb / 2)) * 2;
      const int j = jc + jj < j1 ? jc + jj : j1 - 1;  // rows past j1 meet zero A columns
      cp_async16(sb + (uint32_t)(jj * BST + i2) * 8u, Ek + (int64_t)j * R + i2);
    }
    cp_commit();
  };

  double acc[4][8][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

  issue(0, 0);
  for (int it = 0; it < niter; ++it) {
    const int buf = it & 1;
    if (it + 1 < niter) {
      issue(it + 1, buf ^ 1);
      cp_wait_one();
    } else {
      cp_wait_all();
    }
    __syncthreads();
    if (active) {
      const double *A = smem + buf * STAGE_DOUBLES;
      const double *B = A + BK * AST;
#pragma unroll
      for (int ks = 0; ks < BK / 4; ++ks) {
        const int k = ks * 4 + (lane & 3);
        double af[4], bf[8];
#pragma unroll
        for (int mf = 0; mf < 4; ++mf) af[mf] = A[k * AST + wm * 32 + mf * 8 + (lane >> 2)];
#pragma unroll
        for (int nf = 0; nf < 8; ++nf) bf[nf] = B[k * BST + wn * 64 + nf * 8 + (lane >> 2)];
#pragma unroll
        for (int mf = 0; mf < 4; ++mf)
#pragma unroll
          for (int nf = 0; nf < 8; ++nf) dmma(acc[mf][nf][0], acc[mf][nf][1], af[mf], bf[nf]);
      }
    }
    __syncthreads();
  }
  if (!active) return;
  // D fragment: row = lane >> 2, columns 2 (lane & 3) + {0, 1}
#pragma unroll
  for (int mf = 0; mf < 4; ++mf) {
    const int t = wm * 32 + mf * 8 + (lane >> 2);
    int sb, px, py, pz;
    bool wr;
    cell(t, sb, px, py, pz, wr);
    if (!wr) continue;
    double *dst = Lout + ((int64_t)(sb + (c & 7)) * P3 + ((int64_t)pz * P + py) * P + px) * R;
#pragma unroll
    for (int nf = 0; nf < 8; ++nf) {
      const int i = wn * 64 + nf * 8 + 2 * (lane & 3);
      if (i < ni) *reinterpret_cast<double2 *>(dst + i) = make_double2(acc[mf][nf][0], acc[mf][nf][1]);
    }
  }
}

// Leading block only (outputs i < NI <= 64, components j < j1 <= 64): a tile of NT targets
// of one class (NT = 64: a bw^3 box, bw = min(P, 4); NT = 128: an 8x4x4 box, P >= 8); every
// warp owns NT/64 8-target fragment rows and all NI/8 output fragments, so each B fragment
// feeds NT/64 DMMAs; a 4-stage cp.async pipeline over the (offset, 16-component chunk)
// sequence keeps the small per-offset tiles in flight. A is stored [target][j] (stride 20
// doubles, conflict-free fragment reads, 16-byte copies).
namespace lead {
constexpr int BK = 16, STAGES = 4, AST = BK + 4;
template <int NI, int NT>
struct Cfg {
  static constexpr int BST = NI + 4;
  static constexpr int STAGE = NT * AST + BK * BST;
  static constexpr int SMEM = STAGES * STAGE * 8;
};
}  // namespace lead

template <int NI, int NT>
__global__ void __launch_bounds__(256) m2l_lead_kernel(const double *__restrict__ M, const double *__restrict__ Ecol,
                                                       double *__restrict__ Lout, int level, int j1,
                                                       const int4 *__restrict__ offs) {
  constexpr int BST = lead::Cfg<NI, NT>::BST, STAGE = lead::Cfg<NI, NT>::STAGE, NF = NI / 8, MF = NT / 64;
  extern __shared__ __align__(16) double smem[];
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;
  const int bwx = NT == 128 ? 8 : bw;  // box extent in x (y and z: bw)
  const int nbx = P / bwx, nbox = P / bw;
  const int tiles_per_class = nbx * nbox * nbox;
  // sibling class fastest (the set above it): the CTAs resident at one time are the 8 classes
  // of neighbouring boxes, which read one source region that stays in L2
  const int set_ = (int)(blockIdx.x / (8 * tiles_per_class)), loc_ = (int)(blockIdx.x % (8 * tiles_per_class));
  const int c = set_ * 8 + loc_ % 8;
  const int tb = loc_ / 8;
  const int bxo = (tb % nbx) * bwx, byo = ((tb / nbx) % nbox) * bw, bzo = (tb / (nbx * nbox)) * bw;
  const int cbx = (c >> 2) & 1, cby = (c >> 1) & 1, cbz = c & 1;
  const int nt = bwx * bw * bw;
  const int64_t P3 = (int64_t)P * P * P;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = (j1 + lead::BK - 1) / lead::BK;
  const int niter = 189 * nchunk;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);

  // the targets and component pairs this thread copies are the same for every (offset,
  // chunk): their box coordinates and shared-memory slots are computed once
  constexpr int PER = (NT * (lead::BK / 2) + 255) / 256;
  int cx[PER], cy[PER], cz[PER], j2s[PER];
  uint32_t soff[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int e = tid + 256 * k;
    const int t = e / (lead::BK / 2);
    j2s[k] = (e % (lead::BK / 2)) * 2;
    const bool valid = e < NT * (lead::BK / 2) && t < nt;
    cx[k] = valid ? bxo + (t % bwx) : -(1 << 20);  // invalid slots fall outside every grid
    cy[k] = byo + ((t / bwx) % bw);
    cz[k] = bzo + (t / (bwx * bw));
    soff[k] = (uint32_t)(t * lead::AST + j2s[k]) * 8u;
  }
  auto issue = [&](int it) {
    if (it < niter) {
      const int o = it / nchunk, jc = (it % nchunk) * lead::BK;
      const int4 ov = offs[(c & 7) * 189 + o];
      const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
      const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
      const int shx = (gx - scx) / 2, shy = (gy - scy) / 2, shz = (gz - scz) / 2;
      const int sc = (scx << 2) | (scy << 1) | scz;
      const uint32_t sa = sbase + (uint32_t)((it % lead::STAGES) * STAGE) * 8u;
      const uint32_t sb = sa + (uint32_t)(NT * lead::AST) * 8u;
      const double *Mc = M + (int64_t)((c & ~7) + sc) * P3 * R + jc;
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        if (tid + 256 * k >= NT * (lead::BK / 2)) break;
        const int px = cx[k] + shx, py = cy[k] + shy, pz = cz[k] + shz;
        const bool ok = jc + j2s[k] < j1 && (unsigned)px < (unsigned)P && (unsigned)py < (unsigned)P &&
                        (unsigned)pz < (unsigned)P;
        const double *src = ok ? Mc + (((int64_t)pz * P + py) * P + px) * R + j2s[k] : M;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa + soff[k]), "l"(src),
                     "r"(ok ? 16 : 0)
                     : "memory");
      }
      const double *Ek = Ecol + (int64_t)ov.x * R * R;
      for (int e = tid; e < lead::BK * (NI / 2); e += 256) {  // 16 rows j x NI/2 pairs of i
        const int jj = e / (NI / 2), i2 = (e % (NI / 2)) * 2;
        const int j = jc + jj < j1 ? jc + jj : j1 - 1;
        cp_async16(sb + (uint32_t)(jj * BST + i2) * 8u, Ek + (int64_t)j * R + i2);
      }
    }
    cp_commit();  // (possibly empty) group keeps the wait counts uniform
  };

  double acc[MF][NF][2];
#pragma unroll
  for (int m = 0; m < MF; ++m)
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[m][f][0] = acc[m][f][1] = 0.0;
#pragma unroll
  for (int s = 0; s < lead::STAGES - 1; ++s) issue(s);
  for (int it = 0; it < niter; ++it) {
    asm volatile("cp.async.wait_group %0;" ::"n"(lead::STAGES - 2) : "memory");
    __syncthreads();
    issue(it + lead::STAGES - 1);  // refills the stage consumed in iteration it - 1
    const double *A = smem + (it % lead::STAGES) * STAGE;
    const double *B = A + NT * lead::AST;
#pragma unroll
    for (int ks = 0; ks < lead::BK / 4; ++ks) {
      const int k = ks * 4 + (lane & 3);
      double af[MF];
#pragma unroll
      for (int m = 0; m < MF; ++m) af[m] = A[(warp * 8 * MF + m * 8 + (lane >> 2)) * lead::AST + k];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double bf = B[k * BST + f * 8 + (lane >> 2)];
#pragma unroll
        for (int m = 0; m < MF; ++m) dmma(acc[m][f][0], acc[m][f][1], af[m], bf);
      }
    }
  }
  cp_wait_all();
#pragma unroll
  for (int m = 0; m < MF; ++m) {
    const int t = warp * 8 * MF + m * 8 + (lane >> 2);
    if (t >= nt) continue;
    const int px = bxo + (t % bwx), py = byo + ((t / bwx) % bw), pz = bzo + (t / (bwx * bw));
    double *dst = Lout + ((int64_t)c * P3 + ((int64_t)pz * P + py) * P + px) * R;
#pragma unroll
    for (int f = 0; f < NF; ++f)
      *reinterpret_cast<double2 *>(dst + f * 8 + 2 * (lane & 3)) = make_double2(acc[m][f][0], acc[m][f][1]);
  }
}

// Lout[e] = sum_g part[g][e], in a fixed order.
__global__ void sum_parts_kernel(int64_t count, int ng, const double *__restrict__ part, double *__restrict__ Lout) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x) {
    double v = 0.0;
    for (int g = 0; g < ng; ++g) v += part[(int64_t)g * count + e];
    Lout[e] = v;
  }
}

}  // namespace dm

// Target tiles (CTAs) of the full FP64 M2L of one level.
static int64_t dmma_tiles(int level, int nsets) {
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;
  const int nbox = P / bw;
  return 8 * (int64_t)nsets * nbox * nbox * nbox;
}

// Offset groups (CTAs per target tile) that fill about two waves of the 148 SMs.
int dmma_default_groups(int level, int nsets) {
  const int64_t tiles = dmma_tiles(level, nsets);
  int64_t g = (2 * 148 + tiles - 1) / tiles;
  return (int)(g < 1 ? 1 : (g > DMMA_PARTS ? DMMA_PARTS : g));
}

// Doubles of partial-sum scratch a level needs with `groups` offset groups (0 when 1).
int64_t dmma_part_elems(int level, int nsets, int groups, int r) {
  return groups > 1 ? (int64_t)groups * nsets * pow8i(level) * r : 0;
}

// Writes Lout[cell][0:ni) for every cell of the level (assign); entries i >= ni untouched.
// The full M2L (ni = r) may split the 189 offsets into `ngroups` CTAs per target tile
// (0: dmma_default_groups) whose partials go to `part` (part_elems doubles) and are then
// summed in a fixed order; with too little scratch the groups are reduced to fit.
int launch_m2l_dmma(int r, const double *M, const double *Ecol, double *Lout, int level, int j0, int j1, int ni,
                    const int4 *offs, double *part, int64_t part_elems, cudaStream_t s, int nsets, int ngroups,
                    const int4 *boxes, int nboxes) {
  if (r != dm::R) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "FP64 tensor M2L is built for r = 256");
  if (j0 < 0 || j1 > r || j0 >= j1 || ni < 2 || ni > r || ni % 2)
    return bbfmm_set_error(BBFMM_ERR_ARG, "bad contraction / output range");
  const int P = 1 << (level - 1);
  const int bw = P < 4 ? P : 4;
  const int nbox = P / bw;
  const int grid = 8 * nsets * nbox * nbox * nbox;
  if (boxes && (j0 != 0 || j1 != r || ni != r))
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "box lists are for the full FP64 M2L");
  if (boxes && (nboxes < 0 || nboxes > (int64_t)nsets * P * P * P / 8 || P < 2))
    return bbfmm_set_error(BBFMM_ERR_ARG, "box list longer than the level");
  if (boxes && nboxes == 0) return BBFMM_OK;
  if (j0 == 0 && j1 <= 64 && (ni == 32 || ni == 64)) {  // the FP64 leading block
    static bool lattr = false;
    if (!lattr) {
      cudaFuncSetAttribute(dm::m2l_lead_kernel<32, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           dm::lead::Cfg<32, 64>::SMEM);
      cudaFuncSetAttribute(dm::m2l_lead_kernel<64, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           dm::lead::Cfg<64, 64>::SMEM);
      cudaFuncSetAttribute(dm::m2l_lead_kernel<32, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           dm::lead::Cfg<32, 128>::SMEM);
      lattr = true;
    }
    if (ni == 32 && P >= 8)  // 128-target tiles (8x4x4 boxes)
      dm::m2l_lead_kernel<32, 128><<<grid / 2, 256, dm::lead::Cfg<32, 128>::SMEM, s>>>(M, Ecol, Lout, level, j1, offs);
    else if (ni == 32)
      dm::m2l_lead_kernel<32, 64><<<grid, 256, dm::lead::Cfg<32, 64>::SMEM, s>>>(M, Ecol, Lout, level, j1, offs);
    else
      dm::m2l_lead_kernel<64, 64><<<grid, 256, dm::lead::Cfg<64, 64>::SMEM, s>>>(M, Ecol, Lout, level, j1, offs);
    return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_lead", __FILE__, __LINE__);
  }
  static bool attr = false;
  if (!attr) {
    cudaError_t e =
        cudaFuncSetAttribute(dm::m2l_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dm::SMEM_BYTES);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "m2l_dmma smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  int ng = ngroups > 0 ? ngroups : dmma_default_groups(level, nsets);
  if (ng > DMMA_PARTS) ng = DMMA_PARTS;
  const int64_t count = 8 * (int64_t)nsets * P * P * P * r;
  if (!part || boxes) ng = 1;
  else if ((int64_t)ng * count > part_elems) ng = (int)(part_elems / count);
  if (ng > 1) {
    // few target tiles: spread the offsets over ng CTAs per tile, then sum the partials
    dm::m2l_dmma_kernel<<<dim3(grid, ng), 256, dm::SMEM_BYTES, s>>>(M, Ecol, part, level, j0, j1, ni, offs, nullptr, 0,
                                                                   nsets);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "m2l_dmma", __FILE__, __LINE__);
    dm::sum_parts_kernel<<<(int)((count + 255) / 256), 256, 0, s>>>(count, ng, part, Lout);
    return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_dmma parts", __FILE__, __LINE__);
  }
  dm::m2l_dmma_kernel<<<boxes ? 8 * ((nboxes + 7) / 8) : grid, 256, dm::SMEM_BYTES, s>>>(M, Ecol, Lout, level, j0, j1,
                                                                                        ni, offs, boxes, nboxes, nsets);
  return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_dmma", __FILE__, __LINE__);
}

}  // namespace bbfmm
