// Mixed-precision M2L on tcgen05 tensor cores (sm_100a).
//
// For one level, everything outside the leading block (i < lead_rows, j < lead) of
//   L_i(F) = sum_{v in IL(F)} sum_j E_v(i, j) M_j(F + v)
// is computed as three-term split products: with x = x_hi + x_lo (bf16 each),
//   E M ~= E_hi M_hi + E_hi M_lo + E_lo M_hi,
// accumulated in FP32 in tensor memory over all 189 offsets. The leading block (default
// 32 outputs x 16 components), whose FP32 accumulation would dominate the error, is
// computed in FP64 beforehand (m2l_dmma.cu) and this kernel adds its result to it: the
// split operator copy holds zeros in that block, so the tensor cores skip nothing but
// contribute nothing there. With lead_rows = r the whole j < lead strip is left out and
// its K-steps are skipped.
//
// Tile: 128 targets of one sibling class forming an 8x4x4 box of its parent grid
// (GEMM M = 128) x all 256 outputs i (N = 256) in a 128 x 256 FP32 TMEM accumulator.
// For an offset v the 128 sources form the same box in one class grid, shifted by a
// whole number of parent cells, so each K-chunk of the A operand (32 bf16 of j per row)
// is ONE 5-D TMA box load from the class-major multipole grid; out-of-grid sources are
// zero-filled by TMA. The B operand chunk is rows i of E_v for the same 32 j. Operand
// tiles are K-major with 64-byte rows in the 64-byte swizzle.
//
// Warp roles (192 threads): warp 0 = TMA producer (and TMEM allocator), warp 1 = MMA
// issuer, warps 2-5 = epilogue (tcgen05.ld of the accumulator, FP64 update of L).
// Four pipeline stages of 48 KB (A_hi, A_lo 8 KB each; B_hi, B_lo 16 KB each): three
// chunks are in flight while the MMA warp consumes the fourth, which hides the TMA latency
// that two stages of 96 KB left exposed (tensor pipe idle ~20% of active cycles).
// Every mbarrier wait is bounded; on timeout the kernel records an error code in a
// device status word, skips the remaining work, frees its tensor memory and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdio>
#include <vector>

#include "solver.cuh"

namespace bbfmm {

namespace tc {

constexpr int BM = 128, BN = 256, BK = 32;  // targets, outputs, bf16 per K-chunk (64 B rows)
constexpr int KS = BK / 16;                 // MMA K-steps per chunk
constexpr int STAGES = 4;                   // three chunks in flight while one is consumed
constexpr int A_BYTES = BM * BK * 2;        // 8 KB
constexpr int B_BYTES = BN * BK * 2;        // 16 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
constexpr int BOX_X = 8, BOX_Y = 4, BOX_Z = 4;
constexpr uint32_t WAIT_LIMIT = 1u << 26;

__device__ int g_tc_status = 0;  // 0 = ok; else code of the first failed wait

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false (and the status word set) if the phase did not complete in time.
// FP64 tensor-core step D += A B (m8n8k4): A row lane >> 2, column lane & 3; B row lane & 3,
// column lane >> 2; D row lane >> 2, columns 2 (lane & 3) + {0, 1}.
__device__ __forceinline__ void dmma_f64(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int code) {
  for (uint32_t i = 0; i < WAIT_LIMIT; ++i)
    if (mbar_try(bar, parity)) return true;
  atomicCAS(&g_tc_status, 0, code);
  return false;
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1,
                                            int c2, int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(dst),
      "l"((uint64_t)map), "r"(bar), "r"(c0), "r"(c1)
      : "memory");
}

// K-major, 64-byte swizzled operand tile: rows of 64 B (32 bf16), 8-row groups 512 B apart.
__device__ __forceinline__ uint64_t sw64_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);        // start address
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;                // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                         // 64-byte swizzle
  return d;
}

// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N columns
// (a multiple of 16 up to 256; the accumulator columns [0, N) of the tile are updated).
__host__ __device__ constexpr uint32_t idesc(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
constexpr uint32_t IDESC = idesc(BN);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t acc,
                                         uint32_t id = IDESC) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(id), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Grid: one CTA per tile (class c, 8x4x4 box). Lacc: the level's FP64 output, cpg layout
// [cell][256]; entries i < ilead hold the FP64 leading block and are added to, the others
// are overwritten.
__global__ void __launch_bounds__(192, 1)
    m2l_tc_kernel(const __grid_constant__ CUtensorMap mapAhi, const __grid_constant__ CUtensorMap mapAlo,
                  const __grid_constant__ CUtensorMap mapBhi, const __grid_constant__ CUtensorMap mapBlo,
                  double *__restrict__ Lacc, int level, const int4 *__restrict__ offs, int kfirst, int ilead,
                  int split_chunks, int split_rows, int ncols) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *gbase = smem_raw + (base - raw);
  const uint32_t bar_base = base + STAGES * STAGE_BYTES;
  uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + STAGES * STAGE_BYTES);
  // bars[0..S-1] = full, bars[S..2S-1] = empty, bars[2S] = accumulator ready; tmem slot after
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 1);
  auto full_bar = [&](int s) { return bar_base + 8u * s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (STAGES + s); };
  const uint32_t acc_bar = bar_base + 8u * (2 * STAGES);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int P = 1 << (level - 1);
  const int nbx = P / BOX_X, nby = P / BOX_Y, nbz = P / BOX_Z;
  const int tiles_per_class = nbx * nby * nbz;
  // sibling class fastest (the set above it): the CTAs resident at one time are the 8 classes
  // of neighbouring boxes, which read one source region that stays in L2
  const int set_ = (int)(blockIdx.x / (8 * tiles_per_class)), loc_ = (int)(blockIdx.x % (8 * tiles_per_class));
  const int c = set_ * 8 + loc_ % 8;
  const int tb = loc_ / 8;
  const int bx0 = (tb % nbx) * BOX_X, by0 = ((tb / nbx) % nby) * BOX_Y, bz0 = (tb / (nbx * nby)) * BOX_Z;
  const int cbx = (c >> 2) & 1, cby = (c >> 1) & 1, cbz = c & 1;
  const int nchunk = ncols / BK;  // K-chunks per offset: the effective rank / 32 (8 for r = 256)
  const int chunk0 = kfirst / KS;  // whole chunks skipped
  const int kstep0 = kfirst % KS;  // K-steps skipped in the first used chunk
  const int used_chunks = nchunk - chunk0;
  const int niter = 189 * used_chunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(256)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    for (int it = 0; it < niter; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (!mbar_wait(empty_bar(s), ph ^ 1u, 1)) break;
      const int o = it / used_chunks, kc = chunk0 + it % used_chunks;
      const int4 ov = offs[(c & 7) * 189 + o];
      const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
      const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
      const int sc = (scx << 2) | (scy << 1) | scz;
      const int sx = bx0 + (gx - scx) / 2, sy = by0 + (gy - scy) / 2, sz = bz0 + (gz - scz) / 2;
      const uint32_t st = base + s * STAGE_BYTES;
      // chunks kc < split_chunks take three products and need the lo halves (of B only its
      // first split_rows rows, the box of mapBlo); the others take hi x hi alone
      const bool three = kc < split_chunks;
      const uint32_t bhi_bytes = (uint32_t)ncols * BK * 2;  // the B box holds the first ncols rows i
      mbar_expect_tx(full_bar(s), three ? 2 * A_BYTES + bhi_bytes + (uint32_t)split_rows * BK * 2 : A_BYTES + bhi_bytes);
      tma_load_5d(st, &mapAhi, full_bar(s), kc * BK, sx, sy, sz, (c & ~7) + sc);
      tma_load_3d(st + 2 * A_BYTES, &mapBhi, full_bar(s), kc * BK, 0, ov.x);
      if (three) {
        tma_load_5d(st + A_BYTES, &mapAlo, full_bar(s), kc * BK, sx, sy, sz, (c & ~7) + sc);
        tma_load_3d(st + 2 * A_BYTES + B_BYTES, &mapBlo, full_bar(s), kc * BK, 0, ov.x);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    uint32_t acc = 0;
    for (int it = 0; it < niter; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (!mbar_wait(full_bar(s), ph, 2)) break;
      tc_fence_after();
      const uint32_t st = base + s * STAGE_BYTES;
      const int k0 = (it % used_chunks == 0) ? kstep0 : 0;
      const bool three = chunk0 + it % used_chunks < split_chunks;
      const uint32_t id_part = idesc(split_rows), id_all = idesc(ncols);
      for (int ks = k0; ks < KS; ++ks) {
        const uint64_t ahi = sw64_desc(st + ks * 32), alo = sw64_desc(st + A_BYTES + ks * 32);
        const uint64_t bhi = sw64_desc(st + 2 * A_BYTES + ks * 32);
        const uint64_t blo = sw64_desc(st + 2 * A_BYTES + B_BYTES + ks * 32);
        mma_bf16(tmem, ahi, bhi, acc, id_all);  // all ncols outputs (the first MMA initialises them)
        if (three) {                    // corrections for the outputs i < split_rows
          mma_bf16(tmem, ahi, blo, 1u, id_part);
          mma_bf16(tmem, alo, bhi, 1u, id_part);
        }
        acc = 1u;
      }
      mma_commit(empty_bar(s));
    }
    mma_commit(acc_bar);  // also after an early exit: the epilogue must not wait forever
  } else if (warp >= 2) {
    // ---------------- epilogue: TMEM -> registers -> Lacc
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const bool ok = mbar_wait(acc_bar, 0, 3);
    tc_fence_after();
    if (ok) {
      const int tx = row % BOX_X, ty = (row / BOX_X) % BOX_Y, tz = row / (BOX_X * BOX_Y);
      const int64_t P3 = (int64_t)P * P * P;
      const int64_t cell = (int64_t)c * P3 + ((int64_t)(bz0 + tz) * P + (by0 + ty)) * P + (bx0 + tx);
      double *dst = Lacc + cell * BN;
      for (int col = 0; col < ncols; col += 32) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)col, v);
        const bool add = col < ilead;  // ilead is a multiple of 32
#pragma unroll
        for (int i = 0; i < 32; i += 2) {
          double2 o = add ? *reinterpret_cast<const double2 *>(dst + col + i) : make_double2(0.0, 0.0);
          o.x += (double)v[i];
          o.y += (double)v[i + 1];
          *reinterpret_cast<double2 *>(dst + col + i) = o;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256) : "memory");
  }
}

// Two target boxes per CTA for the adaptive product map: one 8x8x4 box of a class (256
// targets) as two M = 128 halves, each with its own 128 x 256 FP32 accumulator in TMEM (all
// 512 columns), so every operator chunk loaded into shared memory serves 256 targets and the
// operator traffic from L2 is halved. The lo halves of B cover the first TC_SPLIT_ROWS rows.
// At levels 3 and 2, whose class grids are only 4 x 4 x 4 and 2 x 2 x 2, the 256 targets are
// that whole grid in 4 or 32 consecutive stacked sets (one box load of 4 KB or 512 B per set
// and operand half; slots past the last set load the last set again and write nothing), so a
// batch of small trees runs its upper levels on the tensor cores as well. Rows: x fastest,
// then y, z, set. With a box list (a target region) a tile is instead 256 / (bx by bz) listed
// bx x by x bz blocks of parent cells (2 x 2 x 2 or 4 x 4 x 2: lgeom), each of its own set and
// origin (one box load per block and operand half; slots past the list's end load its last
// block and write nothing), so the tiles follow the region. The box of slot k is loaded by
// lane k of the producer warp, so the small boxes of a stage go out together.
// Stage: A_hi 16 KB | A_lo 16 KB | B_hi 16 KB | B_lo TC_SPLIT_ROWS x 32 BF16 (4 KB).
// With Mlead and Erow given (leading block i < 32, j < 16), the four epilogue warps, idle
// while the tensor cores run the ~1 ms mainloop of a CTA, compute that block in FP64 for the
// rows they later read from tensor memory: DMMA m8n8k4 with fragments loaded straight from
// global memory (shared memory is taken by the stages), k-slot u of step ks standing for
// component 4u + ks so that each fragment load is one contiguous 32-byte run of M or of
// Erow[k][i][j] = E_k(i, j). The block is written to Lacc (assign) before the accumulator
// wait, and the tensor-memory epilogue adds to it as it adds to a separately computed block.
// With Lsplit (one whole level, mixed projections) the epilogue writes the FP64 output only
// for i < 32 and, for every i < ncols, its [hi | lo] BF16 split into the Morton row of the
// cell (planes of `nrows` rows of 256), components i < DNZ zero: the input of the fused down
// projection, which otherwise gathers and splits the rows in a separate pass.
constexpr int A2_BYTES = 2 * A_BYTES, BLO2_BYTES = TC_SPLIT_ROWS * BK * 2;
constexpr int STAGE2_BYTES = 2 * A2_BYTES + B_BYTES + BLO2_BYTES;
constexpr int SMEM2_BYTES = STAGES * STAGE2_BYTES + 1024 /*align*/ + 256 /*barriers*/;
static_assert(SMEM2_BYTES <= 232448, "two-box stages exceed the shared memory of a CTA");

__global__ void __launch_bounds__(192, 1)
    m2l_tc2_kernel(const __grid_constant__ CUtensorMap mapAhi, const __grid_constant__ CUtensorMap mapAlo,
                   const __grid_constant__ CUtensorMap mapBhi, const __grid_constant__ CUtensorMap mapBlo,
                   double *__restrict__ Lacc, int level, const int4 *__restrict__ offs, int kfirst, int ilead,
                   int split_chunks, int ncols, const double *__restrict__ Mlead, const double *__restrict__ Erow,
                   __nv_bfloat16 *__restrict__ Lsplit, int64_t nrows, const int4 *__restrict__ boxes,
                   int nboxes, int lgeom, int nsets) {
  constexpr int STAGE_BYTES = STAGE2_BYTES;
  constexpr int DNZ = 16;  // components the fused down projection takes in FP64
  constexpr int split_rows = TC_SPLIT_ROWS;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *gbase = smem_raw + (base - raw);
  const uint32_t bar_base = base + STAGES * STAGE_BYTES;
  uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + STAGES * STAGE_BYTES);
  // bars[0..S-1] = full, bars[S..2S-1] = empty, bars[2S] = accumulator ready; tmem slot after
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 1);
  auto full_bar = [&](int s) { return bar_base + 8u * s; };
  auto empty_bar = [&](int s) { return bar_base + 8u * (STAGES + s); };
  const uint32_t acc_bar = bar_base + 8u * (2 * STAGES);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int P = 1 << (level - 1);
  const bool listed = boxes != nullptr;
  const Tc2Box g = listed ? Tc2Box{lgeom & 15, (lgeom >> 4) & 15, (lgeom >> 8) & 15} : tc2_box(level);
  const int nbx = P >> g.lx, nby = P >> g.ly, nbz = P >> g.lz;
  const int tiles_per_class = listed ? 1 : nbx * nby * nbz;
  // sibling class fastest (the set group or list group above it): the CTAs resident at one
  // time are the 8 classes of neighbouring boxes, which read one source region that stays in L2
  const int bid_ = (int)blockIdx.x;
  const int sg_ = bid_ / (8 * tiles_per_class), loc_ = bid_ % (8 * tiles_per_class);
  const int cls = loc_ % 8, tb = loc_ / 8;
  const int set0 = sg_ << (8 - g.lb());  // first set (or list entry) of the tile
  const int bx0 = (tb % nbx) << g.lx, by0 = ((tb / nbx) % nby) << g.ly, bz0 = (tb / (nbx * nby)) << g.lz;
  const int cbx = (cls >> 2) & 1, cby = (cls >> 1) & 1, cbz = cls & 1;
  // slot k of the tile (rows k 2^lb ..): its set, the origin of its box in the class grid, and
  // whether its rows are written (a slot past the last set or list entry loads a valid box)
  __shared__ int4 s_box[32];  // listed: (set, or -1 - set for a slot past the list; x0, y0, z0)
  if (listed && threadIdx.x < (1 << (8 - g.lb()))) {
    const int bi = set0 + threadIdx.x;
    int4 b = boxes[bi < nboxes ? bi : nboxes - 1];
    if (bi >= nboxes) b.x = -1 - b.x;
    s_box[threadIdx.x] = b;
  }
  auto slot = [&](int k, int &set, int &x0, int &y0, int &z0, bool &ok) {
    if (listed) {
      const int4 b = s_box[k];
      ok = b.x >= 0;
      set = ok ? b.x : -1 - b.x;
      x0 = b.y;
      y0 = b.z;
      z0 = b.w;
    } else {
      set = set0 + k;
      ok = set < nsets;
      if (!ok) set = nsets - 1;
      x0 = bx0;
      y0 = by0;
      z0 = bz0;
    }
  };
  // row of the tile -> its cell's set and class-grid position
  auto row_cell = [&](int row, int &set, int &x, int &y, int &z, bool &ok) {
    int k, x0, y0, z0;
    g.pos(row, x, y, z, k);
    slot(k, set, x0, y0, z0, ok);
    x += x0;
    y += y0;
    z += z0;
  };
  const int nchunk = ncols / BK;  // K-chunks per offset: the effective rank / 32 (8 for r = 256)
  const int chunk0 = kfirst / KS;  // whole chunks skipped
  const int kstep0 = kfirst % KS;  // K-steps skipped in the first used chunk
  const int used_chunks = nchunk - chunk0;
  const int niter = 189 * used_chunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(acc_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer: lane 0 takes the stage and loads the operator; the box of
    // slot k of the tile is loaded by lane k
    const int nslot = 1 << (8 - g.lb());
    int set_k = 0, x0_k = 0, y0_k = 0, z0_k = 0;  // this lane's slot
    if (lane < nslot) {
      bool ok;
      slot(lane, set_k, x0_k, y0_k, z0_k, ok);
    }
    const uint32_t box_bytes = (uint32_t)BK * 2u << g.lb();
    for (int it = 0; it < niter; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      const bool got = lane == 0 ? mbar_wait(empty_bar(s), ph ^ 1u, 1) : true;
      if (!__shfl_sync(0xffffffffu, got ? 1 : 0, 0)) break;
      const int o = it / used_chunks, kc = chunk0 + it % used_chunks;
      const int4 ov = offs[cls * 189 + o];
      const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
      const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
      const int sc = (scx << 2) | (scy << 1) | scz;
      const int shx = (gx - scx) / 2, shy = (gy - scy) / 2, shz = (gz - scz) / 2;  // parent-grid step
      const uint32_t st = base + s * STAGE_BYTES;
      // chunks kc < split_chunks take three products and need the lo halves (of B only its
      // first split_rows rows, the box of mapBlo); the others take hi x hi alone
      const bool three = kc < split_chunks;
      const uint32_t bhi_bytes = (uint32_t)ncols * BK * 2;  // the B box holds the first ncols rows i
      if (lane == 0) {
        mbar_expect_tx(full_bar(s), three ? 2 * A2_BYTES + bhi_bytes + BLO2_BYTES : A2_BYTES + bhi_bytes);
        tma_load_3d(st + 2 * A2_BYTES, &mapBhi, full_bar(s), kc * BK, 0, ov.x);
        if (three) tma_load_3d(st + 2 * A2_BYTES + B_BYTES, &mapBlo, full_bar(s), kc * BK, 0, ov.x);
      }
      __syncwarp();
      // a slot past the last set or list entry loads a valid box: the same bytes
      if (lane < nslot) {
        const int sidx = set_k * 8 + sc;
        tma_load_5d(st + lane * box_bytes, &mapAhi, full_bar(s), kc * BK, x0_k + shx, y0_k + shy, z0_k + shz, sidx);
        if (three)
          tma_load_5d(st + A2_BYTES + lane * box_bytes, &mapAlo, full_bar(s), kc * BK, x0_k + shx, y0_k + shy,
                      z0_k + shz, sidx);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    uint32_t acc = 0;
    for (int it = 0; it < niter; ++it) {
      const int s = it % STAGES;
      const uint32_t ph = (uint32_t)(it / STAGES) & 1u;
      if (!mbar_wait(full_bar(s), ph, 2)) break;
      tc_fence_after();
      const uint32_t st = base + s * STAGE_BYTES;
      const int k0 = (it % used_chunks == 0) ? kstep0 : 0;
      const bool three = chunk0 + it % used_chunks < split_chunks;
      const uint32_t id_part = idesc(split_rows), id_all = idesc(ncols);
      for (int ks = k0; ks < KS; ++ks) {
        const uint64_t bhi = sw64_desc(st + 2 * A2_BYTES + ks * 32);
        const uint64_t blo = sw64_desc(st + 2 * A2_BYTES + B_BYTES + ks * 32);
#pragma unroll
        for (int h = 0; h < 2; ++h) {  // the two 128-target halves of the box, accumulators h * 256
          const uint64_t ahi = sw64_desc(st + h * A_BYTES + ks * 32);
          const uint64_t alo = sw64_desc(st + A2_BYTES + h * A_BYTES + ks * 32);
          mma_bf16(tmem + h * 256, ahi, bhi, acc, id_all);  // all ncols outputs (the first initialises)
          if (three) {                              // corrections for the outputs i < split_rows
            mma_bf16(tmem + h * 256, ahi, blo, 1u, id_part);
            mma_bf16(tmem + h * 256, alo, bhi, 1u, id_part);
          }
        }
        acc = 1u;
      }
      mma_commit(empty_bar(s));
    }
    mma_commit(acc_bar);  // also after an early exit: the epilogue must not wait forever
  } else if (warp >= 2) {
    // ---------------- epilogue: TMEM -> registers -> Lacc
    const int q = warp & 3;  // TMEM lane quarter this warp may access
    const int row = q * 32 + lane;
    const int64_t P3 = (int64_t)P * P * P;
    if (Mlead) {
      // FP64 leading block of rows h * 128 + q * 32 + [0, 32): fragment m holds the 8 rows
      // 8m .. 8m + 7 of that range, this lane's A row being 8m + (lane >> 2)
      const int u = lane & 3, tr = lane >> 2;
      for (int h = 0; h < 2; ++h) {
        double acc[4][4][2];
        int ax[4], ay[4], az[4], aset[4];  // grid position and set of this lane's A rows
        bool aok[4];                       // whether those rows are written
#pragma unroll
        for (int m = 0; m < 4; ++m) {
#pragma unroll
          for (int f = 0; f < 4; ++f) acc[m][f][0] = acc[m][f][1] = 0.0;
          row_cell(h * 128 + q * 32 + 8 * m + tr, aset[m], ax[m], ay[m], az[m], aok[m]);
        }
        __syncwarp();
        for (int o = 0; o < 189; ++o) {
          const int4 ov = offs[cls * 189 + o];
          const int gx = cbx + ov.y, gy = cby + ov.z, gz = cbz + ov.w;
          const int scx = gx & 1, scy = gy & 1, scz = gz & 1;
          const int sc = (scx << 2) | (scy << 1) | scz;
          const int shx = (gx - scx) / 2, shy = (gy - scy) / 2, shz = (gz - scz) / 2;
          double2 a[4][2], b[4][2];
#pragma unroll
          for (int m = 0; m < 4; ++m) {
            const int px = ax[m] + shx, py = ay[m] + shy, pz = az[m] + shz;
            if ((unsigned)px < (unsigned)P && (unsigned)py < (unsigned)P && (unsigned)pz < (unsigned)P) {
              const double *Mc = Mlead + (int64_t)(aset[m] * 8 + sc) * P3 * BN + 4 * u;
              const double2 *src = reinterpret_cast<const double2 *>(Mc + (((int64_t)pz * P + py) * P + px) * BN);
              a[m][0] = src[0];
              a[m][1] = src[1];
            } else {
              a[m][0] = a[m][1] = make_double2(0.0, 0.0);
            }
          }
          const double *Ek = Erow + (int64_t)ov.x * BN * BN + 4 * u;
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            const double2 *src = reinterpret_cast<const double2 *>(Ek + (int64_t)(8 * f + tr) * BN);
            b[f][0] = src[0];
            b[f][1] = src[1];
          }
#pragma unroll
          for (int ks = 0; ks < 4; ++ks)
#pragma unroll
            for (int m = 0; m < 4; ++m) {
              const double av = (ks & 1) ? a[m][ks >> 1].y : a[m][ks >> 1].x;
#pragma unroll
              for (int f = 0; f < 4; ++f)
                dmma_f64(acc[m][f][0], acc[m][f][1], av, (ks & 1) ? b[f][ks >> 1].y : b[f][ks >> 1].x);
            }
        }
        // D fragment: row tr of fragment m (the A row of this lane), columns 8f + 2u + {0, 1}
#pragma unroll
        for (int m = 0; m < 4; ++m) {
          if (aok[m]) {
            const int64_t cell = (int64_t)(aset[m] * 8 + cls) * P3 + ((int64_t)az[m] * P + ay[m]) * P + ax[m];
            double *dst = Lacc + cell * BN;
#pragma unroll
            for (int f = 0; f < 4; ++f)
              *reinterpret_cast<double2 *>(dst + 8 * f + 2 * u) = make_double2(acc[m][f][0], acc[m][f][1]);
          }
        }
        __syncwarp();
      }
      __threadfence_block();
      __syncwarp();  // the rows written here are read back below by other lanes of this warp
    }
    const bool ok = mbar_wait(acc_bar, 0, 3);
    tc_fence_after();
    for (int h = 0; h < 2 && ok; ++h) {
      int tx, ty, tz, set;
      bool valid;  // rows of slots past the last set or list entry: read from TMEM, not written
      row_cell(h * 128 + row, set, tx, ty, tz, valid);
      const int64_t cell = (int64_t)(set * 8 + cls) * P3 + ((int64_t)tz * P + ty) * P + tx;
      double *dst = Lacc + cell * BN;
      int64_t mrow = 0;  // Morton row of the cell: set base + Morton index of its grid position
      if (Lsplit) mrow = (int64_t)set * 8 * P3 + grid_to_morton(2 * tx + cbx, 2 * ty + cby, 2 * tz + cbz, level);
      for (int col = 0; col < ncols; col += 32) {
        float v[32];
        __syncwarp();
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * 256 + col), v);
        if (!valid) continue;
        const bool add = col < ilead;  // ilead is a multiple of 32
        const bool fp = !Lsplit || col < 32;
        __align__(16) __nv_bfloat16 sh[32], sl[32];
#pragma unroll
        for (int i = 0; i < 32; i += 2) {
          double2 o = add ? *reinterpret_cast<const double2 *>(dst + col + i) : make_double2(0.0, 0.0);
          o.x += (double)v[i];
          o.y += (double)v[i + 1];
          if (fp) *reinterpret_cast<double2 *>(dst + col + i) = o;
          const double x0 = col + i < DNZ ? 0.0 : o.x, x1 = col + i + 1 < DNZ ? 0.0 : o.y;
          sh[i] = __double2bfloat16(x0);
          sl[i] = __double2bfloat16(x0 - (double)__bfloat162float(sh[i]));
          sh[i + 1] = __double2bfloat16(x1);
          sl[i + 1] = __double2bfloat16(x1 - (double)__bfloat162float(sh[i + 1]));
        }
        if (Lsplit) {
          uint4 *oh = reinterpret_cast<uint4 *>(Lsplit + mrow * BN + col);
          uint4 *ol = reinterpret_cast<uint4 *>(Lsplit + (nrows + mrow) * BN + col);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            oh[e] = reinterpret_cast<const uint4 *>(sh)[e];
            ol[e] = reinterpret_cast<const uint4 *>(sl)[e];
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// ---------------------------------------------------------------- wait probe
// Failure detection without a fault: an mbarrier that nothing arrives at, waited on with the
// bounded wait of the kernels above (at most `limit` try_wait polls). The wait must give up,
// record `code` in the status word and return, leaving the context usable.
__global__ void wait_probe_kernel(uint32_t limit, int code) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    mbar_init(b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (uint32_t i = 0; i < limit; ++i)
      if (mbar_try(b, 0)) return;  // cannot happen: no thread arrives
    atomicCAS(&g_tc_status, 0, code);
  }
}

// ---------------------------------------------------------------- splitting
// hi/lo bf16 split of src; for operators (r > 0) entries with i < zrows and j < zcols of
// each row-major r x r block are zeroed (the FP64 leading block).
__global__ void split_kernel(int64_t count, const double *__restrict__ src, __nv_bfloat16 *__restrict__ hi,
                             __nv_bfloat16 *__restrict__ lo, int r, int zrows, int zcols) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count; e += (int64_t)gridDim.x * blockDim.x) {
    double x = src[e];
    if (r > 0) {
      const int j = (int)(e % r), i = (int)((e / r) % r);
      if (i < zrows && j < zcols) x = 0.0;
    }
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[e] = h;
    lo[e] = __double2bfloat16(x - (double)__bfloat162float(h));
  }
}

// ---------------------------------------------------------------- projections
// Projection passes with double-buffered accumulators (mixed mode). Down projection in one
// pass: for the rows t < rows of a level (or slab),
//   F[t][n] = scale cs[n] (sum_{j < 16} L[cpg(row0 + t)][j] Dn(n, j)  +  sum_{16 <= j < 32 kc1} L'[t][j] Dn(n, j))
// the first sum in FP64 (DMMA, the epilogue warps), the second from the split-BF16 rows L'
// (Morton order) on the tensor cores, F written once. Persistent CTAs walk tiles of 128 rows
// x 256 columns (tile = 2 row-tile + column block); two 256-column accumulators in tensor
// memory let the MMA of a CTA's next tile run while its epilogue drains the previous one.
// The up projection (UP) runs the same kernel without the FP64 part (its FP64 columns come
// from proj_narrow_kernel): M[cpg(row0 + t)][j] for j >= col_skip from the split S rows, one
// 256-column block, output rows in the class-major parent grid.
// Eight epilogue warps, two per tensor-memory lane quarter q (rows 32q .. 32q + 31 of the
// tile), so that each SM sub-partition interleaves two of them: per 32-column chunk, warp half
// h computes the FP64 part of rows 32q + 16h + [0, 16) as DMMA fragments (k-slot u of step ks
// standing for component 4u + ks, so that a thread's A and B fragments are 32 contiguous
// bytes) into the quarter's staging tile; after a barrier of the pair it adds the
// tensor-memory columns 16h .. 16h + 15 of all 32 rows, and after a second barrier it writes
// its 16 rows of the chunk (256 coalesced bytes per store). Two staging tiles alternate by
// chunk.
constexpr int PD_STAGES = 3, PD_SROW = 33;  // staging rows of 33 doubles: few bank conflicts
constexpr int PD_STAGING = 4 * 2 * 32 * PD_SROW * 8;
constexpr int PD_THREADS = 320;
constexpr int DN_LEAD = 16;  // FP64 components of the down projection (the split rows zero them)
constexpr int PD_SMEM = PD_STAGES * STAGE_BYTES + PD_STAGING + 1024 /*align*/ + 256 /*barriers*/;
static_assert(PD_SMEM <= 232448, "down-projection stages exceed the shared memory of a CTA");

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void pair_bar(int q) {  // the two epilogue warps of lane quarter q
  asm volatile("bar.sync %0, 64;" ::"r"(1 + q) : "memory");
}

template <bool UP>
__global__ void __launch_bounds__(PD_THREADS, 1)
    proj_fused_kernel(const __grid_constant__ CUtensorMap mapAhi, const __grid_constant__ CUtensorMap mapAlo,
                      const __grid_constant__ CUtensorMap mapBhi, const __grid_constant__ CUtensorMap mapBlo,
                      const double *__restrict__ Lfp, int ldl, const double *__restrict__ Dlead,
                      double *__restrict__ F, int ldf, int64_t rows, int level, int64_t row0, int kc0, int kc1,
                      const double *__restrict__ cs, double scale, int64_t ntiles, int col_skip,
                      const int64_t *__restrict__ rowlist) {
  constexpr int ncb = UP ? 1 : 2;  // 256-column blocks: r = 256 outputs up, n3 = 512 down
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *gbase = smem_raw + (base - raw);
  double *staging = reinterpret_cast<double *>(gbase + PD_STAGES * STAGE_BYTES);
  const uint32_t bar_base = base + PD_STAGES * STAGE_BYTES + PD_STAGING;
  uint64_t *bars = reinterpret_cast<uint64_t *>(gbase + PD_STAGES * STAGE_BYTES + PD_STAGING);
  // bars: full[S], empty[S], acc_full[2], acc_empty[2]; then the tmem slot and the pair flags
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * PD_STAGES + 4);
  volatile int *pair_ok = reinterpret_cast<volatile int *>(tmem_slot + 4);
  auto full_bar = [&](int st) { return bar_base + 8u * st; };
  auto empty_bar = [&](int st) { return bar_base + 8u * (PD_STAGES + st); };
  auto accf_bar = [&](int b) { return bar_base + 8u * (2 * PD_STAGES + b); };
  auto acce_bar = [&](int b) { return bar_base + 8u * (2 * PD_STAGES + 2 + b); };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int st = 0; st < PD_STAGES; ++st) {
      mbar_init(full_bar(st), 1);
      mbar_init(empty_bar(st), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf_bar(b), 1);  // tcgen05.commit of the tile's last MMA
      mbar_init(acce_bar(b), 8);  // one arrival per epilogue warp
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(512)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int nk = kc1 - kc0;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    int it = 0;
    bool alive = true;
    for (int64_t tile = blockIdx.x; tile < ntiles && alive; tile += gridDim.x) {
      const int t0 = (int)((tile / ncb) * BM), col0 = (int)(tile % ncb) * BN;
      for (int kc = kc0; kc < kc1; ++kc, ++it) {
        const int st = it % PD_STAGES;
        const uint32_t ph = (uint32_t)(it / PD_STAGES) & 1u;
        if (!mbar_wait(empty_bar(st), ph ^ 1u, 21)) {
          alive = false;
          break;
        }
        const uint32_t sa = base + st * STAGE_BYTES;
        mbar_expect_tx(full_bar(st), STAGE_BYTES);
        tma_load_2d(sa, &mapAhi, full_bar(st), kc * BK, t0);
        tma_load_2d(sa + A_BYTES, &mapAlo, full_bar(st), kc * BK, t0);
        tma_load_2d(sa + 2 * A_BYTES, &mapBhi, full_bar(st), kc * BK, col0);
        tma_load_2d(sa + 2 * A_BYTES + B_BYTES, &mapBlo, full_bar(st), kc * BK, col0);
      }
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    int it = 0, lt = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++lt) {
      const int b = lt & 1;
      const uint32_t use = (uint32_t)(lt >> 1) & 1u;
      if (!mbar_wait(acce_bar(b), use ^ 1u, 22)) break;  // the epilogue has drained accumulator b
      tc_fence_after();
      bool ok = true;
      for (int kc = 0; kc < nk; ++kc, ++it) {
        const int st = it % PD_STAGES;
        const uint32_t ph = (uint32_t)(it / PD_STAGES) & 1u;
        if (!mbar_wait(full_bar(st), ph, 23)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t sa = base + st * STAGE_BYTES;
        for (int ks = 0; ks < KS; ++ks) {
          const uint64_t ahi = sw64_desc(sa + ks * 32), alo = sw64_desc(sa + A_BYTES + ks * 32);
          const uint64_t bhi = sw64_desc(sa + 2 * A_BYTES + ks * 32);
          const uint64_t blo = sw64_desc(sa + 2 * A_BYTES + B_BYTES + ks * 32);
          const uint32_t acc = (kc > 0 || ks > 0) ? 1u : 0u;
          mma_bf16(tmem + b * BN, ahi, bhi, acc);
          mma_bf16(tmem + b * BN, ahi, blo, 1u);
          mma_bf16(tmem + b * BN, alo, bhi, 1u);
        }
        mma_commit(empty_bar(st));
      }
      mma_commit(accf_bar(b));
      if (!ok) break;
    }
  } else if (warp >= 2) {
    // ---------------- epilogue: FP64 leading part + tensor-memory rows -> F
    const int q = warp & 3, h = (warp - 2) >> 2;
    const int u = lane & 3, tr = lane >> 2;
    double *stg0 = staging + q * 2 * 32 * PD_SROW;
    int lt = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++lt) {
      const int b = lt & 1;
      const uint32_t use = (uint32_t)(lt >> 1) & 1u;
      const int64_t tq = (tile / ncb) * BM + q * 32;  // first row of the quarter
      const int col0 = (int)(tile % ncb) * BN;
      // output row of row 16h + (lane & 15) of the quarter (up: read back by shuffles)
      int64_t orow = tq + 16 * h + (lane & 15);
      if (UP && orow < rows) orow = morton_to_cpg_row(pass_cell(rowlist, row0, orow), level);
      // A fragments: rows tq + 16h + 8m + tr, components 4u .. 4u + 3 (FP64 L in cpg order)
      double2 a[2][2];
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int64_t t = tq + 16 * h + 8 * m + tr;
        if (!UP && t < rows) {
          const int64_t crow = morton_to_cpg_row(pass_cell(rowlist, row0, t), level);
          const double2 *src = reinterpret_cast<const double2 *>(Lfp + crow * ldl + 4 * u);
          a[m][0] = src[0];
          a[m][1] = src[1];
        } else {
          a[m][0] = a[m][1] = make_double2(0.0, 0.0);
        }
      }
      // a wait that gave up (status word set) ends the tiles of both warps of the pair
      const bool okw = __all_sync(0xffffffffu, mbar_wait(accf_bar(b), use, 24));
      if (lane == 0) pair_ok[2 * q + h] = okw ? 1 : 0;
      pair_bar(q);
      if (!(pair_ok[2 * q] && pair_ok[2 * q + 1])) break;
      tc_fence_after();
      const int nrow = rows - tq < 32 ? (int)(rows - tq) : 32;  // valid rows of the quarter
      for (int cc = 0; cc < BN / 32; ++cc) {
        const int n0 = col0 + cc * 32;
        if (n0 + 32 <= col_skip) continue;  // the same for both warps of the pair
        double *stg = stg0 + (cc & 1) * 32 * PD_SROW;
        double acc[2][4][2];
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
          for (int f = 0; f < 4; ++f) acc[m][f][0] = acc[m][f][1] = 0.0;
#pragma unroll
        for (int f = 0; f < (UP ? 0 : 4); ++f) {
          const double2 *src =
              reinterpret_cast<const double2 *>(Dlead + (int64_t)(n0 + 8 * f + tr) * DN_LEAD + 4 * u);
          const double2 bf[2] = {src[0], src[1]};
#pragma unroll
          for (int ks = 0; ks < 4; ++ks) {
            const double bv = (ks & 1) ? bf[ks >> 1].y : bf[ks >> 1].x;
#pragma unroll
            for (int m = 0; m < 2; ++m)
              dmma_f64(acc[m][f][0], acc[m][f][1], (ks & 1) ? a[m][ks >> 1].y : a[m][ks >> 1].x, bv);
          }
        }
        // stage the FP64 part: row 16h + 8m + tr, columns 8f + 2u + {0, 1}
#pragma unroll
        for (int m = 0; m < 2; ++m)
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            stg[(16 * h + 8 * m + tr) * PD_SROW + 8 * f + 2 * u] = acc[m][f][0];
            stg[(16 * h + 8 * m + tr) * PD_SROW + 8 * f + 2 * u + 1] = acc[m][f][1];
          }
        pair_bar(q);
        float v[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN + cc * 32 + 16 * h), v);  // every lane
#pragma unroll
        for (int c = 0; c < 16; ++c) stg[lane * PD_SROW + 16 * h + c] += (double)v[c];
        pair_bar(q);
        const double sc = cs ? scale * cs[n0 + lane] : scale;
        if (nrow == 32) {
#pragma unroll
          for (int rr = 0; rr < 16; ++rr) {
            const int64_t o = UP ? __shfl_sync(0xffffffffu, orow, rr) : tq + 16 * h + rr;
            F[o * ldf + n0 + lane] = sc * stg[(16 * h + rr) * PD_SROW + lane];
          }
        } else {
          for (int rr = 0; rr < 16; ++rr) {
            const int64_t o = UP ? __shfl_sync(0xffffffffu, orow, rr) : tq + 16 * h + rr;
            if (16 * h + rr < nrow) F[o * ldf + n0 + lane] = sc * stg[(16 * h + rr) * PD_SROW + lane];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce_bar(b));
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512) : "memory");
  }
}

// Dlead[n][j] = B[j][n] for j < lead: the leading rows of a K x N operator, transposed.
__global__ void lead_transpose_kernel(int K, int N, int lead, const double *__restrict__ B, double *__restrict__ Dlead) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N * lead; e += gridDim.x * blockDim.x)
    Dlead[e] = B[(int64_t)(e % lead) * N + e / lead];
}

// dst = [hi | lo] split of rows x K values; row t comes from src row cpg(row0 + t) of
// `level` when gather != 0 (Morton order from the class-major grid), else from row t.
// One warp per row (grid-stride), 8 consecutive values per lane and step: two 32-byte
// loads, one 16-byte store per plane. K is a multiple of 256.
__global__ void split_rows_kernel(int64_t rows, int K, const double *__restrict__ src, int gather, int level,
                                  int64_t row0, __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo,
                                  int zlead, const int64_t *__restrict__ rowlist) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t t = warp; t < rows; t += nwarps) {
    const int64_t sr = gather ? morton_to_cpg_row(pass_cell(rowlist, row0, t), level) : t;
    const double4 *in = reinterpret_cast<const double4 *>(src + sr * K);
    uint4 *oh = reinterpret_cast<uint4 *>(hi + t * K), *ol = reinterpret_cast<uint4 *>(lo + t * K);
    for (int c = lane; c < K / 8; c += 32) {
      const double4 a = in[2 * c], b = in[2 * c + 1];
      double x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
      if (8 * c < zlead) {  // components below zlead are computed elsewhere (FP64)
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = 8 * c + i < zlead ? 0.0 : x[i];
      }
      __align__(16) __nv_bfloat16 h[8], l[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        h[i] = __double2bfloat16(x[i]);
        l[i] = __double2bfloat16(x[i] - (double)__bfloat162float(h[i]));
      }
      oh[c] = *reinterpret_cast<const uint4 *>(h);
      ol[c] = *reinterpret_cast<const uint4 *>(l);
    }
  }
}

// out[c][r] = split(src[r][c]) for an R x Cn row-major FP64 matrix (hi, lo: Cn x R bf16);
// rows c < zero_rows of the output are zero.
__global__ void transpose_split_kernel(int R, int Cn, const double *__restrict__ src, __nv_bfloat16 *__restrict__ hi,
                                       __nv_bfloat16 *__restrict__ lo, int zero_rows) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < R * Cn; e += gridDim.x * blockDim.x) {
    const int c = e / R, r = e % R;
    const double x = c < zero_rows ? 0.0 : src[(int64_t)r * Cn + c];
    const __nv_bfloat16 h = __double2bfloat16(x);
    hi[e] = h;
    lo[e] = __double2bfloat16(x - (double)__bfloat162float(h));
  }
}

}  // namespace tc

// --------------------------------------------------------------------- host side
using PFN_encodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled encode_fn() {
  static PFN_encodeTiled fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_encodeTiled)p;
  }
  return fn;
}

struct TcOps {
  int r = 0, lead = 0, lead_rows = 0;
  __nv_bfloat16 *Ehi = nullptr, *Elo = nullptr;
  CUtensorMap mapBhi, mapBlo;
  CUtensorMap mapBlo_part;  // the first TC_SPLIT_ROWS rows i of the lo operator chunk
};

int tc_supported() {
  int dev = 0, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return 0;
  return major == 10 && encode_fn() != nullptr;
}

static int make_map(CUtensorMap *m, void *ptr, int rank, const cuuint64_t *dims, const cuuint64_t *strides_bytes,
                    const cuuint32_t *box) {
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult rc = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, ptr, dims, strides_bytes, box, es,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (rc != CUDA_SUCCESS) {
    char buf[96];
    snprintf(buf, sizeof(buf), "cuTensorMapEncodeTiled failed (%d)", (int)rc);
    return bbfmm_set_error(BBFMM_ERR_CUDA, buf);
  }
  return BBFMM_OK;
}

int tc_prepare_operators(int r, const double *Ert, int lead, int lead_rows, void **out, cudaStream_t s) {
  *out = nullptr;
  if (r != 256) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core M2L is built for r = 256 (n = 8)");
  if (lead < 0 || lead > 64 || lead % 16) return bbfmm_set_error(BBFMM_ERR_ARG, "lead must be 0, 16, 32, 48 or 64");
  if (lead_rows < 32 || lead_rows > r || lead_rows % 32)
    return bbfmm_set_error(BBFMM_ERR_ARG, "lead_rows must be a multiple of 32 in [32, 256]");
  if (!encode_fn()) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  TcOps *ops = new TcOps();
  ops->r = r;
  ops->lead = lead;
  ops->lead_rows = lead_rows;
  const size_t cnt = (size_t)BBFMM_NUM_OFFSETS * r * r;
  if (cudaMalloc(&ops->Ehi, cnt * 2) != cudaSuccess || cudaMalloc(&ops->Elo, cnt * 2) != cudaSuccess) {
    tc_free_operators(ops);
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "operator split allocation failed");
  }
  tc::split_kernel<<<148 * 8, 256, 0, s>>>((int64_t)cnt, Ert, ops->Ehi, ops->Elo, r, lead_rows < r ? lead_rows : 0,
                                           lead);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    tc_free_operators(ops);
    return bbfmm_set_cuda_error(e, "split operators", __FILE__, __LINE__);
  }
  const cuuint64_t dims[3] = {(cuuint64_t)r, (cuuint64_t)r, (cuuint64_t)BBFMM_NUM_OFFSETS};
  const cuuint64_t strides[2] = {(cuuint64_t)r * 2, (cuuint64_t)r * r * 2};
  const cuuint32_t box[3] = {tc::BK, (cuuint32_t)tc::BN, 1};
  int rc = make_map(&ops->mapBhi, ops->Ehi, 3, dims, strides, box);
  if (rc == BBFMM_OK) rc = make_map(&ops->mapBlo, ops->Elo, 3, dims, strides, box);
  const cuuint32_t box_part[3] = {tc::BK, (cuuint32_t)TC_SPLIT_ROWS, 1};
  if (rc == BBFMM_OK) rc = make_map(&ops->mapBlo_part, ops->Elo, 3, dims, strides, box_part);
  if (rc != BBFMM_OK) {
    tc_free_operators(ops);
    return rc;
  }
  *out = ops;
  return BBFMM_OK;
}

void tc_free_operators(void *p) {
  TcOps *ops = (TcOps *)p;
  if (!ops) return;
  if (ops->Ehi) cudaFree(ops->Ehi);
  if (ops->Elo) cudaFree(ops->Elo);
  delete ops;
}

size_t tc_split_bytes(int r, int64_t ncell) { return (size_t)ncell * r * 2 * 2; }

// Split, transposed copies of the projection operators for proj_fused_kernel.
struct TcProj {
  int n3 = 0, r = 0, lead = 0;
  __nv_bfloat16 *up = nullptr;  // [hi | lo] of Bup^T: r x n3, rows j < lead zero
  __nv_bfloat16 *dn = nullptr;  // [hi | lo] of Bdn^T: n3 x r
  double *dn_lead = nullptr;    // FP64 Bdn^T for j < DN_LEAD: n3 x DN_LEAD
  CUtensorMap up_hi, up_lo, dn_hi, dn_lo;
};

static int map2d(CUtensorMap *m, const void *ptr, int64_t rows, int K, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)K * 2};
  const cuuint32_t box[2] = {tc::BK, (cuuint32_t)box_rows};
  return make_map(m, (void *)ptr, 2, dims, strides, box);
}

int tc_prepare_projections(int n3, int r, const double *Bup, const double *Bdn, int lead, void **out,
                           cudaStream_t s) {
  *out = nullptr;
  if (r != tc::BN || n3 % tc::BN || lead % 16 || lead <= 0 || lead >= r)
    return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core projections need n = 8 (r = 256)");
  if (!encode_fn()) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  TcProj *p = new TcProj();
  p->n3 = n3; p->r = r; p->lead = lead;
  const size_t cnt = (size_t)n3 * r;
  if (cudaMalloc(&p->up, cnt * 4) != cudaSuccess || cudaMalloc(&p->dn, cnt * 4) != cudaSuccess ||
      cudaMalloc(&p->dn_lead, (size_t)n3 * tc::DN_LEAD * 8) != cudaSuccess) {
    tc_free_projections(p);
    return bbfmm_set_error(BBFMM_ERR_NOMEM, "projection operator split allocation failed");
  }
  tc::transpose_split_kernel<<<148, 256, 0, s>>>(n3, r, Bup, p->up, p->up + cnt, lead);  // Bup: n3 x r
  tc::transpose_split_kernel<<<148, 256, 0, s>>>(r, n3, Bdn, p->dn, p->dn + cnt, 0);     // Bdn: r x n3
  tc::lead_transpose_kernel<<<64, 256, 0, s>>>(r, n3, tc::DN_LEAD, Bdn, p->dn_lead);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    tc_free_projections(p);
    return bbfmm_set_cuda_error(e, "split projection operators", __FILE__, __LINE__);
  }
  int rc = map2d(&p->up_hi, p->up, r, n3, tc::BN);
  if (rc == BBFMM_OK) rc = map2d(&p->up_lo, p->up + cnt, r, n3, tc::BN);
  if (rc == BBFMM_OK) rc = map2d(&p->dn_hi, p->dn, n3, r, tc::BN);
  if (rc == BBFMM_OK) rc = map2d(&p->dn_lo, p->dn + cnt, n3, r, tc::BN);
  if (rc != BBFMM_OK) {
    tc_free_projections(p);
    return rc;
  }
  *out = p;
  return BBFMM_OK;
}

void tc_free_projections(void *v) {
  TcProj *p = (TcProj *)v;
  if (!p) return;
  if (p->up) cudaFree(p->up);
  if (p->dn) cudaFree(p->dn);
  if (p->dn_lead) cudaFree(p->dn_lead);
  delete p;
}

// Down projection of `rows` Morton rows (row0 ..) of `level` in one pass: F[t][l] = scale Kw[l]
// (sum_{j < 16} L[cpg(row0 + t)][j] Bdn[j][l] in FP64 + sum_{16 <= j < rank} L'[t][j] Bdn[j][l]
// from the split rows L' = Asplit, whose components j < 16 are zero), F rows n3 apart, assigned.
int launch_proj_down(const void *pv, const void *Asplit, const double *Lfp, int64_t rows, double *F, int level,
                     int64_t row0, const double *cs, double scale, cudaStream_t s, int rank, const int64_t *rowlist) {
  const TcProj *p = (const TcProj *)pv;
  if (!p) return bbfmm_set_error(BBFMM_ERR_STATE, "tensor-core projections not prepared");
  if (rows <= 0) return BBFMM_OK;
  if (p->n3 != 2 * tc::BN) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "fused down projection: n3 = 512");
  const __nv_bfloat16 *hi = (const __nv_bfloat16 *)Asplit;
  const __nv_bfloat16 *lo = hi + (size_t)rows * p->r;
  CUtensorMap ahi, alo;
  int rc = map2d(&ahi, hi, rows, p->r, tc::BM);
  if (rc == BBFMM_OK) rc = map2d(&alo, lo, rows, p->r, tc::BM);
  if (rc != BBFMM_OK) return rc;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc::proj_fused_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc::PD_SMEM);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "proj_fused smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  const int64_t ntiles = ((rows + tc::BM - 1) / tc::BM) * (p->n3 / tc::BN);
  const int grid = (int)(ntiles < 148 ? ntiles : 148);
  tc::proj_fused_kernel<false><<<grid, tc::PD_THREADS, tc::PD_SMEM, s>>>(
      ahi, alo, p->dn_hi, p->dn_lo, Lfp, p->r, p->dn_lead, F, p->n3, rows, level, row0, 0,
      (rank > 0 ? rank : p->r) / tc::BK, cs, scale, ntiles, 0, rowlist);
  return bbfmm_set_cuda_error(cudaGetLastError(), "proj_down", __FILE__, __LINE__);
}

// Up projection of `rows` Morton rows (row0 ..) of `level`: M[cpg(row0 + t)][j] = sum_l S'[t][l]
// Bup[l][j] from the split S rows (Asplit, rows x n3), assigned for every j; the split operator
// is zero for j < lead, whose FP64 values proj_narrow_kernel writes afterwards.
int launch_proj_up(const void *pv, const void *Asplit, int64_t rows, double *M, int level, int64_t row0,
                   cudaStream_t s, const int64_t *rowlist) {
  const TcProj *p = (const TcProj *)pv;
  if (!p) return bbfmm_set_error(BBFMM_ERR_STATE, "tensor-core projections not prepared");
  if (rows <= 0) return BBFMM_OK;
  const __nv_bfloat16 *hi = (const __nv_bfloat16 *)Asplit;
  const __nv_bfloat16 *lo = hi + (size_t)rows * p->n3;
  CUtensorMap ahi, alo;
  int rc = map2d(&ahi, hi, rows, p->n3, tc::BM);
  if (rc == BBFMM_OK) rc = map2d(&alo, lo, rows, p->n3, tc::BM);
  if (rc != BBFMM_OK) return rc;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc::proj_fused_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tc::PD_SMEM);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "proj_fused smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  const int64_t ntiles = (rows + tc::BM - 1) / tc::BM;
  const int grid = (int)(ntiles < 148 ? ntiles : 148);
  tc::proj_fused_kernel<true><<<grid, tc::PD_THREADS, tc::PD_SMEM, s>>>(
      ahi, alo, p->up_hi, p->up_lo, nullptr, 0, nullptr, M, p->r, rows, level, row0, 0, p->n3 / tc::BK, nullptr, 1.0,
      ntiles, 0, rowlist);
  return bbfmm_set_cuda_error(cudaGetLastError(), "proj_up", __FILE__, __LINE__);
}

// [hi | lo] split of rows x K FP64 values; gather != 0 reads row t from the cpg row of Morton
// cell row0 + t of `level`.
int tc_split_rows(int64_t rows, int K, const double *src, int gather, int level, int64_t row0, void *dst,
                  cudaStream_t s, int zlead, const int64_t *rowlist) {
  if (K % 256) return bbfmm_set_error(BBFMM_ERR_ARG, "split rows: K must be a multiple of 256");
  __nv_bfloat16 *hi = (__nv_bfloat16 *)dst;
  tc::split_rows_kernel<<<148 * 16, 256, 0, s>>>(rows, K, src, gather, level, row0, hi, hi + rows * K, zlead,
                                                 rowlist);
  return bbfmm_set_cuda_error(cudaGetLastError(), "split", __FILE__, __LINE__);
}

// Msplit = [hi plane | lo plane], each ncell_total * r bf16, same cell order as M.
int tc_split_multipoles(int r, int64_t ncell, const double *M, int lead, void *Msplit, cudaStream_t s) {
  (void)lead;
  __nv_bfloat16 *hi = (__nv_bfloat16 *)Msplit;
  __nv_bfloat16 *lo = hi + (size_t)ncell * r;
  tc::split_kernel<<<148 * 8, 256, 0, s>>>(ncell * r, M, hi, lo, 0, 0, 0);
  return bbfmm_set_cuda_error(cudaGetLastError(), "split multipoles", __FILE__, __LINE__);
}

// Whether launch_m2l_tc runs the two-box kernel with the FP64 leading block inside it (given
// the FP64 multipoles and operators): the adaptive product map at full split rows and a
// leading block of i < 32, j < 16.
bool tc_fuses_lead(const void *opsv, int nprod, int rank) {
  const TcOps *ops = (const TcOps *)opsv;
  if (rank <= 0) rank = tc::BN;
  return ops && nprod == 0 && rank >= TC_SPLIT_ROWS && ops->lead == 16 && ops->lead_rows == 32;
}

int launch_m2l_tc(int r, const void *Msplit, int64_t ncell_total, int64_t cell_offset, const void *opsv, double *Lacc,
                  int level, const int4 *offs, cudaStream_t s, int nsets, int nprod, int rank, const double *Mlead,
                  const double *Erow, void *Lsplit, const int4 *boxes, int nboxes, int lgeom) {
  const TcOps *ops = (const TcOps *)opsv;
  if (nprod != 0 && nprod != 1 && nprod != 3)
    return bbfmm_set_error(BBFMM_ERR_ARG, "tensor-core products must be 0 (adaptive), 1 or 3");
  // 3: three products everywhere; 1: one everywhere; 0: three only where one would not do
  if (rank <= 0) rank = tc::BN;
  if (rank % tc::BK || rank > tc::BN) return bbfmm_set_error(BBFMM_ERR_ARG, "rank must be a multiple of 32 <= 256");
  const int nchunk = rank / tc::BK;
  int split_chunks = nprod == 3 ? nchunk : (nprod == 1 ? 0 : TC_SPLIT_CHUNKS);
  if (split_chunks > nchunk) split_chunks = nchunk;
  int split_rows = nprod == 0 ? TC_SPLIT_ROWS : rank;
  if (split_rows > rank) split_rows = rank;
  if (!ops || r != 256) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "tensor-core M2L needs r = 256 operators");
  const int P = 1 << (level - 1);
  // the adaptive map runs two 128-target halves of a 256-target box per CTA (m2l_tc2_kernel)
  const bool two = nprod == 0 && split_rows == TC_SPLIT_ROWS;
  if (level < (two ? TC2_MIN_LEVEL : TC_MIN_LEVEL))
    return bbfmm_set_error(BBFMM_ERR_ARG, two ? "tensor-core M2L needs level >= 2" : "tensor-core M2L needs level >= 4");
  if (nsets < 1) return bbfmm_set_error(BBFMM_ERR_ARG, "tensor-core M2L needs a set");
  const Tc2Box g2 = boxes ? Tc2Box{lgeom & 15, (lgeom >> 4) & 15, (lgeom >> 8) & 15} : tc2_box(level);
  if (boxes && (g2.lb() < 3 || g2.lb() > 8 || (1 << g2.lx) > P || (1 << g2.ly) > P || (1 << g2.lz) > P))
    return bbfmm_set_error(BBFMM_ERR_ARG, "box-list geometry: 8 to 256 rows inside the class grid");
  const __nv_bfloat16 *hi = (const __nv_bfloat16 *)Msplit + (size_t)cell_offset * r;
  const __nv_bfloat16 *lo = (const __nv_bfloat16 *)Msplit + (size_t)(ncell_total + cell_offset) * r;
  CUtensorMap mapAhi, mapAlo;
  // the class dimension runs over the 8 sibling classes of every stacked set
  const cuuint64_t dims[5] = {(cuuint64_t)r, (cuuint64_t)P, (cuuint64_t)P, (cuuint64_t)P, (cuuint64_t)8 * nsets};
  const cuuint64_t strides[4] = {(cuuint64_t)r * 2, (cuuint64_t)r * 2 * P, (cuuint64_t)r * 2 * P * P,
                                 (cuuint64_t)r * 2 * P * P * P};
  const cuuint32_t box[5] = {tc::BK, two ? 1u << g2.lx : (cuuint32_t)tc::BOX_X,
                             two ? 1u << g2.ly : (cuuint32_t)tc::BOX_Y, two ? 1u << g2.lz : (cuuint32_t)tc::BOX_Z, 1};
  int rc = make_map(&mapAhi, (void *)hi, 5, dims, strides, box);
  if (rc == BBFMM_OK) rc = make_map(&mapAlo, (void *)lo, 5, dims, strides, box);
  if (rc != BBFMM_OK) return rc;
  // with a full-width leading strip its K-steps are skipped; otherwise every K-step runs
  const int kfirst = ops->lead_rows >= r ? ops->lead / 16 : 0;
  const int ilead = ops->lead > 0 ? ops->lead_rows : 0;
  // B boxes of the first `rank` operator rows (the effective rank); the lo box keeps its
  // split_rows rows (box maps built here when they differ from the prepared ones)
  CUtensorMap mapBhi = ops->mapBhi, mapBlo = split_rows < tc::BN ? ops->mapBlo_part : ops->mapBlo;
  {
    const cuuint64_t bd[3] = {(cuuint64_t)r, (cuuint64_t)r, (cuuint64_t)BBFMM_NUM_OFFSETS};
    const cuuint64_t bs[2] = {(cuuint64_t)r * 2, (cuuint64_t)r * r * 2};
    if (rank != tc::BN) {
      const cuuint32_t bb[3] = {tc::BK, (cuuint32_t)rank, 1};
      rc = make_map(&mapBhi, ops->Ehi, 3, bd, bs, bb);
    }
    if (rc == BBFMM_OK && split_rows != tc::BN && split_rows != TC_SPLIT_ROWS) {
      const cuuint32_t bl[3] = {tc::BK, (cuuint32_t)split_rows, 1};
      rc = make_map(&mapBlo, ops->Elo, 3, bd, bs, bl);
    }
    if (rc != BBFMM_OK) return rc;
  }
  if (two) {
    static bool attr2 = false;
    if (!attr2) {
      cudaError_t e =
          cudaFuncSetAttribute(tc::m2l_tc2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM2_BYTES);
      if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "m2l_tc2 smem attribute", __FILE__, __LINE__);
      attr2 = true;
    }
    const bool fuse = Mlead && Erow && tc_fuses_lead(ops, nprod, rank) && kfirst == 0 && ilead == 32;
    if (Lsplit && !fuse) return bbfmm_set_error(BBFMM_ERR_ARG, "split M2L output needs the fused leading block");
    const int spl = 1 << (8 - g2.lb());  // listed blocks per tile
    if (boxes && (nboxes < 0 || nboxes > (int64_t)nsets * (P >> g2.lx) * (P >> g2.ly) * (P >> g2.lz)))
      return bbfmm_set_error(BBFMM_ERR_ARG, "box list longer than the level");
    if (boxes && nboxes == 0) return BBFMM_OK;
    const int64_t tiles2 = boxes ? 8 * (int64_t)((nboxes + spl - 1) / spl) : tc2_tiles(level, nsets);
    tc::m2l_tc2_kernel<<<(unsigned)tiles2, 192, tc::SMEM2_BYTES, s>>>(
        mapAhi, mapAlo, mapBhi, mapBlo, Lacc, level, offs, kfirst, ilead, split_chunks, rank, fuse ? Mlead : nullptr,
        fuse ? Erow : nullptr, (__nv_bfloat16 *)Lsplit, 8 * (int64_t)nsets * P * P * P, boxes, nboxes, lgeom, nsets);
    return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_tc2", __FILE__, __LINE__);
  }
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tc::m2l_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
    if (e != cudaSuccess) return bbfmm_set_cuda_error(e, "m2l_tc smem attribute", __FILE__, __LINE__);
    attr = true;
  }
  if (boxes) return bbfmm_set_error(BBFMM_ERR_UNSUPPORTED, "box lists are for the two-box tensor-core M2L");
  const int tiles = 8 * nsets * (P / tc::BOX_X) * (P / tc::BOX_Y) * (P / tc::BOX_Z);
  tc::m2l_tc_kernel<<<tiles, 192, tc::SMEM_BYTES, s>>>(mapAhi, mapAlo, mapBhi, mapBlo, Lacc, level, offs, kfirst,
                                                       ilead, split_chunks, split_rows, rank);
  return bbfmm_set_cuda_error(cudaGetLastError(), "m2l_tc", __FILE__, __LINE__);
}

// Runs the wait probe; returns the status word it left (then cleared), or -1 on a CUDA error.
int tc_wait_probe(unsigned limit, int code) {
  tc_status(1);
  tc::wait_probe_kernel<<<1, 32>>>(limit, code);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return -1;
  return tc_status(1);
}

// Reads and clears the kernel status word (0 = every bounded wait completed).
int tc_status(int clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, tc::g_tc_status, sizeof(int)) != cudaSuccess) return -1;
  if (clear && v) {
    int z = 0;
    cudaMemcpyToSymbol(tc::g_tc_status, &z, sizeof(int));
  }
  return v;
}

}  // namespace bbfmm
