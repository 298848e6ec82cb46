// Device-resident FMM solver (internal C++ interface shared by the handle C-ABI and by
// the reference-compatible drop-in entry points).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/bbfmm_b200.h"
#include "common.cuh"

struct __nv_bfloat16;

namespace bbfmm {

enum Mode { MODE_D = 0, MODE_S = 1, MODE_MIXED = 2 };

enum Stage {
  ST_GATHER = 0, ST_P2M, ST_M2M, ST_PROJ_UP, ST_M2L, ST_PROJ_DOWN, ST_L2L, ST_L2P, ST_P2P, ST_SCATTER,
  ST_COUNT
};

// Launchers (passes.cu, p2p.cu, m2l_simt.cu, m2l_tc.cu)
// nsets: number of particle sets of the same depth stacked in one launch (cells of set k
// are the Morton indices [k 8^l, (k+1) 8^l) of each level; see common.cuh).
// first, count: a range of cells (P2M, L2P: leaves; M2M, L2L: parents) whose per-cell n^3
// arrays (S of P2M, F of L2P; the children in M2M and L2L) start at the pointer given, so a
// level can be processed in slabs; count < 0 means every cell from `first` on.
template <typename T>
int build_tree_device(int N, const T *xyz, T L, int maxlev, int *perm, int *leaf_start, cudaStream_t s);
// The same for nseg stacked sets, set j the particles xyz[off[j] .. off[j] + count[j]) (off and
// count on the host, every range inside the positions array): perm holds indices into xyz.
template <typename T>
int build_tree_device_sets(int nseg, const int *off, const int *count, const T *xyz, T L, int maxlev, int *perm,
                           int *leaf_start, cudaStream_t s);
template <typename T> int launch_p2m(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, T *S, cudaStream_t s, int nsets = 1, int64_t first = 0, int64_t count = -1, void *Ssplit = nullptr, const int64_t *rows = nullptr);
template <typename T> int launch_m2m(int n, const T *Sc, T *Sp, int level, const Tables &t, cudaStream_t s, int nsets = 1, int64_t first = 0, int64_t count = -1);
template <typename T> int launch_l2l(int n, const T *Fp, T *Fc, int level, const Tables &t, cudaStream_t s, int nsets = 1, int64_t first = 0, int64_t count = -1);
template <typename T> int launch_l2p(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, const T *F, T *phi, cudaStream_t s, int nsets = 1, int64_t first = 0, int64_t count = -1, const int64_t *rows = nullptr);
// rows are a slab of the level starting at cell row0 (the cpg side is indexed by level cell)
template <typename T> int launch_proj(int64_t M, int K, int N, const T *A, const float *A2, const T *B, const T *cs, T scale, T *C, int level, int mapmode, cudaStream_t s, int64_t row0 = 0, int ldc = 0, int lda = 0, const int64_t *rows = nullptr);
template <typename T, typename TI> int launch_gather(int N, const int *perm, const TI *xyz, const TI *q, T *pos4, cudaStream_t s);
template <typename T> int launch_charges_of(int N, const T *pos4, T *q, cudaStream_t s);  // sorted charges
template <typename T> int launch_add(int64_t n, const T *x, T *y, cudaStream_t s);        // y += x
template <typename T, typename TO> int launch_scatter(int N, const int *perm, const T *phis, TO *phi, cudaStream_t s);
template <typename T> int launch_morton_cpg(int level, int r, const T *src, T *dst, int inverse, cudaStream_t s);
// Near field (p2p.cu): a work list built on the device from the leaf offsets (near_work_build,
// into near_work_bytes of scratch), then one CTA per item of `threads` threads (64, 128 or
// 256; the list depends on it). mode: MODE_D / MODE_S / MODE_MIXED (pos4 and pot in FP64,
// FP32, FP64); homogen 1, 2 or 4; fld != null adds the gradient (1/r only, no target factor
// on pot then). nitems_host / flag_host: synchronise and return the item count and whether
// the offsets were malformed.
size_t near_work_bytes(int N, int maxlev, int nsets);
// mask (optional, device): the near field computes only the targets of leaves whose ancestor at
// mask_level (<= maxlev) has its mask byte set (stacked cell numbering); the others are not written.
int near_work_build(int N, const int *leaf_start, int maxlev, int nsets, int threads, void *scratch, cudaStream_t s,
                    int *nitems_host, int *flag_host, const unsigned char *mask = nullptr, int mask_level = 0);
int launch_near(int mode, int homogen, int N, const void *pos4, const int *leaf_start, int maxlev, const void *work,
                int nsets, int nitems, int threads, void *pot, void *fld, cudaStream_t s,
                const unsigned char *mask = nullptr, int mask_level = 0);
int near_status(int clear);
int launch_near2(int mode, int N, const void *pos4, const int *leaf_start, int maxlev, const void *work, int nsets,
                 int nitems, int threads, const void *q2, void *pot, void *fld, void *pot2, void *fld2, cudaStream_t s,
                 const unsigned char *mask = nullptr, int mask_level = 0);
int pass_status(int clear);  // the passes' bounded waits (L2P leaf copies)
template <typename T> int launch_l2p_field(int n, const T *pos4, const int *leaf_start, int maxlev, T L, const Tables &t, const T *F, T *pot, T *fld, cudaStream_t s, int nsets = 1, int64_t first = 0, int64_t count = -1, const int64_t *rows = nullptr);
template <typename T, typename TO> int launch_scatter_field(int N, const int *perm, const T *pot, const T *fld, TO *pot_out, TO *fld_out, cudaStream_t s);
template <typename T> int launch_m2l_simt(int r, const T *M, const T *Ert, T *Lout, int level, int j0, int j1, const int4 *offs, int accumulate, cudaStream_t s, int nsets = 1, int ngroups = 1, T *part = nullptr, int64_t part_elems = 0, const int4 *boxes = nullptr, int nboxes = 0);
void build_offset_table(int *out);
constexpr int DMMA_PARTS = 21;  // most offset groups of the FP64 M2L (189 = 9 x 21)
int launch_m2l_dmma(int r, const double *M, const double *Ecol, double *Lout, int level, int j0, int j1, int ni,
                    const int4 *offs, double *part, int64_t part_elems, cudaStream_t s, int nsets = 1,
                    int ngroups = 0, const int4 *boxes = nullptr, int nboxes = 0);
int dmma_default_groups(int level, int nsets);
int64_t dmma_part_elems(int level, int nsets, int groups, int r);
int launch_proj_dmma(int64_t M, int K, int N, const double *A, const double *B, const double *cs, double scale,
                     double *C, int level, int mapmode, cudaStream_t s, int64_t row0 = 0, int lda = 0,
                     const int64_t *rows = nullptr);
// C[out(m)][0:32] = sum_k A[m][k] B[k][0:32] on the FP64 tensor path (B: K x 32 contiguous).
int launch_proj_narrow(int64_t M, int K, const double *A, const double *B, double *C, int ldc, int level,
                       int mapmode, cudaStream_t s, int64_t row0, const int64_t *rows = nullptr);
int launch_direct_fp64(int N, const double *xyz, const double *q, int nt, const int *targets, double *out, cudaStream_t s);
int launch_direct_field_fp64(int N, const double *xyz, const double *q, int nt, const int *targets, double *pot,
                             double *fld, cudaStream_t s);

template <typename T> int bbfmm_weights_t(int n, T *Tkz, int *Ktable, T *Kweights, T *Cweights);

// Mixed-precision tensor-core M2L (m2l_tc.cu).
struct TcOperators;
int tc_supported();
int tc_prepare_operators(int r, const double *Ert, int lead, int lead_rows, void **out, cudaStream_t s);
void tc_free_operators(void *ops);
int tc_split_multipoles(int r, int64_t ncell, const double *M, int lead, void *Msplit, cudaStream_t s);
size_t tc_split_bytes(int r, int64_t ncell);
// nprod: 3 = hi*hi + hi*lo + lo*hi (split BF16) for every term, 1 = hi*hi only (plain BF16
// products), 0 = adaptive: the three products for components j < 32 TC_SPLIT_CHUNKS and
// outputs i < TC_SPLIT_ROWS, hi*hi alone elsewhere. With the SVD-ordered operators those
// other terms are small enough for one BF16 product: on 4M uniform particles (n = 8, depth 7)
// the error against the FP64 direct sum is 1.0453x that of the FP64 FMM with the 64 x 64
// three-product block, 1.0450x with 96 x 96, 1.075x with 64 x 48 and 1.9x with 64 x 32 or
// 32 x 64.
constexpr int TC_SPLIT_CHUNKS = 2, TC_SPLIT_ROWS = 64;
// rank: the effective rank (outputs i and components j below it; 0 = r).
// boxes (nboxes entries of set, x0, y0, z0): run only the targets of these blocks of parent
// cells, of 2^lx x 2^ly x 2^lz cells (lgeom = lx | ly << 4 | lz << 8, 8 to 256 cells, origins
// multiples of the extents), 256 / cells per tile; the outputs of the other cells are not
// written.
int launch_m2l_tc(int r, const void *Msplit, int64_t ncell_total, int64_t cell_offset, const void *ops, double *Lacc,
                  int level, const int4 *offs, cudaStream_t s, int nsets = 1, int nprod = 3, int rank = 0,
                  const double *Mlead = nullptr, const double *Erow = nullptr, void *Lsplit = nullptr,
                  const int4 *boxes = nullptr, int nboxes = 0, int lgeom = 0x111);
bool tc_fuses_lead(const void *ops, int nprod, int rank);
// Whether launch_m2l_tc runs the two-box kernel (the adaptive product map at full split rows).
inline bool tc_two_box(int nprod, int rank) { return nprod == 0 && (rank <= 0 || rank >= TC_SPLIT_ROWS); }
int tc_status(int clear);
int tc_wait_probe(unsigned limit, int code);
// Tensor-core projections (m2l_tc.cu): the components j >= lead of the up projection and the
// contraction over j >= lead of the down projection, as split-BF16 products.
int tc_prepare_projections(int n3, int r, const double *Bup, const double *Bdn, int lead, void **out, cudaStream_t s);
void tc_free_projections(void *p);
int launch_proj_down(const void *p, const void *Asplit, const double *Lfp, int64_t rows, double *F, int level,
                     int64_t row0, const double *cs, double scale, cudaStream_t s, int rank = 0,
                     const int64_t *rowlist = nullptr);
int launch_proj_up(const void *p, const void *Asplit, int64_t rows, double *M, int level, int64_t row0, cudaStream_t s,
                   const int64_t *rowlist = nullptr);
// rowlist (optional): the pass's Morton rows, row t being rowlist[t] instead of row0 + t
int tc_split_rows(int64_t rows, int K, const double *src, int gather, int level, int64_t row0, void *dst,
                  cudaStream_t s, int zlead = 0, const int64_t *rowlist = nullptr);
constexpr int TC_MIN_LEVEL = 4;   // the one-box tensor-core M2L needs a parent grid of >= 8 per axis
constexpr int TC2_MIN_LEVEL = 2;  // the two-box kernel tiles every level (stacked sets below 4)

// Target box of the two-box tensor-core M2L at one level: 2^lx x 2^ly x 2^lz parent cells of
// one sibling class grid in each of 2^(8 - lb()) consecutive stacked sets, 256 target rows in
// all, x fastest, then y, z, set. Level >= 4: an 8 x 8 x 4 box of one set; level 3: the whole
// 4 x 4 x 4 grid of four sets; level 2: the whole 2 x 2 x 2 grid of 32 sets.
struct Tc2Box {
  int lx, ly, lz;
  __host__ __device__ int lb() const { return lx + ly + lz; }
  __host__ __device__ void pos(int row, int &x, int &y, int &z, int &set) const {
    x = row & ((1 << lx) - 1);
    y = (row >> lx) & ((1 << ly) - 1);
    z = (row >> (lx + ly)) & ((1 << lz) - 1);
    set = row >> lb();
  }
};
__host__ __device__ inline Tc2Box tc2_box(int level) {
  const int p = level - 1;  // log2 of the class grid's cells per axis
  return Tc2Box{p < 3 ? p : 3, p < 3 ? p : 3, p < 2 ? p : 2};
}
// Tiles of the two-box kernel over a whole level: 8 classes x set groups x boxes per class grid.
inline int64_t tc2_tiles(int level, int nsets) {
  const Tc2Box g = tc2_box(level);
  const int P = 1 << (level - 1), spt = 1 << (8 - g.lb());
  return 8 * (int64_t)((nsets + spt - 1) / spt) * (P >> g.lx) * (P >> g.ly) * (P >> g.lz);
}

// Degree of homogeneity of a BBFMM_B200_KERNEL_* value (bbfmm.c:109-144), 0 for an unknown one.
inline int kernel_homogen(int kernel) {
  return kernel == BBFMM_B200_KERNEL_LAPLACIAN         ? 1
         : kernel == BBFMM_B200_KERNEL_LAPLACIAN_FORCE ? 2
         : kernel == BBFMM_B200_KERNEL_ONEOVERR4       ? 4
                                                       : 0;
}

// Launch choices of one solver, per level (index = level): what the autotuner sets.
struct Tuning {
  // 0: default (the tensor-core split M2L where the mode has it, from level 4, and at levels
  // 2-3 for stacked sets), 1: FP64/SIMT M2L, 2: the tensor-core M2L wherever it tiles the level
  int m2l_kind[11] = {};
  int m2l_groups[11] = {};  // offset groups of the FP64 DMMA M2L (0: dmma_default_groups)
  int p2p_threads = 128;    // threads per block of the near-field kernel
};

template <typename T>
struct Solver {
  int n = 0, r = 0, n3 = 0, maxlev = 0, mode = MODE_D, lead = 16, lead_rows = 32, device = 0;
  int nsets = 1;  // particle sets of this depth stacked in every launch (set k = cells [k 8^l, (k+1) 8^l))
  // kernel: degree of homogeneity, 1 (1/r, LAPLACIAN), 2 (x/r^3, LAPLACIANFORCE) or 4 (1/r^4,
  // ONEOVERR4), in every mode: the near-field pair value and the per-level scale
  // (1/L_l)^homogen after the M2L
  int homogen = 1;
  // Effective rank (0 = r): the operators hold a rank-rank_eff truncation zero-padded to r,
  // and the M2L and the down projection skip the zero components j >= rank_eff and outputs
  // i >= rank_eff (a tolerance-rank SVD cut, bbfmm_b200_set_rank).
  int rank_eff = 0;
  int rk() const { return rank_eff > 0 ? rank_eff : r; }
  // Leaf cells per slab of the leaf level (multiple of 64): P2M -> up projection -> M2M and
  // down projection -> L2L -> L2P run slab by slab through one slab-sized S / F buffer, so
  // the leaf level's n^3 arrays never exist in full. 0: automatic (slabs only when a full
  // leaf-level array would exceed 16 GiB); slab_request > 0 forces that size.
  int64_t slab = 0, slab_request = 0;
  double L = 1.0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool own_ops = true;  // false: tables and operators borrowed from another solver (share_operators)
  Tuning tune;
  int tc_products = 0;  // mixed mode: tensor-core M2L products (0 adaptive, 3 split everywhere, 1 plain BF16)
  // tables and operators (device)
  T *tkz = nullptr, *cw = nullptr, *kw = nullptr;
  T *Ert = nullptr;  // [316][r][r] row-major
  T *Ecol = nullptr; // [316][r][r] column-major (the reference's K-file layout)
  T *Bup = nullptr;  // [n3][r]  Kweights[l] U(l, i)
  T *Bdn = nullptr;  // [r][n3]  U(l, j)
  T *kwcol = nullptr;
  int4 *offs = nullptr;
  void *tcops = nullptr;  // mixed mode: split operators for the tensor-core kernel
  // mixed mode, n = 8: projections with the leading PROJ_LEAD components in FP64 and the rest
  // as split-BF16 tensor-core products (tcproj: split, transposed U operators)
  static constexpr int PROJ_LEAD = 16;
  bool mixed_proj = true;
  void *tcproj = nullptr;
  T *Bup_lead = nullptr;  // [n3][PROJ_LEAD] leading columns of Bup
  void *Ssplit = nullptr, *Lsplit = nullptr;  // bf16 [hi | lo] copies of S rows / L rows
  int64_t Ssplit_rows = 0, Lsplit_rows = 0;
  // particles (sorted by leaf, Morton leaf order)
  int N = 0;
  int *perm = nullptr, *leaf_start = nullptr;
  void *near_work = nullptr;  // near-field work list (near_work_build) for near_threads
  int near_items = 0, near_threads = 0;
  // Target region (bbfmm_b200_set_target_region): results are wanted only at the
  // particles inside the active cells of region_level. The near field skips the other targets,
  // and the tensor-core M2L of every level above region_level runs only on the two-box tiles
  // that hold descendants of active cells (the rest of that level's output is zero).
  int region_level = -1;                       // < 0: every particle
  unsigned char *region_mask = nullptr;        // device, nsets 8^region_level bytes (stacked numbering)
  std::vector<unsigned char> region_host;
  int4 *region_boxes[11] = {};                 // per level: active 2 x 2 x 2 parent blocks (set, x0, y0, z0)
  int region_nboxes[11] = {};
  int4 *region_tcboxes[11] = {};               // per level: the tensor-core M2L's active blocks,
  int region_ntcboxes[11] = {}, region_tcgeom[11] = {};  // of geometry region_tcgeom (lgeom)
  // First level whose M2L runs (bbfmm_b200_set_first_m2l_level): the local expansions start
  // there (no L2L from the level above), so the solve gathers, for every target, only the
  // sources inside the neighbourhood of its ancestor one level up.
  int m2l_first = BBFMM_MINLEV;
  // Local solve (a target region and m2l_first > region_level): every source that a target of
  // the region gathers lies in an active cell of region_level or in one of its neighbours, so
  // the passes at the levels >= m2l_first run only over those cells' descendants -- the upward
  // ones over src_runs (active cells and their neighbours), the downward ones over tgt_runs
  // (active cells) -- and the levels below m2l_first are skipped. Runs: Morton rows [a, a + c)
  // of region_level over the stacked sets, neighbouring rows merged. Targets outside the
  // region get zero.
  bool local_solve = false;
  std::vector<std::pair<int64_t, int64_t>> src_runs, tgt_runs;
  // the runs' cells at each level >= m2l_first, in order (device lists): the passes of a local
  // solve keep S and F rows in this compact order, the children of compact row p at 8p .. 8p + 7
  int64_t *src_list[11] = {}, *tgt_list[11] = {};
  int64_t n_src[11] = {}, n_tgt[11] = {};
  T *pos4 = nullptr;
  // expansions
  T *S[2] = {nullptr, nullptr};
  T *F[2] = {nullptr, nullptr};
  T *Mall = nullptr;
  std::vector<int64_t> Moff;  // offset (elements) of level l in Mall, cpg layout
  T *Lbuf = nullptr;
  T *Lpart = nullptr;  // partial sums of the offset-group FP64 M2L
  int64_t Lpart_elems = 0;
  void *Msplit = nullptr;
  T *phis = nullptr;
  T *flds = nullptr;  // 3 N, sorted field of the last solve_fields
  T *phis2 = nullptr, *flds2 = nullptr, *qs2 = nullptr;  // solve_fields2: second potential, field, charges
  T *phisn = nullptr, *fldsn = nullptr;  // solve_fields2: near field of the second vector
  cudaStream_t side = nullptr;           // solve_fields2: the near field beside the far field
  cudaEvent_t side_ev[2] = {};
  void *io_q = nullptr, *io_phi = nullptr;  // device staging of the host-buffer solve (N each)
  // timing
  bool timing = false;
  cudaEvent_t ev[ST_COUNT + 1] = {};
  float stage_ms[ST_COUNT] = {};
  int kernel_launches = 0;

  Tables tables() const;
  int64_t cells(int l) const { return nsets * pow8i(l); }
  int64_t leaf_slab() const { return slab > 0 && slab < cells(maxlev) ? slab : cells(maxlev); }
  bool slabbed() const { return leaf_slab() < cells(maxlev); }
  int leaf_down(bool field);  // down projection, L2L and L2P (or L2P with field) of the leaf level
  int64_t Mcells() const { return (Moff[maxlev] + cells(maxlev) * r) / r; }
  int init(int n_, int maxlev_, double L_, int mode_, int lead_, int lead_rows_, int device_, cudaStream_t s);
  int set_tables(const T *Tkz, const T *Cweights, const T *Kweights);  // host arrays
  int set_operators(const T *U, const T *E);                              // host, reference layout
  // positions already on the device ([N][3], this solver's precision): the tree is built there
  int set_particles_device(int N_, const T *xyz_dev);
  // nsets_ stacked sets whose positions are on the device: set j is the particles
  // xyz_dev[off_host[j] .. off_host[j] + count_host[j]) of an array of Nxyz (the tree of every set
  // built there, one sort for all; perm indexes that array, as for set_particles_global)
  int set_particles_sets_device(int nsets_, const int *off_host, const int *count_host, int Nxyz, const T *xyz_dev);
  int set_particles_sorted(int N_, const int *perm_host, const int *leaf_start_host, const T *xyz_host);
  // N_ particles of nsets_ stacked sets: perm_host[k] indexes the caller's arrays of Nxyz
  // particles (positions xyz_host, and later q and phi); leaf_start_host has nsets_ 8^maxlev + 1
  // entries over the sorted order.
  int set_particles_global(int nsets_, int N_, const int *perm_host, const int *leaf_start_host, int Nxyz,
                           const T *xyz_host);
  int share_operators(const Solver<T> &from);  // borrow tables and operators (same n, mode, lead)
  int alloc_partials();                          // Lpart for the current tuning
  int near(T *pot, T *fld);                      // P2P (add) into sorted pot (and field)
  int build_near_work();                         // the work list for tune.p2p_threads
  int set_target_region(int level, const unsigned char *active_host);  // level < 0 clears
  int set_m2l_first(int level);                                        // m2l_first, then the runs
  int build_local();                                                   // runs and row lists
  void free_local();
  bool chunked() const { return slabbed() || local_solve; }  // leaf passes run per leaf chunk
  int build_region_tiles();                      // region_boxes from region_host
  bool proj_tc() const { return mode == MODE_MIXED && mixed_proj && tcproj != nullptr; }
  // level l has a tensor-core M2L under the current product map and rank (mixed mode), and
  // the solve runs it there (the level's tuning keeps the default kind)
  bool tc_level(int l) const {
    return mode == MODE_MIXED && tcops &&
           (l >= TC_MIN_LEVEL || (l >= TC2_MIN_LEVEL && tc_two_box(tc_products, rk())));
  }
  // The default keeps a single set's levels 2-3 in FP64: they are a few tiles either way, and
  // their split-BF16 M2L raised the 4M uniform solve's error ratio against the FP64 direct sum
  // from 1.05 to 1.10; stacked sets take the tensor cores there (the FP64 M2L of a batch's
  // levels 2-3 took tens of ms).
  bool tc_default(int l) const { return tc_level(l) && (l >= TC_MIN_LEVEL || nsets > 1); }
  bool tc_m2l(int l) const {
    const int k = tune.m2l_kind[l];
    return k == 2 ? tc_level(l) : (k == 0 && tc_default(l));
  }
  // S rows -> Mall (cpg); F rows <- Lbuf (Morton, assign). Row t is cell row0 + t, or
  // rowlist[t] when a row list is given.
  int proj_up(int64_t rows, const T *S_rows, int level, int64_t row0, bool presplit = false,
              const int64_t *rowlist = nullptr);
  int proj_down(int level, int64_t rows, int64_t row0, T *F_rows, bool presplit = false,
                const int64_t *rowlist = nullptr);
  // Times the launch choices of every level's M2L and of the near field on this solver's
  // own tree (after an upward pass with q_dev) and keeps the fastest; results are cached per
  // (mode, n, level, target tiles) and (mode, particles, leaves) for later solvers.
  int autotune(const void *q_dev, int io_double);
  int alloc_work();
  int upward(const void *q_dev, int q_is_double);   // gather q, P2M, M2M, projections -> Mall
  int interaction(int level_lo, int level_hi);       // M2L + post projection + L2L into F
  int m2l_post(int level);                           // M2L + post projection of one level
  int downward_finish(void *phi_dev, int phi_is_double, bool near);  // L2P, P2P, scatter
  int solve(const void *q_dev, void *phi_dev, int io_double);
  int solve_fields(const void *q_dev, void *pot_dev, void *fld_dev);  // potential and its gradient
  // solve_fields for two charge vectors, the near-field pairs evaluated once for both
  int solve_fields2(const void *q1_dev, const void *q2_dev, void *pot1_dev, void *fld1_dev, void *pot2_dev,
                    void *fld2_dev);
  int copy_multipoles_morton(int level, T *host_out);  // level's M in reference (Morton) order
  int copy_m2l_morton(int level, T *host_out);         // level's M2L output, recomputed, Morton order
  void mark(int stage, int launches = 1);
  int time_m2l(int level, int reps, float *ms);
  int m2l_fp(const T *Ml, int level, int j0, int j1, int ni,  // FP64 (DMMA) / FP32 (SIMT) M2L part
             const int4 *boxes = nullptr, int nboxes = 0);
  int proj(int64_t M, int K, int N, const T *A, const T *B, const T *cs, T scale, T *C, int level, int mapmode,
           int64_t row0 = 0, int lda = 0, const int64_t *rowlist = nullptr);
  void release();
};

}  // namespace bbfmm
