/*
 * bbfmm_b200 -- B200 (sm_100a) implementation of the bbFMM hot path: the SVD-compressed
 * Chebyshev M2L, the near-field P2P and the P2M/M2M/L2L/L2P passes, with expansions
 * resident in device memory.
 *
 * Two C-ABI surfaces are exported:
 *
 *  1. The reference's own entry points (m2l_drv, m2l_host_*, anotherFMMCompute,
 *     anotherUpwardPass, anotherFMMInteraction, anotherDownwardPass, anotherNearField,
 *     kernel_exec_time), declared in bbfmm_b200_reference.h with the reference's
 *     signatures so that its host objects link against this library unchanged.
 *
 *  2. The handle API below: tree, operators and expansions stay on the device and one
 *     call runs one whole solve. This surface has no counterpart in the reference, whose
 *     GPU path copies every array to and from the host around each kernel.
 *
 * Conventions shared with the reference: the root cell is the cube [-L/2, L/2]^3 centred
 * at the origin (anotherFMMDistribute.c:321-324); the result is q_i * phi_i, the target
 * charge times the potential (bbfmm.c:501, anotherDownwardPassX.c:330); leaves sit at
 * level maxlev of a full uniform octree; the rank of the compressed operators is the
 * reference's fixed cutoff r = n^3 / 2 (bbfmm.c:1340-1343); operator arrays use the
 * layouts of the reference's [s]laplacian{K,U}{n}.bin files: U is n^3 x r column-major,
 * E ("K") holds 316 r x r column-major blocks (bbfmm.c:1361-1405).
 *
 * Every function returns 0 on success or a positive BBFMM_B200_ERR_* code; the message of
 * the last failure on the calling thread is available from bbfmm_b200_last_error().
 */
#ifndef BBFMM_B200_H
#define BBFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BBFMM_B200_API __attribute__((visibility("default")))
#else
#define BBFMM_B200_API
#endif

#define BBFMM_B200_VERSION 1

#define BBFMM_B200_OK 0
#define BBFMM_B200_ERR_ARG 1
#define BBFMM_B200_ERR_CUDA 2
#define BBFMM_B200_ERR_NOMEM 3
#define BBFMM_B200_ERR_UNSUPPORTED 4
#define BBFMM_B200_ERR_STATE 5

/* Precision modes.
 *  D      FP64 storage and arithmetic in every stage (the reference's double build).
 *  S      FP32 storage and arithmetic in every stage (the reference's SINGLE build).
 *  MIXED  FP64 passes; M2L with the leading block of every operator (outputs i < lead_rows,
 *         contraction components j < lead) in FP64 and everything else as split-BF16
 *         products on tcgen05 tensor cores accumulated in FP32 (three products for the
 *         leading 64 x 64 block, one elsewhere; bbfmm_b200_set_tc_products); U-projections
 *         with their 16 leading components in FP64 and the rest as split-BF16 products;
 *         P2P with FP64 pair separations, FP32 reciprocal distances and compensated FP32
 *         sums added to FP64 potentials. */
#define BBFMM_B200_MODE_D 0
#define BBFMM_B200_MODE_S 1
#define BBFMM_B200_MODE_MIXED 2

typedef struct {
  int n;        /* Chebyshev nodes per dimension: 4 (r = 32) or 8 (r = 256) */
  int maxlev;   /* level of the leaves, >= 2 (the reference's maxlev) */
  double L;     /* edge of the root cube */
  int mode;     /* BBFMM_B200_MODE_* */
  int lead;     /* MIXED: leading contraction components j kept in FP64 (0, 16, 32, 48, 64) */
  int lead_rows;/* MIXED: ... for the outputs i < lead_rows only (multiple of 32; 0 = all r) */
  int device;   /* CUDA device ordinal */
  void *stream; /* cudaStream_t to run on, or NULL for a private stream */
} bbfmm_b200_config;

typedef struct bbfmm_b200_solver bbfmm_b200_solver;

/* Stage indices of bbfmm_b200_stage_times(). */
enum {
  BBFMM_B200_STAGE_GATHER = 0,
  BBFMM_B200_STAGE_P2M,
  BBFMM_B200_STAGE_M2M,
  BBFMM_B200_STAGE_PROJ_UP,
  BBFMM_B200_STAGE_M2L,
  BBFMM_B200_STAGE_PROJ_DOWN,
  BBFMM_B200_STAGE_L2L,
  BBFMM_B200_STAGE_L2P,
  BBFMM_B200_STAGE_P2P,
  BBFMM_B200_STAGE_SCATTER,
  BBFMM_B200_NUM_STAGES
};

BBFMM_B200_API const char *bbfmm_b200_last_error(void);
BBFMM_B200_API int bbfmm_b200_version(void);

/* Chebyshev tables of ComputeWeights (bbfmm.c:922-1028) in FP64 (fp32 = 0) or FP32:
 * Tkz[n*n], Ktable[343], Kweights[n^3], Cweights[2*n*n]. */
BBFMM_B200_API int bbfmm_b200_weights(int n, int fp32, void *Tkz, int *Ktable, void *Kweights, void *Cweights);

/* Leaf assignment and stable counting sort (anotherFMMDistribute.c:258-473):
 * perm[k] = index of the k-th particle in leaf-sorted order, leaf_start[8^maxlev + 1] =
 * CSR offsets of the leaves in Morton (reference) order. xyz is N x 3, FP64 or FP32. */
BBFMM_B200_API int bbfmm_b200_sort_particles(int N, int fp32, const void *xyz, double L, int maxlev, int *perm,
                              int *leaf_start);

/* Create a solver: uploads tables and operators (U, E in the reference file layouts,
 * FP64 unless operators_fp32). */
BBFMM_B200_API int bbfmm_b200_create(const bbfmm_b200_config *cfg, const void *U, const void *E, int operators_fp32,
                      bbfmm_b200_solver **out);

/* Positions (host, N x 3; FP32 in mode S, FP64 otherwise), inside [-L/2, L/2]^3. Builds
 * the leaf order on the host and keeps the sorted particles on the device. */
BBFMM_B200_API int bbfmm_b200_set_particles(bbfmm_b200_solver *s, int N, const void *xyz);
/* The same for positions already on the solver's device (xyz_dev: N x 3 in the solver's
 * precision, float in mode S, double otherwise): the octree is built on the GPU (leaf
 * assignment and a stable radix sort by Morton leaf), with the same particle order and leaf
 * ranges as bbfmm_b200_set_particles (anotherFMMDistribute.c:258-298, 431-473). */
BBFMM_B200_API int bbfmm_b200_set_particles_device(bbfmm_b200_solver *s, int N, const void *xyz_dev);

/* One solve with device-resident charges and result (original particle order; FP32 in
 * mode S, FP64 otherwise): phi[i] = q_i * sum_{j != i} q_j / |x_i - x_j| (FMM-approximated).
 * Runs on the solver's stream and returns without synchronising. */
BBFMM_B200_API int bbfmm_b200_solve(bbfmm_b200_solver *s, const void *q_dev, void *phi_dev);

/* Potential and its gradient at every particle, without the target-charge factor:
 * pot[i] = sum_{j != i} q_j / r_ij, field[3i + a] = d pot / d x_{i,a} (FMM-approximated, both
 * device arrays in the caller's order; either may be NULL). With phi = q o pot this gives a
 * backward pass in one extra solve: dL/dq = g o pot(q) + pot(g o q),
 * dL/dx = q o (g o field(q) + field(g o q)) for L with dL/dphi = g. The reference has no
 * derivative code; the gradient of the Chebyshev interpolant (S_n of bbfmm.c:1682-1690) is
 * new. Runs on the solver's stream without synchronising. */
BBFMM_B200_API int bbfmm_b200_solve_fields(bbfmm_b200_solver *s, const void *q_dev, void *pot_dev, void *field_dev);
/* bbfmm_b200_solve_fields for two charge vectors q1 and q2 (device, N each) in one call, the
 * same results as two calls: the two far fields run one after the other and one near-field pass
 * evaluates each pair once for both (no counterpart in the reference, which has no derivative
 * code; it serves the backward of bbfmm_b200.autograd.fmm_phi with save="recompute"). Either
 * output of each pair may be NULL, not both. */
BBFMM_B200_API int bbfmm_b200_solve_fields2(bbfmm_b200_solver *s, const void *q1_dev, const void *q2_dev,
                                            void *pot1_dev, void *field1_dev, void *pot2_dev, void *field2_dev);

/* The same with host buffers: copies q in, solves, copies phi out and synchronises. The
 * device staging (2 N values) is allocated on the first call and kept until the particles
 * change or the solver is destroyed; pinned host buffers make the copies direct. */
BBFMM_B200_API int bbfmm_b200_solve_host(bbfmm_b200_solver *s, const void *q_host, void *phi_host);

/* Per-stage device times (ms) of the last solve run with timing on; returns the number of
 * kernel launches of that solve. Timing inserts a synchronisation after every stage. */
BBFMM_B200_API int bbfmm_b200_set_timing(bbfmm_b200_solver *s, int on);
BBFMM_B200_API int bbfmm_b200_stage_times(const bbfmm_b200_solver *s, float *ms, int count);

/* The multipole (proxy source) coefficients of one level after a solve, r per cell in
 * the reference's Morton cell order (the level's slice of proxysval). */
BBFMM_B200_API int bbfmm_b200_copy_multipoles(bbfmm_b200_solver *s, int level, void *host_out);

/* The M2L output of one level -- the level's slice of what the reference's m2l_drv writes
 * into L (m2l_drv.cu:14-19; PF of anotherFMMInteraction): L(F) = sum_{S in IL(F)} E_k M(S),
 * before the post-M2L projection and its (1/L_l)^homogeneity scale -- recomputed from the
 * multipoles of the last solve with that solve's kernels (MIXED: the tensor-core kernel with
 * its full FP64 output), r values per cell in the reference's Morton cell order. */
BBFMM_B200_API int bbfmm_b200_copy_m2l(bbfmm_b200_solver *s, int level, void *host_out);

/* Re-run the M2L of one level `reps` times (inputs of the last solve), each launch as the
 * solve makes it, between CUDA events on the solver's stream: ms[0] = mean time of the main
 * M2L kernel per launch, ms[1] = mean time of a separate FP64 leading-component kernel
 * (MIXED where the tensor-core kernel does not compute that block itself, else 0). */
BBFMM_B200_API int bbfmm_b200_time_m2l(bbfmm_b200_solver *s, int level, int reps, float *ms);

/* FP64 direct sum on the device (DirectCalc3D, bbfmm.c:471-504): out[t] =
 * q_i sum_{x_j != x_i} q_j / |x_j - x_i| for i = targets[t]; xyz (N x 3), q, targets, out are
 * device pointers; runs on `stream` (cudaStream_t, may be NULL). */
BBFMM_B200_API int bbfmm_b200_direct(int N, const double *xyz_dev, const double *q_dev, int ntarget,
                                     const int *targets_dev, double *out_dev, void *stream);

/* FP64 direct potential and gradient at the targets, without the target-charge factor (the
 * exact counterpart of bbfmm_b200_solve_fields): pot[t] = sum_{x_j != x_i} q_j / r_ij,
 * field[3t + a] = sum q_j (x_j - x_i)_a / r_ij^3 for i = targets[t]; either output may be
 * NULL. The reference has no gradient code; this is the analytic derivative of its kernel. */
BBFMM_B200_API int bbfmm_b200_direct_field(int N, const double *xyz_dev, const double *q_dev, int ntarget,
                                           const int *targets_dev, double *pot_dev, double *field_dev,
                                           void *stream);

/* Status word of the device kernels: 0 when every bounded wait of every tensor-core launch and
 * of every L2P launch (its leaf copies) so far completed and every near-field launch found
 * well-formed leaf offsets, else the code of the first failure: the code of a wait that gave
 * up (the launch then skipped its remaining work and returned; 31 for an L2P leaf copy), or
 * BBFMM_B200_LEAF_RANGE_CODE when a near-field call was given leaf
 * offsets that are out of [0, N] or decrease (the kernels clamp every offset, so nothing was
 * read or written outside the caller's arrays). Synchronises the device; clear != 0 resets
 * the word. */
#define BBFMM_B200_LEAF_RANGE_CODE 98
BBFMM_B200_API int bbfmm_b200_device_status(int clear);

/* Failure-detection self test (no counterpart in the reference): one kernel waits, with the
 * bounded mbarrier wait of the tensor-core kernels (at most `limit` polls, 1 .. 2^24), on a
 * barrier that nothing arrives at. The wait gives up, the kernel records
 * BBFMM_B200_WAIT_SELFTEST_CODE in the status word and returns; the call synchronises,
 * returns the status word it found (BBFMM_B200_WAIT_SELFTEST_CODE when the mechanism works)
 * and clears it. No fault, trap or hang is involved; the context stays usable. */
#define BBFMM_B200_WAIT_SELFTEST_CODE 99
BBFMM_B200_API int bbfmm_b200_wait_selftest(unsigned limit);

/* Near-field (P2P) part of the solve on caller-owned device arrays, the work of
 * anotherNearField (anotherNearField.c:219-346) and of the reference GPU kernel `direct`
 * (direct.cu:69-209): phi[k] += q_k sum_{B in N(A)} sum_{j in B, r != 0} q_j / r_kj over the
 * <= 27 neighbour leaves. xyzq is N x 4 (x, y, z, q) FP64 sorted by leaf in Morton order
 * (as bbfmm_b200_sort_particles orders them), leaf_start holds the 8^maxlev + 1 leaf
 * offsets, phi is added to; all three are device pointers. The offsets must start at
 * leaf_start[0] = 0, never decrease and end at leaf_start[8^maxlev] = N; other offsets make
 * the call return BBFMM_B200_ERR_ARG (and set BBFMM_B200_LEAF_RANGE_CODE in the status word)
 * without any access outside the arrays, phi then being unspecified. mode BBFMM_B200_MODE_D
 * computes in FP64 like the reference; BBFMM_B200_MODE_MIXED takes each pair's separation in
 * FP64 and the reciprocal distance, product and compensated sum in FP32. L is checked (> 0)
 * but the leaf geometry needs only maxlev. Allocates a device work list for the call (8 bytes
 * per particle plus 8 bytes per 256 cells of level maxlev - 2), runs on `stream`
 * (cudaStream_t, may be NULL) and synchronises it. */
BBFMM_B200_API int bbfmm_b200_near_field(int N, int maxlev, double L, const double *xyzq, const int *leaf_start,
                                         double *phi, int mode, void *stream);

/* The same near field without any device allocation. This entry point has no counterpart
 * in the reference. It is for callers that must not call cudaMalloc: code whose device
 * memory is handed out by another framework's allocator (which may hold all of it), and
 * time-critical loops that cannot afford the device-wide synchronisation cudaMalloc and
 * cudaFree imply. Inputs, output and the leaf-offset rules are as above; the work list
 * lives in one fixed array of device memory inside the library,
 * BBFMM_B200_NOALLOC_SCRATCH_BYTES (2.5 MiB) long, room for BBFMM_B200_NOALLOC_MAX_PARTICLES
 * particles at any maxlev up to 10, which every GPU that loads the library keeps until the
 * process exits. Larger N is rejected with BBFMM_B200_ERR_ARG. The first call on a device
 * looks up that array's device address (with the device current), so make the first call
 * on each device before any stream capture; the address stays valid for the life of the
 * device's primary context, so do not call it across a cudaDeviceReset. All calls share
 * the array: calls that overlap on the GPU (other streams, other host threads) race on it,
 * so order them. Each call clears the list's counters and rewrites every entry it reads. Runs
 * on `stream` and synchronises that stream (not the device) to check the leaf offsets. */
#define BBFMM_B200_NOALLOC_MAX_PARTICLES 262144
#define BBFMM_B200_NOALLOC_SCRATCH_BYTES 2621696
BBFMM_B200_API int bbfmm_b200_near_field_noalloc(int N, int maxlev, double L, const double *xyzq,
                                                 const int *leaf_start, double *phi, int mode, void *stream);

BBFMM_B200_API void *bbfmm_b200_stream(bbfmm_b200_solver *s);
BBFMM_B200_API void bbfmm_b200_destroy(bbfmm_b200_solver *s);

/* Leaf cells per slab of the leaf level (a multiple of 64; 0 = automatic). The leaf level's
 * P2M -> up projection -> M2M and down projection -> L2L -> L2P run slab by slab through one
 * slab-sized buffer of Chebyshev node values, so those per-leaf arrays (n^3 values per leaf)
 * never exist for the whole level; results are bitwise the same for every slab size.
 * Automatic: slabs of 16 GiB when a whole-level array would be larger (n = 8, FP64: depth 8
 * and deeper). Reallocates the work buffers when particles are already set. */
BBFMM_B200_API int bbfmm_b200_set_leaf_slab(bbfmm_b200_solver *s, long long cells);

/* Effective rank (0 = r, else a multiple of 32 in [32, r]): for operators that hold a rank-k
 * truncation of the SVD basis zero-padded to r (the leading k singular vectors in U, the
 * leading k x k block of every E_k; an SVD cut at a relative singular value), the M2L and the
 * down projection skip the zero components j >= k and outputs i >= k. Results equal the
 * rank-k bbFMM; the reference fixes r = n^3 / 2 (bbfmm.c:1340-1343), this tolerance-rank mode
 * is new. */
BBFMM_B200_API int bbfmm_b200_set_rank(bbfmm_b200_solver *s, int rank);

/* Kernel of the solver (the reference's compile-time kernels, bbfmm.c:109-144, 798-849):
 * BBFMM_B200_KERNEL_LAPLACIAN (1/r, the default), BBFMM_B200_KERNEL_LAPLACIAN_FORCE (x / r^3,
 * x the first component of source - target, homogeneity 2) or BBFMM_B200_KERNEL_ONEOVERR4
 * (1/r^4, homogeneity 4), in every mode; the operators given at create must be that kernel's,
 * e.g. the reference's laplacianforce{K,U}{n}.bin or oneoverr4{K,U}{n}.bin. It sets the
 * near-field pair value (MIXED: x / r^3 with the separation in FP64 and dx r^-3 in FP32 with
 * the compensated sum; 1/r^4 in FP64, its potentials being near-field dominated) and the
 * per-level scale (1/L_l)^homogeneity after the M2L. Field solves are for 1/r. */
#define BBFMM_B200_KERNEL_LAPLACIAN 0
#define BBFMM_B200_KERNEL_LAPLACIAN_FORCE 1
#define BBFMM_B200_KERNEL_ONEOVERR4 2
BBFMM_B200_API int bbfmm_b200_set_kernel(bbfmm_b200_solver *s, int kernel);

/* Adaptive refinement support (no counterpart in the reference, whose trees are uniform,
 * anotherBuildFMMHierachy.c:44-55). A target region marks the cells of one level whose
 * particles' results are wanted: active[m] != 0 for the Morton cells m of `level` (8^level
 * bytes, host; level < 0 clears). The solve then computes the near field only for particles
 * in active cells (others keep what the far field gives them), and the M2L of every level
 * above `level` runs only on the tiles holding descendants of active cells. The first M2L
 * level (default 2) starts the local expansions at that level: with first = l + 1 the solve
 * gathers, for every target, only the sources inside the 3 x 3 x 3 neighbourhood of its
 * level-l ancestor -- exactly the near field of a level-l leaf, computed by a deeper FMM.
 * With both (first > region level: a local solve) every pass runs only below the active cells
 * (downward) and below them and their neighbours (upward), the levels above the first M2L
 * level are skipped, and particles outside the region get 0. bbfmm_b200.AdaptiveSolver
 * composes a coarse and a refined solver this way. Single-set solvers only. */
BBFMM_B200_API int bbfmm_b200_set_target_region(bbfmm_b200_solver *s, int level, const unsigned char *active);
BBFMM_B200_API int bbfmm_b200_set_first_m2l_level(bbfmm_b200_solver *s, int level);

/* MIXED mode: products per term of the tensor-core M2L. 0 (default, adaptive): the three
 * split-BF16 products hi*hi + hi*lo + lo*hi for the contraction components j < 64 and the
 * outputs i < 64 of every operator, hi*hi alone for the rest, whose terms are small enough
 * (singular-value ordered operators) for one BF16 product; 3: the three products
 * everywhere; 1: hi*hi everywhere (plain BF16, for precision comparisons). */
BBFMM_B200_API int bbfmm_b200_set_tc_products(bbfmm_b200_solver *s, int nprod);

/* Autotuner (no counterpart in the reference): runs an upward pass with q_dev, then times the
 * launch choices of every level's M2L (mixed mode: tensor-core split vs FP64; FP64 DMMA: the
 * 189 offsets split over 1, 3, 7 or 21 CTAs per target tile) and of the near field (64, 128
 * or 256 threads per block) on this solver's tree, and keeps the fastest. Choices are cached
 * in the process per (mode, n, level, cell count) and (mode, particles, leaves), so solvers
 * of similar shape reuse them without timing. Synchronises the device. */
BBFMM_B200_API int bbfmm_b200_autotune(bbfmm_b200_solver *s, const void *q_dev);
/* Current choices: info[0] = P2P threads per block, info[1 + l] = M2L kind of level l
 * (0 default: mixed mode on the tensor cores from level 4, and at levels 2-3 in batches;
 * 1 FP64/SIMT; 2 the tensor cores wherever they tile the level), info[12 + l] = offset groups
 * of level l (0 = default); 23 ints. */
BBFMM_B200_API int bbfmm_b200_tuning(const bbfmm_b200_solver *s, int *info);
/* Sets the choices (same 23 ints; for replaying a tuning or for tests). */
BBFMM_B200_API int bbfmm_b200_set_tuning(bbfmm_b200_solver *s, const int *info);

/* ---------------------------------------------------------------- batches
 * Many independent particle sets of uneven size, each with its own order n (4 or 8) and leaf
 * depth, solved together (no counterpart in the reference, which solves one set per call).
 * Sets of equal (n, depth) are stacked into one group whose every pass is one launch over all
 * its sets; groups of the same n share one copy of the operators; the groups run on streams
 * forked from the batch stream, and the batch solve is captured into a CUDA graph on first use
 * (and again whenever q_dev or phi_dev changes). cfg supplies mode, L, lead, lead_rows and
 * device (cfg->n, cfg->maxlev and cfg->stream are not used). Positions, charges and results
 * hold the sets back to back in set order: set s starts at counts[0] + ... + counts[s-1].
 * U4/E4 and U8/E8 are the operators of n = 4 and n = 8 (reference file layouts, FP64 unless
 * operators_fp32); the pair of an order no set uses may be NULL. */
typedef struct bbfmm_b200_batch bbfmm_b200_batch;
BBFMM_B200_API int bbfmm_b200_batch_create(const bbfmm_b200_config *cfg, int nsets, const int *n, const int *maxlev,
                                           const int *counts, const void *xyz, const void *U4, const void *E4,
                                           const void *U8, const void *E8, int operators_fp32,
                                           bbfmm_b200_batch **out);
/* The same with the positions in device memory on cfg->device (xyz_dev, the sets back to back,
 * in the batch's precision: FP32 for BBFMM_B200_MODE_S, else FP64): every group's octrees are
 * built there by one stable radix sort over (set, Morton leaf) keys -- per set the particle order
 * and leaf ranges of the host sort, bit for bit, so every solve is the same. Particles outside
 * [-L/2, L/2]^3 are rejected with BBFMM_B200_ERR_ARG. Synchronises the device. */
BBFMM_B200_API int bbfmm_b200_batch_create_device(const bbfmm_b200_config *cfg, int nsets, const int *n,
                                                  const int *maxlev, const int *counts, const void *xyz_dev,
                                                  const void *U4, const void *E4, const void *U8, const void *E8,
                                                  int operators_fp32, bbfmm_b200_batch **out);
/* One solve of every set (phi as in bbfmm_b200_solve), on the batch stream, without
 * synchronising; use_graph != 0 replays the captured graph. */
BBFMM_B200_API int bbfmm_b200_batch_solve(bbfmm_b200_batch *b, const void *q_dev, void *phi_dev, int use_graph);
/* bbfmm_b200_autotune for every group (drops the captured graph). */
BBFMM_B200_API int bbfmm_b200_batch_autotune(bbfmm_b200_batch *b, const void *q_dev);
/* Target regions of a batch (bbfmm_b200_set_target_region for every set): active holds, set
 * after set in set order, the mask bytes of the cells of level depth_s - levels_up of set s
 * (8^(depth_s - levels_up) each; NULL clears); first_m2l != 0 also starts each set's local
 * expansions one level below its region level (bbfmm_b200_set_first_m2l_level). Drops the
 * captured graph. bbfmm_b200.AdaptiveBatch refines the heavy leaves of a batch with it. */
BBFMM_B200_API int bbfmm_b200_batch_set_target_regions(bbfmm_b200_batch *b, int levels_up,
                                                       const unsigned char *active, int first_m2l);
/* Kernel of every set of the batch (as bbfmm_b200_set_kernel; the operators given at create
 * must be that kernel's). Drops the captured graph. */
BBFMM_B200_API int bbfmm_b200_batch_set_kernel(bbfmm_b200_batch *b, int kernel);
BBFMM_B200_API int bbfmm_b200_batch_groups(const bbfmm_b200_batch *b);
/* Nodes of the captured graph (0 before the first graph solve). */
BBFMM_B200_API long long bbfmm_b200_batch_graph_nodes(const bbfmm_b200_batch *b);
/* Group g: info[0] = n, info[1] = depth, info[2] = sets, info[3] = particles, info[4] = P2P
 * threads, info[5 + l] = M2L kind of level l, info[16 + l] = offset groups; 27 ints. */
BBFMM_B200_API int bbfmm_b200_batch_group_info(const bbfmm_b200_batch *b, int g, int *info);
/* Group g solved alone with per-stage timing (see bbfmm_b200_stage_times); synchronises. */
BBFMM_B200_API int bbfmm_b200_batch_group_stage_times(bbfmm_b200_batch *b, int g, const void *q_dev, void *phi_dev,
                                                      float *ms, int count);
BBFMM_B200_API void *bbfmm_b200_batch_stream(bbfmm_b200_batch *b);
BBFMM_B200_API void bbfmm_b200_batch_destroy(bbfmm_b200_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* BBFMM_B200_H */
