/*
 * The reference's own entry points (takahashitoru/bbFMMonGPU), served by the B200 library.
 *
 * Two layers:
 *  - libbbfmm_b200.so exports bbfmm_b200_ref_<name>_d / _s: the implementations for
 *    real = double / float, returning a status code (0 = success; the message is in
 *    bbfmm_b200_last_error()).
 *  - libbbfmm_b200_ref_d.so / libbbfmm_b200_ref_s.so (built from reference_shim.c) export the
 *    reference's names with its exact signatures and the global kernel_exec_time, so that
 *    the reference's host objects (main, bbfmm, tree build, interaction lists) link against
 *    them in place of the replaced objects. Define BBFMM_B200_SINGLE for the float build.
 *
 * Semantics kept from the reference: host arrays in and out; the ownership side effects of
 * the passes (proxysval allocated by the upward pass and freed by the interaction,
 * fieldval allocated by the interaction and freed by the downward pass); m2l_drv returns
 * M2L_EXIT_SUCCESS (0) or M2L_EXIT_FAIL (1) (m2l_drv.h:4-5) and accepts schemes 0-3, all of
 * which run the same B200 M2L. Differences: the tree must be the full uniform octree the
 * reference builds (its lists are implied and not read); dof = 1; the kernels with homogen 1
 * (LAPLACIAN, 1/r), 2 (LAPLACIANFORCE, x/r^3) and 4 (ONEOVERR4, 1/r^4), the caller's K and U
 * files being that kernel's;
 * void entry points report failures on stderr and through bbfmm_b200_last_error() instead
 * of aborting.
 */
#ifndef BBFMM_B200_REFERENCE_H
#define BBFMM_B200_REFERENCE_H

#include "bbfmm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define BBFMM_B200_REF_API __attribute__((visibility("default")))
#else
#define BBFMM_B200_REF_API
#endif

#ifdef BBFMM_B200_SINGLE
typedef float bbfmm_b200_real;
#else
typedef double bbfmm_b200_real;
#endif

/* real3, cell and anotherTree of the reference (vec234.h, cell.h:10-22, anotherTree.h:7-20),
 * non-periodic build. */
typedef struct { bbfmm_b200_real x, y, z; } bbfmm_b200_real3;
typedef struct {
  int *neighbors, *interaction;
  bbfmm_b200_real3 *center;
  int *fieldsta, *fieldend, *sourcesta, *sourceend;
  int *ineigh, *iinter;
  int pitch_neighbors, pitch_interaction;
} bbfmm_b200_cell;
typedef struct {
  int ncell, minlev, maxlev;
  int *levsta, *levend;
  bbfmm_b200_real *celeng;
  bbfmm_b200_cell *c;
  bbfmm_b200_real *fieldval, *sourceval, *proxysval;
  int ncell0;
  int Nf, Ns, *fieldlist, *sourcelist;
} bbfmm_b200_tree;

/* ---- implementations in libbbfmm_b200.so (atree is a bbfmm_b200_tree ** of the matching
 * precision; secs receives the M2L kernel time the reference stores in kernel_exec_time) */

/* m2l_drv.cu:14-93 and m2l_host_*: L[r A + i] for the cells A of levels lo..hi. */
BBFMM_B200_API int bbfmm_b200_ref_m2l_levels_d(int lo, int hi, int r, double *L, double *K, double *M, double *secs);
BBFMM_B200_API int bbfmm_b200_ref_m2l_levels_s(int lo, int hi, int r, float *L, float *K, float *M, double *secs);
/* anotherUpwardPass.c:20-571 */
BBFMM_B200_API int bbfmm_b200_ref_upward_d(void *atree, void *source, double *Cweights, double *Tkz, double *q,
                                           double *V, double *Kweights, int cutoff, int n, int dof);
BBFMM_B200_API int bbfmm_b200_ref_upward_s(void *atree, void *source, float *Cweights, float *Tkz, float *q,
                                           float *V, float *Kweights, int cutoff, int n, int dof);
/* anotherFMMInteraction.cu:29-126 */
BBFMM_B200_API int bbfmm_b200_ref_interaction_d(void *atree, double *E, int *Ktable, double *U, double *Kweights,
                                                int n, int dof, int cutoff, double homogen, double *secs);
BBFMM_B200_API int bbfmm_b200_ref_interaction_s(void *atree, float *E, int *Ktable, float *U, float *Kweights,
                                                int n, int dof, int cutoff, float homogen, double *secs);
/* anotherDownwardPass.cu:41-411 (far field + near field) */
BBFMM_B200_API int bbfmm_b200_ref_downward_d(void *atree, void *field, void *source, double *Cweights, double *Tkz,
                                             double *q, double *U, int cutoff, int n, int dof, double homogen,
                                             double *phi);
BBFMM_B200_API int bbfmm_b200_ref_downward_s(void *atree, void *field, void *source, float *Cweights, float *Tkz,
                                             float *q, float *U, int cutoff, int n, int dof, float homogen,
                                             float *phi);
/* anotherDownwardPassX.c:7-435 (L2L + L2P only) */
BBFMM_B200_API int bbfmm_b200_ref_downward_far_d(void *atree, void *field, double *Cweights, double *Tkz, double *q,
                                                 double *U, int cutoff, int n, int dof, double homogen, double *phi);
BBFMM_B200_API int bbfmm_b200_ref_downward_far_s(void *atree, void *field, float *Cweights, float *Tkz, float *q,
                                                 float *U, int cutoff, int n, int dof, float homogen, float *phi);
/* anotherNearField.c:219-346 */
BBFMM_B200_API int bbfmm_b200_ref_near_field_d(void *atree, int dof, double homogen, void *field, void *source,
                                               double *phi, double *q);
BBFMM_B200_API int bbfmm_b200_ref_near_field_s(void *atree, int dof, float homogen, void *field, void *source,
                                               float *phi, float *q);
/* anotherFMMCompute.cu:48-85 (one device-resident solve) */
BBFMM_B200_API int bbfmm_b200_ref_compute_d(void *atree, void *field, void *source, double *q, double *K, double *U,
                                            double *Tkz, int *Ktable, double *Kweights, double *Cweights,
                                            double homogen, int cutoff, int n, int dof, double *phi, double *secs);
BBFMM_B200_API int bbfmm_b200_ref_compute_s(void *atree, void *field, void *source, float *q, float *K, float *U,
                                            float *Tkz, int *Ktable, float *Kweights, float *Cweights, float homogen,
                                            int cutoff, int n, int dof, float *phi, double *secs);

/* ---- the reference's own names, exported by libbbfmm_b200_ref_{d,s}.so */

/* Seconds of M2L kernel time of the last M2L call (m2l_host.h:24). */
extern BBFMM_B200_REF_API double kernel_exec_time;

/* m2l_drv.cu:14-19 */
BBFMM_B200_REF_API int m2l_drv(int r, bbfmm_b200_real *L, bbfmm_b200_real *K, bbfmm_b200_real *M, int minlev,
                               int maxlev, bbfmm_b200_real L0, bbfmm_b200_real3 *center, int *ineigh,
                               int pitch_neighbors, int *neighbors, int *iinter, int pitch_interaction,
                               int *interaction, int scheme);
/* m2l_host_basic.cu:18-19 */
BBFMM_B200_REF_API void m2l_host_basic(int level_start, int level_end, int r, bbfmm_b200_real *L,
                                       bbfmm_b200_real *K, bbfmm_b200_real *M, int pitch_interaction,
                                       int *interaction, int *iinter, int *Kindex);
/* m2l_host_sibling_blocking.cu:22-23 */
BBFMM_B200_REF_API void m2l_host_sibling_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L,
                                                  bbfmm_b200_real *K, bbfmm_b200_real *M, int pitch_sourceclusters,
                                                  int *sourceclusters, int *Ktable);
/* m2l_host_cluster_blocking.cu:29-30 */
BBFMM_B200_REF_API void m2l_host_cluster_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L,
                                                  bbfmm_b200_real *K, bbfmm_b200_real *M, int pitch_sourceclusters,
                                                  int *sourceclusters, int *Ktable);
/* m2l_host_ij_blocking.cu:166-167 */
BBFMM_B200_REF_API void m2l_host_ij_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L,
                                             bbfmm_b200_real *K, bbfmm_b200_real *M, int *Ktable,
                                             bbfmm_b200_real3 *center, bbfmm_b200_real L0);
/* another.h:42-45 */
BBFMM_B200_REF_API void anotherFMMCompute(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field,
                                          bbfmm_b200_real3 *source, bbfmm_b200_real *q, bbfmm_b200_real *K,
                                          bbfmm_b200_real *U, bbfmm_b200_real *Tkz, int *Ktable,
                                          bbfmm_b200_real *Kweights, bbfmm_b200_real *Cweights,
                                          bbfmm_b200_real homogen, int cutoff, int n, int dof,
                                          bbfmm_b200_real *phi);
/* another.h:47-49 */
BBFMM_B200_REF_API void anotherFMMInteraction(bbfmm_b200_tree **atree, bbfmm_b200_real *E, int *Ktable,
                                              bbfmm_b200_real *U, bbfmm_b200_real *Kweights, int n, int dof,
                                              int cutoff, bbfmm_b200_real homogen);
/* another.h:50-51 */
BBFMM_B200_REF_API void anotherUpwardPass(bbfmm_b200_tree **atree, bbfmm_b200_real3 *source,
                                          bbfmm_b200_real *Cweights, bbfmm_b200_real *Tkz, bbfmm_b200_real *q,
                                          bbfmm_b200_real *V, bbfmm_b200_real *Kweights, int cutoff, int n, int dof);
/* another.h:52-54 */
BBFMM_B200_REF_API void anotherDownwardPass(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field,
                                            bbfmm_b200_real3 *source, bbfmm_b200_real *Cweights,
                                            bbfmm_b200_real *Tkz, bbfmm_b200_real *q, bbfmm_b200_real *U, int cutoff,
                                            int n, int dof, bbfmm_b200_real homogen, bbfmm_b200_real *phi);
/* another.h:63-65 */
BBFMM_B200_REF_API void anotherDownwardPassX(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field,
                                             bbfmm_b200_real *Cweights, bbfmm_b200_real *Tkz, bbfmm_b200_real *q,
                                             bbfmm_b200_real *U, int cutoff, int n, int dof,
                                             bbfmm_b200_real homogen, bbfmm_b200_real *phi);
/* another.h:72-73 */
BBFMM_B200_REF_API void anotherNearField(bbfmm_b200_tree **atree, int dof, bbfmm_b200_real homogen,
                                         bbfmm_b200_real3 *field, bbfmm_b200_real3 *source, bbfmm_b200_real *phi,
                                         bbfmm_b200_real *q);

#ifdef __cplusplus
}
#endif

#endif /* BBFMM_B200_REFERENCE_H */
