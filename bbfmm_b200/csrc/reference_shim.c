/* The reference's own entry-point names and signatures (include/bbfmm_b200_reference.h),
 * forwarding to the implementations in libbbfmm_b200.so. Compiled once per precision:
 * plain for real = double, -DBBFMM_B200_SINGLE for real = float. */
#include <stdio.h>

#include "bbfmm_b200_reference.h"

#ifdef BBFMM_B200_SINGLE
#define IMPL(name) bbfmm_b200_ref_##name##_s
#else
#define IMPL(name) bbfmm_b200_ref_##name##_d
#endif

double kernel_exec_time = 0.0;

/* The reference's void entry points abort or stay silent on errors; these report them. */
static void report(const char *fn, int rc)
{
  if (rc != 0) fprintf(stderr, "# %s: bbfmm_b200 error %d: %s\n", fn, rc, bbfmm_b200_last_error());
}

int m2l_drv(int r, bbfmm_b200_real *L, bbfmm_b200_real *K, bbfmm_b200_real *M, int minlev, int maxlev,
            bbfmm_b200_real L0, bbfmm_b200_real3 *center, int *ineigh, int pitch_neighbors, int *neighbors,
            int *iinter, int pitch_interaction, int *interaction, int scheme)
{
  (void)L0; (void)center; (void)ineigh; (void)pitch_neighbors; (void)neighbors; (void)iinter;
  (void)pitch_interaction; (void)interaction;
  if (scheme < 0 || scheme > 3) return 1; /* M2L_EXIT_FAIL, m2l_drv.cu:77-83 */
  int rc = IMPL(m2l_levels)(minlev, maxlev, r, L, K, M, &kernel_exec_time);
  report("m2l_drv", rc);
  return rc == 0 ? 0 : 1;
}

static void m2l_host(const char *fn, int lo, int hi, int r, bbfmm_b200_real *L, bbfmm_b200_real *K,
                     bbfmm_b200_real *M)
{
  report(fn, IMPL(m2l_levels)(lo, hi, r, L, K, M, &kernel_exec_time));
}

void m2l_host_basic(int level_start, int level_end, int r, bbfmm_b200_real *L, bbfmm_b200_real *K,
                    bbfmm_b200_real *M, int pitch_interaction, int *interaction, int *iinter, int *Kindex)
{
  (void)pitch_interaction; (void)interaction; (void)iinter; (void)Kindex;
  m2l_host("m2l_host_basic", level_start, level_end, r, L, K, M);
}

void m2l_host_sibling_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L, bbfmm_b200_real *K,
                               bbfmm_b200_real *M, int pitch_sourceclusters, int *sourceclusters, int *Ktable)
{
  (void)pitch_sourceclusters; (void)sourceclusters; (void)Ktable;
  m2l_host("m2l_host_sibling_blocking", level_start, level_end, r, L, K, M);
}

void m2l_host_cluster_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L, bbfmm_b200_real *K,
                               bbfmm_b200_real *M, int pitch_sourceclusters, int *sourceclusters, int *Ktable)
{
  (void)pitch_sourceclusters; (void)sourceclusters; (void)Ktable;
  m2l_host("m2l_host_cluster_blocking", level_start, level_end, r, L, K, M);
}

void m2l_host_ij_blocking(int level_start, int level_end, int r, bbfmm_b200_real *L, bbfmm_b200_real *K,
                          bbfmm_b200_real *M, int *Ktable, bbfmm_b200_real3 *center, bbfmm_b200_real L0)
{
  (void)Ktable; (void)center; (void)L0;
  m2l_host("m2l_host_ij_blocking", level_start, level_end, r, L, K, M);
}

void anotherFMMCompute(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field, bbfmm_b200_real3 *source,
                       bbfmm_b200_real *q, bbfmm_b200_real *K, bbfmm_b200_real *U, bbfmm_b200_real *Tkz,
                       int *Ktable, bbfmm_b200_real *Kweights, bbfmm_b200_real *Cweights, bbfmm_b200_real homogen,
                       int cutoff, int n, int dof, bbfmm_b200_real *phi)
{
  report("anotherFMMCompute", IMPL(compute)(atree, field, source, q, K, U, Tkz, Ktable, Kweights, Cweights,
                                            homogen, cutoff, n, dof, phi, &kernel_exec_time));
}

void anotherFMMInteraction(bbfmm_b200_tree **atree, bbfmm_b200_real *E, int *Ktable, bbfmm_b200_real *U,
                           bbfmm_b200_real *Kweights, int n, int dof, int cutoff, bbfmm_b200_real homogen)
{
  report("anotherFMMInteraction",
         IMPL(interaction)(atree, E, Ktable, U, Kweights, n, dof, cutoff, homogen, &kernel_exec_time));
}

void anotherUpwardPass(bbfmm_b200_tree **atree, bbfmm_b200_real3 *source, bbfmm_b200_real *Cweights,
                       bbfmm_b200_real *Tkz, bbfmm_b200_real *q, bbfmm_b200_real *V, bbfmm_b200_real *Kweights,
                       int cutoff, int n, int dof)
{
  report("anotherUpwardPass", IMPL(upward)(atree, source, Cweights, Tkz, q, V, Kweights, cutoff, n, dof));
}

void anotherDownwardPass(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field, bbfmm_b200_real3 *source,
                         bbfmm_b200_real *Cweights, bbfmm_b200_real *Tkz, bbfmm_b200_real *q, bbfmm_b200_real *U,
                         int cutoff, int n, int dof, bbfmm_b200_real homogen, bbfmm_b200_real *phi)
{
  report("anotherDownwardPass",
         IMPL(downward)(atree, field, source, Cweights, Tkz, q, U, cutoff, n, dof, homogen, phi));
}

void anotherDownwardPassX(bbfmm_b200_tree **atree, bbfmm_b200_real3 *field, bbfmm_b200_real *Cweights,
                          bbfmm_b200_real *Tkz, bbfmm_b200_real *q, bbfmm_b200_real *U, int cutoff, int n, int dof,
                          bbfmm_b200_real homogen, bbfmm_b200_real *phi)
{
  report("anotherDownwardPassX",
         IMPL(downward_far)(atree, field, Cweights, Tkz, q, U, cutoff, n, dof, homogen, phi));
}

void anotherNearField(bbfmm_b200_tree **atree, int dof, bbfmm_b200_real homogen, bbfmm_b200_real3 *field,
                      bbfmm_b200_real3 *source, bbfmm_b200_real *phi, bbfmm_b200_real *q)
{
  report("anotherNearField", IMPL(near_field)(atree, dof, homogen, field, source, phi, q));
}
