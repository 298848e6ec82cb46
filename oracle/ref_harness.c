/*
 * Harness around the REFERENCE implementation, compiled from the reference's own
 * sources by oracle/build_ref.sh into oracle/_ref/. TEST INFRASTRUCTURE ONLY: it
 * exists so that the CPU oracle (bbfmm_oracle.c) and the product can be pinned
 * against the reference itself on identical, seeded inputs.
 *
 * The reference generates its own particles (bbfmm.c:401-463) and chooses the depth
 * from N (bbfmm.c:151-160); this harness instead feeds caller-owned arrays and an
 * explicit maxlev to the reference's own set-up and pass functions:
 *   ComputeWeights (bbfmm.c:922), ComputeKernelSVD (bbfmm.c:1209),
 *   FMMReadMatrices (bbfmm.c:216), anotherBuildFMMHierachy (anotherBuildFMMHierachy.c:24),
 *   anotherUpwardPass, anotherFMMInteraction, anotherDownwardPass (another.h:42-73),
 *   DirectCalc3D (bbfmm.c:471), SetSources (bbfmm.c:401).
 *
 * Heap hygiene: the reference reads memory it never wrote (proxysval is malloc'd and
 * then accumulated into, anotherUpwardPass.c:50 with atransx.c:48-86; non-leaf
 * sourcesta/sourceend are read by M2M, anotherUpwardPass.c:388). Its results are the
 * intended ones only when fresh allocations read as zero, which holds for large
 * (mmap'd) blocks. Every call below therefore runs with glibc's M_PERTURB set to 0xff,
 * which makes every malloc return zero bytes, and restores it afterwards.
 */
#include <malloc.h>
#include <string.h>
#include "bbfmm.h"

static int g_timers_ready = 0;

static void harness_begin(void)
{
  mallopt(M_PERTURB, 0xff);
  if (!g_timers_ready) {
    allocTimer(&timer_main); initTimer(timer_main);
    allocTimer(&timer_run); initTimer(timer_run);
    allocTimer(&timer_setup); initTimer(timer_setup);
    allocTimer(&timer_comp); initTimer(timer_comp);
    allocTimer(&timer_upward); initTimer(timer_upward);
    allocTimer(&timer_interact); initTimer(timer_interact);
    allocTimer(&timer_downward); initTimer(timer_downward);
    allocTimer(&timer_output); initTimer(timer_output);
    allocTimer(&timer_cuda); initTimer(timer_cuda);
    g_timers_ready = 1;
  }
}

static void harness_end(void) { mallopt(M_PERTURB, 0); }

/* Reference's own operator precompute: writes K and U files at the given paths. */
int ref_compute_operators(int n, char *Kpath, char *Upath)
{
  harness_begin();
  int n2 = n * n, n3 = n2 * n;
  real *Kweights = (real *)malloc(n3 * sizeof(real));
  real *Cweights = (real *)malloc(2 * n2 * sizeof(real));
  real *Tkz = (real *)malloc(n2 * sizeof(real));
  int Ktable[343];
  ComputeWeights(Tkz, Ktable, Kweights, Cweights, n);
  ComputeKernelSVD(Kweights, n, 1, Kpath, Upath);
  free(Kweights); free(Cweights); free(Tkz);
  harness_end();
  return 0;
}

/* Reference's weight tables in its own precision. */
void ref_weights(int n, real *Tkz, int *Ktable, real *Kweights, real *Cweights)
{
  harness_begin();
  ComputeWeights(Tkz, Ktable, Kweights, Cweights, n);
  harness_end();
}

/* Reference's own input generator (glibc rand(), alternating +-1 charges), started from
   glibc's initial state (srand(1)) as in a fresh process of the reference executable. */
void ref_set_sources(int N, real L, real *xyz, real *q)
{
  harness_begin();
  srand(1);
  SetSources((real3 *)xyz, (real3 *)xyz, q, N, 1, L, 0);
  harness_end();
}

/* Tree and lists exactly as the reference builds them. Outputs as in orc_build_tree;
   sta/end of non-leaf cells are reported as 0/0. */
int ref_build_tree(int N, real *xyz, real L, int n, int maxlev, real *center, int *fieldlist,
                   int *sta, int *end, int *ineigh, int *neighbors, int *iinter, int *interaction)
{
  harness_begin();
  anotherTree *atree;
  anotherBuildFMMHierachy(L, n, 1, maxlev, n * n * n / 2, &atree, N, N, (real3 *)xyz,
                          (real3 *)xyz);
  cell *c = atree->c;
  int ncell = atree->ncell;
  memcpy(center, c->center, sizeof(real) * 3 * ncell);
  memcpy(fieldlist, atree->fieldlist, sizeof(int) * N);
  for (int A = 0; A < ncell; A++) {
    int leaf = A >= atree->levsta[maxlev];
    sta[A] = leaf ? c->fieldsta[A] : 0;
    end[A] = leaf ? c->fieldend[A] : 0;
  }
  memcpy(ineigh, c->ineigh, sizeof(int) * ncell);
  memcpy(iinter, c->iinter, sizeof(int) * ncell);
  for (int A = 0; A < ncell; A++) {
    memcpy(&neighbors[64 * A], &c->neighbors[c->pitch_neighbors * A], sizeof(int) * 64);
    memcpy(&interaction[192 * A], &c->interaction[c->pitch_interaction * A], sizeof(int) * 192);
  }
  anotherFMMCleanup(&atree);
  harness_end();
  return c ? 0 : 1;
}

/* One FMM solve through the reference's pass functions. Optional copies of the
   proxy source values (after the upward pass, ncell*r) and of the field values at
   the Chebyshev nodes (after M2L + post-M2L, before L2L; ncell*n^3). */
int ref_fmm(int N, real *xyz, real *q, real L, int n, int maxlev, char *Kpath, char *Upath,
            real *phi, real *proxysval_out, real *fieldval_out)
{
  harness_begin();
  int n2 = n * n, n3 = n2 * n, cutoff;
  real *Kweights = (real *)malloc(n3 * sizeof(real));
  real *Cweights = (real *)malloc(2 * n2 * sizeof(real));
  real *Tkz = (real *)malloc(n2 * sizeof(real));
  int Ktable[343];
  ComputeWeights(Tkz, Ktable, Kweights, Cweights, n);
  FILE *f = fopen(Upath, "rb");
  if (!f) { harness_end(); return 1; }
#ifdef ENABLE_ASCII_IO
  /* the text form starts with the cutoff on its own line (bbfmm.c:1361-1364) */
  if (fscanf(f, "%d", &cutoff) != 1) { fclose(f); harness_end(); return 1; }
#else
  if (fread(&cutoff, sizeof(int), 1, f) != 1) { fclose(f); harness_end(); return 1; }
#endif
  fclose(f);
  if (cutoff < 1 || cutoff > n3) { harness_end(); return 1; }
  real *K = (real *)malloc((size_t)316 * cutoff * cutoff * sizeof(real));
  real *U = (real *)malloc((size_t)cutoff * n3 * sizeof(real));
  FMMReadMatrices(K, U, cutoff, n, 1, Kpath, Upath);
  anotherTree *atree;
  anotherBuildFMMHierachy(L, n, 1, maxlev, cutoff, &atree, N, N, (real3 *)xyz, (real3 *)xyz);
#if defined(ONEOVERR4)
  real homogen = 4;  /* bbfmm.c:133-143 */
#elif defined(LAPLACIANFORCE)
  real homogen = 2;  /* bbfmm.c:122-131 */
#else
  real homogen = 1;
#endif
  anotherUpwardPass(&atree, (real3 *)xyz, Cweights, Tkz, q, U, Kweights, cutoff, n, 1);
  if (proxysval_out) memcpy(proxysval_out, atree->proxysval, sizeof(real) * atree->ncell * cutoff);
  anotherFMMInteraction(&atree, K, Ktable, U, Kweights, n, 1, cutoff, homogen);
  if (fieldval_out) memcpy(fieldval_out, atree->fieldval, sizeof(real) * atree->ncell * n3);
  anotherDownwardPass(&atree, (real3 *)xyz, (real3 *)xyz, Cweights, Tkz, q, U, cutoff, n, 1,
                      homogen, phi);
  anotherFMMCleanup(&atree);
  free(K); free(U); free(Kweights); free(Cweights); free(Tkz);
  harness_end();
  return 0;
}

/* Reference direct O(N^2) code (q_i * sum_{x_j != x_i} q_j / r_ij) on all targets. */
void ref_direct(int N, real *xyz, real *q, real L, real *phi)
{
  harness_begin();
  DirectCalc3D((real3 *)xyz, (real3 *)xyz, q, N, N, 1, 0, L, phi);
  harness_end();
}

int ref_real_size(void) { return (int)sizeof(real); }
