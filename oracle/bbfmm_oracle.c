/*
 * CPU ORACLE for the bbFMM hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker against which the CUDA path is compared. Only tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it; the product
 * library never links or calls it.
 *
 * It restates, in plain C, the reference implementation's CPU algorithm for every
 * stage of one FMM solve, in the same loop and summation order wherever the order
 * changes floating-point results, so that it can be pinned bit-for-bit against the
 * reference code compiled from its own sources (oracle/build_ref.sh):
 *
 *   tree + lists   anotherBuildFMMHierachy.c:24-122, anotherFMMDistribute.c:191-484,
 *                  anotherInteractionList.c:11-111
 *   weights        bbfmm.c:922-1028 (ComputeWeights), 1626-1733 (ComputeTk, ComputeSn2)
 *   P2M            anotherUpwardPass.c:61-330, atransx.c:48-86
 *   M2M            anotherUpwardPass.c:345-560 (all eight children are always present)
 *   M2L            m2l_kern_basic.cu:82-130 semantics: L(F) = sum_S E_k(F,S) M(S),
 *                  k from m2l_aux.c:1135-1191 (Kindex), E column-major per offset
 *   post-M2L       auxAnotherFMMInteraction.c:364-416, anotherFMMInteraction.cu:98-113
 *   L2L, L2P       anotherDownwardPassX.c:40-431
 *   P2P            anotherNearField.c:141-206 (CPU8A) and 219-316 (driver)
 *   direct         bbfmm.c:880-913 semantics (q_i * sum_{x_j != x_i} q_j / r_ij),
 *                  evaluated here in FP64 with compensated summation on sampled targets.
 *   kernels        1/r (LAPLACIAN), x/r^3 (LAPLACIANFORCE) and 1/r^4 (ONEOVERR4):
 *                  bbfmm.c:109-144 (homogeneity), anotherNearField.c:111-124 (pair value),
 *                  selected at run time by orc_set_kernel.
 *
 * Compiled twice: -DORC_SINGLE gives real = float (the reference's SINGLE build),
 * otherwise real = double. Every exported symbol carries the suffix _s or _d.
 *
 * Full-tree convention: the reference's M2M and L2L decide which children to visit
 * from fieldsta/fieldend, which it sets only for leaves (anotherFMMDistribute.c:318-319,
 * 842-843); on a zero-filled or pattern-filled heap every non-leaf reads as non-empty.
 * The oracle always visits all eight children, which is the mathematically exact
 * result (an empty child contributes zeros) and equals the reference on such heaps.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef ORC_SINGLE
typedef float real;
#define SFX(name) name##_s
#define SQRT(x) sqrtf(x)
#define POW(x, y) powf(x, y)
#define COS(x) cosf(x)
#define RINT(x) rintf(x)
#define ZERO 0.0f
#define ONE 1.0f
#define TWO 2.0f
#else
typedef double real;
#define SFX(name) name##_d
#define SQRT(x) sqrt(x)
#define POW(x, y) pow(x, y)
#define COS(x) cos(x)
#define RINT(x) rint(x)
#define ZERO 0.0
#define ONE 1.0
#define TWO 2.0
#endif

#define PITCH_NEIGHBORS 64     /* FLOORUP(27, 64), anotherBuildFMMHierachy.c:90-97 */
#define PITCH_INTERACTION 192  /* FLOORUP(189, 64) */
#define MINLEV 2

static int pow8(int i) { return 1 << (3 * i); }

/* Kernel: degree of homogeneity 1 (1/r, LAPLACIAN), 2 (x / r^3, LAPLACIANFORCE: the x
   component of the separation source - field over r^3) or 4 (1/r^4, ONEOVERR4); the pair value
   as the reference's near field forms it from rinv = 1/r and dx = x_s - x_f
   (anotherNearField.c:111-124). */
static int g_homogen = 1;
void SFX(orc_set_kernel)(int homogen) { g_homogen = homogen; }
static real kern(real rinv, real dx)
{
  if (g_homogen == 4) return rinv * rinv * rinv * rinv;
  if (g_homogen == 2) return dx * rinv * rinv * rinv;
  return rinv;
}

int SFX(orc_ncell)(int maxlev) { return (pow8(maxlev + 1) - 1) / 7; }
int SFX(orc_levsta)(int level) { return (pow8(level) - 1) / 7; }

/* ---------------------------------------------------------------- weights --- */

static void tk(real x, int n, real *vec)
{
  vec[0] = 1;
  vec[1] = x;
  for (int k = 2; k < n; k++) vec[k] = 2 * x * vec[k - 1] - vec[k - 2];
}

static real sn_each(const real *vec, real *d, int n, real x)
{
  d[n] = d[n + 1] = 0;
  for (int j = n - 1; j > 0; j--) d[j] = 2 * x * d[j + 1] - d[j + 2] + vec[j];
  return x * d[1] - d[2] + (real)0.5 * vec[0];
}

/* Tkz[n*n], Ktable[343], Kweights[n^3], Cweights[2 n^2] (bbfmm.c:922-1028). */
void SFX(orc_weights)(int n, real *Tkz, int *Ktable, real *Kweights, real *Cweights)
{
  real nodes[32], vec[32], d[34];
  real pi = (real)3.1415926535897932384626433832795;
  for (int i = 0; i < 343; i++) Ktable[i] = -1;
  int ncell = 0, ninteract = 0;
  for (int l1 = -3; l1 < 4; l1++)
    for (int l2 = -3; l2 < 4; l2++)
      for (int l3 = -3; l3 < 4; l3++) {
        if (abs(l1) > 1 || abs(l2) > 1 || abs(l3) > 1) Ktable[ncell] = ninteract++;
        ncell++;
      }
  for (int m = 0; m < n; m++) nodes[m] = COS(pi * (real)(2 * m + 1) / (real)(2 * n));
  for (int m = 0; m < n; m++) {
    tk(nodes[m], n, vec);
    for (int k = 0; k < n; k++) Tkz[m * n + k] = vec[k];
  }
  int count = 0;
  for (int l1 = 0; l1 < n; l1++) {
    real t1 = 1 / SQRT(1 - nodes[l1] * nodes[l1]);
    for (int l2 = 0; l2 < n; l2++) {
      real t2 = t1 / SQRT(1 - nodes[l2] * nodes[l2]);
      for (int l3 = 0; l3 < n; l3++) Kweights[count++] = t2 / SQRT(1 - nodes[l3] * nodes[l3]);
    }
  }
  /* Cweights[side n^2 + p n + c] = S(x_p, (x_c -/+ 1)/2): the z-component of
     ComputeSn over the mapped child nodes, of which only the first n matter. */
  for (int side = 0; side < 2; side++)
    for (int p = 0; p < n; p++)
      for (int c = 0; c < n; c++) {
        real z = (real)0.5 * (nodes[c] + (side ? (real)1 : (real)-1));
        Cweights[side * n * n + p * n + c] = sn_each(&Tkz[p * n], d, n, z);
      }
}

/* ------------------------------------------------------------------- tree --- */

/* Cell centres, leaf particle lists and neighbour/interaction lists of the full
   uniform octree with leaves at maxlev; xyz is N x 3 (AoS). Outputs:
   center[ncell*3], fieldlist[N], sta/end[ncell] (leaves only; others set to 0/0),
   ineigh[ncell], neighbors[ncell*64], iinter[ncell], interaction[ncell*192]. */
void SFX(orc_build_tree)(int N, const real *xyz, real L, int maxlev, real *center,
                         int *fieldlist, int *sta, int *end, int *ineigh, int *neighbors,
                         int *iinter, int *interaction)
{
  int ncell = SFX(orc_ncell)(maxlev);
  real celeng[32];
  real length = L;
  for (int level = 0; level <= maxlev; level++) {
    celeng[level] = length;
    length *= 0.5;
  }
  center[0] = center[1] = center[2] = ZERO;
  for (int level = 1; level <= maxlev; level++) {
    real Lhalf = celeng[level] / 2;
    for (int A = SFX(orc_levsta)(level); A < SFX(orc_levsta)(level + 1); A++) {
      int P = (A - 1) >> 3;
      int s = A - (8 * P + 1);
      center[3 * A + 0] = center[3 * P + 0] + (s < 4 ? -Lhalf : Lhalf);
      center[3 * A + 1] = center[3 * P + 1] + (s % 4 < 2 ? -Lhalf : Lhalf);
      center[3 * A + 2] = center[3 * P + 2] + (s % 2 == 0 ? -Lhalf : Lhalf);
    }
  }
  for (int A = 0; A < ncell; A++) sta[A] = end[A] = 0;
  /* Counting sort into leaves, stable in particle index. */
  int Asta = SFX(orc_levsta)(maxlev), nc = pow8(maxlev), ncpd = 1 << maxlev;
  int *map = (int *)malloc(sizeof(int) * nc);
  int *cnt = (int *)calloc(nc, sizeof(int));
  int *leaf = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
  real L0half = celeng[0] / 2, iLm = 1 / celeng[maxlev];
  for (int A = Asta; A < Asta + nc; A++) {
    int ix = (int)((center[3 * A] + L0half) * iLm);
    int iy = (int)((center[3 * A + 1] + L0half) * iLm);
    int iz = (int)((center[3 * A + 2] + L0half) * iLm);
    map[(iz * ncpd + iy) * ncpd + ix] = A;
  }
  for (int i = 0; i < N; i++) {
    int ix = (int)((xyz[3 * i] + L0half) * iLm);
    int iy = (int)((xyz[3 * i + 1] + L0half) * iLm);
    int iz = (int)((xyz[3 * i + 2] + L0half) * iLm);
    if (ix > ncpd - 1) ix = ncpd - 1;
    if (iy > ncpd - 1) iy = ncpd - 1;
    if (iz > ncpd - 1) iz = ncpd - 1;
    leaf[i] = map[(iz * ncpd + iy) * ncpd + ix] - Asta;
    cnt[leaf[i]]++;
  }
  int l = 0;
  for (int k = 0; k < nc; k++) {
    sta[Asta + k] = l;
    int c = cnt[k];
    cnt[k] = l;
    l += c;
    end[Asta + k] = l - 1;
  }
  for (int i = 0; i < N; i++) fieldlist[cnt[leaf[i]]++] = i;
  free(map);
  free(cnt);
  free(leaf);
  /* Lists (anotherInteractionList.c:41-110). */
  for (int A = 0; A < ncell; A++) ineigh[A] = iinter[A] = 0;
  neighbors[0] = 0;
  ineigh[0] = 1;
  for (int level = 1; level <= maxlev; level++) {
    real Lsafe = celeng[level] * (real)1.5;
    real Lsafe2 = Lsafe * Lsafe;
    for (int A = SFX(orc_levsta)(level); A < SFX(orc_levsta)(level + 1); A++) {
      int P = (A - 1) >> 3;
      for (int i = 0; i < ineigh[P]; i++) {
        int U = neighbors[PITCH_NEIGHBORS * P + i];
        for (int j = 0; j < 8; j++) {
          int C = 8 * U + 1 + j;
          real dx = center[3 * C] - center[3 * A];
          real dy = center[3 * C + 1] - center[3 * A + 1];
          real dz = center[3 * C + 2] - center[3 * A + 2];
          if (dx * dx <= Lsafe2 && dy * dy <= Lsafe2 && dz * dz <= Lsafe2)
            neighbors[PITCH_NEIGHBORS * A + ineigh[A]++] = C;
          else
            interaction[PITCH_INTERACTION * A + iinter[A]++] = C;
        }
      }
    }
  }
}

/* ----------------------------------------------------------------- upward --- */

static void sn2(const real *xt, int Ns, const real *Tkz, int n, real *Sx, real *Sy, real *Sz)
{
  real d[34];
  for (int m = 0; m < n; m++)
    for (int i = 0; i < Ns; i++) {
      Sx[m * Ns + i] = sn_each(&Tkz[m * n], d, n, xt[3 * i + 0]);
      Sy[m * Ns + i] = sn_each(&Tkz[m * n], d, n, xt[3 * i + 1]);
      Sz[m * Ns + i] = sn_each(&Tkz[m * n], d, n, xt[3 * i + 2]);
    }
}

/* y[i] = 0 + sum_j A^T ... (atransx.c:48-86 with y zero on entry), from the transposed
   copy ut[nn j + i] = at[m i + j]: every y[i] still sums its terms in the order j = 0 .. m-1
   from +0 (a sum started at +0 is never -0 under round-to-nearest, so the final 0 + sum of
   the reference changes nothing), and the inner loop runs over contiguous i. */
static void atransx_t(int m, int nn, const real *ut, const real *x, real *y)
{
  for (int i = 0; i < nn; i++) y[i] = ZERO;
  for (int j = 0; j < m; j++) {
    const real xj = x[j];
    const real *u = &ut[(size_t)nn * j];
    for (int i = 0; i < nn; i++) y[i] += u[i] * xj;
  }
}

static real xdot(int n, const real *x, int incx, const real *y, int incy)
{
  real sum = ZERO;
  for (int i = 0; i < n; i++) sum += x[i * incx] * y[i * incy];
  return sum;
}

/* P2M at maxlev then M2M up to minlev. sourceval[ncell n^3], proxysval[ncell r]
   (entries of levels < minlev are left untouched). */
void SFX(orc_upward)(int maxlev, int n, int r, const real *xyz, const real *q,
                     const real *center, const int *fieldlist, const int *sta, const int *end,
                     const real *Tkz, const real *Kweights, const real *Cweights, const real *U,
                     real L, real *sourceval, real *proxysval)
{
  int n2 = n * n, n3 = n2 * n;
  real prefac = TWO / (real)n, prefac3 = prefac * prefac * prefac;
  real celeng[32];
  real length = L;
  for (int level = 0; level <= maxlev; level++) {
    celeng[level] = length;
    length *= 0.5;
  }
  real *Sw = (real *)malloc(sizeof(real) * n3);
  real *Ut = (real *)malloc(sizeof(real) * (size_t)n3 * r);  /* Ut[r l + i] = U[n3 i + l] */
  for (int i = 0; i < r; i++)
    for (int l = 0; l < n3; l++) Ut[(size_t)r * l + i] = U[(size_t)n3 * i + l];
  {
    real Lc = celeng[maxlev], halfL = Lc / TWO, ihalfL = ONE / halfL;
    for (int A = SFX(orc_levsta)(maxlev); A < SFX(orc_levsta)(maxlev + 1); A++) {
      int Ns = end[A] - sta[A] + 1;
      real *xt = (real *)malloc(sizeof(real) * 3 * (Ns > 0 ? Ns : 1));
      real *qt = (real *)malloc(sizeof(real) * (Ns > 0 ? Ns : 1));
      real *Sx = (real *)malloc(sizeof(real) * n * (Ns > 0 ? Ns : 1));
      real *Sy = (real *)malloc(sizeof(real) * n * (Ns > 0 ? Ns : 1));
      real *Sz = (real *)malloc(sizeof(real) * n * (Ns > 0 ? Ns : 1));
      for (int j = 0; j < Ns; j++) {
        int k = fieldlist[sta[A] + j];
        xt[3 * j + 0] = ihalfL * (xyz[3 * k + 0] - center[3 * A + 0]);
        xt[3 * j + 1] = ihalfL * (xyz[3 * k + 1] - center[3 * A + 1]);
        xt[3 * j + 2] = ihalfL * (xyz[3 * k + 2] - center[3 * A + 2]);
        qt[j] = q[k];
      }
      sn2(xt, Ns, Tkz, n, Sx, Sy, Sz);
      real *S = &sourceval[(size_t)n3 * A];
      int l = 0;
      for (int l1 = 0; l1 < n; l1++)
        for (int l2 = 0; l2 < n; l2++)
          for (int l3 = 0; l3 < n; l3++) {
            real sum = ZERO;
            for (int j = 0; j < Ns; j++) {
              real w = qt[j] * Sx[l1 * Ns + j] * Sy[l2 * Ns + j];
              sum += w * Sz[l3 * Ns + j];
            }
            S[l] = prefac3 * sum;
            Sw[l] = S[l] * Kweights[l];
            l++;
          }
      atransx_t(n3, r, Ut, Sw, &proxysval[(size_t)r * A]);
      free(xt); free(qt); free(Sx); free(Sy); free(Sz);
    }
  }
  real *Sy = (real *)malloc(sizeof(real) * 2 * n3);
  real *Sz = (real *)malloc(sizeof(real) * 4 * n3);
  for (int level = maxlev - 1; level >= MINLEV; level--) {
    for (int A = SFX(orc_levsta)(level); A < SFX(orc_levsta)(level + 1); A++) {
      memset(Sy, 0, sizeof(real) * 2 * n3);
      memset(Sz, 0, sizeof(real) * 4 * n3);
      real *S = &sourceval[(size_t)n3 * A];
      for (int l = 0; l < n3; l++) S[l] = ZERO;
      for (int j = 0; j < 8; j++) {
        int l = (j / 2) * n3;
        const real *Sc = &sourceval[(size_t)n3 * (8 * A + 1 + j)];
        int wstart = (j % 2) ? n2 : 0;
        for (int l1 = 0; l1 < n2; l1++)
          for (int l3 = 0; l3 < n; l3++) {
            Sz[l] += xdot(n, &Sc[l1 * n], 1, &Cweights[wstart + l3 * n], 1);
            l++;
          }
      }
      for (int j = 0; j < 4; j++) {
        int l = (j / 2) * n3;
        int wstart = (j % 2) ? n2 : 0;
        for (int l1 = 0; l1 < n; l1++)
          for (int l2 = 0; l2 < n; l2++)
            for (int l3 = 0; l3 < n; l3++) {
              Sy[l] += xdot(n, &Sz[j * n3 + l1 * n2 + l3], n, &Cweights[wstart + l2 * n], 1);
              l++;
            }
      }
      for (int j = 0; j < 2; j++) {
        int l = 0;
        int wstart = j ? n2 : 0;
        for (int l1 = 0; l1 < n; l1++)
          for (int l2 = 0; l2 < n; l2++)
            for (int l3 = 0; l3 < n; l3++) {
              S[l] += xdot(n, &Sy[j * n3 + l2 * n + l3], n2, &Cweights[wstart + l1 * n], 1);
              l++;
            }
      }
      for (int l = 0; l < n3; l++) {
        S[l] *= prefac3;
        Sw[l] = S[l] * Kweights[l];
      }
      atransx_t(n3, r, Ut, Sw, &proxysval[(size_t)r * A]);
    }
  }
  free(Sy);
  free(Sz);
  free(Sw);
  free(Ut);
}

/* -------------------------------------------------------------------- M2L --- */

/* PF[r*F + i] = sum_{S in IL(F)} sum_j E_k[j r + i] M[r S + j] for levels
   minlev..maxlev; the operator index k comes from the rounded centre difference. */
void SFX(orc_m2l)(int maxlev, int r, const real *E, const real *M, const real *center,
                  const int *iinter, const int *interaction, const int *Ktable, real L,
                  real *PF)
{
  real *acc = (real *)malloc(sizeof(real) * r), *tmp = (real *)malloc(sizeof(real) * r);
  for (int level = MINLEV; level <= maxlev; level++) {
    real Lc = L;
    for (int i = 0; i < level; i++) Lc *= 0.5;
    real iL = ONE / Lc;
    for (int F = SFX(orc_levsta)(level); F < SFX(orc_levsta)(level + 1); F++) {
      for (int i = 0; i < r; i++) acc[i] = ZERO;
      for (int t = 0; t < iinter[F]; t++) {
        int S = interaction[PITCH_INTERACTION * F + t];
        int vx = (int)RINT((center[3 * S] - center[3 * F]) * iL);
        int vy = (int)RINT((center[3 * S + 1] - center[3 * F + 1]) * iL);
        int vz = (int)RINT((center[3 * S + 2] - center[3 * F + 2]) * iL);
        int k = Ktable[49 * (vx + 3) + 7 * (vy + 3) + (vz + 3)];
        const real *Ek = &E[(size_t)r * r * k];
        const real *Ms = &M[(size_t)r * S];
        /* sum_j Ek(i, j) M_S[j] for every i, each in the order j = 0 .. r-1, then added to
           acc[i]; the loop over i is the inner one so that it reads Ek contiguously */
        for (int i = 0; i < r; i++) tmp[i] = ZERO;
        for (int j = 0; j < r; j++) {
          const real mj = Ms[j];
          const real *col = &Ek[(size_t)j * r];
          for (int i = 0; i < r; i++) tmp[i] += col[i] * mj;
        }
        for (int i = 0; i < r; i++) acc[i] += tmp[i];
      }
      for (int i = 0; i < r; i++) PF[(size_t)r * F + i] = acc[i];
    }
  }
  free(acc);
  free(tmp);
}

/* The same (target, source) products from a list of pairs: acc[r cell[p] + i] += sum_j
   E_{k[p]}(i, j) M[r src[p] + j], the pairs taken in the order given (a caller that sorts them
   by operator reads each r x r block once per run of equal k). Each product sums over j in
   order, as orc_m2l; only the order in which a cell's products are added can differ. */
void SFX(orc_m2l_pairs)(int r, const real *E, const real *M, long long npairs, const int *cell,
                        const long long *src, const int *k, real *acc)
{
  real *tmp = (real *)malloc(sizeof(real) * r);
  for (long long p = 0; p < npairs; p++) {
    const real *Ek = &E[(size_t)r * r * k[p]];
    const real *Ms = &M[(size_t)r * src[p]];
    for (int i = 0; i < r; i++) tmp[i] = ZERO;
    for (int j = 0; j < r; j++) {
      const real mj = Ms[j];
      const real *col = &Ek[(size_t)j * r];
      for (int i = 0; i < r; i++) tmp[i] += col[i] * mj;
    }
    real *a = &acc[(size_t)r * cell[p]];
    for (int i = 0; i < r; i++) a[i] += tmp[i];
  }
  free(tmp);
}

/* fieldval[n3 A + i] = (scale * Kweights[i]) * sum_j U(i, j) PF[r A + j], scale =
   (1/L_level)^homogeneity (anotherFMMInteraction.c:7545-7549), for levels minlev..maxlev. */
void SFX(orc_postm2l)(int maxlev, int n, int r, const real *U, const real *Kweights,
                      const real *PF, real L, real *fieldval)
{
  int n3 = n * n * n;
  real *tmp = (real *)malloc(sizeof(real) * n3);
  for (int level = MINLEV; level <= maxlev; level++) {
    real Lc = L;
    for (int i = 0; i < level; i++) Lc *= 0.5;
    real scale = POW(ONE / Lc, (real)g_homogen);
    for (int A = SFX(orc_levsta)(level); A < SFX(orc_levsta)(level + 1); A++) {
      /* every sum over j in order, the loop over i inner (contiguous columns of U) */
      for (int i = 0; i < n3; i++) tmp[i] = ZERO;
      for (int j = 0; j < r; j++) {
        const real pj = PF[(size_t)r * A + j];
        const real *col = &U[(size_t)n3 * j];
        for (int i = 0; i < n3; i++) tmp[i] += col[i] * pj;
      }
      for (int i = 0; i < n3; i++) fieldval[(size_t)n3 * A + i] = scale * Kweights[i] * tmp[i];
    }
  }
  free(tmp);
}

/* --------------------------------------------------------------- downward --- */

/* L2L (minlev..maxlev-1, accumulate into children; fieldval is modified) and L2P
   (assign phi[k] = q_k prefac^3 sum F S S S at every particle). */
void SFX(orc_downward)(int maxlev, int n, const real *xyz, const real *q, const real *center,
                       const int *fieldlist, const int *sta, const int *end, const real *Tkz,
                       const real *Cweights, real L, real *fieldval, real *phi)
{
  int n2 = n * n, n3 = n2 * n;
  real prefac = TWO / (real)n, prefac3 = prefac * prefac * prefac;
  real *Fx = (real *)malloc(sizeof(real) * 2 * n3);
  real *Fy = (real *)malloc(sizeof(real) * 4 * n3);
  for (int level = MINLEV; level < maxlev; level++) {
    for (int A = SFX(orc_levsta)(level); A < SFX(orc_levsta)(level + 1); A++) {
      const real *F = &fieldval[(size_t)n3 * A];
      for (int j = 0; j < 2; j++) {
        int l = j * n3, wstart = j ? n2 : 0;
        for (int l1 = 0; l1 < n; l1++)
          for (int l2 = 0; l2 < n; l2++)
            for (int l3 = 0; l3 < n; l3++)
              Fx[l++] = xdot(n, &F[l2 * n + l3], n2, &Cweights[wstart + l1], n);
      }
      for (int j = 0; j < 4; j++) {
        int l = j * n3, wstart = (j % 2) ? n2 : 0;
        for (int l1 = 0; l1 < n; l1++)
          for (int l2 = 0; l2 < n; l2++)
            for (int l3 = 0; l3 < n; l3++)
              Fy[l++] = xdot(n, &Fx[(j / 2) * n3 + l1 * n2 + l3], n, &Cweights[wstart + l2], n);
      }
      for (int j = 0; j < 8; j++) {
        real *Fc = &fieldval[(size_t)n3 * (8 * A + 1 + j)];
        int l = 0, wstart = (j % 2) ? n2 : 0;
        for (int l1 = 0; l1 < n2; l1++)
          for (int l3 = 0; l3 < n; l3++) {
            Fc[l] += prefac3 * xdot(n, &Fy[(j / 2) * n3 + l1 * n], 1, &Cweights[wstart + l3], n);
            l++;
          }
      }
    }
  }
  free(Fx);
  free(Fy);
  real Lc = L;
  for (int i = 0; i < maxlev; i++) Lc *= 0.5;
  real halfL = Lc / TWO, ihalfL = ONE / halfL;
  for (int A = SFX(orc_levsta)(maxlev); A < SFX(orc_levsta)(maxlev + 1); A++) {
    int Nf = end[A] - sta[A] + 1;
    if (Nf <= 0) continue;
    const real *F = &fieldval[(size_t)n3 * A];
    real *xt = (real *)malloc(sizeof(real) * 3 * Nf);
    real *Sx = (real *)malloc(sizeof(real) * n * Nf);
    real *Sy = (real *)malloc(sizeof(real) * n * Nf);
    real *Sz = (real *)malloc(sizeof(real) * n * Nf);
    real *sum = (real *)calloc(Nf, sizeof(real));
    for (int i = 0; i < Nf; i++) {
      int k = fieldlist[sta[A] + i];
      for (int a = 0; a < 3; a++) xt[3 * i + a] = ihalfL * (xyz[3 * k + a] - center[3 * A + a]);
    }
    sn2(xt, Nf, Tkz, n, Sx, Sy, Sz);
    int l = 0;
    for (int l1 = 0; l1 < n; l1++)
      for (int l2 = 0; l2 < n; l2++) {
        if (n % 4 == 0) {
          for (int l3 = 0; l3 < n; l3 += 4) {
            for (int i = 0; i < Nf; i++)
              sum[i] += Sx[l1 * Nf + i] * Sy[l2 * Nf + i] *
                        (Sz[l3 * Nf + i] * F[l] + Sz[(l3 + 1) * Nf + i] * F[l + 1] +
                         Sz[(l3 + 2) * Nf + i] * F[l + 2] + Sz[(l3 + 3) * Nf + i] * F[l + 3]);
            l += 4;
          }
        } else {
          for (int l3 = 0; l3 < n; l3++) {
            for (int i = 0; i < Nf; i++)
              sum[i] += Sx[l1 * Nf + i] * Sy[l2 * Nf + i] * Sz[l3 * Nf + i] * F[l];
            l++;
          }
        }
      }
    for (int i = 0; i < Nf; i++) {
      int k = fieldlist[sta[A] + i];
      phi[k] = q[k] * prefac3 * sum[i];
    }
    free(xt); free(Sx); free(Sy); free(Sz); free(sum);
  }
}

/* -------------------------------------------------------------------- P2P --- */

/* phi[k] += q_k sum_{B in N(A)} sum_{j in B, r != 0} q_j K(x_j - x_k), K = kern() above
   (anotherNearField.c). */
void SFX(orc_nearfield)(int maxlev, int N, const real *xyz, const real *q, const int *fieldlist,
                        const int *sta, const int *end, const int *ineigh, const int *neighbors,
                        real *phi)
{
  real *x = (real *)malloc(sizeof(real) * (N > 0 ? N : 1));
  real *y = (real *)malloc(sizeof(real) * (N > 0 ? N : 1));
  real *z = (real *)malloc(sizeof(real) * (N > 0 ? N : 1));
  real *p = (real *)malloc(sizeof(real) * (N > 0 ? N : 1));
  real *qs = (real *)malloc(sizeof(real) * (N > 0 ? N : 1));
  int Asta = SFX(orc_levsta)(maxlev), Aend = SFX(orc_levsta)(maxlev + 1);
  for (int A = Asta; A < Aend; A++)
    for (int i = sta[A]; i <= end[A]; i++) {
      int k = fieldlist[i];
      x[i] = xyz[3 * k]; y[i] = xyz[3 * k + 1]; z[i] = xyz[3 * k + 2];
      p[i] = phi[k]; qs[i] = q[k];
    }
  for (int A = Asta; A < Aend; A++)
    for (int i = sta[A]; i <= end[A]; i++) {
      real fx = x[i], fy = y[i], fz = z[i], v = ZERO;
      for (int t = 0; t < ineigh[A]; t++) {
        int B = neighbors[PITCH_NEIGHBORS * A + t];
        int jsta = sta[B], nj = end[B] - sta[B] + 1;
        for (int j = 0; j < nj; j++) {
          real dx = x[jsta + j] - fx, dy = y[jsta + j] - fy, dz = z[jsta + j] - fz;
          real rr = dx * dx + dy * dy + dz * dz;
          real rinv = (rr != ZERO ? ONE / SQRT(rr) : ZERO);
          v += kern(rinv, dx) * qs[jsta + j];
        }
      }
      p[i] += qs[i] * v;
    }
  for (int A = Asta; A < Aend; A++)
    for (int i = sta[A]; i <= end[A]; i++) phi[fieldlist[i]] = p[i];
  free(x); free(y); free(z); free(p); free(qs);
}

/* ------------------------------------------------------------------- solve --- */

/* One whole solve (upward, M2L, post-M2L, downward, near field) on the tree built by
   orc_build_tree. E: 316 r^2 column-major blocks, U: n^3 x r column-major. */
void SFX(orc_fmm)(int N, const real *xyz, const real *q, real L, int n, int r, int maxlev,
                  const real *E, const real *U, real *phi)
{
  int ncell = SFX(orc_ncell)(maxlev), n3 = n * n * n;
  real *center = (real *)malloc(sizeof(real) * 3 * ncell);
  int *fieldlist = (int *)malloc(sizeof(int) * (N > 0 ? N : 1));
  int *sta = (int *)malloc(sizeof(int) * ncell), *end = (int *)malloc(sizeof(int) * ncell);
  int *ineigh = (int *)malloc(sizeof(int) * ncell), *iinter = (int *)malloc(sizeof(int) * ncell);
  int *neighbors = (int *)malloc(sizeof(int) * (size_t)ncell * PITCH_NEIGHBORS);
  int *interaction = (int *)malloc(sizeof(int) * (size_t)ncell * PITCH_INTERACTION);
  SFX(orc_build_tree)(N, xyz, L, maxlev, center, fieldlist, sta, end, ineigh, neighbors,
                      iinter, interaction);
  real Tkz[1024], Kweights[32768], Cweights[2048];
  int Ktable[343];
  SFX(orc_weights)(n, Tkz, Ktable, Kweights, Cweights);
  real *sourceval = (real *)calloc((size_t)ncell * n3, sizeof(real));
  real *proxysval = (real *)calloc((size_t)ncell * r, sizeof(real));
  real *PF = (real *)calloc((size_t)ncell * r, sizeof(real));
  real *fieldval = (real *)calloc((size_t)ncell * n3, sizeof(real));
  SFX(orc_upward)(maxlev, n, r, xyz, q, center, fieldlist, sta, end, Tkz, Kweights, Cweights, U,
                  L, sourceval, proxysval);
  SFX(orc_m2l)(maxlev, r, E, proxysval, center, iinter, interaction, Ktable, L, PF);
  SFX(orc_postm2l)(maxlev, n, r, U, Kweights, PF, L, fieldval);
  SFX(orc_downward)(maxlev, n, xyz, q, center, fieldlist, sta, end, Tkz, Cweights, L, fieldval,
                    phi);
  SFX(orc_nearfield)(maxlev, N, xyz, q, fieldlist, sta, end, ineigh, neighbors, phi);
  free(center); free(fieldlist); free(sta); free(end); free(ineigh); free(iinter);
  free(neighbors); free(interaction); free(sourceval); free(proxysval); free(PF); free(fieldval);
}

/* FP64 direct sum on sampled targets: out[t] = q_i sum_{x_j != x_i} q_j K(x_j - x_i) (K = 1/r,
   x/r^3 or 1/r^4 as set by orc_set_kernel),
   i = targets[t], with Neumaier-compensated summation. Positions are given in FP64
   whatever the build precision. */
void SFX(orc_direct_fp64)(int N, const double *xyz, const double *q, int ntarget,
                          const int *targets, double *out)
{
  for (int t = 0; t < ntarget; t++) {
    int i = targets[t];
    double fx = xyz[3 * i], fy = xyz[3 * i + 1], fz = xyz[3 * i + 2];
    double s = 0.0, c = 0.0;
    for (int j = 0; j < N; j++) {
      double dx = xyz[3 * j] - fx, dy = xyz[3 * j + 1] - fy, dz = xyz[3 * j + 2] - fz;
      if (dx == 0.0 && dy == 0.0 && dz == 0.0) continue;
      double rr = dx * dx + dy * dy + dz * dz;
      double v = g_homogen == 4   ? q[j] * (1.0 / rr) * (1.0 / rr)
                 : g_homogen == 2 ? q[j] * dx / (rr * sqrt(rr))
                                  : q[j] / sqrt(rr);
      double tsum = s + v;
      if (fabs(s) >= fabs(v)) c += (s - tsum) + v; else c += (v - tsum) + s;
      s = tsum;
    }
    out[t] = q[i] * (s + c);
  }
}

/* The reference's own input generator (bbfmm.c:401-463, RANDOM_SEED off): alternating
   +1/-1 charges and positions uniform in [-L/2, L/2)^3 drawn with glibc rand() from its
   default state, x then y then z per particle. Restarts the sequence with srand(1), which
   is glibc's initial state. */
void SFX(orc_ref_sources)(int N, real L, real *xyz, real *q)
{
  srand(1);
  real halfp = L / 2, halfm = -halfp;
  real inv_rand_max = 1.0 / RAND_MAX;
  for (int i = 0; i < N; i++) {
    q[i] = 1 - 2 * (i % 2);
    xyz[3 * i + 0] = halfm + (halfp - halfm) * rand() * inv_rand_max;
    xyz[3 * i + 1] = halfm + (halfp - halfm) * rand() * inv_rand_max;
    xyz[3 * i + 2] = halfm + (halfp - halfm) * rand() * inv_rand_max;
  }
}

/* FP64 potential and its gradient on sampled targets, without the target-charge factor:
   pot[t] = sum_{x_j != x_i} q_j / r_ij, fld[3t + a] = sum_j q_j (x_j - x_i)_a / r_ij^3,
   i = targets[t] (the derivative of the direct sum of bbfmm.c:880-913; the reference has
   no gradient code). Neumaier-compensated sums. */
void SFX(orc_direct_field_fp64)(int N, const double *xyz, const double *q, int ntarget, const int *targets,
                                double *pot, double *fld)
{
  for (int t = 0; t < ntarget; t++) {
    int i = targets[t];
    double fx = xyz[3 * i], fy = xyz[3 * i + 1], fz = xyz[3 * i + 2];
    double s[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};
    for (int j = 0; j < N; j++) {
      double dx = xyz[3 * j] - fx, dy = xyz[3 * j + 1] - fy, dz = xyz[3 * j + 2] - fz;
      double rr = dx * dx + dy * dy + dz * dz;
      if (rr == 0.0) continue;
      double rinv = 1.0 / sqrt(rr), v[4];
      v[0] = q[j] * rinv;
      v[1] = v[0] * rinv * rinv * dx;
      v[2] = v[0] * rinv * rinv * dy;
      v[3] = v[0] * rinv * rinv * dz;
      for (int a = 0; a < 4; a++) {
        double y = s[a] + v[a];
        c[a] += (fabs(s[a]) >= fabs(v[a])) ? ((s[a] - y) + v[a]) : ((v[a] - y) + s[a]);
        s[a] = y;
      }
    }
    pot[t] = s[0] + c[0];
    for (int a = 0; a < 3; a++) fld[3 * t + a] = s[a + 1] + c[a + 1];
  }
}
