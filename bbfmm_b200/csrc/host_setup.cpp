// Host-side set-up that stays in C++: Chebyshev tables and the leaf sort.
//
//  * bbfmm_weights<T>: the tables of ComputeWeights (bbfmm.c:922-1028) computed in the
//    working precision T, with the same operations, so that a float build produces the
//    same tables as the reference's SINGLE build.
//  * bbfmm_sort_particles<T>: the leaf assignment of anotherFMMDistribute.c:258-298
//    (truncating (x + L/2) / leaf_length, clamped to the last leaf) and a stable counting
//    sort into leaves in Morton (reference) order, i.e. the particle order of the
//    reference's fieldlist (anotherFMMDistribute.c:431-473).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace {

template <typename T>
void tk(T x, int n, T *vec) {
  vec[0] = 1;
  vec[1] = x;
  for (int k = 2; k < n; k++) vec[k] = 2 * x * vec[k - 1] - vec[k - 2];
}

template <typename T>
T sn_clenshaw(const T *vec, int n, T x) {
  T d[40];
  d[n] = d[n + 1] = 0;
  for (int j = n - 1; j > 0; j--) d[j] = 2 * x * d[j + 1] - d[j + 2] + vec[j];
  return x * d[1] - d[2] + (T)0.5 * vec[0];
}

template <typename T> T tcos(T x);
template <> float tcos<float>(float x) { return cosf(x); }
template <> double tcos<double>(double x) { return cos(x); }
template <typename T> T tsqrt(T x);
template <> float tsqrt<float>(float x) { return sqrtf(x); }
template <> double tsqrt<double>(double x) { return sqrt(x); }

}  // namespace

template <typename T>
int bbfmm_weights(int n, T *Tkz, int *Ktable, T *Kweights, T *Cweights) {
  if (n < 2 || n > 32) return bbfmm_set_error(BBFMM_ERR_ARG, "order n must be in [2, 32]");
  T nodes[32], vec[32];
  const T pi = (T)3.1415926535897932384626433832795;
  for (int i = 0; i < 343; i++) Ktable[i] = -1;
  int c = 0, k = 0;
  for (int l1 = -3; l1 < 4; l1++)
    for (int l2 = -3; l2 < 4; l2++)
      for (int l3 = -3; l3 < 4; l3++) {
        if (std::abs(l1) > 1 || std::abs(l2) > 1 || std::abs(l3) > 1) Ktable[c] = k++;
        c++;
      }
  for (int m = 0; m < n; m++) nodes[m] = tcos<T>(pi * (T)(2 * m + 1) / (T)(2 * n));
  for (int m = 0; m < n; m++) {
    tk<T>(nodes[m], n, vec);
    for (int j = 0; j < n; j++) Tkz[m * n + j] = vec[j];
  }
  int cnt = 0;
  for (int l1 = 0; l1 < n; l1++) {
    T t1 = 1 / tsqrt<T>(1 - nodes[l1] * nodes[l1]);
    for (int l2 = 0; l2 < n; l2++) {
      T t2 = t1 / tsqrt<T>(1 - nodes[l2] * nodes[l2]);
      for (int l3 = 0; l3 < n; l3++) Kweights[cnt++] = t2 / tsqrt<T>(1 - nodes[l3] * nodes[l3]);
    }
  }
  for (int side = 0; side < 2; side++)
    for (int p = 0; p < n; p++)
      for (int q = 0; q < n; q++) {
        T z = (T)0.5 * (nodes[q] + (side ? (T)1 : (T)-1));
        Cweights[side * n * n + p * n + q] = sn_clenshaw<T>(&Tkz[p * n], n, z);
      }
  return BBFMM_OK;
}

template <typename T>
int bbfmm_sort_particles(int N, const T *xyz, T L, int maxlev, int *perm, int *leaf_start) {
  if (N < 0 || maxlev < BBFMM_MINLEV || maxlev > 10)
    return bbfmm_set_error(BBFMM_ERR_ARG, "need N >= 0 and 2 <= maxlev <= 10");
  const int ncpd = 1 << maxlev;
  const int64_t nleaf = pow8i(maxlev);
  T celeng_max = L;
  for (int l = 1; l <= maxlev; ++l) celeng_max *= (T)0.5;
  const T L0half = L / 2, iLm = 1 / celeng_max;
  std::vector<int> leaf(N > 0 ? N : 1);
  std::vector<int> cnt(nleaf + 1, 0);
  for (int i = 0; i < N; i++) {
    const T x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
    if (!(x >= -L0half && x <= L0half && y >= -L0half && y <= L0half && z >= -L0half &&
          z <= L0half))
      return bbfmm_set_error(BBFMM_ERR_ARG, "particle outside the root cell [-L/2, L/2]^3");
    int ix = (int)((x + L0half) * iLm), iy = (int)((y + L0half) * iLm), iz = (int)((z + L0half) * iLm);
    if (ix > ncpd - 1) ix = ncpd - 1;
    if (iy > ncpd - 1) iy = ncpd - 1;
    if (iz > ncpd - 1) iz = ncpd - 1;
    leaf[i] = (int)grid_to_morton(ix, iy, iz, maxlev);
    cnt[leaf[i] + 1]++;
  }
  for (int64_t k = 0; k < nleaf; k++) cnt[k + 1] += cnt[k];
  std::memcpy(leaf_start, cnt.data(), sizeof(int) * (nleaf + 1));
  for (int i = 0; i < N; i++) perm[cnt[leaf[i]]++] = i;
  return BBFMM_OK;
}

template int bbfmm_weights<float>(int, float *, int *, float *, float *);
template int bbfmm_weights<double>(int, double *, int *, double *, double *);
template int bbfmm_sort_particles<float>(int, const float *, float, int, int *, int *);
template int bbfmm_sort_particles<double>(int, const double *, double, int, int *, int *);
